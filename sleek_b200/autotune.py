"""Autotuner for the launch shape.

The 16 KB chunk is part of the stream format (``SLEEK_CS``, enforced by
``sleek_system_checks`` in the reference), so what is tuned is how the work is
laid on the GPU, where the reference uses fixed constants (``SLEEK_TPB`` = 512
threads and a grid from ``sleek_thread_blocks``, include/sleek_common_gpu.h:54-56,
108-119):

- single-buffer calls: the kernel shape -- threads per CTA, compute warps (and so
  subchunks per warp) and shared-memory chunk stages, from the shapes the library
  is built with (``sleek_launch_shape_info``) -- and the CTAs per SM, per kind
  (element size, lossless / lossy, compress / decompress) and per input-size
  bucket (base-2 logarithm of the bytes), applied with ``sleek_set_launch_shape``;
- batched plans: CTAs per SM (``sleek_batch_plan_set_grid``).

Candidates are timed with CUDA events on the caller's data (outputs are identical
for every candidate), and the winner is cached per device name and key in a JSON
file.
"""
from __future__ import annotations

import ctypes as C
import json
import os
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np
import torch

from . import _capi

CANDIDATES = (1, 2, 3)


def _cache_path() -> str:
    return os.environ.get("SLEEK_TUNING_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "sleek_b200", "tuning.json"))


def _load() -> Dict[str, object]:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save(d: Dict[str, object]) -> None:
    p = _cache_path()
    os.makedirs(os.path.dirname(p), exist_ok=True)
    with open(p, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)


def _time(fn: Callable[[], None], reps: int = 5) -> float:
    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def tune(key: str, run_with: Callable, candidates: Sequence = CANDIDATES, use_cache: bool = True) -> dict:
    """Times ``run_with(candidate)`` for each candidate and returns
    {"best": c, "ms": {str(c): ms}}; cached under ``key`` + device name."""
    full = f"{torch.cuda.get_device_name()}|{key}"
    cache = _load() if use_cache else {}
    if full in cache:
        best = cache[full]
        return {"best": tuple(best) if isinstance(best, list) else best, "ms": {}, "cached": True}
    ms = {c: _time(lambda c=c: run_with(c)) for c in candidates}
    best = min(ms, key=ms.get)
    if use_cache:
        cache[full] = list(best) if isinstance(best, tuple) else best
        _save(cache)
    return {"best": best, "ms": {str(c): round(v, 4) for c, v in ms.items()}, "cached": False}


def shapes(decompress: bool) -> List[dict]:
    """The launch shapes the library is built with for one direction."""
    L = _capi.lib()
    out = []
    k = 0
    while True:
        t, w, s, c = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        if L.sleek_launch_shape_info(int(decompress), k, C.byref(t), C.byref(w), C.byref(s), C.byref(c)) != 0:
            return out
        out.append({"shape": k, "threads": t.value, "warps": w.value, "stages": s.value, "ctas_per_sm": c.value})
        k += 1


def single_candidates(decompress: bool) -> List[tuple]:
    """(shape, CTAs per SM) pairs: every shape at as many CTAs as fit (0) and at one fewer."""
    out = []
    for sh in shapes(decompress):
        out.append((sh["shape"], 0))
        if sh["ctas_per_sm"] > 1:
            out.append((sh["shape"], sh["ctas_per_sm"] - 1))
    return out


def size_log2(nbytes: int) -> int:
    return max(0, int(nbytes).bit_length() - 1)


def tune_single(x: torch.Tensor, eb: Optional[float], decompress: bool = False, use_cache: bool = True) -> dict:
    """Tunes and applies the launch shape and CTAs per SM of the single-buffer kernel
    of x's kind for inputs in x's size bucket.  Candidates are timed on the device:
    C-ABI calls into preallocated buffers, back to back on the current stream (no
    host wait between calls, so small inputs are not timed by the host's latency)."""
    from . import api

    L = _capi.lib()
    w = x.element_size()
    lossy = int(eb is not None)
    x = x.contiguous().view(-1)
    nbytes = x.numel() * w
    bucket = size_log2(nbytes)
    t = "f32" if w == 4 else "f64"
    enc = api.compress(x, eb)
    out = torch.empty_like(x)
    buf = torch.empty(api.sleek_upper_bound_size(nbytes), dtype=torch.uint8, device=x.device)
    size = torch.zeros(1, dtype=torch.int64, device=x.device)
    pre = (api.sleek_error_bound(eb, np.float32 if w == 4 else np.float64).c_struct(),) if lossy else ()
    mid = "_lossy" if lossy else ""
    fc = getattr(L, f"sleek_compress{mid}_{t}")
    fd = getattr(L, f"sleek_decompress{mid}_{t}")

    def apply(c):
        _capi.check(L.sleek_set_launch_shape(int(decompress), w, lossy, bucket, c[0], c[1]), "sleek_set_launch_shape")

    def run(c):
        apply(c)
        sh = torch.cuda.current_stream().cuda_stream
        for _ in range(4):
            if decompress:
                rc = fd(*pre, enc.data_ptr(), enc.numel(), out.data_ptr(), nbytes, size.data_ptr(), None, 0, sh)
            else:
                rc = fc(*pre, x.data_ptr(), x.numel(), buf.data_ptr(), size.data_ptr(), None, 0, sh)
            _capi.check(rc)

    key = f"single|{'dec' if decompress else 'enc'}|{w}|{lossy}|2^{bucket}"
    r = tune(key, run, single_candidates(decompress), use_cache=use_cache)
    apply(r["best"])
    r.update({"bucket_log2": bucket, "shape": shapes(decompress)[r["best"][0]]})
    return r


def tune_plan(plan, key: str, use_cache: bool = True) -> dict:
    """Tunes and applies CTAs per SM for a batched plan."""
    L = _capi.lib()

    def run(c):
        L.sleek_batch_plan_set_grid(plan._h, c)
        plan.run()

    r = tune("batch|" + key, run, use_cache=use_cache)
    L.sleek_batch_plan_set_grid(plan._h, r["best"])
    return r
