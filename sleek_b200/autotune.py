"""Autotuner for the launch shape.

The 16 KB chunk is part of the stream format (``SLEEK_CS``, enforced by
``sleek_system_checks`` in the reference), so what is tuned is how the work is
laid on the GPU: CTAs per SM of the persistent kernels (each CTA is 10 warps and
keeps a 4-deep pipeline of chunks), for the single-buffer kernels of each kind and
for batched plans.  Candidates are timed with CUDA events on the caller's data
(outputs are identical for every candidate), and the winner is cached per device
name and workload key in a JSON file.
"""
from __future__ import annotations

import json
import os
from typing import Callable, Dict, Optional

import torch

from . import _capi

CANDIDATES = (1, 2, 3)


def _cache_path() -> str:
    return os.environ.get("SLEEK_TUNING_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "sleek_b200", "tuning.json"))


def _load() -> Dict[str, int]:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save(d: Dict[str, int]) -> None:
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


def tune(key: str, run_with: Callable[[int], None], candidates=CANDIDATES, use_cache: bool = True) -> dict:
    """Times ``run_with(ctas_per_sm)`` for each candidate and returns
    {"best": c, "ms": {c: ms}}; cached under ``key`` + device name."""
    full = f"{torch.cuda.get_device_name()}|{key}"
    cache = _load() if use_cache else {}
    if full in cache:
        return {"best": cache[full], "ms": {}, "cached": True}
    ms = {c: _time(lambda c=c: run_with(c)) for c in candidates}
    best = min(ms, key=ms.get)
    if use_cache:
        cache[full] = best
        _save(cache)
    return {"best": best, "ms": ms, "cached": False}


def tune_single(x: torch.Tensor, eb: Optional[float], decompress: bool = False, use_cache: bool = True) -> dict:
    """Tunes and applies CTAs per SM for the single-buffer kernel of x's kind."""
    from . import api

    L = _capi.lib()
    w = x.element_size()
    lossy = int(eb is not None)
    enc = api.compress(x, eb)
    dt = torch.float32 if w == 4 else torch.float64
    out = torch.empty_like(x)

    def run(c):
        L.sleek_set_ctas_per_sm(int(decompress), w, lossy, c)
        if decompress:
            api.decompress(enc, dt, eb, out=out)
        else:
            api.compress(x, eb)

    key = f"single|{'dec' if decompress else 'enc'}|{w}|{lossy}|{x.numel() * w >> 24}"
    r = tune(key, run, use_cache=use_cache)
    L.sleek_set_ctas_per_sm(int(decompress), w, lossy, r["best"])
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
