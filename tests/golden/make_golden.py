"""Generates the golden fixtures in tests/golden/ from the REFERENCE's own CPU
codec (oracle/_ref/libsleek_ref_cpu.so, compiled from the SLEEK headers by
oracle/Makefile).  Run once where the reference sources exist:

    make -C oracle ref && python tests/golden/make_golden.py

Each case stores its input (``<name>.in.npy``), the reference's compressed
stream (``<name>.sleek``) and, in ``manifest.json``, the dtype, the error bound
(null = lossless) and SHA-256 digests of the stream and of the reference's
decoded output.  Inputs are stored rather than regenerated so the fixtures do
not depend on any floating-point library of the machine that reads them.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

CS = 16384


def smooth(n, dt, seed):
    rng = np.random.default_rng(seed)
    i = np.arange(n, dtype=np.float64)
    x = np.zeros(n)
    for _ in range(4):
        f = 10 ** rng.uniform(-5, -2)
        x += 1e3 * np.sin(2 * np.pi * f * i + rng.uniform(0, 2 * np.pi))
    x += rng.normal(0, 1e-3, n)
    x = x.astype(dt)
    k = max(1, n // 1000)
    idx = rng.choice(n, k, replace=False)
    tiny = np.float32(3e-41) if dt == np.float32 else np.float64(5e-320)
    sp = np.array([np.nan, np.inf, -np.inf, tiny], dt)
    x[idx] = sp[np.arange(k) % 4]
    return x


def random_bits(n, dt, seed):
    rng = np.random.default_rng(seed)
    it = np.uint32 if dt == np.float32 else np.uint64
    return rng.integers(0, np.iinfo(it).max, n, dtype=it, endpoint=True).view(dt)


def wide(n, dt, seed):
    """Alternating huge positive / tiny negative values: bit width TB in every subchunk."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(1, 2, n).astype(dt)
    x[0::2] *= (np.float32(3e38) if dt == np.float32 else 1e308)
    x[1::2] *= -(np.float32(1e-38) if dt == np.float32 else 1e-307)
    return x


def build_cases():
    cases = []
    for dt, tag in ((np.float32, "f32"), (np.float64, "f64")):
        w = np.dtype(dt).itemsize
        vpc = CS // w
        s = smooth(vpc * 3 + vpc // 2 + 3, dt, 11 if tag == "f32" else 12)
        cases += [
            (f"{tag}_smooth_lossless", s, None),
            (f"{tag}_smooth_eb1e-2", s, 1e-2),
            (f"{tag}_smooth_eb1e-4", s, 1e-4),
            (f"{tag}_smooth_eb1e-6", s, 1e-6),
            (f"{tag}_smooth_ebneg1e-3", s, -1e-3),
            (f"{tag}_smooth_ebdenormal", s, 1e-40 if tag == "f32" else 1e-310),
            (f"{tag}_smooth_eb0", s, 0.0),
            (f"{tag}_randbits_lossless", random_bits(vpc * 2 + 5, dt, 21), None),
            (f"{tag}_randbits_eb1e-3", random_bits(vpc * 2 + 5, dt, 22), 1e-3),
            (f"{tag}_zeros_lossless", np.zeros(vpc + 1, dt), None),
            (f"{tag}_zeros_eb1e-3", np.zeros(vpc + 1, dt), 1e-3),
            (f"{tag}_one_value", np.array([1.5], dt), None),
            (f"{tag}_one_value_eb1e-1", np.array([-2.75], dt), 0.1),
            (f"{tag}_exact_chunk", smooth(vpc, dt, 31), None),
            (f"{tag}_wide", wide(vpc + 7, dt, 41), None),
            (f"{tag}_wide_eb1e-5", wide(vpc + 7, dt, 42), 1e-5),
        ]
    return cases


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def main():
    if O.ref_cpu() is None:
        raise SystemExit("reference CPU build missing: run `make -C oracle ref` first")
    manifest = []
    for name, x, eb in build_cases():
        stream = O.ref_encode(x, eb)
        dec = O.ref_decode(stream, x.dtype, eb)
        np.save(os.path.join(HERE, f"{name}.in.npy"), x)
        with open(os.path.join(HERE, f"{name}.sleek"), "wb") as f:
            f.write(stream)
        manifest.append({
            "name": name, "dtype": str(x.dtype), "eb": eb, "n": int(x.size),
            "stream_bytes": len(stream), "stream_sha256": sha(stream), "decoded_sha256": sha(dec.tobytes()),
        })
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump({"generator": "reference CPU codec (include/sleek_common_cpu.h) via oracle/_ref",
                   "cases": manifest}, f, indent=1)
    print(f"{len(manifest)} cases written")


if __name__ == "__main__":
    main()
