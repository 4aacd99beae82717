"""Loader for the parity checkers (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.  It wraps three shared libraries built by
``oracle/Makefile``:

* ``oracle/_lib/libsleek_oracle.so`` -- the C restatement in ``sleek_oracle.c``
  (rebuilt with ``gcc`` on demand, so it is available on any box with a C
  compiler);
* ``oracle/_ref/libsleek_ref_cpu.so`` -- the reference's own CPU codec
  (``include/sleek_common_cpu.h``), compiled from the reference sources;
* ``oracle/_ref/libsleek_ref_gpu.so`` -- the reference's own GPU codec
  (``include/sleek_common_gpu.h``) for sm_100a.

The reference libraries only exist where they were built (they are carried
with the working tree, not the git history); callers must treat them as
optional and skip when absent.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "_lib")
REF_DIR = os.path.join(HERE, "_ref")
CS = 16384

_c = ctypes
_i64 = _c.c_longlong
_vp = _c.c_void_p


def _build_oracle() -> str:
    path = os.path.join(LIB_DIR, "libsleek_oracle.so")
    src = os.path.join(HERE, "sleek_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        os.makedirs(LIB_DIR, exist_ok=True)
        subprocess.check_call(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-o", path, src])
    return path


_oracle = None


def lib():
    """The C restatement (always available; built with gcc if missing)."""
    global _oracle
    if _oracle is None:
        L = _c.CDLL(_build_oracle())
        L.oracle_encode.restype = _i64
        L.oracle_encode.argtypes = [_c.c_int, _c.c_int, _vp, _i64, _vp, _c.c_int, _c.c_int, _c.c_ulonglong]
        L.oracle_decode.restype = _c.c_int
        L.oracle_decode.argtypes = [_c.c_int, _c.c_int, _vp, _i64, _vp, _i64, _c.POINTER(_i64), _c.c_int, _c.c_ulonglong]
        L.oracle_upper_bound_size.restype = _i64
        L.oracle_upper_bound_size.argtypes = [_i64]
        L.oracle_error_bound_f32.restype = _c.c_int
        L.oracle_error_bound_f32.argtypes = [_c.c_float, _c.POINTER(_c.c_int), _c.POINTER(_c.c_int), _c.POINTER(_c.c_uint)]
        L.oracle_error_bound_f64.restype = _c.c_int
        L.oracle_error_bound_f64.argtypes = [_c.c_double, _c.POINTER(_c.c_int), _c.POINTER(_c.c_int), _c.POINTER(_c.c_ulonglong)]
        for n, rt, at in [
            ("oracle_fwd32", _c.c_uint, [_c.c_uint]), ("oracle_inv32", _c.c_uint, [_c.c_uint]),
            ("oracle_fwd64", _c.c_ulonglong, [_c.c_ulonglong]), ("oracle_inv64", _c.c_ulonglong, [_c.c_ulonglong]),
            ("oracle_quant32", _c.c_uint, [_c.c_uint, _c.c_int, _c.c_int, _c.c_uint]),
            ("oracle_dequant32", _c.c_uint, [_c.c_uint, _c.c_int, _c.c_uint]),
            ("oracle_quant64", _c.c_ulonglong, [_c.c_ulonglong, _c.c_int, _c.c_int, _c.c_ulonglong]),
            ("oracle_dequant64", _c.c_ulonglong, [_c.c_ulonglong, _c.c_int, _c.c_ulonglong]),
        ]:
            f = getattr(L, n)
            f.restype = rt
            f.argtypes = at
        _oracle = L
    return _oracle


def upper_bound_size(insize: int) -> int:
    return int(lib().oracle_upper_bound_size(insize))


def error_bound(eb: float, dtype) -> tuple[int, int, int]:
    """(eb_e, thr_e, offs_e) as the reference derives them, or raises ValueError."""
    a, b = _c.c_int(), _c.c_int()
    if np.dtype(dtype) == np.float32:
        o = _c.c_uint()
        rc = lib().oracle_error_bound_f32(float(eb), a, b, o)
    else:
        o = _c.c_ulonglong()
        rc = lib().oracle_error_bound_f64(float(eb), a, b, o)
    if rc != 0:
        raise ValueError("error bound too large")
    return a.value, b.value, o.value


def encode(x: np.ndarray, eb: float | None = None) -> bytes:
    """Compress a float32/float64 array; eb=None means lossless."""
    x = np.ascontiguousarray(x)
    width = x.dtype.itemsize
    assert x.dtype in (np.float32, np.float64)
    out = np.zeros(max(upper_bound_size(x.nbytes), 16), np.uint8)
    if eb is None:
        n = lib().oracle_encode(width, 0, x.ctypes.data, x.nbytes, out.ctypes.data, 0, 0, 0)
    else:
        e, t, o = error_bound(eb, x.dtype)
        n = lib().oracle_encode(width, 1, x.ctypes.data, x.nbytes, out.ctypes.data, e, t, o)
    if n < 0:
        raise ValueError("oracle encode failed")
    return out[:n].tobytes()


def decode(stream: bytes, dtype, eb: float | None = None) -> np.ndarray:
    """Decompress; raises ValueError on a malformed stream (trailer, sizes)."""
    dtype = np.dtype(dtype)
    s = np.frombuffer(stream, np.uint8)
    insize = int(np.frombuffer(stream[:8], np.int64)[0]) if len(stream) >= 8 else -1
    if insize < 0:
        raise ValueError("corrupt stream")
    out = np.zeros(insize // dtype.itemsize + 1, dtype)
    got = _i64()
    if eb is None:
        rc = lib().oracle_decode(dtype.itemsize, 0, s.ctypes.data, len(s), out.ctypes.data, out.nbytes, got, 0, 0)
    else:
        _, t, o = error_bound(eb, dtype)
        rc = lib().oracle_decode(dtype.itemsize, 1, s.ctypes.data, len(s), out.ctypes.data, out.nbytes, got, t, o)
    if rc != 0:
        raise ValueError(f"corrupt stream (status {rc})")
    return out[: got.value // dtype.itemsize]


# ---- the reference's own CPU codec (optional) --------------------------------

_ref_cpu = None


def ref_cpu_path() -> str:
    return os.path.join(REF_DIR, "libsleek_ref_cpu.so")


def ref_cpu():
    """The reference CPU codec, or None when it was not built here."""
    global _ref_cpu
    if _ref_cpu is None and os.path.exists(ref_cpu_path()):
        L = _c.CDLL(ref_cpu_path())
        for t, ct in (("f32", _c.c_float), ("f64", _c.c_double)):
            f = getattr(L, f"ref_cpu_compress_{t}"); f.restype = _i64; f.argtypes = [_vp, _i64, _vp]
            f = getattr(L, f"ref_cpu_decompress_{t}"); f.restype = _i64; f.argtypes = [_vp, _vp]
            f = getattr(L, f"ref_cpu_compress_lossy_{t}"); f.restype = _i64; f.argtypes = [ct, _vp, _i64, _vp]
            f = getattr(L, f"ref_cpu_decompress_lossy_{t}"); f.restype = _i64; f.argtypes = [ct, _vp, _vp]
        _ref_cpu = L
    return _ref_cpu


def ref_encode(x: np.ndarray, eb: float | None = None) -> bytes:
    L = ref_cpu()
    x = np.ascontiguousarray(x)
    t = "f32" if x.dtype == np.float32 else "f64"
    out = np.zeros(max(upper_bound_size(x.nbytes), 16), np.uint8)
    if eb is None:
        n = getattr(L, f"ref_cpu_compress_{t}")(x.ctypes.data, x.size, out.ctypes.data)
    else:
        n = getattr(L, f"ref_cpu_compress_lossy_{t}")(eb, x.ctypes.data, x.size, out.ctypes.data)
    return out[:n].tobytes()


def ref_decode(stream: bytes, dtype, eb: float | None = None) -> np.ndarray:
    L = ref_cpu()
    dtype = np.dtype(dtype)
    s = np.frombuffer(stream, np.uint8)
    insize = int(np.frombuffer(stream[:8], np.int64)[0])
    out = np.zeros(insize // dtype.itemsize + 1, dtype)
    t = "f32" if dtype == np.float32 else "f64"
    if eb is None:
        n = getattr(L, f"ref_cpu_decompress_{t}")(s.ctypes.data, out.ctypes.data)
    else:
        n = getattr(L, f"ref_cpu_decompress_lossy_{t}")(eb, s.ctypes.data, out.ctypes.data)
    return out[: n // dtype.itemsize]


# ---- the reference's own GPU codec (optional; needs a GPU) --------------------

_ref_gpu = None


def ref_gpu_path() -> str:
    return os.path.join(REF_DIR, "libsleek_ref_gpu.so")


def ref_gpu():
    """The reference GPU codec, or None when it was not built here."""
    global _ref_gpu
    if _ref_gpu is None and os.path.exists(ref_gpu_path()):
        L = _c.CDLL(ref_gpu_path())
        L.ref_gpu_blocks.restype = _c.c_int
        for t, ct in (("f32", _c.c_float), ("f64", _c.c_double)):
            f = getattr(L, f"ref_gpu_compress_{t}"); f.restype = None; f.argtypes = [_c.c_int, _vp, _i64, _vp, _vp]
            f = getattr(L, f"ref_gpu_decompress_{t}"); f.restype = None; f.argtypes = [_c.c_int, _vp, _vp, _vp]
            f = getattr(L, f"ref_gpu_compress_lossy_{t}"); f.restype = None; f.argtypes = [_c.c_int, ct, _vp, _i64, _vp, _vp]
            f = getattr(L, f"ref_gpu_decompress_lossy_{t}"); f.restype = None; f.argtypes = [_c.c_int, ct, _vp, _vp, _vp]
            f = getattr(L, f"ref_gpu_encode_prealloc_{t}"); f.restype = None
            f.argtypes = [_c.c_int, _vp, _i64, _vp, _vp, _vp, _c.c_int, _c.c_double]
            f = getattr(L, f"ref_gpu_decode_prealloc_{t}"); f.restype = None
            f.argtypes = [_c.c_int, _vp, _vp, _vp, _vp, _c.c_int, _c.c_double]
        _ref_gpu = L
    return _ref_gpu
