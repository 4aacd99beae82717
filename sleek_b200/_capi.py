"""ctypes binding of the C ABI in ``include/sleek_capi.h``.

Loads ``sleek_b200/_lib/libsleek_b200.so`` (built by ``sleek_b200/build.py``).
There is no fallback: if the library is missing or cannot be loaded, importing
the binding raises, so a box without the CUDA build fails loudly instead of
silently computing something else.
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

LIB_PATH = _build.LIB

SLEEK_OK = 0
SLEEK_ERR_INVALID_ARG = 1
SLEEK_ERR_ALIGNMENT = 2
SLEEK_ERR_CUDA = 3
SLEEK_ERR_ERROR_BOUND = 4
SLEEK_ERR_CORRUPT_STREAM = 5
SLEEK_ERR_TIMEOUT = 6
SLEEK_ERR_WORKSPACE = 7
SLEEK_ERR_NO_DEVICE = 8
SLEEK_ERR_CAPACITY = 9
SLEEK_ERR_TOO_LARGE = 10
SLEEK_SELFTEST_VALUE_CHECKS = 6


class EbInfoF32(C.Structure):
    _fields_ = [("eb_e", C.c_int), ("thr_e", C.c_int), ("offs_e", C.c_uint)]


class EbInfoF64(C.Structure):
    _fields_ = [("eb_e", C.c_int), ("thr_e", C.c_int), ("offs_e", C.c_ulonglong)]


class BatchItem(C.Structure):
    _fields_ = [("input", C.c_void_p), ("output", C.c_void_p), ("size_out", C.c_void_p),
                ("num_elements", C.c_longlong), ("stream_bytes", C.c_longlong),
                ("elem_bytes", C.c_int), ("lossy", C.c_int), ("error_bound", C.c_double)]


class ServerRequest(C.Structure):
    _fields_ = [("input", C.c_void_p), ("num_elements", C.c_longlong), ("stream_bytes", C.c_longlong),
                ("arrival_s", C.c_double), ("error_bound", C.c_double), ("tag", C.c_longlong),
                ("op", C.c_int), ("elem_bytes", C.c_int), ("lossy", C.c_int), ("keep", C.c_int)]


class ServerCompletion(C.Structure):
    _fields_ = [("tag", C.c_longlong), ("result_bytes", C.c_longlong), ("output", C.c_void_p),
                ("arrival_s", C.c_double), ("done_s", C.c_double)]


# every symbol the header declares: name -> (restype, argtypes)
_i64 = C.c_longlong
class StreamInfo(C.Structure):
    _fields_ = [("insize", C.c_longlong), ("chunks", C.c_longlong), ("stream_bytes", C.c_longlong),
                ("raw_chunks", C.c_longlong), ("bad_chunk", C.c_longlong), ("reason", C.c_int), ("pad_", C.c_int)]


_vp = C.c_void_p
_sz = C.c_size_t
SIGNATURES = {
    "sleek_status_string": (C.c_char_p, [C.c_int]),
    "sleek_upper_bound_size": (_i64, [_i64]),
    "sleek_system_checks": (C.c_int, []),
    "sleek_thread_blocks": (C.c_int, []),
    "sleek_compress_workspace_size": (_sz, [_i64]),
    "sleek_decompress_workspace_size": (_sz, []),
    "sleek_error_bound_f32": (C.c_int, [C.c_float, C.POINTER(EbInfoF32)]),
    "sleek_error_bound_f64": (C.c_int, [C.c_double, C.POINTER(EbInfoF64)]),
    "sleek_compress_f32": (C.c_int, [_vp, _i64, _vp, _vp, _vp, _sz, _vp]),
    "sleek_compress_f64": (C.c_int, [_vp, _i64, _vp, _vp, _vp, _sz, _vp]),
    "sleek_decompress_f32": (C.c_int, [_vp, _i64, _vp, _i64, _vp, _vp, _sz, _vp]),
    "sleek_decompress_f64": (C.c_int, [_vp, _i64, _vp, _i64, _vp, _vp, _sz, _vp]),
    "sleek_compress_lossy_f32": (C.c_int, [EbInfoF32, _vp, _i64, _vp, _vp, _vp, _sz, _vp]),
    "sleek_compress_lossy_f64": (C.c_int, [EbInfoF64, _vp, _i64, _vp, _vp, _vp, _sz, _vp]),
    "sleek_decompress_lossy_f32": (C.c_int, [EbInfoF32, _vp, _i64, _vp, _i64, _vp, _vp, _sz, _vp]),
    "sleek_decompress_lossy_f64": (C.c_int, [EbInfoF64, _vp, _i64, _vp, _i64, _vp, _vp, _sz, _vp]),
    "sleek_workspace_status": (C.c_int, [_vp, _vp, C.POINTER(C.c_int)]),
    "sleek_compress_f32_static": (C.c_int, [_vp, _i64, _vp, _vp, _vp]),
    "sleek_set_ctas_per_sm": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int]),
    "sleek_launch_shape_info": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                          C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "sleek_set_launch_shape": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    "sleek_compress_to_host": (C.c_int, [_vp, C.c_longlong, C.c_int, C.c_int, C.c_double, _vp, C.c_longlong,
                                         C.POINTER(C.c_longlong), C.c_longlong, _vp]),
    "sleek_decompress_from_host": (C.c_int, [_vp, C.c_longlong, C.c_int, C.c_int, C.c_double, _vp, C.c_longlong,
                                             C.POINTER(C.c_longlong), C.c_longlong, _vp]),
    "sleek_validate_stream": (C.c_int, [_vp, C.c_longlong, C.c_int, _vp]),
    "sleek_stream_reason_string": (C.c_char_p, [C.c_int]),
    "sleek_selftest_bounded_waits": (C.c_int, [C.c_longlong, C.POINTER(C.c_longlong)]),
    "sleek_selftest_value_maps": (C.c_int, [C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "sleek_minmax_f32": (C.c_int, [_vp, C.c_longlong, C.POINTER(C.c_float), C.POINTER(C.c_float), _vp]),
    "sleek_minmax_f64": (C.c_int, [_vp, C.c_longlong, C.POINTER(C.c_double), C.POINTER(C.c_double), _vp]),
    "sleek_batch_plan_create": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "sleek_batch_plan_workspace_size": (_sz, [_vp]),
    "sleek_batch_plan_create_reusable": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "sleek_batch_plan_set_items": (C.c_int, [_vp, C.c_void_p, C.c_int, _vp]),
    "sleek_batch_plan_set_grid": (C.c_int, [_vp, C.c_int]),
    "sleek_batch_plan_run": (C.c_int, [_vp, _vp, _sz, _vp]),
    "sleek_batch_plan_destroy": (C.c_int, [_vp]),
    "sleek_compress_batch": (C.c_int, [C.c_void_p, C.c_int, _vp, _sz, _vp]),
    "sleek_decompress_batch": (C.c_int, [C.c_void_p, C.c_int, _vp, _sz, _vp]),
    "sleek_server_create": (C.c_int, [_vp, C.c_longlong, C.c_int, C.c_int, C.c_longlong, C.POINTER(C.c_void_p)]),
    "sleek_server_now": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "sleek_server_submit": (C.c_int, [_vp, C.c_void_p, C.c_longlong]),
    "sleek_server_poll": (C.c_int, [_vp, C.c_void_p, C.c_longlong, C.POINTER(C.c_longlong), C.c_int]),
    "sleek_server_outstanding": (C.c_int, [_vp, C.POINTER(C.c_longlong)]),
    "sleek_server_arena_info": (C.c_int, [_vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "sleek_server_release": (C.c_int, [_vp, _vp]),
    "sleek_server_destroy": (C.c_int, [_vp]),
    "sleek_server_arena_replay": (C.c_int, [C.c_longlong, C.c_void_p, C.c_longlong, C.c_void_p]),
}

_lib = None


def lib() -> C.CDLL:
    """The loaded library; raises OSError when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing: build it with `python -m sleek_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (rt, at) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = rt
            f.argtypes = at
        _lib = L
    return _lib


class SleekError(RuntimeError):
    def __init__(self, status: int, where: str = ""):
        self.status = int(status)
        msg = lib().sleek_status_string(self.status).decode()
        super().__init__(f"{where}: {msg} (status {self.status})" if where else f"{msg} (status {self.status})")


def check(status: int, where: str = "") -> None:
    if status != SLEEK_OK:
        raise SleekError(status, where)
