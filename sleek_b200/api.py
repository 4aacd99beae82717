"""Python mirror of SLEEK's GPU API, backed by the sm_100a C ABI.

Names and argument order follow the reference headers
(``include/sleek_lossless_gpu.h``, ``include/sleek_lossy_gpu.h``,
``include/sleek_common_gpu.h``); device buffers are torch CUDA tensors.  The
differences from the reference are in error behaviour only: where the
reference calls ``exit(-1)`` or traps on the device, these functions raise
``SleekError`` (host-detected errors immediately; device-detected errors when
``check=True`` or when the size output is read and found negative).

Calls are asynchronous on the current torch CUDA stream unless ``check=True``.
"""
from __future__ import annotations

import ctypes as C
from typing import NamedTuple, Optional

import numpy as np
import torch

from . import _capi
from ._capi import SleekError, check

CS = 16384  # chunk bytes, fixed by the stream format (sleek_common_gpu.h:54)


class ErrorBoundInfo(NamedTuple):
    """Quantizer parameters; mirrors sleek_error_bound_info<T> (sleek_lossy_gpu.h:47-53)."""

    eb_e: int
    thr_e: int
    offs_e: int
    dtype: np.dtype

    def c_struct(self):
        if self.dtype == np.float32:
            return _capi.EbInfoF32(self.eb_e, self.thr_e, self.offs_e)
        return _capi.EbInfoF64(self.eb_e, self.thr_e, self.offs_e)


def sleek_upper_bound_size(insize: int) -> int:
    """Bytes to allocate for the stream of an insize-byte input (sleek_common_gpu.h:79-83)."""
    return int(_capi.lib().sleek_upper_bound_size(int(insize)))


def sleek_system_checks() -> int:
    """0 on a supported host, -1 otherwise (sleek_common_gpu.h:86-105)."""
    return int(_capi.lib().sleek_system_checks())


def sleek_thread_blocks() -> int:
    """Persistent grid size used on the current device (sleek_common_gpu.h:108-119)."""
    return int(_capi.lib().sleek_thread_blocks())


def sleek_error_bound(eb, dtype=None) -> ErrorBoundInfo:
    """Derives the quantizer parameters of an absolute error bound
    (sleek_lossy_gpu.h:56-71).  ``dtype`` defaults to the type of ``eb`` when it
    is a numpy float32/float64 scalar, else float32.  Raises SleekError with
    SLEEK_ERR_ERROR_BOUND where the reference exits."""
    if dtype is None:
        dtype = eb.dtype if isinstance(eb, np.floating) else np.float32
    dtype = np.dtype(dtype)
    if dtype == np.float32:
        info = _capi.EbInfoF32()
        check(_capi.lib().sleek_error_bound_f32(float(np.float32(eb)), C.byref(info)), "sleek_error_bound")
    elif dtype == np.float64:
        info = _capi.EbInfoF64()
        check(_capi.lib().sleek_error_bound_f64(float(eb), C.byref(info)), "sleek_error_bound")
    else:
        raise TypeError("error bounds exist for float32 and float64 only")
    return ErrorBoundInfo(info.eb_e, info.thr_e, info.offs_e, dtype)


def _np_dtype(t: torch.Tensor) -> np.dtype:
    if t.dtype == torch.float32:
        return np.dtype(np.float32)
    if t.dtype == torch.float64:
        return np.dtype(np.float64)
    raise TypeError("SLEEK compresses float32 and float64 data")


def _stream_handle(stream) -> int:
    if stream is None:
        stream = torch.cuda.current_stream()
    return int(stream.cuda_stream) if isinstance(stream, torch.cuda.Stream) else int(stream)


def _ws(workspace):
    if workspace is None:
        return None, 0
    return workspace.data_ptr(), workspace.numel() * workspace.element_size()


def _check_device(*ts):
    for t in ts:
        if not (isinstance(t, torch.Tensor) and t.is_cuda):
            raise TypeError("device buffers must be CUDA tensors")


def _raise_if_negative(size_tensor: torch.Tensor, where: str) -> int:
    v = int(size_tensor.view(-1)[0].item())
    if v < 0:
        raise SleekError(-v, where)
    return v


def sleek_compress_gpu(blocks: int, *args, stream=None, workspace=None, check: bool = False) -> None:
    """``sleek_compress_gpu(blocks, d_input, num_elements, d_encoded, d_encsize)`` or,
    lossy, ``sleek_compress_gpu(blocks, eb_info, d_input, num_elements, d_encoded, d_encsize)``
    (sleek_lossless_gpu.h:47-60, 75-88; sleek_lossy_gpu.h:74-88, 102-116).

    ``blocks`` is accepted for compatibility and ignored (the grid is sized from
    the kernels' occupancy).  ``d_encoded`` is a uint8 CUDA tensor of at least
    ``sleek_upper_bound_size`` bytes; ``d_encsize`` an int64 CUDA tensor that
    receives the stream size."""
    eb_info = None
    if args and isinstance(args[0], ErrorBoundInfo):
        eb_info, args = args[0], args[1:]
    d_input, num_elements, d_encoded, d_encsize = args
    _check_device(d_input, d_encoded, d_encsize)
    dt = _np_dtype(d_input)
    if num_elements > d_input.numel():
        raise SleekError(_capi.SLEEK_ERR_INVALID_ARG, "sleek_compress_gpu: num_elements exceeds the input")
    if d_encoded.numel() * d_encoded.element_size() < sleek_upper_bound_size(num_elements * dt.itemsize):
        raise SleekError(_capi.SLEEK_ERR_CAPACITY, "sleek_compress_gpu: d_encoded smaller than the upper bound")
    if d_encsize.dtype != torch.int64:
        raise TypeError("d_encsize must be an int64 tensor")
    L = _capi.lib()
    wp, wb = _ws(workspace)
    st = _stream_handle(stream)
    t = "f32" if dt == np.float32 else "f64"
    if eb_info is None:
        rc = getattr(L, f"sleek_compress_{t}")(d_input.data_ptr(), int(num_elements), d_encoded.data_ptr(),
                                               d_encsize.data_ptr(), wp, wb, st)
    else:
        if eb_info.dtype != dt:
            raise TypeError("eb_info dtype does not match the input dtype")
        rc = getattr(L, f"sleek_compress_lossy_{t}")(eb_info.c_struct(), d_input.data_ptr(), int(num_elements),
                                                     d_encoded.data_ptr(), d_encsize.data_ptr(), wp, wb, st)
    _capi.check(rc, "sleek_compress_gpu")
    if check:
        _raise_if_negative(d_encsize, "sleek_compress_gpu")


def sleek_decompress_gpu(blocks: int, *args, stream=None, workspace=None, check: bool = False,
                         encoded_bytes: int = -1) -> None:
    """``sleek_decompress_gpu(blocks, d_encoded, d_decoded, d_decsize)`` or, lossy,
    ``sleek_decompress_gpu(blocks, eb_info, d_encoded, d_decoded, d_decsize)``
    (sleek_lossless_gpu.h:63-72, 91-100; sleek_lossy_gpu.h:90-99, 118-127).

    The stream's length bounds every read when ``encoded_bytes`` is given (the
    reference trusts the stream); the output tensor's size always bounds the
    writes."""
    eb_info = None
    if args and isinstance(args[0], ErrorBoundInfo):
        eb_info, args = args[0], args[1:]
    d_encoded, d_decoded, d_decsize = args
    _check_device(d_encoded, d_decoded, d_decsize)
    dt = _np_dtype(d_decoded)
    if d_decsize.dtype != torch.int64:
        raise TypeError("d_decsize must be an int64 tensor")
    if encoded_bytes is None or encoded_bytes < 0:
        encoded_bytes = -1
    cap = d_decoded.numel() * d_decoded.element_size()
    L = _capi.lib()
    wp, wb = _ws(workspace)
    st = _stream_handle(stream)
    t = "f32" if dt == np.float32 else "f64"
    if eb_info is None:
        rc = getattr(L, f"sleek_decompress_{t}")(d_encoded.data_ptr(), int(encoded_bytes), d_decoded.data_ptr(),
                                                 cap, d_decsize.data_ptr(), wp, wb, st)
    else:
        if eb_info.dtype != dt:
            raise TypeError("eb_info dtype does not match the output dtype")
        rc = getattr(L, f"sleek_decompress_lossy_{t}")(eb_info.c_struct(), d_encoded.data_ptr(), int(encoded_bytes),
                                                       d_decoded.data_ptr(), cap, d_decsize.data_ptr(), wp, wb, st)
    _capi.check(rc, "sleek_decompress_gpu")
    if check:
        _raise_if_negative(d_decsize, "sleek_decompress_gpu")


# ---- convenience layer ----------------------------------------------------------

def stream_size(encoded: torch.Tensor) -> int:
    """Original byte count recorded in a stream's 8-byte header."""
    return int(encoded[:8].cpu().numpy().view(np.int64)[0])


def compress(x: torch.Tensor, eb: Optional[float] = None, stream=None) -> torch.Tensor:
    """Compresses a float32/float64 CUDA tensor; returns the stream as a uint8
    CUDA tensor of its exact size (synchronises to read the size)."""
    x = x.contiguous().view(-1)
    dt = _np_dtype(x)
    enc = torch.empty(sleek_upper_bound_size(x.numel() * dt.itemsize), dtype=torch.uint8, device=x.device)
    size = torch.empty(1, dtype=torch.int64, device=x.device)
    if eb is None:
        sleek_compress_gpu(0, x, x.numel(), enc, size, stream=stream)
    else:
        sleek_compress_gpu(0, sleek_error_bound(eb, dt), x, x.numel(), enc, size, stream=stream)
    n = _raise_if_negative(size, "compress")
    return enc[:n]


def decompress(encoded: torch.Tensor, dtype, eb: Optional[float] = None, stream=None,
               out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Decompresses a stream produced by ``compress`` (or by the reference)."""
    dt = np.dtype(dtype)
    tdt = torch.float32 if dt == np.float32 else torch.float64
    n = stream_size(encoded)
    if n < 0 or n % dt.itemsize:
        raise SleekError(_capi.SLEEK_ERR_CORRUPT_STREAM, "decompress")
    if out is None:
        out = torch.empty(max(n // dt.itemsize, 1), dtype=tdt, device=encoded.device)
    size = torch.empty(1, dtype=torch.int64, device=encoded.device)
    if eb is None:
        sleek_decompress_gpu(0, encoded, out, size, stream=stream, encoded_bytes=encoded.numel())
    else:
        sleek_decompress_gpu(0, sleek_error_bound(eb, dt), encoded, out, size, stream=stream,
                             encoded_bytes=encoded.numel())
    m = _raise_if_negative(size, "decompress")
    return out[: m // dt.itemsize]


def value_range(x: torch.Tensor, stream=None) -> tuple:
    """(min, max) of a float32/float64 CUDA tensor on the device, NaNs ignored
    (NaN, NaN when it holds no other value)."""
    x = x.contiguous().view(-1)
    _check_device(x)
    dt = _np_dtype(x)
    if dt == np.float32:
        lo, hi = C.c_float(), C.c_float()
        check(_capi.lib().sleek_minmax_f32(x.data_ptr(), x.numel(), C.byref(lo), C.byref(hi), _stream_handle(stream)),
              "sleek_minmax_f32")
    else:
        lo, hi = C.c_double(), C.c_double()
        check(_capi.lib().sleek_minmax_f64(x.data_ptr(), x.numel(), C.byref(lo), C.byref(hi), _stream_handle(stream)),
              "sleek_minmax_f64")
    return lo.value, hi.value


def range_relative_error_bound(x: torch.Tensor, parameter: float) -> float:
    """The absolute error bound of the reference's range-relative drivers,
    (max - min) * parameter, computed in the array's own precision."""
    lo, hi = value_range(x)
    if x.dtype == torch.float32:
        return float(np.float32(np.float32(hi) - np.float32(lo)) * np.float32(parameter))
    return float((hi - lo) * parameter)


def validate_stream(stream, dtype) -> dict:
    """Checks a stream held in host memory (bytes, bytearray, numpy or CPU
    tensor) against every rule the device decoders enforce, without a device
    call.  Returns ``{"valid", "reason", "reason_text", "bad_chunk", "insize",
    "chunks", "stream_bytes", "raw_chunks"}``."""
    if isinstance(stream, torch.Tensor):
        if stream.is_cuda:
            raise TypeError("validate_stream reads host memory")
        stream = stream.contiguous().numpy()
    buf = np.frombuffer(bytes(stream), dtype=np.uint8) if not isinstance(stream, np.ndarray) else \
        np.ascontiguousarray(stream).view(np.uint8).reshape(-1)
    info = _capi.StreamInfo()
    L = _capi.lib()
    rc = L.sleek_validate_stream(buf.ctypes.data if buf.size else None, buf.size, np.dtype(dtype).itemsize,
                                 C.byref(info))
    if rc not in (0, _capi.SLEEK_ERR_CORRUPT_STREAM):
        check(rc, "sleek_validate_stream")
    return {"valid": rc == 0, "reason": info.reason,
            "reason_text": L.sleek_stream_reason_string(info.reason).decode(),
            "bad_chunk": info.bad_chunk, "insize": info.insize, "chunks": info.chunks,
            "stream_bytes": info.stream_bytes, "raw_chunks": info.raw_chunks}


def compress_to_host(x: torch.Tensor, eb: Optional[float] = None, out: Optional[torch.Tensor] = None,
                     segment_bytes: int = 0, stream=None) -> torch.Tensor:
    """Compresses a float32/float64 CUDA tensor and returns its stream in pinned
    host memory (a uint8 CPU tensor of the exact size): only the stream's bytes
    cross PCIe, segment by segment, overlapped with the encoding of the next."""
    x = x.contiguous().view(-1)
    _check_device(x)
    dt = _np_dtype(x)
    cap = sleek_upper_bound_size(x.numel() * dt.itemsize)
    if out is None:
        out = torch.empty(max(cap, 16), dtype=torch.uint8, pin_memory=True)
    if out.is_cuda or out.dtype != torch.uint8:
        raise TypeError("out must be a uint8 CPU tensor")
    n = C.c_longlong()
    check(_capi.lib().sleek_compress_to_host(x.data_ptr(), x.numel(), dt.itemsize, int(eb is not None),
                                             float(eb) if eb is not None else 0.0, out.data_ptr(), out.numel(),
                                             C.byref(n), int(segment_bytes), _stream_handle(stream)),
          "sleek_compress_to_host")
    return out[: n.value]


def decompress_from_host(encoded: torch.Tensor, dtype, eb: Optional[float] = None, out: Optional[torch.Tensor] = None,
                         segment_bytes: int = 0, stream=None) -> torch.Tensor:
    """Decompresses a stream held in host memory (a uint8 CPU tensor, ideally
    pinned) into a CUDA tensor; the stream is validated on the host first and
    only its bytes cross PCIe."""
    if encoded.is_cuda or encoded.dtype != torch.uint8:
        raise TypeError("encoded must be a uint8 CPU tensor")
    encoded = encoded.contiguous()
    dt = np.dtype(dtype)
    tdt = torch.float32 if dt == np.float32 else torch.float64
    n = int(encoded[:8].numpy().view(np.int64)[0]) if encoded.numel() >= 8 else -1
    if out is None:
        out = torch.empty(max(n // dt.itemsize, 1), dtype=tdt, device="cuda")
    got = C.c_longlong()
    check(_capi.lib().sleek_decompress_from_host(encoded.data_ptr(), encoded.numel(), dt.itemsize, int(eb is not None),
                                                 float(eb) if eb is not None else 0.0, out.data_ptr(),
                                                 out.numel() * out.element_size(), C.byref(got), int(segment_bytes),
                                                 _stream_handle(stream)),
          "sleek_decompress_from_host")
    return out[: got.value // dt.itemsize]
