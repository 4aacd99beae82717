"""B200-native (sm_100a) SLEEK compress / decompress.

A drop-in for SLEEK's GPU compress / decompress path: same API names, same
compressed byte stream (bit-identical to the reference CPU and GPU code), with
hand-written sm_100a kernels behind a C ABI (``include/sleek_capi.h``).
"""
from .api import (  # noqa: F401
    CS,
    ErrorBoundInfo,
    SleekError,
    compress,
    decompress,
    sleek_compress_gpu,
    sleek_decompress_gpu,
    sleek_error_bound,
    sleek_system_checks,
    sleek_thread_blocks,
    sleek_upper_bound_size,
    stream_size,
)
