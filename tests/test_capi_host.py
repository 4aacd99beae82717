"""C-ABI checks that need no GPU: the library loads, exports every symbol the
headers in include/ declare, and its host-side logic (sizes, error bounds,
argument validation) matches the reference's rules."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from oracle import oracle as O
from sleek_b200 import _capi
from sleek_b200.build import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        # only the C ABI header declares extern "C" functions; the drop-in C++
        # headers are inline forwarders and declare no symbols of their own
        if 'extern "C"' not in src:
            continue
        for m in re.finditer(r"\b(sleek_\w+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_builds_and_loads():
    assert os.path.exists(_capi.LIB_PATH)
    _capi.lib()


def test_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 17
    L = _capi.lib()
    for s in sorted(syms):
        assert hasattr(L, s), s
    assert syms == set(_capi.SIGNATURES), syms ^ set(_capi.SIGNATURES)


@pytest.mark.parametrize("n", [0, 1, 16383, 16384, 16385, 10**9, 3 * 2**30])
def test_upper_bound_size_matches_reference_formula(n):
    chunks = (n + 16383) // 16384
    assert _capi.lib().sleek_upper_bound_size(n) == 12 + 2 * chunks + 16384 * chunks
    assert _capi.lib().sleek_upper_bound_size(n) == O.upper_bound_size(n)


def test_system_checks_and_status_strings():
    L = _capi.lib()
    assert L.sleek_system_checks() == 0
    for s in range(10):
        assert L.sleek_status_string(s)
    assert L.sleek_status_string(0) == b"ok"


@pytest.mark.parametrize("eb", [1e-1, 1e-2, 1e-4, 1e-6, 3e-41, 0.0, -1e-3, 1e20, 1e38, float("inf"), float("nan")])
def test_error_bound_f32_matches_oracle(eb):
    info = _capi.EbInfoF32()
    rc = _capi.lib().sleek_error_bound_f32(eb, C.byref(info))
    try:
        e, t, o = O.error_bound(eb, np.float32)
    except ValueError:
        assert rc == _capi.SLEEK_ERR_ERROR_BOUND
        return
    assert rc == 0 and (info.eb_e, info.thr_e, info.offs_e) == (e, t, o)


@pytest.mark.parametrize("eb", [1e-1, 1e-6, 1e-12, 1e-310, 0.0, -2.0, 1e300, 1.7e308])
def test_error_bound_f64_matches_oracle(eb):
    info = _capi.EbInfoF64()
    rc = _capi.lib().sleek_error_bound_f64(eb, C.byref(info))
    try:
        e, t, o = O.error_bound(eb, np.float64)
    except ValueError:
        assert rc == _capi.SLEEK_ERR_ERROR_BOUND
        return
    assert rc == 0 and (info.eb_e, info.thr_e, info.offs_e) == (e, t, o)


def test_workspace_sizes():
    L = _capi.lib()
    assert L.sleek_compress_workspace_size(0) == 8 * 32
    assert L.sleek_compress_workspace_size(16384 * 10) == 8 * (32 + 10)
    assert L.sleek_decompress_workspace_size() >= 8 * 33


def test_host_argument_validation_before_any_device_call():
    L = _capi.lib()
    fake = 0x10000  # never dereferenced: every case below fails a host check first
    assert L.sleek_compress_f32(None, 10, fake, fake, None, 0, None) == _capi.SLEEK_ERR_INVALID_ARG
    assert L.sleek_compress_f32(fake, 10, None, fake, None, 0, None) == _capi.SLEEK_ERR_INVALID_ARG
    assert L.sleek_compress_f32(fake, -1, fake, fake, None, 0, None) == _capi.SLEEK_ERR_INVALID_ARG
    assert L.sleek_compress_f32(fake + 2, 10, fake, fake, None, 0, None) == _capi.SLEEK_ERR_ALIGNMENT
    assert L.sleek_compress_f64(fake + 4, 10, fake, fake, None, 0, None) == _capi.SLEEK_ERR_ALIGNMENT
    assert L.sleek_compress_f32(fake, 10, fake + 4, fake, None, 0, None) == _capi.SLEEK_ERR_ALIGNMENT
    assert L.sleek_decompress_f32(None, 100, fake, 100, fake, None, 0, None) == _capi.SLEEK_ERR_INVALID_ARG
    assert L.sleek_decompress_f32(fake + 4, 100, fake, 100, fake, None, 0, None) == _capi.SLEEK_ERR_ALIGNMENT
    assert L.sleek_decompress_f64(fake, 100, fake + 4, 100, fake, None, 0, None) == _capi.SLEEK_ERR_ALIGNMENT
    assert L.sleek_decompress_f32(fake, 4, fake, 100, fake, None, 0, None) == _capi.SLEEK_ERR_CORRUPT_STREAM
    bad = _capi.EbInfoF32(10, 99, 0)  # thr_e inconsistent with eb_e
    assert L.sleek_compress_lossy_f32(bad, fake, 10, fake, fake, None, 0, None) == _capi.SLEEK_ERR_ERROR_BOUND


def test_no_device_is_a_status_not_a_crash():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = _capi.lib()
    fake = 0x10000
    assert L.sleek_compress_f32(fake, 10, fake, fake, None, 0, None) == _capi.SLEEK_ERR_NO_DEVICE


@pytest.mark.parametrize("elem", [4, 8])
def test_batch_items_beyond_the_largest_input_are_rejected_on_the_host(elem):
    # 2^52 bytes is the largest input any entry point accepts; one element more
    # would overflow the plan's byte and chunk arithmetic
    L = _capi.lib()
    fake = 0x10000  # never dereferenced: the item fails a host check first
    it = _capi.BatchItem(fake, fake, fake, (1 << 52) // elem + 1, -1, elem, 0, 0.0)
    plan = C.c_void_p()
    for decompress in (0, 1):
        rc = L.sleek_batch_plan_create(C.byref(it), 1, decompress, C.byref(plan))
        assert rc == _capi.SLEEK_ERR_INVALID_ARG
        assert not plan.value
    it.num_elements = -1
    assert L.sleek_batch_plan_create(C.byref(it), 1, 0, C.byref(plan)) == _capi.SLEEK_ERR_INVALID_ARG


def test_launch_shapes_are_described_and_validated_on_the_host():
    L = _capi.lib()
    t, w, s, c = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    for dec in (0, 1):
        n = 0
        while L.sleek_launch_shape_info(dec, n, C.byref(t), C.byref(w), C.byref(s), C.byref(c)) == 0:
            assert t.value % 32 == 0 and 1 <= w.value <= t.value // 32 and s.value >= 2 and c.value >= 1
            n += 1
        assert n >= 2  # shape 0 (the default) and at least one alternative
        assert L.sleek_launch_shape_info(dec, -1, None, None, None, None) == _capi.SLEEK_ERR_INVALID_ARG
        assert L.sleek_set_launch_shape(dec, 4, 0, 20, n, 0) == _capi.SLEEK_ERR_INVALID_ARG
        assert L.sleek_set_launch_shape(dec, 2, 0, 20, 0, 0) == _capi.SLEEK_ERR_INVALID_ARG
        assert L.sleek_set_launch_shape(dec, 4, 0, 64, 0, 0) == _capi.SLEEK_ERR_INVALID_ARG
        assert L.sleek_set_launch_shape(dec, 4, 0, 20, 0, -1) == _capi.SLEEK_ERR_INVALID_ARG
