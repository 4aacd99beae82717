"""The kernels' value maps, checked on the device against the reference's own
integer steps (include/sleek_common_gpu.h: forward transform :356-374, inverse
:614-632, quantize :776-802, dequantize :1077-1108).

The codec computes the transform's exponent step as one conditional add, the
64-bit maps on 32-bit halves, and the quantizer's and dequantizer's rounding
division in floating point.  sleek_selftest_value_maps runs those device forms
beside a literal restatement of the reference's integer arithmetic: for float32
over every 32-bit word (and every code) at eight error-bound exponents from the
smallest to the largest legal one, for float64 over every sign/exponent field
with 2^20 seeded mantissas each, every code below 2^32 and codes of every bit
length at nine exponents.  Every count must be zero."""
import ctypes as C

import pytest

from sleek_b200 import _capi

pytestmark = pytest.mark.gpu

CHECKS = ["f32 transform + inverse", "f32 quantize", "f32 dequantize",
          "f64 transform + inverse", "f64 quantize", "f64 dequantize"]


def test_value_maps_equal_the_reference_integer_steps(cuda):
    n = _capi.SLEEK_SELFTEST_VALUE_CHECKS
    assert n == len(CHECKS)
    counts = (C.c_longlong * n)()
    first = (C.c_longlong * n)()
    _capi.check(_capi.lib().sleek_selftest_value_maps(counts, first))
    bad = {CHECKS[k]: (counts[k], first[k]) for k in range(n) if counts[k]}
    assert not bad, bad
    assert all(first[k] == -1 for k in range(n))


def test_value_map_selftest_rejects_null(cuda):
    assert _capi.lib().sleek_selftest_value_maps(None, None) == _capi.SLEEK_ERR_INVALID_ARG
