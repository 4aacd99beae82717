"""The device kernels compute three steps of the reference's value maps in a
rewritten form (sleek_b200/csrc/sleek_device.cuh).  Each rewrite is checked
here against the reference's own formulation (include/sleek_common_gpu.h:
lossless forward :356-374, quantize :776-802), restated in numpy / exact
rational arithmetic:

1. the forward transform's exponent step as one conditional add;
2. the quantizer's sign step `e2 = (enc << 1) | !sign; e2 ? e2 - 1 : 0` as
   `(enc << 1) - (enc ? sign : 0)`;
3. the quantizer's "below eb_e gives 0" case left to the rounding of
   `trunc(round_down(|v| 2^(bias + m - thr_e) + 1/2))`.

The device code itself is covered by the GPU parity tests; these pin the
algebra on the CPU.  (The first identity also holds exhaustively over all 2^32
words, which takes a couple of minutes; the sample here covers every exponent
field value and both ends of each.)"""
from fractions import Fraction

import numpy as np


def _words32(rng):
    """Every 8-bit and 11-bit exponent-field boundary plus random words."""
    edges = []
    for top in range(1 << 11):
        base = top << 21
        edges += [base, base + 1, base + (1 << 21) - 1, base + (1 << 20)]
    for top in range(1 << 8):
        base = top << 24
        edges += [base, base + 1, base + (1 << 24) - 1]
    rnd = rng.integers(0, 1 << 32, size=1 << 20, dtype=np.uint64)
    return np.concatenate([np.array(edges, dtype=np.uint64), rnd]).astype(np.uint32)


def _ref_step(v, top_mask, unit):
    """The reference's exponent step on the rotated word (field under `top_mask`)."""
    m = (v & top_mask) != 0
    v2 = np.where(m, v - np.uint32(0x80000000), v).astype(np.uint32)
    c = m & (((v2 & top_mask) == 0) | (v2 >= 0x80000000))
    return np.where(c, v2 - np.uint32(unit), v2).astype(np.uint32)


def _new_step(v, unit):
    """The rewritten step: add 0, 2^31 - unit or 2^31 (mod 2^32)."""
    lo, mid = np.uint32(unit), np.uint32(0x80000000 + unit)
    add = np.where(v < lo, 0, np.where(v < mid, 0x80000000 - unit, 0x80000000)).astype(np.uint32)
    return (v + add).astype(np.uint32)


def test_forward_exponent_step_f32():
    v = _words32(np.random.default_rng(20261203))
    assert np.array_equal(_ref_step(v, np.uint32(0xff000000), 0x01000000), _new_step(v, 0x01000000))


def test_forward_exponent_step_f64_high_word():
    # the 64-bit transform's step touches only the high word of the rotated value
    v = _words32(np.random.default_rng(20261204))
    assert np.array_equal(_ref_step(v, np.uint32(0xffe00000), 0x00200000), _new_step(v, 0x00200000))


def test_quantizer_sign_step():
    rng = np.random.default_rng(20261205)
    for bits, dt in ((32, np.uint32), (64, np.uint64)):
        enc = np.concatenate([np.array([0, 1, 2, (1 << (bits - 1)) - 1], dtype=dt),
                              rng.integers(0, 1 << (bits - 2), size=1 << 16, dtype=np.uint64).astype(dt)])
        for sign in (0, 1):
            s = dt(sign)
            e2 = (enc << dt(1)) | dt(1 - sign)
            ref = np.where(e2 != 0, e2 - dt(1), dt(0)).astype(dt)
            new = ((enc << dt(1)) - np.where(enc != 0, s, dt(0))).astype(dt)
            assert np.array_equal(ref, new), (bits, sign)


def test_quantizer_below_eb_e_rounds_to_zero():
    """For 1 <= eb_e, thr_e = eb_e + m + 1 and any value with biased exponent
    ve < eb_e (denormals included), y = |v| 2^(bias + m - thr_e) satisfies
    y + 1/2 < 1 exactly, so its round-down truncates to 0."""
    rng = np.random.default_rng(20261206)
    for m, bias, emax in ((23, 127, 255), (52, 1023, 2047)):
        for eb_e in sorted(set([1, 2, 3, m, emax - m - 3] + [int(e) for e in rng.integers(1, emax - m - 2, 20)])):
            thr_e = eb_e + m + 1
            for ve in sorted(set([0, eb_e - 1, max(0, eb_e - 2)])):
                for mant in (0, 1, (1 << m) - 1, int(rng.integers(0, 1 << m))):
                    frac = Fraction(mant, 1 << m)
                    x = frac * Fraction(2) ** (1 - bias) if ve == 0 else (1 + frac) * Fraction(2) ** (ve - bias)
                    y = x * Fraction(2) ** (bias + m - thr_e)
                    assert y + Fraction(1, 2) < 1, (m, eb_e, ve, mant)
