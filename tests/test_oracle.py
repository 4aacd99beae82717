"""The oracle (C restatement in oracle/sleek_oracle.c) pinned against the
reference: the golden fixtures made by the reference's own CPU codec, and --
where oracle/_ref was built here -- the reference CPU codec itself on seeded
inputs."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.golden_io import cases, load, sha

CASES = cases()


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_matches_golden_stream(case):
    x, stream = load(case)
    assert sha(stream) == case["stream_sha256"]
    got = O.encode(x, case["eb"])
    assert got == stream


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_decodes_golden_stream(case):
    x, stream = load(case)
    dec = O.decode(stream, x.dtype, case["eb"])
    assert sha(dec.tobytes()) == case["decoded_sha256"]
    if case["eb"] is None:
        assert dec.tobytes() == x.tobytes()


def test_golden_covers_edge_cases():
    names = {c["name"] for c in CASES}
    for t in ("f32", "f64"):
        for suffix in ("smooth_lossless", "randbits_lossless", "zeros_lossless", "one_value", "exact_chunk",
                       "wide", "smooth_ebdenormal", "smooth_eb0", "smooth_ebneg1e-3"):
            assert f"{t}_{suffix}" in names


def _seeded(n, dt, seed):
    rng = np.random.default_rng(seed)
    x = (np.cumsum(rng.normal(0, 1, n)) * 0.01).astype(dt)
    k = max(1, n // 500)
    idx = rng.choice(n, k, replace=False)
    x[idx] = np.array([np.nan, np.inf, -np.inf, 0.0, -0.0], dt)[np.arange(k) % 5]
    return x


@pytest.mark.skipif(O.ref_cpu() is None, reason="reference CPU build (oracle/_ref) not present")
@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("n", [1, 2, 1023, 4096, 4097, 8192 + 3, 100_003])
@pytest.mark.parametrize("eb", [None, 1e-1, 1e-3, 1e-7, 1e-39, 0.0])
def test_oracle_equals_reference_cpu(dt, n, eb):
    x = _seeded(n, dt, n * 7 + (0 if eb is None else 1))
    a = O.encode(x, eb)
    b = O.ref_encode(x, eb)
    assert a == b
    assert O.decode(a, dt, eb).tobytes() == O.ref_decode(b, dt, eb).tobytes()


@pytest.mark.parametrize("width", [32, 64])
def test_lossless_transform_is_bijective(width):
    L = O.lib()
    rng = np.random.default_rng(5)
    if width == 32:
        vals = list(rng.integers(0, 2**32, 20000, dtype=np.uint64)) + [0, 1, 0x7F800000, 0xFF800000, 0x80000000,
                                                                       0x00FFFFFF, 0x01000000, 0xFFFFFFFF]
        for v in vals:
            v = int(v) & 0xFFFFFFFF
            assert L.oracle_inv32(L.oracle_fwd32(v)) == v
    else:
        vals = list(rng.integers(0, 2**63, 20000, dtype=np.uint64)) + [0, 1, 0x7FF0000000000000, 2**64 - 1, 2**63]
        for v in vals:
            v = int(v)
            assert L.oracle_inv64(L.oracle_fwd64(v)) == v


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("eb", [1e-1, 1e-3, 1e-6])
def test_lossy_roundtrip_within_bound(dt, eb):
    x = _seeded(50_000, dt, 99)
    y = O.decode(O.encode(x, eb), dt, eb)
    fin = np.isfinite(x)
    assert np.array_equal(x[~fin].view(np.uint32 if dt == np.float32 else np.uint64),
                          y[~fin].view(np.uint32 if dt == np.float32 else np.uint64)) or \
        np.all(np.isnan(x[~fin]) == np.isnan(y[~fin]))
    err = np.abs(x[fin].astype(np.float64) - y[fin].astype(np.float64))
    assert err.max() <= eb


def test_error_bound_matches_reference_rule():
    # eb_e = biased exponent of |eb|; thr_e = eb_e + m + 1; offs = (thr_e << m) - (1 << m)
    for eb in (1e-1, 1e-3, 3e-41, -2.5, 1e30):
        e, t, o = O.error_bound(eb, np.float32)
        bits = np.array([eb], np.float32).view(np.uint32)[0]
        assert e == (bits >> 23) & 0xFF and t == e + 24 and o == (t << 23) - (1 << 23)
    with pytest.raises(ValueError):
        O.error_bound(1e38, np.float32)
    with pytest.raises(ValueError):
        O.error_bound(1e300, np.float64)


def test_oracle_rejects_corrupt_stream():
    x, s = load(next(c for c in CASES if c["name"] == "f32_smooth_lossless"))
    b = bytearray(s)
    b[8] ^= 0x01  # first chunk size entry
    with pytest.raises(ValueError):
        O.decode(bytes(b), np.float32, None)
    with pytest.raises(ValueError):
        O.decode(s[: len(s) // 2], np.float32, None)
