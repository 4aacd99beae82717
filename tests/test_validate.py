"""Stream validation (sleek_validate_stream, host only): every golden fixture and
oracle stream is valid and fully accounted for; each planted defect is reported
with its reason and chunk; and on random corruptions a stream the validator
accepts always decodes with the oracle (the validator's rules are the device
decoders' rules, which are at least as strict as the reference's)."""
import os
import subprocess

import numpy as np
import pytest

import golden_io
from oracle import oracle as O
from sleek_b200 import api, build as B
from sleek_b200 import _capi



def _stream(dtype, n, eb=None, seed=0):
    rng = np.random.default_rng(seed)
    x = (np.cumsum(rng.normal(0, 1, n)) * 0.3).astype(dtype)
    if n > 100:
        x[rng.integers(0, n, n // 100)] = np.nan
    return x, bytearray(O.encode(x, eb))


@pytest.mark.parametrize("case", golden_io.cases(), ids=lambda c: c["name"])
def test_golden_fixtures_are_valid(case):
    x, s = golden_io.load(case)
    v = api.validate_stream(s, x.dtype)
    assert v["valid"], v
    assert v["stream_bytes"] == len(s) and v["insize"] == x.nbytes
    assert v["chunks"] == (x.nbytes + 16383) // 16384


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("eb", [None, 1e-2, 1e-6])
def test_oracle_streams_are_valid(dtype, eb):
    for n in (0, 1, 4095, 4096, 4097, 40000):
        x, s = _stream(dtype, n, eb, n)
        v = api.validate_stream(s, dtype)
        assert v["valid"] and v["stream_bytes"] == len(s), (n, v)


def _first_compressed(s, dtype):
    """(chunk, payload offset, csize) of the first compressed chunk"""
    insize = int(np.frombuffer(bytes(s[:8]), np.int64)[0])
    chunks = (insize + 16383) // 16384
    cs = np.frombuffer(bytes(s[8:8 + 2 * chunks]), np.uint16)
    off = 8 + 2 * chunks
    for c in range(chunks):
        os_ = min(16384, insize - c * 16384)
        if cs[c] < os_:
            return c, off, int(cs[c])
        off += int(cs[c])
    raise AssertionError("no compressed chunk")


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_planted_defects(dtype):
    x, s = _stream(dtype, 5 * 16384 // np.dtype(dtype).itemsize + 7, 1e-3, 3)
    tb = 8 * np.dtype(dtype).itemsize
    c, off, cs = _first_compressed(s, dtype)

    def check(buf, reason, chunk=-1):
        v = api.validate_stream(buf, dtype)
        assert not v["valid"] and v["reason"] == reason and v["bad_chunk"] == chunk, v

    check(s[:7], 1)
    b = bytearray(s); b[:8] = np.int64(-4).tobytes(); check(b, 2)
    b = bytearray(s); b[:8] = np.int64(len(x) * x.itemsize + 2).tobytes(); check(b, 2)
    b = bytearray(s); b[:8] = np.int64(1 << 40).tobytes(); check(b, 3)
    b = bytearray(s); b[8 + 2 * c:10 + 2 * c] = np.uint16(0).tobytes(); check(b, 4, c)
    b = bytearray(s); b[8 + 2 * c:10 + 2 * c] = np.uint16(16385).tobytes(); check(b, 4, c)
    b = bytearray(s); b[8 + 2 * c:10 + 2 * c] = np.uint16(20).tobytes(); check(b, 4, c)
    check(s[:off + cs - 1], 5, c)
    b = bytearray(s); b[off] = tb + 1; check(b, 6, c)
    b = bytearray(s); b[off] = (b[off] + 1) % (tb + 1); check(b, 7, c)
    b = bytearray(s); b[off + cs - 2] ^= 1; check(b, 8, c)
    # trailing bytes after the last payload are allowed, as the decoders allow them
    assert api.validate_stream(bytes(s) + b"\0" * 5, dtype)["valid"]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("eb", [None, 1e-3])
def test_random_corruptions_valid_implies_decodable(dtype, eb):
    x, s = _stream(dtype, 3 * 16384 // np.dtype(dtype).itemsize + 5, eb, 11)
    rng = np.random.default_rng(5)
    n_valid = n_bad = 0
    for t in range(400):
        b = bytearray(s)
        if t % 5 == 4:
            b = b[: int(rng.integers(0, len(b)))]
        else:
            region = int(rng.integers(0, 3))
            hi = {0: 8, 1: 8 + 2 * 4, 2: len(b)}[region]
            for _ in range(int(rng.integers(1, 4))):
                b[int(rng.integers(0, hi))] = int(rng.integers(0, 256))
        v = api.validate_stream(b, dtype)
        if v["valid"] and 0 <= v["insize"] <= x.nbytes:
            y = O.decode(bytes(b), dtype, eb)  # must not raise
            assert y.nbytes == v["insize"]
            n_valid += 1
        elif not v["valid"]:
            n_bad += 1
    assert n_valid > 20 and n_bad > 20


def test_validate_program(tmp_path):
    progs = B.build_cli()
    prog = [p for p in progs if p.endswith("sleek_validate")][0]
    x, s = _stream(np.float32, 50000, 1e-3, 7)
    f = tmp_path / "s.sleek"
    f.write_bytes(bytes(s))
    r = subprocess.run([prog, str(f), "single"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.splitlines()[-1] == "valid", r.stdout
    s[8], s[9] = 0, 0
    f.write_bytes(bytes(s))
    r = subprocess.run([prog, str(f), "single"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 255 and "INVALID: chunk size out of range at chunk 0" in r.stdout, r.stdout
