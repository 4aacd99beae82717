"""Command-line drivers: this project's programs (sleek_b200/_bin) against the
reference's own GPU drivers built from its sources (oracle/_ref/cli), and the
reference's driver sources rebuilt against this project's drop-in headers
(oracle/_ref/dropin).  On the same input files every program must write the same
output file byte for byte and print the same stdout lines, apart from the banner
and the time / throughput lines; the lines the reference's measurement scripts
parse must parse the same way (compress_decompress_inputs_single.py:176-184,233-235)."""
import os
import subprocess

import numpy as np
import pytest

from sleek_b200 import build as B

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OURS = os.path.join(ROOT, "sleek_b200", "_bin")
REFCLI = os.path.join(ROOT, "oracle", "_ref", "cli")
DROPIN = os.path.join(ROOT, "oracle", "_ref", "dropin")
TIMING = ("encoding time", "encoding throughput", "decoding time", "decoding throughput")
PREC = {np.float32: "single", np.float64: "double"}


@pytest.fixture(scope="module")
def programs():
    B.build_cli()
    return OURS


def _run(prog, *args):
    r = subprocess.run([prog, *map(str, args)], capture_output=True, text=True, timeout=300)
    return r.returncode, r.stdout.splitlines(), r.stderr


def _body(lines, banner=2):
    """stdout without the banner and the timing lines"""
    return [ln for ln in lines[banner:] if not ln.startswith(TIMING)]


def _inputs(tmp_path, dtype, specials):
    rng = np.random.default_rng(20261203 + (8 if dtype == np.float64 else 4) + specials)
    n = 3 * 16384 // np.dtype(dtype).itemsize * 37 + 11  # a ragged last chunk
    i = np.arange(n)
    x = (1e3 * np.sin(2e-4 * i) + 40 * np.cos(3.1e-3 * i + 0.5) + rng.normal(0, 1e-3, n)).astype(dtype)
    if specials:
        k = rng.choice(n, n // 1000, replace=False)
        q = len(k) // 4
        x[k[:q]] = np.nan
        x[k[q:2 * q]] = np.inf
        x[k[2 * q:3 * q]] = -np.inf
        x[k[3 * q:]] = 3e-41 if dtype == np.float32 else 3e-310
    p = tmp_path / f"in_{np.dtype(dtype).name}_{specials}.bin"
    x.tofile(p)
    return p


def _have(d):
    return os.path.isdir(d) and len(os.listdir(d)) >= 8


def _compare(outs):
    ref = outs["ref"]
    for who, got in outs.items():
        assert got[0] == ref[0], who  # stream file
        assert got[1] == ref[1], who  # decoded file
        assert _body(got[2]) == _body(ref[2]), (who, got[2], ref[2])
        assert _body(got[3]) == _body(ref[3]), (who, got[3], ref[3])


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("mode", ["artifact", "standalone"])
def test_lossless_drivers_match_reference(programs, tmp_path, dtype, mode):
    if not _have(REFCLI):
        pytest.skip("reference drivers not built (oracle/Makefile cli)")
    sub = "" if mode == "artifact" else "standalone"
    p = PREC[dtype]
    src = _inputs(tmp_path, dtype, specials=1)
    outs = {}
    for who, base in (("ours", OURS), ("ref", REFCLI), ("dropin", DROPIN)):
        if who == "dropin" and not _have(DROPIN):
            continue
        c, d = tmp_path / f"{who}.sleek", tmp_path / f"{who}.out"
        rc1, o1, e1 = _run(os.path.join(base, sub, f"sleek_{p}_compressor_lossless"), src, c)
        rc2, o2, e2 = _run(os.path.join(base, sub, f"sleek_{p}_decompressor_lossless"), c, d)
        assert rc1 == 0 and rc2 == 0, (who, e1, e2)
        outs[who] = (c.read_bytes(), d.read_bytes(), o1, o2)
    assert outs["ref"][1] == src.read_bytes()
    _compare(outs)
    if mode == "artifact":  # the fields the measurement script reads
        o1, o2 = outs["ours"][2], outs["ours"][3]
        assert float(o1[-3].split()[-1][0:-1]) == float(outs["ref"][2][-3].split()[-1][0:-1])
        assert float(o1[-1].split()[-2]) > 0 and float(o2[-1].split()[-2]) > 0


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("mode,param", [("artifact", "1e-3"), ("artifact", "1e-6"), ("standalone", "0.01")])
def test_lossy_drivers_match_reference(programs, tmp_path, dtype, mode, param):
    if not _have(REFCLI):
        pytest.skip("reference drivers not built (oracle/Makefile cli)")
    sub = "" if mode == "artifact" else "standalone"
    p = PREC[dtype]
    # the reference's range-relative bound depends on its OpenMP schedule when the
    # data hold NaNs, and infinities make the range infinite: plain finite inputs
    src = _inputs(tmp_path, dtype, specials=0)
    outs = {}
    for who, base in (("ours", OURS), ("ref", REFCLI), ("dropin", DROPIN)):
        if who == "dropin" and not _have(DROPIN):
            continue
        c, d = tmp_path / f"{who}.sleek", tmp_path / f"{who}.out"
        rc1, o1, e1 = _run(os.path.join(base, sub, f"sleek_{p}_compressor_lossy"), src, c, param)
        dargs = (c, d, param, src) if mode == "artifact" else (c, d, param)
        rc2, o2, e2 = _run(os.path.join(base, sub, f"sleek_{p}_decompressor_lossy"), *dargs)
        assert rc1 == 0 and rc2 == 0, (who, e1, e2)
        outs[who] = (c.read_bytes(), d.read_bytes(), o1, o2)
    if mode == "artifact":
        assert any("verification passed" in ln for ln in outs["ref"][3])
    _compare(outs)


def test_memcpy_program_line_the_scripts_read(programs, tmp_path):
    src = _inputs(tmp_path, np.float32, specials=0)
    rc, out, err = _run(os.path.join(OURS, "GPUmemcpy"), src)
    assert rc == 0, err
    assert out[7].startswith("DtD throughput:")
    assert float(out[7].split()[-2]) > 0


def test_corrupt_stream_is_an_error_not_a_crash(programs, tmp_path):
    src = _inputs(tmp_path, np.float32, specials=0)
    c, d = tmp_path / "c.sleek", tmp_path / "d.out"
    assert _run(os.path.join(OURS, "sleek_single_compressor_lossless"), src, c)[0] == 0
    b = bytearray(c.read_bytes())
    b[8], b[9] = 0xFF, 0x7F  # first chunk size beyond 16384
    c.write_bytes(bytes(b))
    rc, out, err = _run(os.path.join(OURS, "sleek_single_decompressor_lossless"), c, d)
    assert rc == 255 and "corrupt compressed stream" in err, (rc, err)
