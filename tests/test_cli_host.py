"""Command-line programs without a GPU: every program the reference's build
scripts produce exists under the same name, and a wrong argument count prints
the reference's USAGE line and exits with status 255 before any device call."""
import os
import subprocess

import pytest

from sleek_b200 import build as B


@pytest.fixture(scope="module")
def programs():
    return B.build_cli()


def test_every_reference_program_name_exists(programs):
    names = {os.path.basename(p) for p in programs}
    for prec in ("single", "double"):
        for kind in ("compressor", "decompressor"):
            for mode in ("lossless", "lossy"):
                assert f"sleek_{prec}_{kind}_{mode}" in names
    assert "GPUmemcpy" in names
    assert sorted(programs) == sorted(B.cli_programs())
    for p in programs:
        assert os.access(p, os.X_OK), p


USAGE = {
    "compressor_lossless": "input_file_name compressed_file_name",
    "decompressor_lossless": "compressed_file_name decompressed_file_name",
    "compressor_lossy": "input_file_name compressed_file_name error_bound",
    "decompressor_lossy": "compressed_file_name decompressed_file_name error_bound",
}


@pytest.mark.parametrize("sub", ["", "standalone"])
@pytest.mark.parametrize("kind", sorted(USAGE))
@pytest.mark.parametrize("prec", ["single", "double"])
def test_usage_line(programs, sub, kind, prec):
    prog = os.path.join(B.BIN_DIR, sub, f"sleek_{prec}_{kind}")
    r = subprocess.run([prog], capture_output=True, text=True, timeout=60)
    assert r.returncode == 255
    lines = r.stdout.splitlines()
    assert lines[0].startswith("SLEEK-B200") and f"{prec}-precision" in lines[0]
    want = USAGE[kind]
    if kind == "decompressor_lossy" and sub == "":
        want += " original_file_name"  # the range-relative form also reads the original
    assert lines[3] == f"USAGE: {prog} {want}"
    assert lines[4] == ""
