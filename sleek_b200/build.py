"""Builds the sm_100a shared library ``sleek_b200/_lib/libsleek_b200.so``.

``python -m sleek_b200.build`` (or ``__graft_entry__.build()``) compiles every
CUDA source in ``sleek_b200/csrc`` with nvcc for ``sm_100a`` and links one
C-ABI shared library (entry points declared in ``include/sleek_capi.h``).
nvcc cross-compiles, so this works on a machine without a GPU.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIB_DIR, "libsleek_b200.so")

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
    "--expt-relaxed-constexpr",
]


def _sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps() -> list[str]:
    return _sources() + sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))) + [
        os.path.join(ROOT, "include", "sleek_capi.h"), __file__]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in _deps())


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compiles the library if any source is newer than it; returns its path."""
    if not force and not ptxas_info and up_to_date():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    objs = []
    for src in _sources():
        obj = os.path.join(LIB_DIR, os.path.basename(src)[:-3] + ".o")
        cmd = ["nvcc", *NVCC_FLAGS, "-c", src, "-o", obj]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        objs.append(obj)
    cmd = ["nvcc", "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB, *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    for o in objs:
        os.remove(o)
    return LIB


CLI_DIR = os.path.join(PKG, "cli")
BIN_DIR = os.path.join(PKG, "_bin")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")

# (program name, SLEEK_DOUBLE, SLEEK_LOSSY, SLEEK_DECOMPRESS): the names the
# reference's build scripts give its GPU drivers (compile_compressors_*.sh)
DRIVERS = [
    (f"sleek_{p}_{'decompressor' if x else 'compressor'}_{'lossy' if l else 'lossless'}", d, l, x)
    for d, p in ((0, "single"), (1, "double")) for l in (0, 1) for x in (0, 1)
]


def cli_programs() -> list[str]:
    """Paths of every command-line program: the range-relative, timed drivers in
    ``_bin`` (as the reference's scripts run them), the plain drivers in
    ``_bin/standalone``, ``_bin/GPUmemcpy`` and ``_bin/sleek_validate``."""
    out = [os.path.join(BIN_DIR, n) for n, *_ in DRIVERS]
    out += [os.path.join(BIN_DIR, "standalone", n) for n, *_ in DRIVERS]
    return out + [os.path.join(BIN_DIR, "GPUmemcpy"), os.path.join(BIN_DIR, "sleek_validate")]


def build_cli(force: bool = False, verbose: bool = False) -> list[str]:
    """Compiles the command-line programs (host C++ over the C ABI) against the
    library; a program is rebuilt when its source, the header or the library is newer."""
    lib = build()
    hdr = os.path.join(ROOT, "include", "sleek_capi.h")
    common = ["g++", "-O2", "-std=c++17", "-Wall", f"-I{CUDA_HOME}/include", f"-I{os.path.join(ROOT, 'include')}"]
    jobs = []
    for name, d, l, x in DRIVERS:
        for sub, extra in (("", ["-DARTIFACT"]), ("standalone", [])):
            out = os.path.join(BIN_DIR, sub, name)
            jobs.append((out, os.path.join(CLI_DIR, "sleek_driver.cpp"),
                         [f"-DSLEEK_DOUBLE={d}", f"-DSLEEK_LOSSY={l}", f"-DSLEEK_DECOMPRESS={x}", *extra]))
    jobs.append((os.path.join(BIN_DIR, "GPUmemcpy"), os.path.join(CLI_DIR, "gpu_memcpy.cpp"), []))
    jobs.append((os.path.join(BIN_DIR, "sleek_validate"), os.path.join(CLI_DIR, "sleek_validate.cpp"), []))
    for out, src, defs in jobs:
        deps = [src, hdr, lib, __file__]
        if not force and os.path.exists(out) and all(os.path.getmtime(p) <= os.path.getmtime(out) for p in deps):
            continue
        os.makedirs(os.path.dirname(out), exist_ok=True)
        rel = os.path.relpath(LIB_DIR, os.path.dirname(out))
        cmd = [*common, *defs, src, "-o", out, f"-L{LIB_DIR}", "-lsleek_b200", f"-L{CUDA_HOME}/lib64", "-lcudart",
               f"-Wl,-rpath,$ORIGIN/{rel}:{CUDA_HOME}/lib64"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return [j[0] for j in jobs]


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv))
    print(len(build_cli(force="--force" in sys.argv)), "command-line programs in", BIN_DIR)
