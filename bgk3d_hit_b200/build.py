"""Builds the CUDA library ``libbgk3d.so`` in-tree for sm_100a, and the
program driver ``bgk3d_hit`` (the reference's main loop over the C-ABI).

    python -m bgk3d_hit_b200.build [--force] [--verbose]

The library is plain C-ABI (include/bgk3d.h); nothing here depends on torch.
Host code is compiled with -ffp-contract=off so that the host-side constants
(omega, output times) round exactly as written.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OUT = os.path.join(HERE, "libbgk3d.so")
SOURCES = ["kernels.cu", "rows.cu", "adjoint.cu", "bgk_abi.cu", "noalloc.cu"]
HEADERS = ["lattice.cuh", "kernels.h", "reduce.cuh"]
ARCH = "-gencode=arch=compute_100a,code=sm_100a"


def nvcc_path() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def command(out: str = OUT, extra=()) -> list[str]:
    return [
        nvcc_path(), "-O3", "-std=c++17", ARCH, "-lineinfo",
        "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared",
        f"-I{INCLUDE}", "-o", out,
        *[os.path.join(CSRC, s) for s in SOURCES],
        "-lcufft", *extra,
    ]


DRIVER = os.path.join(HERE, "bgk3d_hit")


def driver_command(out: str = DRIVER) -> list[str]:
    """g++ for the program driver (csrc/driver.cpp) over the C-ABI."""
    cxx = shutil.which("g++") or "g++"
    return [cxx, "-O2", "-std=c++17", f"-I{INCLUDE}", os.path.join(CSRC, "driver.cpp"), "-o", out,
            f"-L{HERE}", "-lbgk3d", "-Wl,-rpath,$ORIGIN"]


def build_driver(force: bool = False) -> str:
    src = os.path.join(CSRC, "driver.cpp")
    if force or not os.path.exists(DRIVER) or max(os.path.getmtime(src), os.path.getmtime(OUT)) > os.path.getmtime(
            DRIVER):
        r = subprocess.run(driver_command(), capture_output=True, text=True)
        if r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("g++ failed on driver.cpp")
    return DRIVER


def _stale(out: str) -> bool:
    if not os.path.exists(out):
        return True
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(INCLUDE, "bgk3d.h"), __file__]
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if force or _stale(OUT):
        cmd = command(extra=["-Xptxas", "-v"] if verbose else [])
        tmp = OUT + ".tmp"
        cmd[cmd.index(OUT)] = tmp
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode:
            raise RuntimeError("nvcc failed")
        os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
    print(build_driver(a.force))
