"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``oracle/lbm_oracle.cpp`` into ``oracle/_build/liblbm_oracle.so``.
``-ffp-contract=off`` keeps every multiply and add separately rounded, as in
the reference's gfortran CPU build (no FMA contraction), so the FP32
instantiation rounds like the reference's single-precision build.  The same
library is used for parity and, with OpenMP threads, as the timed CPU
baseline; OpenMP does not change results because no loop reduces across
cells.

A second library, ``liblbm_oracle_fma.so``, is the same source built with
``-ffp-contract=fast``: multiplies and adds contracted into FMAs wherever the
compiler can, as a GPU build does.  Parity tests compare the GPU against both
to show how far FP32 reordering alone moves the result.

The reference itself (Fortran 90 / CUDA Fortran) cannot be compiled in this
image: there is no gfortran, nvfortran or flang, so there is no ``oracle/_ref``.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "lbm_oracle.cpp")
HDR = os.path.join(HERE, "lbm_oracle.h")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liblbm_oracle.so")
LIB_FMA = os.path.join(OUT_DIR, "liblbm_oracle_fma.so")

CXXFLAGS = ["-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-std=c++17", "-Wall", "-Wno-unknown-pragmas"]


def needs_build(lib: str = LIB) -> bool:
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    return any(os.path.getmtime(s) > t for s in (SRC, HDR))


def build(force: bool = False, verbose: bool = False, contract: bool = False) -> str:
    """Build (when stale) and return the path of the library: separately rounded
    multiplies and adds, or with contract=True FMA-contracted."""
    lib = LIB_FMA if contract else LIB
    if force or needs_build(lib):
        os.makedirs(OUT_DIR, exist_ok=True)
        tmp = lib + ".tmp%d" % os.getpid()
        flag = "-ffp-contract=fast" if contract else "-ffp-contract=off"
        cmd = ["g++", *CXXFLAGS, flag, "-shared", "-o", tmp, SRC]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
    print(build(force="--force" in sys.argv, verbose=True, contract=True))
