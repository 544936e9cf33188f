"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``oracle/lbm_oracle.cpp`` into ``oracle/_build/liblbm_oracle.so``.
``-ffp-contract=off`` keeps every multiply and add separately rounded, as in
the reference's gfortran CPU build (no FMA contraction), so the FP32
instantiation rounds like the reference's single-precision build.  The same
library is used for parity and, with OpenMP threads, as the timed CPU
baseline; OpenMP does not change results because no loop reduces across
cells.

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

CXXFLAGS = ["-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-fPIC",
            "-std=c++17", "-Wall", "-Wno-unknown-pragmas"]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(s) > t for s in (SRC, HDR))


def build(force: bool = False, verbose: bool = False) -> str:
    if force or needs_build():
        os.makedirs(OUT_DIR, exist_ok=True)
        tmp = LIB + ".tmp%d" % os.getpid()
        cmd = ["g++", *CXXFLAGS, "-shared", "-o", tmp, SRC]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
