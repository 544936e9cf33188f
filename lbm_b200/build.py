"""Build the CUDA library ``lbm_b200/liblbmb200.so`` for sm_100a with nvcc.

The library is built in-tree so that it travels with the source tree; it has
no Python or torch dependency (a plain C ABI, ``include/lbm_b200.h``).
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liblbmb200.so")
HEADER = os.path.join(ROOT, "include", "lbm_b200.h")

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
    "-shared", "-cudart", "static", "-lcufft",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build lbm_b200")


def sources():
    return [os.path.join(CSRC, "api.cu")]


def deps():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cuh")) + [HEADER])


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in deps())


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    if force or needs_build():
        tmp = LIB + ".tmp%d" % os.getpid()
        cmd = [nvcc(), *NVCC_FLAGS, *extra, "-o", tmp, *sources()]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(force="--force" in sys.argv, verbose=True, extra=extra))
