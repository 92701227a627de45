"""Build recipe of the engine's shared library (sm_100a, in-tree).

``python -m esdgsem_mpiocca_b200.build_ext`` compiles csrc/*.cu and
csrc/*.cpp with nvcc into esdgsem_mpiocca_b200/libesdg_b200.so.  The build
needs no GPU (nvcc cross-compiles for sm_100a).
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libesdg_b200.so")
SOURCES = ["esdg_engine.cu", "esdg_ensemble.cu", "esdg_setup.cpp"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    # no a*b+c contraction: every FP64 operation rounds as in the reference's
    # Serial/OpenMP build, so results match it bit for bit on the plain path
    "-fmad=false",
    "-Xcompiler", "-fPIC,-O2",
    "-ccbin", "g++",
]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for name in os.listdir(CSRC):
        if name.endswith((".cu", ".cuh", ".cpp", ".hpp")) and os.path.getmtime(os.path.join(CSRC, name)) > t:
            return True
    hdr = os.path.join(os.path.dirname(PKG), "include", "esdg_b200.h")
    return os.path.exists(hdr) and os.path.getmtime(hdr) > t


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile libesdg_b200.so if it is missing or older than its sources."""
    if not force and not _stale():
        return LIB
    srcs = [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    cmd = [_nvcc(), *NVCC_FLAGS, "-shared", "-o", LIB + ".tmp", *srcs, "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
