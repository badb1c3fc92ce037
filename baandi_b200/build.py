"""Build libbaandi_b200.so in-tree for sm_100a (B200) with nvcc.

`python -m baandi_b200.build` compiles every CUDA/C++ source under csrc/ into one
shared library next to this file.  The host compiler keeps every multiply and add
separately rounded (-ffp-contract=off) because the basis sort depends on exact |G|^2.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libbaandi_b200.so")
SOURCES = ["api.cu", "hpsi_kernels.cu", "davidson.cu", "noalloc.cu", "fields.cu", "kset_davidson.cu", "mixer.cu",
           "learned.cu", "gemm_tc.cu", "setup.cpp"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O3,-fopenmp",
    "-Xptxas", "-v",
]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for root, _, files in os.walk(CSRC):
        for f in files:
            if os.path.getmtime(os.path.join(root, f)) > t:
                return True
    inc = os.path.join(HERE, "..", "include", "baandi_gpu.h")
    return os.path.exists(inc) and os.path.getmtime(inc) > t


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *NVCC_FLAGS, "-shared", "-o", tmp] + [os.path.join(CSRC, s) for s in SOURCES] + ["-lcudart", "-lgomp"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libbaandi_b200.so")
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
