"""Builds libnxd_b200.so in-tree with nvcc for sm_100a.

The shared library is the product: the CUDA kernels plus the C ABI of
include/nxd.h.  --fmad=false keeps every FP64 multiply and add separately
rounded (the CPU oracle is compiled with -ffp-contract=off to match).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libnxd_b200.so")
SRCS = [os.path.join(HERE, "csrc", f) for f in ("nxd.cu", "noalloc.cu", "peak.cu")]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--fmad=false",
    "-Xcompiler", "-fPIC", "-shared",
]


def build(verbose: bool = False, extra=()) -> str:
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *NVCC_FLAGS, *extra, "-o", LIB, *SRCS]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
