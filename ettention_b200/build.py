"""Builds the CUDA library in-tree: ettention_b200/libettention_b200.so (sm_100a).

    python -m ettention_b200.build          # or ettention_b200.build.build()

The library is built ahead of time with nvcc for sm_100a only (no JIT, no
other architectures) and loaded with ctypes by ettention_b200._abi.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libettention_b200.so")
SOURCES = ["etcu_api.cu", "etcu_learned.cu", "etcu_io.cpp", "etcu_tiff.cpp", "etcu_stack.cpp"]
HEADERS = ["geometry.hpp", "kernels.cuh", "io_util.hpp", "blobs.cuh", "learned.cuh", "tune.hpp"]

# -fmad=false: no multiply-add is formed implicitly.  The kernels follow the
# reference's operation order step by step and write every intended fused
# multiply-add explicitly (fmaf, __ffma2_rn); the paired FP32 operations
# (__fmul2_rn, __fadd2_rn) are otherwise contracted by the compiler.
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo", "-fmad=false",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-shared", "--expt-relaxed-constexpr", "-cudart", "static", "-lz",
]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "ettention_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    cmd = [_nvcc(), *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-I", CSRC,
           *[os.path.join(CSRC, s) for s in SOURCES], "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
