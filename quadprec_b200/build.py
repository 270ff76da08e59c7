"""Build recipe for libhyperprec_gpu.so (sm_100a) and the test shims.

The library is compiled in-tree with nvcc; no JIT cache is involved, so the
built .so travels with the source tree. -fmad=false keeps every a*b+c in the
kernels unfused unless the source asks for a fused multiply-add explicitly
(the extended-precision arithmetic depends on the exact rounding sequence).
"""
from __future__ import annotations

import glob
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libhyperprec_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "-fmad=false",
    "-ccbin", "/usr/bin/g++",
]


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    deps = sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + [
        os.path.join(REPO, "include", "hyperprec_gpu.h")]
    if force or _stale(LIB, deps):
        cmd = [NVCC, *NVCC_FLAGS, "-o", LIB, *sources()]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
