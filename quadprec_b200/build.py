"""Build recipe for libhyperprec_gpu.so (sm_100a) and the test shims.

The library is compiled in-tree with nvcc; no JIT cache is involved, so the
built .so travels with the source tree. -fmad=false keeps every a*b+c in the
kernels unfused unless the source asks for a fused multiply-add explicitly
(the extended-precision arithmetic depends on the exact rounding sequence).
Each .cu file is compiled to its own object in quadprec_b200/_build (in
parallel; a file is recompiled when it or any header is newer than its
object), then the objects are linked into the shared library.
"""
from __future__ import annotations

import glob
import os
import subprocess
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libhyperprec_gpu.so")
OBJ_DIR = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    *ARCH,
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "-fmad=false",
    "-ccbin", "/usr/bin/g++",
]


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def headers() -> list[str]:
    return glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + [os.path.join(REPO, "include", "hyperprec_gpu.h")]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _obj(src: str) -> str:
    return os.path.join(OBJ_DIR, os.path.basename(src)[:-3] + ".o")


def _compile(src: str, force: bool, verbose: bool) -> str:
    obj = _obj(src)
    if force or _stale(obj, [src, *headers()]):
        cmd = [NVCC, *NVCC_FLAGS, "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
    return obj


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(OBJ_DIR, exist_ok=True)
    srcs = sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose), srcs))
    if force or _stale(LIB, objs):
        subprocess.run([NVCC, *ARCH, "-shared", "-ccbin", "/usr/bin/g++", "-o", LIB, *objs],
                       check=True)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True)
