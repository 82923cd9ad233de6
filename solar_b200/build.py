"""Build the in-tree CUDA library ``solar_b200/libsolar_gpu.so`` for sm_100a.

The library is plain nvcc output (no torch extension): the CUDA kernels, the host-side
FP64 setup and the C-ABI of ``include/solar_gpu.h``.  It is built in the source tree so
that it travels with the repository to the GPU host.

Usage: ``python -m solar_b200.build [--verbose]`` (``-Xptxas -v`` register report).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsolar_gpu.so")
SOURCES = [os.path.join(CSRC, "solar_gpu.cu"), os.path.join(CSRC, "noalloc.cu"), os.path.join(CSRC, "tables.cpp"),
           os.path.join(CSRC, "io.cpp")]
HEADERS = [os.path.join(CSRC, h) for h in ("kernels.cuh", "tma.cuh", "tables.h", "adjoint.cuh", "adjoint_host.cuh",
                                            "split_host.cuh", "io_host.cuh", "forcing.cuh", "curl.cuh")] + [os.path.join(ROOT, "include", "solar_gpu.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def host_compiler() -> list:
    # The system g++ is the one nvcc supports; an inherited $CXX wrapper may not be.
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in SOURCES + HEADERS)


def build(verbose: bool = False, force: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
           "-Xcompiler", "-fPIC", "-shared", *host_compiler(), "-o", LIB, *SOURCES]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.check_call(cmd, cwd=ROOT)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(LIB)
