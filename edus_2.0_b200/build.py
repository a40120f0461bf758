"""Build the CUDA library of the propagator in-tree.

    python edus_2.0_b200/build.py        -> edus_2.0_b200/lib/libedus_gpu.so

nvcc compiles for sm_100a only (B200); the result is loaded through ctypes by
edus.py and by any C/C++ caller of include/edus_gpu.h.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libedus_gpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["edus_gpu.cu", "edus_noalloc.cu", "surrogate.cu"]
HEADERS = ["comm_ws.cuh", "fft_plane.cuh", "kernels.cuh", "packed_kernels.cuh", "plane3.cuh", "plane_plan.hpp", "split_kernels.cuh", "sweep_kernels.cuh", "tma.cuh"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "edus_gpu.h"))
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-o", LIB] + [os.path.join(CSRC, f) for f in SOURCES]
    if verbose:
        cmd.insert(-len(SOURCES), "-Xptxas")
        cmd.insert(-len(SOURCES), "-v")
    env = dict(os.environ)
    # the host compiler must be the system gcc (its OpenMP/libstdc++ match the image)
    env.pop("CC", None)
    env.pop("CXX", None)
    subprocess.run(cmd, check=True, env=env)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
