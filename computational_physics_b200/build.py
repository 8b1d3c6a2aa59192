"""Builds the native libraries of the package in-tree.

  computational_physics_b200/lib/libswb200.so   CUDA kernels + C ABI (include/swb200.h), sm_100a

The reference's own Ising2D program with the nvidia_gpu target is built from the reference
sources by computational_physics_b200/dropin/build_dropin.py (into lib/dropin/).

Usage: python -m computational_physics_b200.build [--verbose]
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I", os.path.join(ROOT, "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    deps = cu + sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + [os.path.join(ROOT, "include", "swb200.h")]
    so = os.path.join(LIB, "libswb200.so")
    if force or _stale(so, deps):
        extra = ["-Xptxas", "-v"] if ptxas_info else []
        _run([nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-shared", "-o", so, *cu, "-lcudart"], verbose)
    return so


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
