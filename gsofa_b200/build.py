"""Builds libgsofa.so (CUDA, sm_100a) and the gsofa CLI in-tree.

    python -m gsofa_b200.build

The library is compiled with nvcc for sm_100a only; the CLI is plain C++ that
links the library through its C ABI (rpath $ORIGIN).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgsofa.so")
CLI = os.path.join(HERE, "gsofa")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libgsofa.so")


def _cxx() -> str:
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("g++ not found")


def _newer(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _sources():
    srcs = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
            if f.endswith((".cu", ".cuh", ".h", ".hpp"))]
    return srcs + [os.path.join(ROOT, "include", "gsofa.h")]


def build_library(force: bool = False, verbose: bool = False) -> str:
    if force or _newer(LIB, _sources()):
        cmd = [_nvcc(), *NVCC_FLAGS, *ARCH, "-shared", "-o", LIB,
               os.path.join(CSRC, "gsofa_api.cu")]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
    return LIB


def build_cli(force: bool = False) -> str:
    src = os.path.join(CSRC, "gsofa_cli.cpp")
    if force or _newer(CLI, [src, LIB, os.path.join(ROOT, "include", "gsofa.h")]):
        cmd = [_cxx(), "-O2", "-std=c++17", "-o", CLI, src, f"-L{HERE}", "-lgsofa",
               "-Wl,-rpath,$ORIGIN", "-Wl,-rpath,/usr/local/cuda/lib64"]
        subprocess.run(cmd, check=True)
    return CLI


def build(force: bool = False, verbose: bool = False) -> None:
    build_library(force, verbose)
    build_cli(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
