"""Build libcatabra_b200.so in-tree for sm_100a (nvcc, no JIT cache).

    python catabrafft.jl_b200/build.py [--force]

The shared library lands next to this file so it travels with the source
tree; Python loads it through ctypes (no torch extension machinery).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcatabra_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "nvcc")

DEVICE_SOURCES = ["kernels.cu", "noalloc.cu", "tables.cu", "real.cu"]
HOST_SOURCES = ["plan.cpp"]
HEADERS = ["engine.cuh", "engine_types.h", "codelets.cuh", "kernels.h"]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    srcs = DEVICE_SOURCES + HOST_SOURCES + HEADERS
    paths = [os.path.join(CSRC, s) for s in srcs]
    paths.append(os.path.join(os.path.dirname(HERE), "include", "catabra_b200.h"))
    return any(os.path.getmtime(p) > t for p in paths if os.path.exists(p))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", CSRC]
    for s in DEVICE_SOURCES:
        o = os.path.join(objdir, s + ".o")
        cmd = [NVCC, *ARCH, "-lineinfo", *common, "-c", os.path.join(CSRC, s), "-o", o]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
        objs.append(o)
    for s in HOST_SOURCES:
        o = os.path.join(objdir, s + ".o")
        subprocess.run([NVCC, *ARCH, *common, "-c", os.path.join(CSRC, s), "-o", o], check=True)
        objs.append(o)
    tmp = LIB + ".tmp"
    subprocess.run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
