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

DEVICE_SOURCES = ["kernels.cu", "queue.cu", "noalloc.cu", "tables.cu", "real.cu"]
HOST_SOURCES = ["plan.cpp"]


def _headers() -> list:
    """Every header under csrc/ plus the public C header: a change to any of
    them rebuilds every object."""
    hs = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(os.path.dirname(HERE), "include", "catabra_b200.h"))
    return hs


def _mtime(p: str) -> float:
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    paths = [os.path.join(CSRC, s) for s in DEVICE_SOURCES + HOST_SOURCES] + _headers()
    return any(_mtime(p) > t for p in paths)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the objects whose source or any header changed (all of them
    with force), then link the library."""
    if not force and not _stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    hdr = max(_mtime(h) for h in _headers())
    objs = []
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", CSRC]
    for s in DEVICE_SOURCES + HOST_SOURCES:
        src = os.path.join(CSRC, s)
        o = os.path.join(objdir, s + ".o")
        objs.append(o)
        if not force and _mtime(o) > max(hdr, _mtime(src)):
            continue
        cmd = [NVCC, *ARCH, *common, "-c", src, "-o", o]
        if s in DEVICE_SOURCES:
            cmd.insert(3, "-lineinfo")
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
    tmp = LIB + ".tmp"
    subprocess.run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
