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


def _obj(s: str) -> str:
    return os.path.join(HERE, "_build", s + ".o")


def _stale_objects(force: bool) -> list:
    """Sources whose object is missing or older than the source or any header
    (a source edited while a build runs stays stale: the check is per object,
    not against the library)."""
    hdr = max(_mtime(h) for h in _headers())
    out = []
    for s in DEVICE_SOURCES + HOST_SOURCES:
        if force or _mtime(_obj(s)) <= max(hdr, _mtime(os.path.join(CSRC, s))):
            out.append(s)
    return out


def _stale() -> bool:
    objs = [_obj(s) for s in DEVICE_SOURCES + HOST_SOURCES]
    return bool(_stale_objects(False)) or not os.path.exists(LIB) or \
        any(_mtime(o) > _mtime(LIB) for o in objs)


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the objects whose source or any header changed (all of them
    with force), then link the library."""
    todo = _stale_objects(force)
    if not todo and not _stale():
        return LIB
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", CSRC]
    for s in todo:
        cmd = [NVCC, *ARCH, *common, "-c", os.path.join(CSRC, s), "-o", _obj(s)]
        if s in DEVICE_SOURCES:
            cmd.insert(3, "-lineinfo")
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
    objs = [_obj(s) for s in DEVICE_SOURCES + HOST_SOURCES]
    tmp = LIB + ".tmp"
    subprocess.run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
