"""ctypes wrapper of the CPU oracle -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module, and only as the checker or the timed CPU baseline.  The
shipped library never calls it.

The oracle restates CatabraFFT.jl's algorithm (see catabra_oracle.c for the
file:line map).  ``fft``/``ifft``/``bfft`` follow CatabraFFT.jl:65-115.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS: dict = {}

FWD, INV, BWD = 0, 1, 2   # fft, ifft (1/n), bfft (unnormalised)


def build() -> None:
    """Compile both oracle variants with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _lib(precision: str):
    if precision in _LIBS:
        return _LIBS[precision]
    name = {"f64": "liboracle_f64.so", "f32": "liboracle_f32.so"}[precision]
    path = os.path.join(_HERE, name)
    if not os.path.exists(path):
        build()
    lib = ctypes.CDLL(path)
    p = "co64_" if precision == "f64" else "co32_"
    i64, vp, ci = ctypes.c_int64, ctypes.c_void_p, ctypes.c_int
    for fn, args, res in [
        ("fft", [i64, vp, vp, ci], ci),
        ("fft_batch", [i64, i64, vp, vp, ci, ci], ci),
        ("prepare", [i64], ci),
        ("describe", [i64, ctypes.c_char_p, ci], ci),
        ("radix_plan_exec", [i64, ctypes.POINTER(ci), ci, vp, vp], ci),
        ("find_closest_factors", [i64, ctypes.POINTER(i64), ctypes.POINTER(i64)], ci),
        ("rader_generator", [i64], i64),
        ("set_rader_mode", [ci], ci),
        ("max_threads", [], ci),
        ("empty_cache", [], None),
    ]:
        f = getattr(lib, p + fn)
        f.argtypes = args
        f.restype = res
    lib._p = p
    _LIBS[precision] = lib
    return lib


def _call(precision, fn, *args):
    lib = _lib(precision)
    return getattr(lib, lib._p + fn)(*args)


def _as(x, precision):
    dt = np.complex128 if precision == "f64" else np.complex64
    return np.ascontiguousarray(x, dtype=dt)


def transform(x, direction=FWD, precision="f64", threads=1):
    """Transform the last axis of ``x`` (1-D or [batch, n]) on the CPU."""
    a = _as(x, precision)
    n = a.shape[-1]
    batch = a.size // n if n else 0
    y = np.empty_like(a)
    if batch:
        rc = _call(precision, "fft_batch", n, batch, a.ctypes.data, y.ctypes.data,
                   int(direction), int(threads))
        if rc != 0:
            raise ValueError(f"oracle rejected n={n}")
    return y


def fft(x, precision="f64", threads=1):
    return transform(x, FWD, precision, threads)


def ifft(x, precision="f64", threads=1):
    return transform(x, INV, precision, threads)


def bfft(x, precision="f64", threads=1):
    return transform(x, BWD, precision, threads)


def prepare(n, precision="f64"):
    return _call(precision, "prepare", int(n))


def describe(n, precision="f64") -> str:
    buf = ctypes.create_string_buffer(4096)
    _call(precision, "describe", int(n), buf, 4096)
    return buf.value.decode()


def radix_plan_exec(x, radices, precision="f64"):
    a = _as(x, precision)
    y = np.empty_like(a)
    arr = (ctypes.c_int * len(radices))(*radices)
    rc = _call(precision, "radix_plan_exec", a.size, arr, len(radices), a.ctypes.data, y.ctypes.data)
    if rc != 0:
        raise ValueError("bad radix plan")
    return y


def find_closest_factors(n):
    p, m = ctypes.c_int64(), ctypes.c_int64()
    _call("f64", "find_closest_factors", int(n), ctypes.byref(p), ctypes.byref(m))
    return p.value, m.value


def rader_generator(n):
    return _call("f64", "rader_generator", int(n))


def set_rader_mode(faithful: bool, precision="f64"):
    _call(precision, "set_rader_mode", 1 if faithful else 0)


def max_threads():
    return _call("f64", "max_threads")
