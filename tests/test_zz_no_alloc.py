"""cfft_fft_twopass_noalloc: the FFT entry point that allocates nothing.

Callers that cannot allocate device memory when they need a transform (a
framework that owns every allocation through its own allocator, a memory pool
that forbids cudaMalloc) use this entry point: its scratch and twiddle tables
live in a fixed array inside the library.  These tests call it
through the C ABI and check it against the planned entry point (cfft_fft) on
two calls in a row, within the parity tolerances of the other GPU tests.
This file is collected last so that a stop-at-first-failure run has already
run every other test; it passes alone in a fresh process as well.
"""
import ctypes

import numpy as np
import pytest

from _pkg import load

pytestmark = pytest.mark.gpu

TOL = {np.complex128: 1e-12, np.complex64: 1e-5}


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _planned(cb, x, direction, dtype_code):
    import torch
    y = torch.empty_like(x)
    n, batch = x.shape[1], x.shape[0]
    cb.check(cb._lib.LIB.cfft_fft(n, batch, dtype_code, 0, ctypes.c_void_p(x.data_ptr()),
                                  ctypes.c_void_p(y.data_ptr()), direction, None))
    return y


def _noalloc(cb, x, direction, dtype_code, stream=None, out=None):
    import torch
    y = torch.empty_like(x) if out is None else out
    n, batch = x.shape[1], x.shape[0]
    cb.check(cb._lib.LIB.cfft_fft_twopass_noalloc(n, batch, dtype_code, ctypes.c_void_p(x.data_ptr()),
                                                  ctypes.c_void_p(y.data_ptr()), direction, stream))
    return y


@pytest.mark.parametrize("dtype", [np.complex128, np.complex64])
def test_noalloc_matches_planned_two_calls(dtype):
    import torch
    cb = load()
    code = cb._lib.C128 if dtype == np.complex128 else cb._lib.C64
    rng = np.random.default_rng(42)
    for n, batch, direction in [(30240, 5, 1), (2 ** 20, 3, 0), (2 ** 18, 4, 2)]:
        x = torch.from_numpy((rng.standard_normal((batch, n))
                              + 1j * rng.standard_normal((batch, n))).astype(dtype)).cuda()
        # the entry point runs before any planned call of this element type, so
        # it must set up everything it launches by itself
        first = _noalloc(cb, x, direction, code)
        second = _noalloc(cb, x, direction, code)      # the array keeps the last call's contents
        ref = _planned(cb, x, direction, code)
        torch.cuda.synchronize()
        r = ref.cpu().numpy()
        assert rel(first.cpu().numpy(), r) < TOL[dtype], (n, dtype)
        assert rel(second.cpu().numpy(), r) < TOL[dtype], (n, dtype)
        # in place (input and output the same buffer), across several chunks
        # of the fixed scratch for the largest case
        t = x.clone()
        _noalloc(cb, t, direction, code, out=t)
        torch.cuda.synchronize()
        assert rel(t.cpu().numpy(), r) < TOL[dtype], (n, dtype, "in place")


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    cb = load()
    lib = cb._lib.LIB
    x = torch.zeros((1, 16), dtype=torch.complex128, device="cuda")
    # 2^22 ComplexF64 elements exceed the 32 MiB scratch; 11 * 4096 is not 7-smooth
    for n in (1 << 22, 11 * 4096):
        rc = lib.cfft_fft_twopass_noalloc(n, 1, cb._lib.C128, ctypes.c_void_p(x.data_ptr()),
                                         ctypes.c_void_p(x.data_ptr()), 0, None)
        assert rc == cb._lib.ERR_UNSUPPORTED
        assert b"cfft_fft_twopass_noalloc" in lib.cfft_last_error()
