"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, rejects bad arguments with status codes, and the host-side
planner makes the expected strategy choices."""
import ctypes
import os
import re

import numpy as np
import pytest

from _pkg import PKG_DIR, ROOT, load

HEADER = os.path.join(ROOT, "include", "catabra_b200.h")


def header_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int64_t|int|const char\*)\s+(cfft_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(os.path.join(PKG_DIR, "libcatabra_b200.so"))
    syms = header_symbols()
    assert len(syms) >= 12
    for s in syms:
        assert hasattr(lib, s), s


def test_binding_covers_header():
    m = load()
    assert set(m._lib.SIGNATURES) == set(header_symbols())
    assert m.version() == 100


def test_invalid_arguments_return_status():
    m = load()
    lib = m._lib.LIB
    h = ctypes.c_void_p()
    assert lib.cfft_plan_create(ctypes.byref(h), 0, 1, 0, 0) == m._lib.ERR_INVALID
    assert b"n and batch" in lib.cfft_last_error()
    assert lib.cfft_plan_create(ctypes.byref(h), 16, 0, 0, 0) == m._lib.ERR_INVALID
    assert lib.cfft_plan_create(ctypes.byref(h), 16, 1, 7, 0) == m._lib.ERR_INVALID
    assert lib.cfft_plan_create(ctypes.byref(h), 16, 1, 0, 3) == m._lib.ERR_INVALID
    assert lib.cfft_plan_create(None, 16, 1, 0, 0) == m._lib.ERR_INVALID
    assert lib.cfft_execute(None, None, None, 0, None) == m._lib.ERR_INVALID
    assert lib.cfft_plan_destroy(None) == m._lib.ERR_INVALID
    assert lib.cfft_plan_launches(None) == -1
    srv = ctypes.c_void_p()
    assert lib.cfft_serve_create(ctypes.byref(srv), 5, 0, 0, 0) == m._lib.ERR_INVALID
    assert lib.cfft_serve_create(ctypes.byref(srv), 0, 0, 0, 9) == m._lib.ERR_INVALID
    assert lib.cfft_serve_create(None, 0, 0, 0, 0) == m._lib.ERR_INVALID
    t = ctypes.c_int64()
    assert lib.cfft_serve_submit(None, 16, None, None, 0, ctypes.byref(t)) == m._lib.ERR_INVALID
    assert lib.cfft_serve_wait(None, 0, None) == m._lib.ERR_INVALID
    assert lib.cfft_serve_drain(None) == m._lib.ERR_INVALID
    assert lib.cfft_serve_destroy(None) == m._lib.ERR_INVALID
    assert lib.cfft_batch_create(None, 1, None, 0, 0) == m._lib.ERR_INVALID
    rp = ctypes.c_void_p()
    assert lib.cfft_rfft_plan_create(None, 16, 1, 0, 0) == m._lib.ERR_INVALID
    assert lib.cfft_rfft_plan_create(ctypes.byref(rp), 0, 1, 0, 0) == m._lib.ERR_INVALID
    assert lib.cfft_rfft_plan_create(ctypes.byref(rp), 16, 1, 9, 0) == m._lib.ERR_INVALID
    assert lib.cfft_rfft_execute(None, None, None, None) == m._lib.ERR_INVALID
    assert lib.cfft_rfft_plan_destroy(None) == m._lib.ERR_INVALID


def test_python_api_argument_errors():
    m = load()
    with pytest.raises(TypeError):
        m.fft(np.zeros(8, dtype=np.float64))
    with pytest.raises(ValueError):
        m.fft(np.zeros((2, 2), dtype=np.complex128), axis=2)
    with pytest.raises(ValueError):
        m.plan_fft(np.zeros(8, dtype=np.complex128), 3)


@pytest.mark.parametrize("n,expect", [
    (1, "rows"), (4096, "rows(V=1)[16,16,16]"), (30240, "cluster(C=9,L=3360 per CTA,threads=240,tma)"), (10007, "rader(n=10007,M=20480)+cluster(C=5"),
    (89, "rader(n=89,M=175)+rows"), (10006, "bluestein(n=10006,M=20160)"),
    (2 ** 20, "pow2(N1=256,N2=4096"), (2 ** 22, "pow2(N1=1024,N2=4096"), (2 ** 23, "twopass(N1=2048,N2=4096)"),
    (2 ** 15, "pow2(N1=8,N2=4096,ctas_per_sm=2,tma)"), (2 ** 14, "pow2cluster(C=4,4096 per CTA,ctas_per_sm=2)"), (60480, "four(C="),
])
def test_strategy_choice(n, expect):
    m = load()
    assert expect in m.describe_strategy(n), m.describe_strategy(n)


@pytest.mark.parametrize("n,expect", [
    (65536, "pow2(N1=16,N2=4096,ctas_per_sm=2,tma)"), (8192, "pow2cluster(C=2,4096 per CTA,ctas_per_sm=2)"), (1 << 17, "pow2(N1=32,N2=4096,ctas_per_sm=2,tma)"), (19683, "four(C=3,"), (4096, "rows"),
])
def test_strategy_choice_complex64(n, expect):
    m = load()
    assert expect in m.describe_strategy(n, np.complex64), m.describe_strategy(n, np.complex64)


def test_strategy_covers_every_length_class():
    # every n in the batching/serving range maps to some strategy
    m = load()
    rng = np.random.default_rng(0)
    for n in rng.integers(16, 2 ** 20, size=200):
        s = m.describe_strategy(int(n))
        assert s, n
