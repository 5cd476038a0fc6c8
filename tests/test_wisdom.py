"""Wisdom (persistent MEASURE/ENCHANT choices): file format and round trip.

The CPU tests check the file handling only; the GPU test checks that a
MEASURE plan rebuilt from imported wisdom has the same shape and results.
"""
import numpy as np
import pytest

import oracle
from _pkg import load


def test_wisdom_file_round_trip(tmp_path):
    m = load()
    m.forget_wisdom()
    good = tmp_path / "w.txt"
    good.write_text("catabra-b200-wisdom 1\n"
                    "30240 64 0 1 | 1 0 30240 168 180 6 1 a 7 3 8 c 9 5 4\n"
                    "# a comment\n"
                    "4096 1 1 2 | 0 0 4096 1 1 1 1 a c 16 16 16\n")
    m.import_wisdom(good)
    assert m.wisdom_entries() == 2
    out = tmp_path / "out.txt"
    m.export_wisdom(out)
    lines = out.read_text().splitlines()
    assert lines[0] == "catabra-b200-wisdom 1"
    assert "30240 64 0 1 | 1 0 30240 168 180 6 1 a 7 3 8 c 9 5 4" in lines
    m.forget_wisdom()
    assert m.wisdom_entries() == 0


@pytest.mark.parametrize("text", ["not wisdom\n", "catabra-b200-wisdom 1\n30240 x 0 1 | 1\n",
                                  "catabra-b200-wisdom 1\n0 1 0 1 | 1 0 1 1 1 1 1 a c\n"])
def test_wisdom_rejects_bad_files(tmp_path, text):
    m = load()
    m.forget_wisdom()
    bad = tmp_path / "bad.txt"
    bad.write_text(text)
    with pytest.raises(m.CatabraError):
        m.import_wisdom(bad)
    assert m.wisdom_entries() == 0
    with pytest.raises(m.CatabraError):
        m.import_wisdom(tmp_path / "missing.txt")


@pytest.mark.gpu
def test_measure_plan_from_wisdom(tmp_path):
    import ctypes
    m = load()
    lib = m._lib.LIB
    m.forget_wisdom()

    def plan_desc():
        h = ctypes.c_void_p()
        m.check(lib.cfft_plan_create(ctypes.byref(h), 30240, 16, m.C128, m.MEASURE))
        buf = ctypes.create_string_buffer(256)
        lib.cfft_plan_describe(h, buf, 256)
        lib.cfft_plan_destroy(h)
        return buf.value.decode()

    d1 = plan_desc()
    assert m.wisdom_entries() == 1
    path = tmp_path / "w.txt"
    m.export_wisdom(path)
    m.forget_wisdom()
    m.import_wisdom(path)
    assert plan_desc() == d1
    x = np.random.default_rng(3).standard_normal((2, 30240)) + 1j * np.random.default_rng(4).standard_normal((2, 30240))
    y = m.plan_fft(x, m.MEASURE) * x
    ref = oracle.fft(x)
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-12
    m.forget_wisdom()


@pytest.mark.gpu
@pytest.mark.parametrize("dtype_name,tol", [("C128", 1e-12), ("C64", 1e-5)])
def test_threads_per_transform_axis_round_trip(tmp_path, dtype_name, tol):
    """The timed planners' thread axis: 30240 runs as 7 CTAs of 288 threads
    (16 x 18 x 15 per CTA) or as 9 CTAs of 240 threads (14 x 16 x 15).  A
    wisdom entry naming the 240-thread build must bring that build back in a
    MEASURE plan (no timing), survive an export, and give the oracle's
    result."""
    import ctypes
    m = load()
    lib = m._lib.LIB
    dtype = getattr(m, dtype_name)
    m.forget_wisdom()
    sig = "7 0 30240 9 3360 9 240 a c v3"
    path = tmp_path / "w.txt"
    path.write_text(f"catabra-b200-wisdom 1\n30240 16 {dtype} {m.MEASURE} | {sig}\n")
    m.import_wisdom(path)
    h = ctypes.c_void_p()
    m.check(lib.cfft_plan_create(ctypes.byref(h), 30240, 16, dtype, m.MEASURE))
    buf = ctypes.create_string_buffer(256)
    lib.cfft_plan_describe(h, buf, 256)
    assert "cluster(C=9,L=3360 per CTA,threads=240)" in buf.value.decode(), buf.value
    out = tmp_path / "out.txt"
    m.export_wisdom(out)
    assert f"30240 16 {dtype} {m.MEASURE} | {sig}" in out.read_text().splitlines()
    import torch
    rng = np.random.default_rng(21)
    x = rng.standard_normal((16, 30240)) + 1j * rng.standard_normal((16, 30240))
    npdt = np.complex128 if dtype_name == "C128" else np.complex64
    xd = torch.from_numpy(x.astype(npdt)).cuda()
    yd = torch.empty_like(xd)
    vp = ctypes.c_void_p
    m.check(lib.cfft_execute(h, vp(xd.data_ptr()), vp(yd.data_ptr()), m.FORWARD, vp(0)))
    torch.cuda.synchronize()
    lib.cfft_plan_destroy(h)
    y = yd.cpu().numpy().astype(np.complex128)
    xr = x.astype(npdt).astype(np.complex128)
    for b in (0, 7, 15):
        ref = oracle.fft(xr[b])
        assert np.linalg.norm(y[b] - ref) / np.linalg.norm(ref) < tol, b
    m.forget_wisdom()
