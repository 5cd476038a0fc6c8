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
