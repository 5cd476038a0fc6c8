"""Host-side check of the n = 4096 register kernel's index plan (k_r4096 in
csrc/engine.cuh): the 16 x 16 x 16 split reproduces the DFT, every
shared-memory index stays inside the buffer the launcher sizes, and each
quarter-warp of 16-byte accesses (half-warp of 8-byte ones) touches distinct
bank groups.  The pitches are read from the kernel source."""
import os
import re

import numpy as np

SRC = os.path.join(os.path.dirname(__file__), "..", "catabrafft.jl_b200", "csrc", "engine.cuh")


def _pitches():
    m = re.search(r"constexpr int R4096_PB = (\d+), R4096_PL = (\d+);", open(SRC).read())
    assert m, "pitch constants not found"
    return int(m.group(1)), int(m.group(2))


def _slot(l):
    return l ^ (l >> 3)        # lo-table slot of entry l (l < 64)


def test_split_reproduces_dft():
    pb, pl = _pitches()
    rng = np.random.default_rng(0)
    x = rng.standard_normal(4096) + 1j * rng.standard_normal(4096)
    lo = np.exp(-2j * np.pi * np.arange(64) / 4096)
    hi = np.exp(-2j * np.pi * np.arange(65) * 64 / 4096)
    slots = np.empty(64, complex)
    slots[[_slot(l) for l in range(64)]] = lo

    def w(e):
        return slots[_slot(e & 63)] * hi[e >> 6]

    buf = np.full(16 * pl, np.nan, complex)
    for t in range(256):                                   # stage A
        v = np.fft.fft(x[t + 256 * np.arange(16)])
        for k1 in range(16):
            buf[k1 * 256 + t] = v[k1] * w(t * k1)
    regs = []
    for t in range(256):                                   # stage B reads
        t1, k1 = t & 15, t >> 4
        regs.append(np.fft.fft(buf[k1 * 256 + t1 + 16 * np.arange(16)]))
    buf[:] = np.nan
    for t in range(256):                                   # stage B writes
        t1, k1 = t & 15, t >> 4
        for k2 in range(16):
            i = k1 * pl + k2 * pb + t1
            assert 0 <= i < 16 * pl and np.isnan(buf[i])
            buf[i] = regs[t][k2] * w(16 * t1 * k2)
    out = np.empty(4096, complex)
    for t in range(256):                                   # stage C
        k1, k2 = t & 15, t >> 4
        v = np.fft.fft(buf[k1 * pl + k2 * pb + np.arange(16)])
        out[t + 256 * np.arange(16)] = v
    ref = np.fft.fft(x)
    assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < 1e-14


def test_shared_accesses_conflict_free():
    pb, pl = _pitches()
    patterns = []
    for k in range(16):
        patterns += [lambda t, k=k: k * 256 + t,                          # A store, own input
                     lambda t, k=k: (t >> 4) * 256 + (t & 15) + 16 * k,  # B load
                     lambda t, k=k: (t >> 4) * pl + k * pb + (t & 15),   # B store
                     lambda t, k=k: (t & 15) * pl + (t >> 4) * pb + k]   # C load
    for f in patterns:
        for group, banks in ((8, 8), (16, 16)):                # 16-byte / 8-byte elements
            for g0 in range(0, 256, group):
                a = [f(t) % banks for t in range(g0, g0 + group)]
                assert len(set(a)) == group


def test_twiddle_lookups_spread():
    # the swizzled lo slots: stride-8 and stride-16 exponents of a quarter-warp
    # (the worst cases in natural order) fall in distinct bank groups
    for step in (8, 16):
        for q in range(0, 64, step * 8 if step * 8 <= 64 else 64):
            slots = {_slot((q + step * i) & 63) % 8 for i in range(min(8, 64 // step))}
            assert len(slots) == min(8, 64 // step)
    assert sorted(_slot(l) for l in range(64)) == list(range(64))


def test_buffer_fits_launcher_size():
    pb, pl = _pitches()
    top = 15 * pl + 15 * pb + 15
    assert top < 16 * pl and 16 * 256 <= 16 * pl
    src = open(os.path.join(os.path.dirname(SRC), "kernels.cu")).read()
    assert "16 * R4096_PL * elem_bytes" in src and "129 * sizeof(double2)" in src
