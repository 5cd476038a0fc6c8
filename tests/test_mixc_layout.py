"""CPU check of the mixed-radix cluster kernel's index plan (mixc.cuh).

Restates the kernel's data movement for n = C x R0 R1 R2 with numpy: CTA c's
stride-C subsequence, the three Stockham stages with the kernel's slot
formulas and twiddles, the natural-order F_c, and the round-robin radix-C
combine.  Checked: the result is the DFT of x; every stage reads and writes
each slot exactly once; the combine covers every k once; and quarter-warps of
16-byte shared accesses (8 consecutive threads of a warp) mostly hit
distinct bank groups (conflicts are counted and bounded).  No GPU is used.
"""
import numpy as np
import pytest

SHAPES = [(7, 16, 18, 15, 288), (9, 14, 16, 15, 240)]          # 30240 two ways


def w(e, L):
    return np.exp(-2j * np.pi * np.asarray(e) / L)


def emulate(x, C, R0, R1, R2, T):
    L = R0 * R1 * R2
    n = C * L
    NB0 = L // R0
    LS1, NB1 = NB0, NB0 // R1
    NBF1, NBF2 = L // R1, L // R2
    F = np.zeros((C, L), dtype=complex)
    acc = {}
    for c in range(C):
        buf = np.full(L, np.nan, dtype=complex)
        buf[:] = x[c::C]                              # slot t = x[c + C t]
        # stage 0
        reads0, writes0 = [], []
        new = buf.copy()
        for b in range(NB0):
            sl = [b + NB0 * m for m in range(R0)]
            reads0.append(sl)
            V = np.fft.fft(buf[sl])
            for k in range(R0):
                new[b + NB0 * k] = V[k] * w(b * k, L)
            writes0.append([b + NB0 * k for k in range(R0)])
        buf = new
        # stage 1
        reads1, writes1 = [], []
        new = np.full(L, np.nan, dtype=complex)
        for b in range(NBF1):
            tp, K = b % NB1, b // NB1
            sl = [K * LS1 + tp + NB1 * m for m in range(R1)]
            reads1.append(sl)
            V = np.fft.fft(buf[sl])
            ws = []
            for k in range(R1):
                s = (K + R0 * k) * NB1 + tp
                new[s] = V[k] * w(tp * k * R0, L)
                ws.append(s)
            writes1.append(ws)
        buf = new
        # stage 2
        reads2, writes2 = [], []
        new = np.full(L, np.nan, dtype=complex)
        for b in range(NBF2):
            sl = [b * R2 + m for m in range(R2)]
            reads2.append(sl)
            V = np.fft.fft(buf[sl])
            for k in range(R2):
                new[b + NBF2 * k] = V[k]
            writes2.append([b + NBF2 * k for k in range(R2)])
        F[c] = new
        acc[c] = dict(reads0=reads0, writes0=writes0, reads1=reads1, writes1=writes1, reads2=reads2,
                      writes2=writes2)
    X = np.full(n, np.nan, dtype=complex)
    seen = np.zeros(L, dtype=int)
    for c in range(C):
        for tid in range(T):
            g = c * T + tid
            for k in range(g, L, C * T):
                seen[k] += 1
                f = F[:, k] * w(np.arange(C) * k, n)
                Y = np.fft.fft(f)
                X[k + L * np.arange(C)] = Y
    assert (seen == 1).all()
    return X, acc


@pytest.mark.parametrize("shape", SHAPES)
def test_mixed_cluster_index_plan(shape):
    C, R0, R1, R2, T = shape
    L = R0 * R1 * R2
    n = C * L
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    X, acc = emulate(x, C, R0, R1, R2, T)
    ref = np.fft.fft(x)
    assert np.linalg.norm(X - ref) / np.linalg.norm(ref) < 1e-12
    a = acc[0]
    conflicts = 0
    groups = 0
    for name in ("reads0", "writes0", "reads1", "writes1", "reads2", "writes2"):
        per = a[name]
        flat = [s for th in per for s in th]
        assert sorted(flat) == list(range(L)), name                 # each slot once
        # quarter-warps: threads 8q .. 8q + 7 (within one warp), same element index
        E = len(per[0])
        for e in range(E):
            for q in range(0, len(per) - 7, 8):
                if q // 32 != (q + 7) // 32:
                    continue
                bank = [per[t][e] % 8 for t in range(q, q + 8)]
                groups += 1
                conflicts += 8 - len(set(bank))
    # the odd last radix and adjacent t' keep conflicts rare
    assert conflicts <= 0.05 * groups * 8, (conflicts, groups)
