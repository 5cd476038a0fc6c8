"""CPU check of the power-of-two passes' index plan (pow2.cuh).

The column pass's per-thread index arithmetic is restated here step by step
for every N1 = 2 .. 1024 and one tile of VC = 4096 / N1 columns: the
shared-memory slots each thread reads and writes in every stage, the stage
twiddles and the output positions.  Checked: the tile's columns come out as
the length-N1 DFT; every slot index is inside the 4096-element buffer; each
stage's writes cover the buffer exactly once; and for VC >= 8 every
quarter-warp of 16-byte accesses (ComplexF64) touches 8 distinct bank groups.
A second test checks the two-pass decomposition itself (pass A's strided
4096-point rows with the four-step twiddle, then pass B's columns).  No GPU
is involved.
"""
import numpy as np
import pytest


def log16(n):
    a = 0
    while n >= 16 and n % 16 == 0:
        n //= 16
        a += 1
    return a


def plan(N1):
    A = log16(N1)
    RL = N1 // 16 ** A
    S = A + (1 if RL > 1 else 0)
    VC = 4096 // N1
    TPC = N1 // 16 if N1 >= 16 else 1
    CPT = 1 if N1 >= 16 else 16 // N1
    return A, RL, S, VC, TPC, CPT


def w(e, L):
    return np.exp(-2j * np.pi * e / L)


def emulate(N1, tile, c0):
    """tile: N1 x VC complex (rows x columns). Returns (Y, accesses) where Y
    is N1 x VC (output row k, column j) and accesses lists, per stage and
    direction, the slot index of every (thread, element)."""
    A, RL, S, VC, TPC, CPT = plan(N1)
    buf = np.zeros(4096, dtype=complex)
    for slot in range(4096):
        buf[slot] = tile[slot // VC, slot % VC]
    Y = np.full((N1, VC), np.nan, dtype=complex)
    acc = []
    regs = [[buf[tid + 256 * k] for k in range(16)] for tid in range(256)]
    acc.append(("stage0-read", [[tid + 256 * k for k in range(16)] for tid in range(256)]))
    if N1 < 16:
        for tid in range(256):
            v = regs[tid]
            for g in range(CPT):
                u = np.array([v[g + CPT * m] for m in range(N1)])
                U = np.fft.fft(u)
                c = c0 + tid + 256 * g
                for k in range(N1):
                    Y[k, c - c0] = U[k]
        return Y, acc
    # stage 0: DFT16 over m, twiddle w_N1^(b k), back into own slots
    writes = []
    for tid in range(256):
        j, b = tid % VC, tid // VC
        V = np.fft.fft(np.array(regs[tid]))
        if S == 1:
            for k in range(16):
                Y[k, j] = V[k]
            continue
        for k in range(16):
            buf[tid + 256 * k] = V[k] * w(b * k, N1)
        writes.append([tid + 256 * k for k in range(16)])
    if S == 1:
        return Y, acc
    acc.append(("stage0-write", writes))
    for s in range(1, S):
        r = 16 if s < A else RL
        Ls = N1 // 16 ** s
        nb = Ls // r
        G = 16 // r
        KR = 16 ** s
        last = s == S - 1
        reads, vals = [], []
        for tid in range(256):
            j, b = tid % VC, tid // VC
            rr, vv = [], []
            for g in range(G):
                beta = b + TPC * g
                tp, K = beta % nb, beta // nb
                for m in range(r):
                    slot = (K * Ls + tp + nb * m) * VC + j
                    rr.append(slot)
                    vv.append(buf[slot])
            reads.append(rr)
            vals.append(vv)
        acc.append((f"stage{s}-read", reads))
        writes = []
        newbuf = np.full(4096, np.nan, dtype=complex)
        for tid in range(256):
            j, b = tid % VC, tid // VC
            ww = []
            for g in range(G):
                grp = np.array(vals[tid][g * r:(g + 1) * r])
                F = np.fft.fft(grp)
                beta = b + TPC * g
                tp, K = beta % nb, beta // nb
                for k in range(r):
                    if last:
                        Y[K + KR * k, j] = F[k]
                    else:
                        slot = ((K + KR * k) * nb + tp) * VC + j
                        newbuf[slot] = F[k] * w(tp * k * (N1 // Ls), N1)
                        ww.append(slot)
            writes.append(ww)
        if not last:
            acc.append((f"stage{s}-write", writes))
            buf = newbuf
    return Y, acc


@pytest.mark.parametrize("N1", [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024])
def test_column_pass_index_plan(N1):
    A, RL, S, VC, TPC, CPT = plan(N1)
    rng = np.random.default_rng(N1)
    tile = rng.standard_normal((N1, VC)) + 1j * rng.standard_normal((N1, VC))
    c0 = VC * (N1 // 2 if N1 > 1 else 0)          # a tile away from column 0
    Y, acc = emulate(N1, tile, c0)
    ref = np.fft.fft(tile, axis=0)
    assert np.allclose(Y, ref, rtol=0, atol=1e-9 * np.abs(ref).max())
    for name, per_thread in acc:
        flat = [s for th in per_thread for s in th]
        assert min(flat) >= 0 and max(flat) < 4096, name
        if name.endswith("write") or name == "stage0-read":
            assert sorted(flat) == list(range(4096)), name       # each slot exactly once
        # bank groups of 16-byte accesses: quarter-warps (8 lanes) of one
        # instruction (same element index e across the lanes)
        if VC >= 8:
            E = len(per_thread[0])
            for e in range(E):
                for q in range(0, 256, 8):
                    groups = {per_thread[t][e] % 8 for t in range(q, q + 8)}
                    assert len(groups) == 8, (name, e, q)


@pytest.mark.parametrize("N1", [2, 16, 64, 1024])
def test_two_pass_decomposition(N1):
    """X[q + 4096 r] = sum_i w_N1^(i r) w_n^(i q) sum_c x[i + N1 c] w_4096^(c q):
    pass A (rows i of the stride-N1 subsequences, twiddled, into Z[i][q]),
    pass B (N1-point DFT down each column q, stored as row r of the output)."""
    n = N1 * 4096
    rng = np.random.default_rng(N1 + 1)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    sub = x.reshape(4096, N1).T                       # sub[i][c] = x[i + N1 c]
    Z = np.fft.fft(sub, axis=1) * w(np.outer(np.arange(N1), np.arange(4096)), n)
    out = np.fft.fft(Z, axis=0)                       # out[r][q] = X[q + 4096 r]
    X = np.fft.fft(x)
    assert np.allclose(out.reshape(-1), X, rtol=0, atol=1e-9 * np.abs(X).max())
    # pass A's twiddle recurrence w_n^(i t) (w_n^(256 i))^k3 against direct powers
    i = N1 - 1
    for t in (0, 1, 255):
        wr, st = w(i * t, n), w(256 * i, n)
        for k3 in range(16):
            assert abs(wr - w(i * (t + 256 * k3), n)) < 1e-14
            wr *= st
