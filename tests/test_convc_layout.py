"""CPU check of the cluster Rader kernel's index plan (convc.cuh).

The kernel's data movement is restated with numpy for one transform: CTA c
gathers a[c + C m] through the permutation table (built as the planner
builds it), F_c = FFT_4096, the per-k combine / spectrum / conjugate / DIF
step that thread t of CTA (k3 mod C) performs for k = t + 256 k3, the second
FFT_4096 per CTA and the scatter y[g^-j] = x0 + conj(U[j]).  The result must
be the DFT of x.  Also checked: every (CTA, slot) of the middle phase is
owned by exactly one thread, and the tables cover the convolution indices
exactly once.  No GPU is involved.
"""
import numpy as np
import pytest


def primitive_root(p):
    phi = p - 1
    fac, m, d = [], phi, 2
    while d * d <= m:
        if m % d == 0:
            fac.append(d)
            while m % d == 0:
                m //= d
        d += 1
    if m > 1:
        fac.append(m)
    g = 2
    while any(pow(g, phi // f, p) == 1 for f in fac):
        g += 1
    return g


def cluster_size(n):
    return next(c for c in (3, 4, 5, 7, 8) if 4096 * c >= 2 * n - 3)


def tables(n, C):
    """perm / iperm in the kernel's order (as plan.cpp builds them)."""
    L, M = n - 1, 4096 * C
    g = primitive_root(n)
    gi = pow(g, n - 2, n)
    fw = [pow(g, j, n) for j in range(L)]
    bw = [pow(gi, j, n) for j in range(L)]
    perm = np.full(M, -1, dtype=np.int64)
    iperm = np.full(M, -1, dtype=np.int64)
    for c in range(C):
        for i in range(4096):
            j = c + C * i
            if j < L:
                perm[c * 4096 + i] = fw[j]
                iperm[c * 4096 + i] = bw[j]
    return perm, iperm, bw


def emulate(x, C):
    n = len(x)
    L, M = n - 1, 4096 * C
    perm, iperm, bw = tables(n, C)
    # kernel vector and spectrum (exact twiddles): b[m] = w_n^(g^-k), cyclic in M
    bL = np.exp(-2j * np.pi * np.array(bw) / n)
    b = np.zeros(M, dtype=complex)
    b[:L] = bL
    b[M - L + 1:] = bL[1:]
    B = np.fft.fft(b) / M
    wM = lambda e: np.exp(-2j * np.pi * e / M)
    # 1-2: gather and F_c
    F = np.zeros((C, 4096), dtype=complex)
    total = 0
    for c in range(C):
        src = perm[c * 4096:(c + 1) * 4096]
        a = np.where(src >= 0, x[np.maximum(src, 0)], 0)
        total += a.sum()
        F[c] = np.fft.fft(a)
    # 3: thread t of CTA (k3 mod C) handles k = t + 256 k3
    Z = np.full((C, 4096), np.nan, dtype=complex)
    owner = np.zeros(4096, dtype=int)
    for cp in range(C):
        for k3 in range(cp, 16, C):
            for t in range(256):
                k = t + 256 * k3
                owner[k] += 1
                q = np.arange(C)
                f = F[:, k] * wM(q * k)
                A = np.fft.fft(f)                     # A[k + 4096 q]
                u = np.conj(A * B[k + 4096 * q])
                v = np.fft.fft(u)                     # sum_r u_r w_C^(r q)
                Z[:, k] = v * wM(q * k)
    assert (owner == 1).all()
    # 4: second FFT per CTA, scatter
    y = np.full(n, np.nan, dtype=complex)
    x0 = x[0]
    for c in range(C):
        U = np.fft.fft(Z[c])
        dst = iperm[c * 4096:(c + 1) * 4096]
        ok = dst >= 0
        y[dst[ok]] = x0 + np.conj(U[ok])
    y[0] = x0 + total
    return y, perm, iperm


@pytest.mark.parametrize("n", [4099, 6151, 10007, 12301, 16381])
def test_cluster_rader_index_plan(n):
    C = cluster_size(n)
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y, perm, iperm = emulate(x, C)
    assert not np.isnan(y).any()
    ref = np.fft.fft(x)
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-12
    # the gather reads x[1:] exactly once and the scatter writes y[1:] exactly once
    assert sorted(perm[perm >= 0].tolist()) == list(range(1, n))
    assert sorted(iperm[iperm >= 0].tolist()) == list(range(1, n))
