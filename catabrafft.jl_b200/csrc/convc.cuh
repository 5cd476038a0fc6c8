// convc.cuh -- Rader's prime-length DFT (src/prime.jl:5-81) with the cyclic
// convolution on a cluster of C CTAs of register 4096-point FFTs.
//
// For a prime n the reference computes
//   y[0] = x[0] + sum_{j>0} x[j],   y[g^-j] = x[0] + (a (*) b)[j],  j < L = n-1,
// with a[j] = x[g^j] and the cyclic convolution (*) of length L.  Here the
// convolution is zero-padded to M = 4096 C >= 2L - 1 and evaluated as
// conj(FFT_M(conj(FFT_M(a) * B))) with B = FFT_M(b) / M precomputed in FP64
// (the same kernel vector and spectrum as the other Rader paths).
//
// One transform per cluster of C CTAs (rank c), 256 threads each, 16
// elements per thread:
//   1. gather: CTA c takes the stride-C subsequence a[c + C m], m < 4096,
//      straight from x through the permutation table (L2-resident x), and
//      sums its part of x[1:] in FP64;
//   2. F_c = FFT_4096 of it in registers (fft4096_regs, two shared-memory
//      exchanges), stored in natural order;
//   3. cluster barrier; thread t of CTA c' then owns k = t + 256 k3 for
//      k3 = c', c' + C, ...: it reads F_c[k] from every CTA (distributed
//      shared memory), applies the decimation-in-time combine
//      A[k + 4096 q] = sum_c w_M^(ck) F_c[k] w_C^(cq), multiplies by B and
//      conjugates (u = conj(A B)), and immediately starts the second FFT by
//      decimation in frequency: Z_c[k] = w_M^(kc) sum_q u[k + 4096 q] w_C^(qc),
//      written back to CTA c's slot k.  Each slot is read and rewritten by
//      the same thread, so this phase needs no barrier inside;
//   4. cluster barrier; U[c + C k''] = FFT_4096(Z_c) in registers; the
//      convolution is c[j] = conj(U[j]) and y[g^-j] = x0 + c[j] is scattered
//      to the output (L2 merges the scattered 16-byte stores), y[0] by CTA 0.
// The inverse directions conjugate on load and conjugate + scale on store
// (CatabraFFT.jl:88-115), like every other kernel here.
#pragma once
#include "engine.cuh"

// w_M^e from the FP64 two-level table
__device__ __forceinline__ double2 convc_w(const TwoLevel& t, unsigned e) {
    return cmul(__ldg(t.lo + (e & ((1u << t.bits) - 1))), __ldg(t.hi + (e >> t.bits)));
}

// KParams: nx = n (prime), M = 4096 C, perm[c 4096 + t + 256 k] = the x
// index of a[c + C (t + 256 k)] or -1 (padding), iperm[c 4096 + t + 256 k] =
// the y index of c[c + C (t + 256 k)] or -1, spec = B (natural order, FP64),
// t4 = two-level table of w_4096, t4n = two-level table of w_M.
// Shared memory: buf (16 R4096_PL elements), w_4096 table (129 FP64), the
// CTA's partial sum of x[1:] (FP64), the block reduction scratch (32) and,
// in CTA 0, the total for y[0].
template <typename V, int C>
__device__ __forceinline__ void convc_rader_body(const KParams& p, unsigned char* smem) {
    cg::cluster_group cl = cg::this_cluster();
    const int c = (int)cl.block_rank();
    const int tr = block_id(p) / C;             // transform of this cluster
    if (tr >= p.batch) return;                  // uniform across the cluster
    V* buf = (V*)smem;
    double2* tlo = after16(buf + 16 * R4096_PL);
    double2* thi = tlo + 64;
    double2* part = thi + 65;                   // this CTA's sum of its x[1:] share
    double2* red = part + 1;                    // block_sum scratch (32 entries), then y[0]'s sum
    {
        const int t = opaque_tid();
        if (t < 64) tlo[t ^ (t >> 3)] = p.t4.lo[t];
        if (t < 65) thi[t] = p.t4.hi[t];
    }
    V v[16];
    {
        // 1. gather a[c + C (t + 256 k)] = x[perm] (zero padding past L)
        const int t = opaque_tid();
        const V* x = (const V*)p.in + (long long)tr * p.in_dist;
        const int* pc = p.perm + c * 4096 + t;
        double2 acc = make_double2(0, 0);
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const int src = __ldg(pc + 256 * k);
            V a = zero<V>();
            if (src >= 0) {
                a = load_in(p, __ldg(x + src));
                const double2 d = tod(a);
                acc.x += d.x;
                acc.y += d.y;
            }
            v[k] = a;
        }
        const double2 s = block_sum(acc, red);  // barriers inside: tables staged too
        if (t == 0) *part = s;
    }
    // 2. F_c, stored in natural order
    fft4096_regs(v, buf, tlo, thi, opaque_tid());
    {
        const int t = opaque_tid();
#pragma unroll
        for (int k3 = 0; k3 < 16; k3++) buf[t + 256 * k3] = v[k3];
    }
    cl.sync();                                  // every F_c and partial sum published
    {
        const int t = opaque_tid();
        if (c == 0 && t == 0) {
            // the sum of x[1:] for y[0], kept in this CTA's own slot
            double2 total = make_double2(0, 0);
            for (int q = 0; q < C; q++) {
                const double2 s = *cl.map_shared_rank(part, q);
                total.x += s.x;
                total.y += s.y;
            }
            red[32] = total;
        }
        // 3. combine, spectrum, conjugate, first DIF step of the second FFT
        for (int k3 = c; k3 < 16; k3 += C) {
            const int k = t + 256 * k3;
            V f[C];
#pragma unroll
            for (int q = 0; q < C; q++) f[q] = cl.map_shared_rank(buf, q)[k];
            // w_M^(q k) as FP64 powers of one table value (the powers'
            // relative error stays near 1e-15), each rounded once where used
            double2 w[C];
            w[0] = make_double2(1, 0);
            w[1] = convc_w(p.t4n, (unsigned)k);
#pragma unroll
            for (int q = 2; q < C; q++) w[q] = cmul(w[q - 1], w[1]);
#pragma unroll
            for (int q = 1; q < C; q++) f[q] = cmul(f[q], fromd<V>(w[q]));
            dft<C>(f);                          // f[q] = A[k + 4096 q]
#pragma unroll
            for (int q = 0; q < C; q++) f[q] = conjv(fromd<V>(cmul(tod(f[q]), __ldg(p.spec + k + 4096 * q))));
            dft<C>(f);                          // f[q] = sum_r u[k + 4096 r] w_C^(rq)
#pragma unroll
            for (int q = 1; q < C; q++) f[q] = cmul(f[q], fromd<V>(w[q]));
#pragma unroll
            for (int q = 0; q < C; q++) cl.map_shared_rank(buf, q)[k] = f[q];
        }
    }
    cl.sync();                                  // every Z_c complete; no remote access follows

    // 4. U = FFT_4096(Z_c); c[j] = conj(U[j]), j = c + C (t + 256 k3)
    {
        const int t = opaque_tid();
#pragma unroll
        for (int k = 0; k < 16; k++) v[k] = buf[t + 256 * k];
    }
    __syncthreads();                            // the buffer is free for the exchanges
    fft4096_regs(v, buf, tlo, thi, opaque_tid());
    {
        const int t = opaque_tid();
        const V* x = (const V*)p.in + (long long)tr * p.in_dist;
        V* y = (V*)p.out + (long long)tr * p.out_dist;
        const V x0 = load_in(p, x[0]);
        const int* ic = p.iperm + c * 4096 + t;
#pragma unroll
        for (int k3 = 0; k3 < 16; k3++) {
            const int dst = __ldg(ic + 256 * k3);
            if (dst >= 0) {
                const V cv = conjv(v[k3]);
                y[dst] = store_out(p, mk<V>(x0.x + cv.x, x0.y + cv.y));
            }
        }
        if (c == 0 && t == 0) {
            const double2 d = tod(x0), total = red[32];
            y[0] = store_out(p, fromd<V>(make_double2(d.x + total.x, d.y + total.y)));
        }
    }
}
