// mixc.cuh -- a mixed-radix length n = C L on a cluster of C CTAs, each
// running an L-point register FFT, joined by one radix-C combine through
// distributed shared memory (the reference splits such lengths four-step
// style, src/mixed_radix.jl:44-78; this is the same decomposition with the
// p = C factor spread over a thread-block cluster).
//
// Decimation in time over the cluster: CTA c transforms the stride-C
// subsequence x[c + C t], t < L, into F_c[k]; then
//   X[k + L q] = sum_c w_n^(c k) F_c[k] w_C^(c q),   k < L, q < C,
// evaluated by the thread that owns k (threads of the whole cluster take k
// round robin), which reads F_c[k] from every CTA and writes the C outputs:
// for fixed q, adjacent k are adjacent addresses, so the stores are whole
// segments.  The strided input (16-byte elements C x 16 bytes apart) is read
// by cp.async; neighbouring CTAs read the other halves of the same sectors,
// which the L2 serves from one DRAM fetch.
//
// The L-point FFT runs as three decimation-in-frequency Stockham stages of
// radices R0 R1 R2 (L = R0 R1 R2): stage s splits every current
// sub-transform of length Ls as t = t' + (Ls / R) m, does DFT_R over m in
// registers (one butterfly per thread; T threads cover the largest butterfly
// count), multiplies by w_Ls^(t' k) and leaves sub-transform K + P k (P = the
// product of the earlier radices) of length Ls / R.  Element (K, t) of a
// stage sits at shared slot K Ls + t; adjacent threads take adjacent t', so
// shared accesses are runs of consecutive 16-byte slots, and the last stage's
// stride-R2 reads are conflict-free for an odd R2.  Stage 0's inputs arrive
// by cp.async in the slots the same thread reads and then overwrites, so the
// load needs no barrier.  Twiddles: FP64 powers of values from two-level
// tables of w_L and w_n in shared memory, each rounded once to the data type.
#pragma once
#include "engine.cuh"

template <int C_, int R0_, int R1_, int R2_, int T_> struct MixShape {
    static constexpr int C = C_, R0 = R0_, R1 = R1_, R2 = R2_, T = T_;
    static constexpr int L = R0 * R1 * R2;
    static constexpr int N = C * L;
    static constexpr int NB0 = L / R0;                 // stage-0 butterflies (t' range)
    static constexpr int LS1 = NB0, NB1 = LS1 / R1;    // stage 1
    static constexpr int NBF1 = L / R1, NBF2 = L / R2; // butterflies of stages 1, 2
    static constexpr int RMAX = R0 > R1 ? (R0 > R2 ? R0 : R2) : (R1 > R2 ? R1 : R2);
    static_assert(NB0 <= T && NBF1 <= T && NBF2 <= T, "a stage has more butterflies than threads");
    static_assert(R2 % 2 == 1, "the last stage's stride-R2 reads are conflict-free for odd R2");
};

// w^e from a two-level FP64 table
__device__ __forceinline__ double2 mx_w(const double2* lo, const double2* hi, int bits, unsigned e) {
    return cmul(lo[e & ((1u << bits) - 1)], hi[e >> bits]);
}
// v[k] w^(e0 k) for k < R, stored at dst[k stride] (mx_tw_store) or kept in
// place (mx_tw_row): the FP64 powers w^(e0 k) = w^(e0 (k-1)) w^e0 of one
// table value, each rounded once to V (the same FP64 work as a table
// product per twiddle, without the per-twiddle table reads; the powers'
// relative error stays near 1e-15)
template <int R, typename V>
__device__ __forceinline__ void mx_tw_store(const V* v, V* dst, int stride, const double2* lo, const double2* hi,
                                            int bits, unsigned e0) {
    const double2 b = mx_w(lo, hi, bits, e0);
    double2 w = b;
    dst[0] = v[0];
#pragma unroll
    for (int k = 1; k < R; k++) {
        dst[k * stride] = cmul(v[k], fromd<V>(w));
        if (k < R - 1) w = cmul(w, b);
    }
}
template <int R, typename V>
__device__ __forceinline__ void mx_tw_row(V* v, const double2* lo, const double2* hi, int bits, unsigned e0) {
    const double2 b = mx_w(lo, hi, bits, e0);
    double2 w = b;
#pragma unroll
    for (int k = 1; k < R; k++) {
        v[k] = cmul(v[k], fromd<V>(w));
        if (k < R - 1) w = cmul(w, b);
    }
}

// rows of one tensor copy of the strided input (TMA): the largest divisor of
// L that a box dimension allows (at most 256)
__host__ __device__ constexpr int mix_box_rows(int L) {
    int r = 1;
    for (int d = 1; d <= 256 && d <= L; d++)
        if (L % d == 0) r = d;
    return r;
}

// KParams: t4 = two-level table of w_L, t4n = two-level table of w_n (both
// staged in shared memory after the buffer unless GTAB), in / out at
// in_dist / out_dist, batch = transforms (one per cluster).
// GTAB: the w_n table is read through L2 instead of being staged (frees
// its shared memory for a third CTA per SM).
// TMA (ComplexF64): the CTA's stride-C subsequence arrives as L / B tensor
// copies of B rows x 16 bytes (tm maps the input as [transform][t < L][2 C
// doubles]) completing on an mbarrier after the tables; per-element cp.async
// of the strided input writes shared memory one sector at a time (measured:
// as many wavefronts as all the FFT exchanges together).  A copy that times
// out records the fault and the CTA still takes every cluster barrier.
template <typename V, class S, bool GTAB = false, bool TMA = false>
__device__ __forceinline__ void mixc_body(const KParams& p, unsigned char* smem, const CUtensorMap* tm = nullptr) {
    cg::cluster_group cl = cg::this_cluster();
    const int c = (int)cl.block_rank();
    const int tr = block_id(p) / S::C;
    if (tr >= p.batch) return;                  // uniform across the cluster
    V* buf = (V*)smem;                          // L slots
    double2* tab = after16(buf + S::L);
    const int bl = p.t4.bits, bn = p.t4n.bits;
    const int nlo = 1 << bl, nhi = (p.t4.N + nlo - 1) / nlo + 1;
    const int mlo = 1 << bn, mhi = (p.t4n.N + mlo - 1) / mlo + 1;
    double2 *llo = tab, *lhi = tab + nlo;
    const double2 *glo = GTAB ? p.t4n.lo : lhi + nhi, *ghi = GTAB ? p.t4n.hi : lhi + nhi + mlo;
    uint64_t* bar = (uint64_t*)(tab + nlo + nhi + (GTAB ? 0 : mlo + mhi));
    if constexpr (TMA) {
        // slot t = x[c + C t]: box k covers t in [B k, B k + B)
        constexpr int B = mix_box_rows(S::L);
        if (opaque_tid() == 0) mbar_init(bar, 1);
        __syncthreads();                        // the barrier is initialised before anyone waits
        if (opaque_tid() == 0) {
            mbar_expect_tx(bar, (unsigned)(S::L * sizeof(V)));
#pragma unroll 1
            for (int k = 0; k < S::L / B; k++) tma_load_3d(buf + B * k, tm, bar, 2 * c, B * k, tr);
        }
    }
    {
        // stage-0 inputs: thread b < NB0 owns slots b + NB0 m = x[c + C (b + NB0 m)]
        const int b = opaque_tid();
        if (!TMA && b < S::NB0) {
            const V* x = (const V*)p.in + (long long)tr * p.in_dist + c + (long long)S::C * b;
#pragma unroll
            for (int m = 0; m < S::R0; m++) cp_async_elem(buf + b + S::NB0 * m, x + (long long)S::C * S::NB0 * m);
        }
        if (!TMA) cp_async_commit();
        for (int i = b; i < nlo + nhi; i += S::T) tab[i] = (i < nlo) ? p.t4.lo[i] : p.t4.hi[i - nlo];
        if (!GTAB) {
            double2* gs = lhi + nhi;
            for (int i = b; i < mlo + mhi; i += S::T) gs[i] = (i < mlo) ? p.t4n.lo[i] : p.t4n.hi[i - mlo];
        }
    }
    V v[S::RMAX];
    {
        // stage 0: DFT_R0 over m, twiddle w_L^(b k), back into the same slots
        const int b = opaque_tid();
        if constexpr (TMA) {
            if (!mbar_wait(bar, 0) && b == 0) record_fault(kFaultTmaTimeout);
        } else {
            cp_async_wait_all();
        }
        if (b < S::NB0) {
#pragma unroll
            for (int m = 0; m < S::R0; m++) v[m] = load_in(p, buf[b + S::NB0 * m]);
            dft<S::R0>(*reinterpret_cast<V(*)[S::R0]>(v));
        }
        __syncthreads();                        // tables staged (the slots are this thread's own)
        if (b < S::NB0) mx_tw_store<S::R0>(v, buf + b, S::NB0, llo, lhi, bl, (unsigned)b);
        __syncthreads();
    }
    {
        // stage 1: sub-transforms K < R0 of length LS1, t' = b % NB1
        const int b = opaque_tid();
        const int tp = b % S::NB1, K = b / S::NB1;
        if (b < S::NBF1) {
#pragma unroll
            for (int m = 0; m < S::R1; m++) v[m] = buf[K * S::LS1 + tp + S::NB1 * m];
        }
        __syncthreads();                        // every read before the writes
        if (b < S::NBF1) {
            dft<S::R1>(*reinterpret_cast<V(*)[S::R1]>(v));
            mx_tw_store<S::R1>(v, buf + K * S::NB1 + tp, S::R0 * S::NB1, llo, lhi, bl, (unsigned)(tp * S::R0));
        }
        __syncthreads();
    }
    {
        // stage 2: sub-transforms K < R0 R1 of length R2; F[K + R0 R1 k]
        const int b = opaque_tid();
        if (b < S::NBF2) {
#pragma unroll
            for (int m = 0; m < S::R2; m++) v[m] = buf[b * S::R2 + m];
        }
        __syncthreads();                        // every read before F overwrites the slots
        if (b < S::NBF2) {
            dft<S::R2>(*reinterpret_cast<V(*)[S::R2]>(v));
#pragma unroll
            for (int k = 0; k < S::R2; k++) buf[b + S::NBF2 * k] = v[k];
        }
    }
    cl.sync();                                  // every F_c published
    {
        // combine: the cluster's threads take k round robin
        const int g = c * S::T + opaque_tid();
        V* out = (V*)p.out + (long long)tr * p.out_dist;
        for (int k = g; k < S::L; k += S::C * S::T) {
            V f[S::C];
#pragma unroll
            for (int q = 0; q < S::C; q++) f[q] = cl.map_shared_rank(buf, q)[k];
            mx_tw_row<S::C>(f, glo, ghi, bn, (unsigned)k);
            dft<S::C>(f);
#pragma unroll
            for (int q = 0; q < S::C; q++) stg_stream(out + k + S::L * q, store_out(p, f[q]));
        }
    }
    cl.sync();                                  // no CTA leaves while a peer reads its F
}
