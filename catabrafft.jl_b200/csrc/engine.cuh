// engine.cuh -- device side of the B200 1D complex FFT.
//
// One transform (or a tile of sub-transforms) is staged in shared memory and
// every radix pass runs there; HBM is touched once on the way in and once on
// the way out.  Four work shapes share the same in-place Stockham core:
//
//   ROWS     V whole transforms per CTA (small n), one row each.
//   FOUR     one transform of length M = N1*N2 split over a thread-block
//            cluster of C CTAs: column FFTs (length N1) in each CTA, twiddle
//            w_M^(i2*k1), exchange through distributed shared memory, row
//            FFTs (length N2).  C = 1 is the single-CTA four-step.
//   COLPASS  / ROWPASS: the two HBM passes of the four-step for lengths that
//            exceed a cluster (tiles of adjacent columns / rows).
//
// Rader (prime n) and Bluestein (other non-smooth n) are fused into ROWS and
// FOUR: the prologue builds the zero-padded convolution input (generator
// permutation or chirp), the convolution runs as FFT_M -> pointwise multiply
// by a precomputed FP64 spectrum -> FFT_M of the conjugate, and the epilogue
// applies the inverse permutation (+x0) or the output chirp.
//
// The Stockham pass is the reference's shell_layered pass
// (src/radix_2_codelets.jl:402-447 and siblings): inputs x[q + s(p + k n1)],
// outputs y[q + s(r p + j)] scaled by w_{n_groups}^{j p}; here x and y are the
// same shared-memory buffer, separated by a barrier with the butterfly inputs
// held in registers.  Twiddles come from tables generated in FP64 on the
// host and rounded once to the data type.
#pragma once
#include <cooperative_groups.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "codelets.cuh"
#include "tma.cuh"

namespace cg = cooperative_groups;

#include "engine_types.h"

// ------------------------------------------------------------------ helpers
// Thread index read through volatile asm: index math derived from it cannot
// be hoisted out of the persistent loops, where the hoisted values would stay
// live across whole transforms and push the FP64 codelets into spills.
__device__ __forceinline__ int opaque_tid() {
    int v;
    asm volatile("mov.u32 %0, %%tid.x;" : "=r"(v));
    return v;
}
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 conjv(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ float2 conjv(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ double2 tod(double2 a) { return a; }
__device__ __forceinline__ double2 tod(float2 a) { return make_double2(a.x, a.y); }
template <typename V> __device__ __forceinline__ V fromd(double2 a);
template <> __device__ __forceinline__ double2 fromd<double2>(double2 a) { return a; }
template <> __device__ __forceinline__ float2 fromd<float2>(double2 a) {
    return make_float2((float)a.x, (float)a.y);
}
template <typename V> __device__ __forceinline__ V zero() { return mk<V>(0, 0); }
// FP64 reduction scratch placed after a V array, rounded up to 16 bytes
template <typename V> __device__ __forceinline__ double2* after16(V* p) {
    return (double2*)(((uintptr_t)p + 15) & ~(uintptr_t)15);
}

// streaming global accesses: inputs and outputs are touched once
__device__ __forceinline__ double2 ldg_stream(const double2* p) { return __ldcs(p); }
__device__ __forceinline__ float2 ldg_stream(const float2* p) { return __ldcs(p); }
__device__ __forceinline__ void stg_stream(double2* p, double2 v) { __stcs(p, v); }
__device__ __forceinline__ void stg_stream(float2* p, float2 v) { __stcs(p, v); }

// The caller's elements (KParams in_fmt / out_fmt, IO_*): a ComplexF16 or
// strided plan reads and writes the caller's layout in its first and last
// kernel, with no widening or gathering sweep of its own.
template <typename V> __device__ __forceinline__ V from_half(__half2 h);
template <> __device__ __forceinline__ float2 from_half<float2>(__half2 h) { return __half22float2(h); }
template <> __device__ __forceinline__ double2 from_half<double2>(__half2 h) {
    const float2 f = __half22float2(h);
    return make_double2(f.x, f.y);
}
template <typename V> __device__ __forceinline__ __half2 to_half(V v) {
    return __floats2half2_rn((float)v.x, (float)v.y);
}
// element j of transform t of the input
template <typename V> __device__ __forceinline__ V user_ld(const KParams& p, long long t, long long j) {
    if (p.in_fmt == IO_PLAIN) return ldg_stream((const V*)p.in + t * p.in_dist + j);
    const long long off = t * p.in_dist + j * p.in_stride;
    if (p.in_fmt == IO_HALF) return from_half<V>(((const __half2*)p.in)[off]);
    return ldg_stream((const V*)p.in + off);
}
// ... staged into shared memory: cp.async for contiguous elements, else a
// load and a shared-memory store (visible after the caller's barrier)
template <typename V> __device__ __forceinline__ void user_cp(const KParams& p, V* dst, long long t, long long j);
// element k of transform t of the output
template <typename V> __device__ __forceinline__ void user_st(const KParams& p, long long t, long long k, V v) {
    if (p.out_fmt == IO_PLAIN) {
        stg_stream((V*)p.out + t * p.out_dist + k, v);
        return;
    }
    const long long off = t * p.out_dist + k * p.out_stride;
    if (p.out_fmt == IO_HALF) ((__half2*)p.out)[off] = to_half(v);
    else stg_stream((V*)p.out + off, v);
}

__device__ __forceinline__ double2 tw_two(const TwoLevel& t, unsigned e) {
    // plain loads: the tables may have been staged in shared memory
    return cmul(t.lo[e & ((1u << t.bits) - 1)], t.hi[e >> t.bits]);
}
// multiply by the four-step twiddle, evaluated in FP64 and rounded once
__device__ __forceinline__ double2 apply_tw(double2 v, const TwoLevel& t, unsigned e) {
    return e ? cmul(v, tw_two(t, e)) : v;
}
// ComplexF32: the twiddle is formed in FP64 and rounded once to FP32, then
// applied in FP32 (the data never leaves FP32)
__device__ __forceinline__ float2 apply_tw(float2 v, const TwoLevel& t, unsigned e) {
    return e ? cmul(v, fromd<float2>(tw_two(t, e))) : v;
}

// block index within this parameter block's launch (batched launches run many
// parameter blocks, each owning a contiguous range of blocks from p.blk0)
__device__ __forceinline__ int block_id(const KParams& p) { return (int)blockIdx.x - p.blk0; }

template <typename V> __device__ __forceinline__ V load_in(const KParams& p, V v) {
    return p.dir ? conjv(v) : v;
}
template <typename V> __device__ __forceinline__ V store_out(const KParams& p, V v);
template <> __device__ __forceinline__ double2 store_out<double2>(const KParams& p, double2 v) {
    if (!p.dir) return v;
    return make_double2(v.x * p.scale, -v.y * p.scale);
}
template <> __device__ __forceinline__ float2 store_out<float2>(const KParams& p, float2 v) {
    if (!p.dir) return v;
    float s = (float)p.scale;
    return make_float2(v.x * s, -v.y * s);
}

// ------------------------------------------------------- fast division
// q = floor(n / d) as (n * m) >> 40 with m = ceil(2^40 / d): exact for
// n < 2^24 and d <= 2^16 (the planner keeps every index and divisor there).
__device__ __forceinline__ int fdiv(unsigned n, unsigned long long m) {
    return (int)(((unsigned long long)n * m) >> 40);
}
__device__ __forceinline__ unsigned long long fdiv_magic(int d) {
    return ((1ULL << 40) + (unsigned long long)d - 1) / (unsigned long long)d;
}

// ------------------------------------------------ asynchronous global->smem
// cp.async (sm_80+ LDGSTS): the copy lands in shared memory without passing
// through registers, so the next transform's input streams in while the
// current one computes.  Both addresses are element aligned (8 or 16 bytes).
template <typename V> __device__ __forceinline__ void cp_async_elem(V* sdst, const V* gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    if constexpr (sizeof(V) == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
template <typename V> __device__ __forceinline__ void user_cp(const KParams& p, V* dst, long long t, long long j) {
    if (p.in_fmt == IO_PLAIN) cp_async_elem(dst, (const V*)p.in + t * p.in_dist + j);
    else *dst = user_ld<V>(p, t, j);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// x / d for 0 <= x < 2^20 and 1 <= d < 2^20 (the block-level indices of the
// radix passes): a fast single-precision quotient, within one of the true
// quotient at these sizes (relative error ~2^-22 on operands exact in
// float), truncated and then corrected by one integer step either way.
__device__ __forceinline__ int udiv_small(int x, int d) {
    int q = (int)__fdividef((float)x, (float)d);
    const int r = x - q * d;
    q += (r >= d) - (r < 0);
    return q;
}

// ----------------------------------------------------- Stockham radix pass
// One pass over Gw sub-transforms of length L held in smem: element i of
// sub-transform g lives at buf[g*gs + i*is].  s = product of earlier radices.
// The team is the whole block (WARP = false) or one warp that owns these
// sub-transforms alone (WARP = true, synchronised with __syncwarp).
// Work item w = b*Gw + g (g fastest: adjacent threads touch adjacent
// sub-transforms), butterfly b = pp*s + q; the items of one thread are
// enumerated with carries instead of divisions.
template <typename V, int EMAX, int R, bool WARP>
__device__ __forceinline__ void spass(V* __restrict__ buf, int L, int Gw, int is, int gs, int s,
                                      const V* __restrict__ twp) {
    constexpr int SL = EMAX / R;
    const int T = WARP ? 32 : (int)blockDim.x;
    const int tid = WARP ? (opaque_tid() & 31) : opaque_tid();
    const int nb = L / R;                  // R is a compile-time constant
    const int n1 = udiv_small(nb, s);  // butterflies per stride class = twiddle block width
    const int W = Gw * nb;
    V v[SL][R];
    int off[SL], pp_[SL];
    int b = udiv_small(tid, Gw), g = tid - b * Gw;
    int pp = udiv_small(b, s), q = b - pp * s;
    const int db = udiv_small(T, Gw), dg = T - db * Gw;
    const int dpp = udiv_small(db, s), dq = db - dpp * s;
#pragma unroll
    for (int i = 0; i < SL; i++) {
        const int w = tid + i * T;
        off[i] = -1;
        if (w < W) {
            const V* src = buf + g * gs + (q + s * pp) * is;
#pragma unroll
            for (int k = 0; k < R; k++) v[i][k] = src[k * nb * is];
            off[i] = g * gs + (q + s * R * pp) * is;
            pp_[i] = pp;
        }
        // advance (g, b) by T and (pp, q) by the resulting change of b
        g += dg;
        int carry = 0;
        if (g >= Gw) { g -= Gw; carry = 1; }
        q += dq + carry;
        pp += dpp;
        if (q >= s) { q -= s; pp += 1; }
    }
    if (WARP) __syncwarp(); else __syncthreads();
#pragma unroll
    for (int i = 0; i < SL; i++) {
        if (off[i] >= 0) {
            dft<R>(v[i]);
            const int p0 = pp_[i];
            if (p0) {
#pragma unroll
                for (int j = 1; j < R; j++) v[i][j] = cmul(v[i][j], twp[(j - 1) * n1 + p0]);
            }
            V* dst = buf + off[i];
#pragma unroll
            for (int j = 0; j < R; j++) dst[j * s * is] = v[i][j];
        }
    }
    if (WARP) __syncwarp(); else __syncthreads();
}

// All passes of `count` sub-transforms, pass-major.  The radix sequence runs
// in CFFT_EXEC_ORDER -- 9^a 7^b 5^c 3^d 16^e 8^f 4^g 2^h, multiplicities in
// P.cnt[] -- as eight fixed-radix loops with runtime trip counts: every pass
// body is a compile-time radix, so no runtime switch widens the register live
// ranges (a switch over radices spills FP64 codelets).
// Block mode: waves of P.G whole sub-transforms (disjoint element sets, so
// each wave's read-barrier-write is a complete in-place pass).
// Warp mode (P.Gwarp > 0): warp w owns groups of P.Gwarp sub-transforms
// (w, w + nwarps, ...) and never waits for the other warps.
// Caller must have synchronised the block after writing buf; returns
// synchronised.
// WM selects the team at compile time (0 block, 1 warp) or at run time from
// P.Gwarp (2).  Kernels that must serve both instantiate 0 and 1 separately:
// with both variants in one FP32 function the compiler demotes the register
// arrays to local memory.
template <typename V, int EMAX, int R, int WM>
__device__ __forceinline__ void radix_loop(V* buf, const SubPlan& P, int count, int is, int gs, int& s,
                                           const V*& twp, int cnt) {
    const bool warp = (WM == 1) || (WM == 2 && P.Gwarp > 0);
    if (WM != 0 && warp) {
        const int nw = blockDim.x >> 5, wid = opaque_tid() >> 5;
        const int step = nw * P.Gwarp;
        for (int i = 0; i < cnt; i++) {
            for (int g0 = wid * P.Gwarp; g0 < count; g0 += step)
                spass<V, EMAX, R, true>(buf + g0 * gs, P.L, min(P.Gwarp, count - g0), is, gs, s, twp);
            twp += (R - 1) * (P.L / (s * R));
            s *= R;
        }
    } else if (WM != 1) {
        for (int i = 0; i < cnt; i++) {
            for (int g0 = 0; g0 < count; g0 += P.G)
                spass<V, EMAX, R, false>(buf + g0 * gs, P.L, min(P.G, count - g0), is, gs, s, twp);
            twp += (R - 1) * (P.L / (s * R));
            s *= R;
        }
    }
}
template <typename V, int EMAX, int WM = 2>
__device__ __forceinline__ void run_subffts(V* buf, const SubPlan& P, const V* tw, int count, int is,
                                            int gs) {
    int s = 1;
    const V* twp = tw;
    // CFFT_EXEC_ORDER
    radix_loop<V, EMAX, 9, WM>(buf, P, count, is, gs, s, twp, P.cnt[0]);
    radix_loop<V, EMAX, 7, WM>(buf, P, count, is, gs, s, twp, P.cnt[1]);
    radix_loop<V, EMAX, 5, WM>(buf, P, count, is, gs, s, twp, P.cnt[2]);
    radix_loop<V, EMAX, 3, WM>(buf, P, count, is, gs, s, twp, P.cnt[3]);
    radix_loop<V, EMAX, 16, WM>(buf, P, count, is, gs, s, twp, P.cnt[4]);
    radix_loop<V, EMAX, 8, WM>(buf, P, count, is, gs, s, twp, P.cnt[5]);
    radix_loop<V, EMAX, 4, WM>(buf, P, count, is, gs, s, twp, P.cnt[6]);
    radix_loop<V, EMAX, 2, WM>(buf, P, count, is, gs, s, twp, P.cnt[7]);
    if (WM == 1 || (WM == 2 && P.Gwarp > 0)) __syncthreads();
}
template <typename V, int EMAX>
__device__ __forceinline__ void run_subffts(V* buf, const SubPlan& P, int count, int is, int gs) {
    run_subffts<V, EMAX, 2>(buf, P, (const V*)P.tw, count, is, gs);
}

// block-wide FP64 complex sum (result valid in every thread)
__device__ __forceinline__ double2 block_sum(double2 v, double2* scratch) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    const int lane = opaque_tid() & 31, wid = opaque_tid() >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    double2 s = make_double2(0, 0);
    for (int i = 0; i < nw; i++) { s.x += scratch[i].x; s.y += scratch[i].y; }
    __syncthreads();
    return s;
}

// ------------------------------------------- n = 4096 held in registers
// 4096-point transforms on CTAs of 256 threads, 16 elements per thread,
// as 4096 = 16 x 256 and 256 = 16 x 16 (three radix-16 stages):
//   A: thread t takes x[t + 256 k] (k < 16; each k is one coalesced row of
//      the transform, copied from HBM by cp.async), DFT_16 over k, twiddle
//      w_4096^(t k1), stores Y[k1][t] to shared memory;
//   B: thread (t1, k1) = (t & 15, t >> 4) reads Y[k1][t1 + 16 t2], DFT_16
//      over t2, twiddle w_256^(t1 k2) = w_4096^(16 t1 k2), stores
//      Z[k1][k2][t1] at k1*273 + k2*17 + t1;
//   C: thread (k1, k2) = (t & 15, t >> 4) reads Z[k1][k2][t1], DFT_16 over
//      t1 and stores X[k1 + 16 k2 + 256 k3] = X[t + 256 k3] straight to HBM.
// Two shared-memory exchanges replace the generic path's three in-place
// passes.  Every shared access is conflict-free: 16-byte
// accesses are served a quarter-warp and 8-byte ones a half-warp at a time,
// and within one of those groups the addresses run with stride 1 or 273
// (odd), so they fall in distinct bank groups.  The FP64 two-level twiddle
// table (w_4096^e = lo[e & 63] hi[e >> 6]) is staged in shared memory, lo
// entry l at l ^ (l >> 3): the exponents t k1 and 16 t1 k2 of a quarter-warp
// step by multiples of 2, 8 or 16, which in natural order land in the same
// bank group.
constexpr int R4096_PB = 17, R4096_PL = 273;
__device__ __forceinline__ double2 r4096_w(const double2* lo, const double2* hi, unsigned e) {
    const unsigned l = e & 63;
    return cmul(lo[l ^ (l >> 3)], hi[e >> 6]);
}
// dst[k stride] = v[k] w_4096^(e0 k), k < 16 (e0 k < 4096): the FP64 powers
// w^(e0 k) = w^(e0 (k-1)) w^e0 of one two-level table value, each rounded
// once to V.  The FP64 power's relative error stays below ~4e-15.  Against
// a table lookup per twiddle the FP64 work is the same (one complex product
// per twiddle) and 28 of 30 shared-memory table reads per thread and stage
// go: measured on B200, 4096-point ComplexF64 0.446 -> 0.376 ms per GiB,
// 1024 x 10007 (Rader) 0.516 -> 0.453 ms, 4096 x 2^16 ComplexF32 2.97 ->
// 2.52 ms (the table reads were most of the shared-memory wavefronts).
template <typename V>
__device__ __forceinline__ void r4096_tw_store(V (&v)[16], V* dst, int stride, const double2* lo,
                                               const double2* hi, unsigned e0) {
    const double2 b = r4096_w(lo, hi, e0);
    double2 w = b;
    dst[0] = v[0];
#pragma unroll
    for (int k = 1; k < 16; k++) {
        dst[k * stride] = cmul(v[k], fromd<V>(w));
        if (k < 15) w = cmul(w, b);
    }
}
// 4096-point DFT of the registers: thread t holds x[t + 256 k] in v[k] and
// gets X[t + 256 k3] in v[k3].  buf (16 planes of R4096_PL elements) must be
// free on entry; on return every thread has finished reading it.
template <typename V>
__device__ __forceinline__ void fft4096_regs(V (&v)[16], V* buf, const double2* tlo, const double2* thi, int t) {
    dft<16>(v);
    r4096_tw_store(v, buf + t, 256, tlo, thi, (unsigned)t);
    __syncthreads();
    {
        const int t1 = t & 15, k1 = t >> 4;
#pragma unroll
        for (int t2 = 0; t2 < 16; t2++) v[t2] = buf[k1 * 256 + t1 + 16 * t2];
        dft<16>(v);
        __syncthreads();                        // every Y read before Z overwrites it
        r4096_tw_store(v, buf + k1 * R4096_PL + t1, R4096_PB, tlo, thi, (unsigned)(16 * t1));
    }
    __syncthreads();
    {
        const int k1 = t & 15, k2 = t >> 4;
#pragma unroll
        for (int t1 = 0; t1 < 16; t1++) v[t1] = buf[k1 * R4096_PL + k2 * R4096_PB + t1];
    }
    __syncthreads();                            // every Z read: the buffer is free
    dft<16>(v);
}

// Persistent: CTA g transforms g, g + gridDim.x, ...  A thread's input
// elements x[t + 256 k] are copied by cp.async to buf[t + 256 k], exactly
// where the same thread later reads them and writes its Y values, so the
// input needs no block barrier.  The next transform's input is issued as soon
// as every thread has read Z (the buffer is free), and lands while stage C
// computes and stores and while the co-resident CTA works.
//
// P2A = true: the first pass of a power-of-two length n = N1 x 4096
// (N1 = 2^p.PA).  Row b is transform b >> PA, i = b & (N1 - 1): the stride-N1
// subsequence x[i + N1 c], c < 4096 (its 16-byte reads share 32-byte sectors
// with the neighbouring rows, which the L2 serves from one DRAM fetch).  Its
// 4096-point DFT is written unscaled as row b of the intermediate
// (contiguous, at b * out_dist); the column pass applies the four-step
// twiddle and finishes.
// Load modes: R4096_PLAIN (cp.async of contiguous transforms), R4096_P2A
// (cp.async of the stride-N1 subsequences), R4096_P2A_TMA (the same
// subsequences as 16 tensor copies of 256 elements each, issued by one
// thread and completing on an mbarrier: the strided gather leaves the
// load/store queue free; ComplexF64 only, whose 16-byte elements are one
// aligned box column of the tensor map)
enum { R4096_PLAIN = 0, R4096_P2A = 1, R4096_P2A_TMA = 2 };
template <typename V, int MODE>
__device__ __forceinline__ void r4096_prefetch(const KParams& p, V* buf, int b, int t, const CUtensorMap* tm,
                                               uint64_t* bar) {
    if (MODE == R4096_P2A_TMA) {
        if (t == 0) {
            const int sh = p.PA;
            const int tt = b >> sh, i = b & ((1 << sh) - 1);
            mbar_expect_tx(bar, 4096 * (unsigned)sizeof(V));
#pragma unroll
            for (int k = 0; k < 16; k++) tma_load_3d(buf + 256 * k, tm, bar, 2 * i, 256 * k, tt);
        }
    } else if (MODE == R4096_P2A) {
        const int sh = p.PA;
        const V* in = (const V*)p.in + (long long)(b >> sh) * p.in_dist + (b & ((1 << sh) - 1)) + (t << sh);
        const long long step = 256LL << sh;
        // a rolled loop: 16 precomputed strided addresses would stay live
        // across the last stage and push the FP64 codelets into spills
#pragma unroll 1
        for (int k = 0; k < 16; k++, in += step) cp_async_elem(buf + t + 256 * k, in);
    } else {
        const V* in = (const V*)p.in + (long long)b * p.in_dist;
#pragma unroll
        for (int k = 0; k < 16; k++) cp_async_elem(buf + t + 256 * k, in + t + 256 * k);
    }
}
template <typename V, int MODE = R4096_PLAIN>
__device__ __forceinline__ void r4096_body(const KParams& p, unsigned char* smem, const CUtensorMap* tm = nullptr) {
    constexpr bool P2A = MODE != R4096_PLAIN;
    constexpr bool TMA = MODE == R4096_P2A_TMA;
    V* buf = (V*)smem;                          // 16 planes of R4096_PL elements
    double2* tlo = after16(buf + 16 * R4096_PL);
    double2* thi = tlo + 64;
    uint64_t* bar = (uint64_t*)(thi + 65);
    int b = block_id(p);
    if (b >= p.batch) return;                   // uniform across the CTA
    {
        const int t = opaque_tid();
        if (TMA && t == 0) mbar_init(bar, 1);
        if (t < 64) tlo[t ^ (t >> 3)] = p.t4.lo[t];
        if (t < 65) thi[t] = p.t4.hi[t];
        if (TMA) __syncthreads();               // the barrier is initialised
        r4096_prefetch<V, MODE>(p, buf, b, t, tm, bar);
        if (!TMA) cp_async_commit();
    }
    __syncthreads();                            // tables staged
    unsigned phase = 0;
    for (; b < p.batch; b += gridDim.x) {
        // re-read per transform: index math hoisted out of the loop would
        // stay live across it and push the FP64 codelets into spills
        const int t = opaque_tid();
        V v[16];
        bool ok = true;
        if (TMA) {
            ok = mbar_wait(bar, phase);         // the row's tensor copies have landed
            phase ^= 1;
        } else {
            cp_async_wait_all();                // this thread's own input elements
        }
#pragma unroll
        for (int k = 0; k < 16; k++) v[k] = load_in(p, buf[t + 256 * k]);
        dft<16>(v);
        r4096_tw_store(v, buf + t, 256, tlo, thi, (unsigned)t);
        if (TMA) {
            // every thread leaves together when a copy timed out
            if (__syncthreads_or(!ok)) {
                if (t == 0) record_fault(kFaultTmaTimeout);
                return;
            }
        } else {
            __syncthreads();
        }
        {
            const int t1 = t & 15, k1 = t >> 4;
#pragma unroll
            for (int t2 = 0; t2 < 16; t2++) v[t2] = buf[k1 * 256 + t1 + 16 * t2];
            dft<16>(v);
            __syncthreads();                    // every Y read before Z overwrites it
            r4096_tw_store(v, buf + k1 * R4096_PL + t1, R4096_PB, tlo, thi, (unsigned)(16 * t1));
        }
        __syncthreads();
        {
            const int k1 = t & 15, k2 = t >> 4;
#pragma unroll
            for (int t1 = 0; t1 < 16; t1++) v[t1] = buf[k1 * R4096_PL + k2 * R4096_PB + t1];
        }
        __syncthreads();                        // every Z read: the buffer is free
        const int bn = b + (int)gridDim.x;
        if (TMA) {
            if (t == 0 && bn < p.batch) {
                fence_proxy_async_smem();       // the reads above precede the copies' writes
                r4096_prefetch<V, MODE>(p, buf, bn, t, tm, bar);
            }
        } else {
            if (bn < p.batch) r4096_prefetch<V, MODE>(p, buf, bn, t, tm, bar);
            cp_async_commit();
        }
        dft<16>(v);
        V* out = (V*)p.out + (long long)b * p.out_dist;
        if (P2A) {
#pragma unroll
            for (int k3 = 0; k3 < 16; k3++) out[t + 256 * k3] = v[k3];
        } else {
#pragma unroll
            for (int k3 = 0; k3 < 16; k3++) stg_stream(out + t + 256 * k3, store_out(p, v[k3]));
        }
    }
}

// ---------------------------------------------------------------- ROWS mode
// smem: buf[V][PC] (+ for Rader: xs[V][XP]) + reduction scratch
template <typename V, int EMAX>
__device__ __forceinline__ void rows_body(const KParams& p, unsigned char* smem) {
    const int T = blockDim.x, tid = opaque_tid();
    V* buf = (V*)smem;
    V* xs = buf + (size_t)p.V * p.PC;
    const int t0 = block_id(p) * p.V;
    const int nrows = min(p.V, p.batch - t0);
    if (nrows <= 0) return;
    const int nx = p.nx, M = p.M;

    if (p.conv == CONV_NONE) {
        if (p.in_fmt == IO_PLAIN) {
            const V* in = (const V*)p.in + (long long)t0 * p.in_dist;
            for (int idx = tid; idx < nrows * nx; idx += T) {
                const int r = fdiv(idx, p.mX), i = idx - r * nx;
                buf[r * p.PC + i] = load_in(p, ldg_stream(in + (long long)r * p.in_dist + i));
            }
        } else {
            for (int idx = tid; idx < nrows * nx; idx += T) {
                const int r = fdiv(idx, p.mX), i = idx - r * nx;
                buf[r * p.PC + i] = load_in(p, user_ld<V>(p, t0 + r, i));
            }
        }
        __syncthreads();
        run_subffts<V, EMAX>(buf, p.pc, nrows, 1, p.PC);
        if (p.out_fmt == IO_PLAIN) {
            V* out = (V*)p.out + (long long)t0 * p.out_dist;
            for (int idx = tid; idx < nrows * nx; idx += T) {
                const int r = fdiv(idx, p.mX), i = idx - r * nx;
                stg_stream(out + (long long)r * p.out_dist + i, store_out(p, buf[r * p.PC + i]));
            }
        } else {
            for (int idx = tid; idx < nrows * nx; idx += T) {
                const int r = fdiv(idx, p.mX), i = idx - r * nx;
                user_st(p, t0 + r, i, store_out(p, buf[r * p.PC + i]));
            }
        }
        return;
    }

    if (p.conv == CONV_RADER) {
        for (int idx = tid; idx < nrows * nx; idx += T) {
            const int r = fdiv(idx, p.mX), i = idx - r * nx;
            xs[r * p.XP + i] = load_in(p, user_ld<V>(p, t0 + r, i));
        }
        __syncthreads();
        const int L = nx - 1;
        for (int idx = tid; idx < nrows * M; idx += T) {
            const int r = fdiv(idx, p.mM), j = idx - r * M;
            buf[r * p.PC + j] = (j < L) ? xs[r * p.XP + __ldg(p.perm + j)] : zero<V>();
        }
    } else {
        for (int idx = tid; idx < nrows * M; idx += T) {
            const int r = fdiv(idx, p.mM), j = idx - r * M;
            V v = zero<V>();
            if (j < nx) {
                V x = load_in(p, user_ld<V>(p, t0 + r, j));
                v = fromd<V>(cmul(tod(x), __ldg(p.chirp + j)));
            }
            buf[r * p.PC + j] = v;
        }
    }
    __syncthreads();
    run_subffts<V, EMAX>(buf, p.pc, nrows, 1, p.PC);
    for (int idx = tid; idx < nrows * M; idx += T) {
        const int r = fdiv(idx, p.mM), k = idx - r * M;
        V* e = buf + r * p.PC + k;
        *e = conjv(fromd<V>(cmul(tod(*e), __ldg(p.spec + k))));
    }
    __syncthreads();
    run_subffts<V, EMAX>(buf, p.pc, nrows, 1, p.PC);

    if (p.conv == CONV_RADER) {
        const int L = nx - 1;
        // y[g^-j] = x0 + c[j]  (prime.jl:76-78), written into the staging rows
        for (int idx = tid; idx < nrows * L; idx += T) {
            const int r = fdiv(idx, p.mL), j = idx - r * L;
            const V x0 = xs[r * p.XP];
            const V c = conjv(buf[r * p.PC + j]);
            buf[r * p.PC + j] = mk<V>(x0.x + c.x, x0.y + c.y);  // park result in place
        }
        __syncthreads();
        // y0 = x0 + sum(x[1:]) per row, reduced in FP64
        double2* red = after16(xs + (size_t)p.V * p.XP);
        for (int r = 0; r < nrows; r++) {
            double2 acc = make_double2(0, 0);
            for (int i = 1 + tid; i < nx; i += T) {
                double2 d = tod(xs[r * p.XP + i]);
                acc.x += d.x; acc.y += d.y;
            }
            double2 s = block_sum(acc, red);
            if (tid == 0) {
                double2 x0 = tod(xs[r * p.XP]);
                xs[r * p.XP] = fromd<V>(make_double2(x0.x + s.x, x0.y + s.y));
            }
        }
        __syncthreads();
        for (int idx = tid; idx < nrows * L; idx += T) {
            const int r = fdiv(idx, p.mL), j = idx - r * L;
            xs[r * p.XP + __ldg(p.iperm + j)] = buf[r * p.PC + j];
        }
        __syncthreads();
        for (int idx = tid; idx < nrows * nx; idx += T) {
            const int r = fdiv(idx, p.mX), i = idx - r * nx;
            user_st(p, t0 + r, i, store_out(p, xs[r * p.XP + i]));
        }
    } else {
        for (int idx = tid; idx < nrows * nx; idx += T) {
            const int r = fdiv(idx, p.mX), k = idx - r * nx;
            const V c = conjv(buf[r * p.PC + k]);
            const V y = fromd<V>(cmul(tod(c), __ldg(p.chirp + k)));
            user_st(p, t0 + r, k, store_out(p, y));
        }
    }
}

// ---------------------------------------------------------------- FOUR mode
// Column layout (step A): (i1, j) at i1*PA + j, j < W = N2/C
// Row layout    (step C): (r, i2) at r*PC + i2, r < N1/C
//
// The body is written once against a shape policy K: DynK<WM> reads the shape
// from KParams (any size the planner picks; WM = 1 when both sub-plans run
// warp-synchronous, 0 when both run block-wide), StatK<...> fixes it at
// compile time for the hot sizes so strides, counts and divisions fold to
// constants.
template <int WM> struct DynK {
    static constexpr bool kSingle = false;     // separate column and row buffers
    static constexpr int kNEf = 1, kNEi = 1;
    __device__ static int N1(const KParams& p) { return p.N1; }
    __device__ static int N2(const KParams& p) { return p.N2; }
    __device__ static int C(const KParams& p) { return p.C; }
    __device__ static int PA(const KParams& p) { return p.PA; }
    __device__ static int PC(const KParams& p) { return p.PC; }
    __device__ static int W(const KParams& p) { return p.N2 / p.C; }
    __device__ static int R1(const KParams& p) { return p.N1 / p.C; }
    __device__ static int dW(const KParams& p, unsigned x) { return fdiv(x, p.mW); }
    __device__ static int dN2(const KParams& p, unsigned x) { return fdiv(x, p.mN2); }
    __device__ static int dR1(const KParams& p, unsigned x) { return fdiv(x, p.mR1); }
    template <typename V, int EMAX> __device__ __forceinline__ static void colA(V* buf, const KParams& p, const V* tw) {
        run_subffts<V, EMAX, WM>(buf, p.pa, tw, p.N2 / p.C, p.PA, 1);
    }
    template <typename V, int EMAX> __device__ __forceinline__ static void rowC(V* buf, const KParams& p, const V* tw) {
        run_subffts<V, EMAX, WM>(buf, p.pc, tw, p.N1 / p.C, 1, p.PC);
    }
};

// compile-time radix sequence (canonical order) and its pass chain
template <int... R> struct Seq {};
template <typename V, int EMAX, bool WARP, int L, int IS, int GS, int COUNT, int GW, int S, int OFF,
          int R, int... Rest>
__device__ __forceinline__ void st_passes(V* buf, const V* tw0) {
    // every butterfly of a wave must have a thread slot: EMAX / R per thread
    static_assert(GW * (L / R) <= (WARP ? 32 : 256) * (EMAX / R),
                  "a static pass has more butterflies than its team has slots");
    const V* tw = tw0 + OFF;
    if constexpr (WARP) {
        const int nw = blockDim.x >> 5, wid = opaque_tid() >> 5;
        for (int g0 = wid * GW; g0 < COUNT; g0 += nw * GW) {
            if constexpr (COUNT % GW == 0)
                spass<V, EMAX, R, true>(buf + g0 * GS, L, GW, IS, GS, S, tw);
            else
                spass<V, EMAX, R, true>(buf + g0 * GS, L, min(GW, COUNT - g0), IS, GS, S, tw);
        }
    } else {
#pragma unroll
        for (int g0 = 0; g0 < COUNT; g0 += GW)
            spass<V, EMAX, R, false>(buf + g0 * GS, L, (COUNT - g0 < GW) ? COUNT - g0 : GW, IS, GS, S, tw);
    }
    if constexpr (sizeof...(Rest) > 0)
        st_passes<V, EMAX, WARP, L, IS, GS, COUNT, GW, S * R, OFF + (R - 1) * (L / (S * R)), Rest...>(buf,
                                                                                                     tw0);
}
template <typename V, int EMAX, bool WARP, int L, int IS, int GS, int COUNT, int GW, int... R>
__device__ __forceinline__ void st_subffts(V* buf, const V* tw, Seq<R...>) {
    st_passes<V, EMAX, WARP, L, IS, GS, COUNT, GW, 1, 0, R...>(buf, tw);
    if constexpr (WARP) __syncthreads();
}

// SB: one shared buffer for both layouts; the exchange stages each thread's
// share in registers between two cluster barriers (FOUR kernels run 256
// threads, so a thread holds ceil(elements / 256) of them)
template <int N1_, int N2_, int C_, class SA, bool WA, int GA, class SC, bool WC, int GC, bool SB = false>
struct StatK {
    static constexpr bool kSingle = SB;
    static constexpr int kNEf = (N1_ * (N2_ / C_) + 255) / 256;
    static constexpr int kNEi = ((N1_ / C_) * N2_ + 255) / 256;
    static constexpr int kW = N2_ / C_, kR1 = N1_ / C_;
    static constexpr int kPC = N2_ + ((N2_ % 2 == 0) ? 1 : 0);
    static constexpr int kPA = (C_ == 1) ? kPC : kW;
    __device__ static constexpr int N1(const KParams&) { return N1_; }
    __device__ static constexpr int N2(const KParams&) { return N2_; }
    __device__ static constexpr int C(const KParams&) { return C_; }
    __device__ static constexpr int PA(const KParams&) { return kPA; }
    __device__ static constexpr int PC(const KParams&) { return kPC; }
    __device__ static constexpr int W(const KParams&) { return kW; }
    __device__ static constexpr int R1(const KParams&) { return kR1; }
    __device__ static int dW(const KParams&, unsigned x) { return (int)(x / (unsigned)kW); }
    __device__ static int dN2(const KParams&, unsigned x) { return (int)(x / (unsigned)N2_); }
    __device__ static int dR1(const KParams&, unsigned x) { return (int)(x / (unsigned)kR1); }
    template <typename V, int EMAX> __device__ __forceinline__ static void colA(V* buf, const KParams&, const V* tw) {
        st_subffts<V, EMAX, WA, N1_, kPA, 1, kW, GA>(buf, tw, SA{});
    }
    template <typename V, int EMAX> __device__ __forceinline__ static void rowC(V* buf, const KParams&, const V* tw) {
        st_subffts<V, EMAX, WC, N2_, 1, kPC, kR1, GC>(buf, tw, SC{});
    }
};

// Exchanges between the column and row layouts, push style: every CTA
// multiplies its own elements by the four-step twiddle and stores them into
// the owning peer's buffer through distributed shared memory (stores do not
// wait for a reply), then one cluster barrier publishes them.  The target
// buffers are idle: bufC is first read after this barrier, and bufA is
// written back only after the forward exchange's barrier, by which time
// every CTA has finished reading its own bufA.
template <typename V, class K>
__device__ __forceinline__ void four_push_fwd(const KParams& p, const V* bufA, V* bufC,
                                              cg::cluster_group& cl, unsigned c, const TwoLevel& t4) {
    // (k1, j) of this CTA's columns -> CTA k1/R1, row k1 % R1, column i2 = c*W + j
    const int W = K::W(p), R1 = K::R1(p), PA = K::PA(p), PC = K::PC(p);
    const int T = blockDim.x, tid = opaque_tid();
    const int total = K::N1(p) * W;
    for (int idx = tid; idx < total; idx += T) {
        const int k1 = K::dW(p, idx), j = idx - k1 * W;
        const int i2 = c * W + j, d = K::dR1(p, k1);
        V* dst = cl.map_shared_rank(bufC, d);
        dst[(k1 - d * R1) * PC + i2] = apply_tw(bufA[k1 * PA + j], t4, (unsigned)(i2 * k1));
    }
    cl.sync();
}
template <typename V, class K>
__device__ __forceinline__ void four_push_inv(const KParams& p, V* bufA, const V* bufC,
                                              cg::cluster_group& cl, unsigned c, const TwoLevel& t4) {
    // (r, i2) of this CTA's rows (k1 = c*R1 + r) -> CTA i2/W, column i2 % W, row k1
    const int W = K::W(p), R1 = K::R1(p), N2 = K::N2(p), PA = K::PA(p), PC = K::PC(p);
    const int T = blockDim.x, tid = opaque_tid();
    const int total = R1 * N2;
    for (int idx = tid; idx < total; idx += T) {
        const int r = K::dN2(p, idx), i2 = idx - r * N2;
        const int k1 = c * R1 + r, d = K::dW(p, i2);
        V* dst = cl.map_shared_rank(bufA, d);
        dst[k1 * PA + (i2 - d * W)] = apply_tw(bufC[r * PC + i2], t4, (unsigned)(i2 * k1));
    }
    cl.sync();
}

// Single-buffer exchanges (K::kSingle): each thread reads its elements of the
// source layout, twiddled, into registers; a cluster barrier (every CTA has
// read its own buffer); remote stores into the owners' buffers in the target
// layout; a cluster barrier publishes them.  Halving the shared memory lets
// the hot shapes run on half as many, twice as large CTAs at two CTAs/SM.
template <typename V, class K>
__device__ __forceinline__ void four_push_fwd_sb(const KParams& p, V* buf, cg::cluster_group& cl,
                                                 unsigned c, const TwoLevel& t4) {
    constexpr int NE = K::kNEf;
    const int W = K::W(p), R1 = K::R1(p), PA = K::PA(p), PC = K::PC(p);
    const int tid = opaque_tid();
    const int total = K::N1(p) * W;
    V v[NE];
#pragma unroll
    for (int m = 0; m < NE; m++) {
        const int idx = tid + m * 256;
        if (idx < total) {
            const int k1 = K::dW(p, idx), j = idx - k1 * W;
            v[m] = apply_tw(buf[k1 * PA + j], t4, (unsigned)((c * W + j) * k1));
        }
    }
    cl.sync();
#pragma unroll
    for (int m = 0; m < NE; m++) {
        const int idx = tid + m * 256;
        if (idx < total) {
            const int k1 = K::dW(p, idx), j = idx - k1 * W;
            const int i2 = c * W + j, d = K::dR1(p, k1);
            V* dst = cl.map_shared_rank(buf, d);
            dst[(k1 - d * R1) * PC + i2] = v[m];
        }
    }
    cl.sync();
}
template <typename V, class K>
__device__ __forceinline__ void four_push_inv_sb(const KParams& p, V* buf, cg::cluster_group& cl,
                                                 unsigned c, const TwoLevel& t4) {
    constexpr int NE = K::kNEi;
    const int W = K::W(p), R1 = K::R1(p), N2 = K::N2(p), PA = K::PA(p), PC = K::PC(p);
    const int tid = opaque_tid();
    const int total = R1 * N2;
    V v[NE];
#pragma unroll
    for (int m = 0; m < NE; m++) {
        const int idx = tid + m * 256;
        if (idx < total) {
            const int r = K::dN2(p, idx), i2 = idx - r * N2;
            v[m] = apply_tw(buf[r * PC + i2], t4, (unsigned)(i2 * (c * R1 + r)));
        }
    }
    cl.sync();
#pragma unroll
    for (int m = 0; m < NE; m++) {
        const int idx = tid + m * 256;
        if (idx < total) {
            const int r = K::dN2(p, idx), i2 = idx - r * N2;
            const int k1 = c * R1 + r, d = K::dW(p, i2);
            V* dst = cl.map_shared_rank(buf, d);
            dst[k1 * PA + (i2 - d * W)] = v[m];
        }
    }
    cl.sync();
}

// single-CTA four-step: twiddle in place (PA == PC, same layout)
template <typename V, class K>
__device__ __forceinline__ void four_twiddle_local(const KParams& p, V* buf, const TwoLevel& t4) {
    const int T = blockDim.x, tid = opaque_tid();
    const int N2 = K::N2(p), total = K::N1(p) * N2;
    for (int idx = tid; idx < total; idx += T) {
        const int k1 = K::dN2(p, idx), i2 = idx - k1 * N2;
        V* e = buf + k1 * K::PA(p) + i2;
        *e = apply_tw(*e, t4, (unsigned)(i2 * k1));
    }
    __syncthreads();
}

// Shared-memory carve-up of a FOUR CTA (host and device agree on it):
//   twA[pa.twlen] twC[pc.twlen] (V)  t4lo[2^bits] t4hi[nhi] (FP64)  bufA[N1*PA]
//   bufC[R1*PC] (C > 1 only; C = 1 works in place)  xs[XP] (Rader)
//   red[48] (FP64, 16-byte aligned)
// One transform per cluster.  The CTA first issues cp.async copies of its
// input slice (they land in shared memory without passing through
// registers), stages the twiddle tables while those are in flight, then
// computes.  A persistent loop over transforms would let the next input
// stream in during compute, but any loop around this body makes the
// compiler keep per-thread index state live across it and the FP64
// codelets spill; two co-resident CTAs per SM provide the overlap instead.
template <typename V, class K>
__device__ __forceinline__ void four_prefetch(const KParams& p, V* dst, int t, unsigned c) {
    const int T = blockDim.x, tid = opaque_tid();
    if (p.conv == CONV_RADER) {
        const int XC = p.XP;                      // staging of this CTA's x chunk
        for (int i = tid; i < XC; i += T) {
            const int gi = c * XC + i;
            if (gi < p.nx) user_cp(p, dst + i, t, gi);
        }
    } else {
        const int N2 = K::N2(p), W = K::W(p), PA = K::PA(p), total = K::N1(p) * W;
        const int lim = (p.conv == CONV_BLUE) ? p.nx : 0x7fffffff;
        if (p.in_fmt == IO_PLAIN) {
            const V* in = (const V*)p.in + (long long)t * p.in_dist;
            for (int idx = tid; idx < total; idx += T) {
                const int i1 = K::dW(p, idx), j = idx - i1 * W;
                const int jj = i1 * N2 + c * W + j;
                if (jj < lim) cp_async_elem(dst + i1 * PA + j, in + jj);
            }
        } else {
            for (int idx = tid; idx < total; idx += T) {
                const int i1 = K::dW(p, idx), j = idx - i1 * W;
                const int jj = i1 * N2 + c * W + j;
                if (jj < lim) dst[i1 * PA + j] = user_ld<V>(p, t, jj);
            }
        }
    }
    cp_async_commit();
}

// One transform of the persistent FOUR loop.  The thread and CTA indices are
// re-read through volatile asm on every call: otherwise the compiler hoists
// every index expression derived from them out of the persistent loop and
// the values it keeps live across the body push the FP64 codelets into
// spills.
template <typename V, int EMAX, class K>
__device__ __forceinline__ void four_transform(const KParams& p, V* buf, V* bufC, V* nxt, V* xs, double2* red,
                                            const V* twA, const V* twC, const TwoLevel& t4, int t,
                                            int tn, unsigned c) {
    cg::cluster_group cl = cg::this_cluster();
    const int C = K::C(p);
    const int T = blockDim.x, tid = opaque_tid();
    const int N1 = K::N1(p), N2 = K::N2(p), W = K::W(p), R1 = K::R1(p), nx = p.nx;
    const int PA = K::PA(p), PC = K::PC(p);
    cp_async_wait_all();
    __syncthreads();

    // ---- prologue fix-ups on the arrived input (column layout)
    double2 xsum = make_double2(0, 0);
    V x0 = zero<V>();
    if (p.conv == CONV_NONE) {
        if (p.dir) {
#pragma unroll 4
            for (int idx = tid; idx < N1 * W; idx += T) {
                const int i1 = K::dW(p, idx), j = idx - i1 * W;
                V* e = buf + i1 * PA + j;
                *e = conjv(*e);
            }
        }
    } else if (p.conv == CONV_BLUE) {
#pragma unroll 4
        for (int idx = tid; idx < N1 * W; idx += T) {
            const int i1 = K::dW(p, idx), j = idx - i1 * W;
            const int jj = i1 * N2 + c * W + j;
            V* e = buf + i1 * PA + j;
            *e = (jj < nx) ? fromd<V>(cmul(tod(load_in(p, *e)), __ldg(p.chirp + jj))) : zero<V>();
        }
    } else {
        // x chunk staged at buf[0..XC): conj, sum x[1:], publish to xs
        const int XC = p.XP;
        double2 acc = make_double2(0, 0);
        for (int i = tid; i < XC; i += T) {
            const int gi = c * XC + i;
            V v = zero<V>();
            if (gi < nx) v = load_in(p, buf[i]);
            xs[i] = v;
            if (gi >= 1 && gi < nx) { double2 d = tod(v); acc.x += d.x; acc.y += d.y; }
        }
        double2 part = block_sum(acc, red);
        if (tid == 0) red[32 + c] = part;
        if (C > 1) cl.sync(); else __syncthreads();
        for (int q = 0; q < C; q++) {
            const double2* rr = (C > 1) ? cl.map_shared_rank(red, q) : red;
            xsum.x += rr[32 + q].x; xsum.y += rr[32 + q].y;
        }
        {
            const V* r0 = (C > 1) ? cl.map_shared_rank(xs, 0) : xs;
            x0 = r0[0];
        }
        // p.perm is in this kernel's order: entry c*N1*W + idx holds
        // (owner << 24 | offset) of x[g^jj] in the owners' x chunks, or -1 for
        // the zero padding (jj >= L)
        const int* pc = p.perm + c * (N1 * W);
#pragma unroll 4
        for (int idx = tid; idx < N1 * W; idx += T) {
            const int i1 = K::dW(p, idx), j = idx - i1 * W;
            const int code = __ldg(pc + idx);
            V v = zero<V>();
            if (code >= 0) {
                const V* rx = (C > 1) ? cl.map_shared_rank(xs, code >> 24) : xs;
                v = rx[code & 0xffffff];
            }
            buf[i1 * PA + j] = v;
        }
    }
    __syncthreads();
    // the idle buffer is free: nobody reads it any more (its last remote
    // reader passed the previous transform's exchange barrier)
    if (tn >= 0) four_prefetch<V, K>(p, nxt, tn, c);

    // ---- forward FFT_M: columns, twiddle + exchange, rows (buf = column layout)
    K::template colA<V, EMAX>(buf, p, twA);
    if constexpr (K::kSingle) four_push_fwd_sb<V, K>(p, buf, cl, c, t4);
    else if (C > 1) four_push_fwd<V, K>(p, buf, bufC, cl, c, t4);
    else four_twiddle_local<V, K>(p, buf, t4);
    K::template rowC<V, EMAX>(bufC, p, twC);

    if (p.conv == CONV_NONE) {
        // X[k1 + N1 k2] from row layout (r, k2), k1 = c*R1 + r
        if (p.out_fmt == IO_PLAIN) {
            V* out = (V*)p.out + (long long)t * p.out_dist;
#pragma unroll 4
            for (int idx = tid; idx < R1 * N2; idx += T) {
                const int k2 = K::dR1(p, idx), r = idx - k2 * R1;
                stg_stream(out + (long long)(c * R1 + r) + (long long)N1 * k2, store_out(p, bufC[r * PC + k2]));
            }
        } else {
            for (int idx = tid; idx < R1 * N2; idx += T) {
                const int k2 = K::dR1(p, idx), r = idx - k2 * R1;
                user_st(p, t, (long long)(c * R1 + r) + (long long)N1 * k2, store_out(p, bufC[r * PC + k2]));
            }
        }
        return;
    }

    // ---- pointwise multiply by spectrum/M and conjugate (inverse via conj)
#pragma unroll 4
    for (int idx = tid; idx < R1 * N2; idx += T) {
        const int r = K::dN2(p, idx), k2 = idx - r * N2;
        // spectrum stored row-major for the cluster kernels: entry (k1, k2)
        // at k1 N2 + k2, so this CTA's rows are contiguous
        V* e = bufC + r * PC + k2;
        *e = conjv(fromd<V>(cmul(tod(*e), __ldg(p.spec + (c * R1) * N2 + idx))));
    }
    __syncthreads();
    // ---- second FFT_M in transposed order: rows, twiddle + exchange, columns
    K::template rowC<V, EMAX>(bufC, p, twC);
    if constexpr (K::kSingle) four_push_inv_sb<V, K>(p, buf, cl, c, t4);
    else if (C > 1) four_push_inv<V, K>(p, buf, bufC, cl, c, t4);
    else four_twiddle_local<V, K>(p, buf, t4);
    K::template colA<V, EMAX>(buf, p, twA);
    // column layout now holds conj(c[j1*N2 + c*W + j])

    if (p.conv == CONV_BLUE) {
#pragma unroll 4
        for (int idx = tid; idx < N1 * W; idx += T) {
            const int j1 = K::dW(p, idx), j = idx - j1 * W;
            const int jj = j1 * N2 + c * W + j;
            if (jj < nx) {
                const V cv = conjv(buf[j1 * PA + j]);
                user_st(p, t, jj, store_out(p, fromd<V>(cmul(tod(cv), __ldg(p.chirp + jj)))));
            }
        }
        return;
    }

    // Rader epilogue: y[g^-j] = x0 + c[j]; y[0] = x0 + sum(x[1:])
    const int XC = p.XP;
    // xs was last read in the prologue (the gather and x0); the exchanges'
    // cluster barriers since then order those reads before these writes
    if (C == 1) __syncthreads();
    // p.iperm in this kernel's order, coded like p.perm: the owner and
    // offset of y[g^-jj] in the x chunks
    const int* ic = p.iperm + c * (N1 * W);
#pragma unroll 4
    for (int idx = tid; idx < N1 * W; idx += T) {
        const int j1 = K::dW(p, idx), j = idx - j1 * W;
        const int code = __ldg(ic + idx);
        if (code >= 0) {
            const V cv = conjv(buf[j1 * PA + j]);
            V* rx = (C > 1) ? cl.map_shared_rank(xs, code >> 24) : xs;
            rx[code & 0xffffff] = mk<V>(x0.x + cv.x, x0.y + cv.y);
        }
    }
    if (C > 1) cl.sync(); else __syncthreads();
    if (c == 0 && tid == 0) {
        double2 d = tod(x0);
        xs[0] = fromd<V>(make_double2(d.x + xsum.x, d.y + xsum.y));
    }
    __syncthreads();
    for (int i = tid; i < XC; i += T) {
        const int gi = c * XC + i;
        if (gi < nx) user_st(p, t, gi, store_out(p, xs[i]));
    }
    // xs is rewritten by the next transform's prologue only after a
    // cluster barrier, so no extra barrier is needed here
    __syncthreads();
}

template <typename V, int EMAX, class K>
__device__ __forceinline__ void four_body(const KParams& p, unsigned char* smem) {
    const int C = K::C(p);
    cg::cluster_group cl = cg::this_cluster();
    const unsigned c = (C > 1) ? cl.block_rank() : 0;
    const int t = block_id(p) / C;
    if (t >= p.batch) return;             // uniform across the cluster
    const int T = blockDim.x, tid = opaque_tid();
    const int N1 = K::N1(p), N2 = K::N2(p);
    const int nlo = 1 << p.t4.bits, nhi = (p.t4.N + nlo - 1) / nlo + 1;

    const int lA = p.pa.twlen, lC = p.pc.twlen;
    V* twA = (V*)smem;
    V* twC = twA + lA;
    double2* t4lo = after16(twC + lC);
    double2* t4hi = t4lo + nlo;
    V* buf = (V*)(t4hi + nhi);            // column layout (N1 x PA)
    // row layout (R1 x PC): its own buffer, or (single buffer) the same one
    V* bufC = (C > 1 && !K::kSingle) ? buf + N1 * K::PA(p) : buf;
    const int lay = (C > 1) ? (K::kSingle ? max(N1 * K::PA(p), K::R1(p) * K::PC(p))
                                          : N1 * K::PA(p) + K::R1(p) * K::PC(p))
                            : N1 * K::PA(p);
    V* xs = buf + lay;                    // Rader x chunk
    double2* red = after16(xs + p.XP);    // reduction scratch (32 + C entries)

    four_prefetch<V, K>(p, buf, t, c);
    // tables -> shared memory while the input is in flight
    for (int i = tid; i < lA; i += T) twA[i] = ((const V*)p.pa.tw)[i];
    for (int i = tid; i < lC; i += T) twC[i] = ((const V*)p.pc.tw)[i];
    for (int i = tid; i < nlo; i += T) t4lo[i] = p.t4.lo[i];
    for (int i = tid; i < nhi; i += T) t4hi[i] = p.t4.hi[i];
    TwoLevel t4 = p.t4;
    t4.lo = t4lo;
    t4.hi = t4hi;
    // no trailing cluster barrier: every path's last access to a peer's
    // shared memory (an exchange, the Rader scatter) is followed by one, so
    // no peer touches this CTA's shared memory after it returns
    four_transform<V, EMAX, K>(p, buf, bufC, nullptr, xs, red, twA, twC, t4, t, -1, c);
}

// ------------------------------------------------------- COLPASS / ROWPASS
// COLPASS: tile of V adjacent columns c0..c0+V of the N1 x N2 view of one
// transform; column FFTs; store the w^(i2 k1)-scaled result to scratch
// row-major.  ROWPASS: tile of V adjacent rows r0..r0+V of the scratch; row
// FFTs; store X[k1 + N1 k2] (natural order), optionally with the Bluestein
// epilogue.  A tile streams into shared memory with cp.async (all of its
// copies in flight at once); pre-multiplications (conjugation, chirp,
// spectrum) are applied in shared memory once it has arrived.  The
// sub-transform twiddle table is staged in shared memory when small.
template <typename V>
__device__ __forceinline__ void colpass_issue(const KParams& p, int tile, V* dst) {
    const int T = blockDim.x, tid = opaque_tid();
    const int tiles = p.N2 / p.V, t = tile / tiles, c0 = (tile - t * tiles) * p.V;
    const int N1 = p.N1, N2 = p.N2, Vw = p.V, PA = p.PA;
    const long long lim = (p.pre == PRE_CHIRP) ? (long long)p.nx : (1LL << 62);
    // the first ks Vw threads (ks = T / Vw) each take one column j of the
    // tile, rows i1 = k0, k0 + ks, ...: no per-element division; a warp
    // still reads runs of Vw consecutive elements of consecutive rows
    const int ks = T / Vw;
    if (tid >= ks * Vw) return;
    const int j = tid % Vw, k0 = tid / Vw;
    if (p.in_fmt == IO_PLAIN) {
        const V* in = (const V*)p.in + (long long)t * p.in_dist + c0 + j;
        for (int i1 = k0; i1 < N1; i1 += ks) {
            const long long jj = (long long)i1 * N2 + c0 + j;
            if (jj < lim) cp_async_elem(dst + i1 * PA + j, in + (long long)i1 * N2);
        }
    } else {
        for (int i1 = k0; i1 < N1; i1 += ks) {
            const long long jj = (long long)i1 * N2 + c0 + j;
            if (jj < lim) dst[i1 * PA + j] = user_ld<V>(p, t, jj);
        }
    }
}
// prologue on the arrived tile; returns whether it wrote (caller syncs)
template <typename V>
__device__ __forceinline__ bool colpass_fix(const KParams& p, int tile, V* buf) {
    if (p.pre == PRE_NONE && !p.dir) return false;
    const int T = blockDim.x, tid = opaque_tid();
    const int tiles = p.N2 / p.V, t = tile / tiles, c0 = (tile - t * tiles) * p.V;
    const int N1 = p.N1, N2 = p.N2, Vw = p.V, PA = p.PA;
    // one column per thread, as in colpass_issue (the caller synchronises)
    const int ks = T / Vw;
    if (tid >= ks * Vw) return true;
    const int j = tid % Vw;
#pragma unroll 4
    for (int i1 = tid / Vw; i1 < N1; i1 += ks) {
        const long long jj = (long long)i1 * N2 + c0 + j;
        V* e = buf + i1 * PA + j;
        if (p.pre == PRE_NONE) {
            *e = conjv(*e);
        } else if (p.pre == PRE_CHIRP) {
            *e = (jj < p.nx) ? fromd<V>(cmul(tod(load_in(p, *e)), __ldg(p.chirp + jj))) : zero<V>();
        } else {
            *e = conjv(fromd<V>(cmul(tod(*e), __ldg(p.spec + jj))));
        }
    }
    return true;
}
// column FFTs and the twiddled store; (c0 + j) * k1 < N2 * N1 = M, so the
// exponent needs no reduction
template <typename V, int EMAX>
__device__ __forceinline__ void colpass_finish(const KParams& p, int tile, V* buf, const V* tw,
                                               const TwoLevel& t4) {
    const int T = blockDim.x, tid = opaque_tid();
    const int tiles = p.N2 / p.V, t = tile / tiles, c0 = (tile - t * tiles) * p.V;
    V* out = (V*)p.out + (long long)t * p.out_dist;
    const int N1 = p.N1, N2 = p.N2, Vw = p.V, PA = p.PA;
    run_subffts<V, EMAX, 2>(buf, p.pa, tw, Vw, PA, 1);
    // the first ks Vw threads (ks = T / Vw; all of them when Vw divides T)
    // each keep one column: no per-element division, and the twiddles
    // w^(c k1), k1 = k0, k0 + ks, ..., are FP64 products with the step
    // w^(c ks), re-seeded from the table every 16 steps (the error stays near
    // 1e-15; the same FP64 work per element as a table product, a sixteenth
    // of its table reads)
    const int ks = T / Vw;
    if (tid < ks * Vw) {
        const int j = tid % Vw, k0 = tid / Vw;
        const unsigned c = (unsigned)(c0 + j);
        V* o = out + c0 + j;
        const double2 st = tw_two(t4, c * (unsigned)ks);
        double2 w = make_double2(1, 0);
        int i = 0;
#pragma unroll 4
        for (int k1 = k0; k1 < N1; k1 += ks, i++) {
            if ((i & 15) == 0) w = tw_two(t4, c * (unsigned)k1);
            o[(long long)k1 * N2] = cmul(buf[k1 * PA + j], fromd<V>(w));
            w = cmul(w, st);
        }
    }
}

template <typename V>
__device__ __forceinline__ void rowpass_issue(const KParams& p, int tile, V* dst) {
    const int T = blockDim.x, tid = opaque_tid();
    const int tiles = p.N1 / p.V, t = tile / tiles, r0 = (tile - t * tiles) * p.V;
    const int N2 = p.N2, PC = p.PC;
    const V* src = (const V*)p.in + (long long)t * p.in_dist + (long long)r0 * N2;
    for (int idx = tid; idx < p.V * N2; idx += T) {
        const int r = fdiv(idx, p.mN2), i2 = idx - r * N2;
        cp_async_elem(dst + r * PC + i2, src + idx);
    }
}
template <typename V, int EMAX>
__device__ __forceinline__ void rowpass_finish(const KParams& p, int tile, V* buf, const V* tw) {
    const int T = blockDim.x, tid = opaque_tid();
    const int tiles = p.N1 / p.V, t = tile / tiles, r0 = (tile - t * tiles) * p.V;
    V* out = (V*)p.out + (long long)t * p.out_dist;
    const int N1 = p.N1, N2 = p.N2, Vw = p.V, PC = p.PC;
    run_subffts<V, EMAX, 2>(buf, p.pc, tw, Vw, 1, PC);
    // the first ks Vw threads (ks = T / Vw) each store one row r of the
    // tile, k2 = k0, k0 + ks, ...: no per-element division; a warp still
    // writes runs of Vw consecutive outputs
    const int ks = T / Vw;
    if (tid >= ks * Vw) return;
    const int r = tid % Vw, k0 = tid / Vw;
    if (p.out_fmt != IO_PLAIN) {
        // the caller's strided or ComplexF16 layout (the last stage of a fused plan)
        for (int k2 = k0; k2 < N2; k2 += ks) {
            const long long k = (long long)(r0 + r) + (long long)N1 * k2;
            const V v = buf[r * PC + k2];
            if (p.post == POST_CHIRP) {
                if (k < p.nx) user_st(p, t, k, store_out(p, fromd<V>(cmul(tod(conjv(v)), __ldg(p.chirp + k)))));
            } else {
                user_st(p, t, k, store_out(p, v));
            }
        }
        return;
    }
#pragma unroll 4
    for (int k2 = k0; k2 < N2; k2 += ks) {
        const long long k = (long long)(r0 + r) + (long long)N1 * k2;
        V v = buf[r * PC + k2];
        if (p.post == POST_CHIRP) {
            if (k < p.nx) stg_stream(out + k, store_out(p, fromd<V>(cmul(tod(conjv(v)), __ldg(p.chirp + k)))));
        } else if (p.post == POST_RAW) {
            out[k] = v;                       // intermediate of a convolution
        } else {
            stg_stream(out + k, store_out(p, v));
        }
    }
}

// one tile per CTA
template <typename V, int EMAX>
__device__ __forceinline__ void colpass_body(const KParams& p, unsigned char* smem) {
    const int T = blockDim.x, tid = opaque_tid();
    const int tile = block_id(p);
    if (tile >= p.batch * (p.N2 / p.V)) return;
    const int lt = cfft_pass_tw_elems(p.pa.twlen, (int)sizeof(V));
    const int nt = cfft_pass_t4_elems(p.t4.bits, p.t4.N), nlo = 1 << p.t4.bits;
    V* tws = (V*)smem;
    double2* t4s = after16(tws + lt);
    V* buf = (V*)(t4s + nt);
    colpass_issue<V>(p, tile, buf);
    cp_async_commit();
    for (int i = tid; i < lt; i += T) tws[i] = ((const V*)p.pa.tw)[i];
    for (int i = tid; i < nt; i += T) t4s[i] = (i < nlo) ? p.t4.lo[i] : p.t4.hi[i - nlo];
    TwoLevel t4 = p.t4;
    if (nt) {
        t4.lo = t4s;
        t4.hi = t4s + nlo;
    }
    cp_async_wait_all();
    __syncthreads();
    if (colpass_fix<V>(p, tile, buf)) __syncthreads();
    colpass_finish<V, EMAX>(p, tile, buf, lt ? (const V*)tws : (const V*)p.pa.tw, t4);
}
template <typename V, int EMAX>
__device__ __forceinline__ void rowpass_body(const KParams& p, unsigned char* smem) {
    const int T = blockDim.x, tid = opaque_tid();
    const int tile = block_id(p);
    if (tile >= p.batch * (p.N1 / p.V)) return;
    const int lt = cfft_pass_tw_elems(p.pc.twlen, (int)sizeof(V));
    V* tws = (V*)smem;
    V* buf = tws + lt;
    rowpass_issue<V>(p, tile, buf);
    cp_async_commit();
    for (int i = tid; i < lt; i += T) tws[i] = ((const V*)p.pc.tw)[i];
    cp_async_wait_all();
    __syncthreads();
    rowpass_finish<V, EMAX>(p, tile, buf, lt ? (const V*)tws : (const V*)p.pc.tw);
}
