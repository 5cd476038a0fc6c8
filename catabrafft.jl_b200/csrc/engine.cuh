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
#include <cuda_runtime.h>
#include <stdint.h>

#include "codelets.cuh"

namespace cg = cooperative_groups;

#include "engine_types.h"

// ------------------------------------------------------------------ helpers
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

__device__ __forceinline__ double2 tw_two(const TwoLevel& t, unsigned e) {
    return cmul(__ldg(t.lo + (e & ((1u << t.bits) - 1))), __ldg(t.hi + (e >> t.bits)));
}
// multiply by the four-step twiddle, evaluated in FP64 and rounded once
__device__ __forceinline__ double2 apply_tw(double2 v, const TwoLevel& t, unsigned e) {
    return e ? cmul(v, tw_two(t, e)) : v;
}
__device__ __forceinline__ float2 apply_tw(float2 v, const TwoLevel& t, unsigned e) {
    return e ? fromd<float2>(cmul(tod(v), tw_two(t, e))) : v;
}

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

// ----------------------------------------------------- Stockham radix pass
// One pass over Gw sub-transforms of length L held in smem: element i of
// sub-transform g lives at buf[g*gs + i*is].  s = product of earlier radices.
template <typename V, int EMAX, int R>
__device__ __noinline__ void spass(V* __restrict__ buf, int L, int Gw, int is, int gs, int s,
                                      const V* __restrict__ tw) {
    constexpr int SL = EMAX / R;
    const int T = blockDim.x, tid = threadIdx.x;
    const int nb = L / R;
    const int W = Gw * nb;
    V v[SL][R];
    int off[SL], pp_[SL];
#pragma unroll
    for (int i = 0; i < SL; i++) {
        const int w = tid + i * T;
        off[i] = -1;
        if (w < W) {
            const int g = w % Gw, b = w / Gw;
            const int pp = b / s, q = b - pp * s;
            const V* src = buf + g * gs + (q + s * pp) * is;
#pragma unroll
            for (int k = 0; k < R; k++) v[i][k] = src[k * nb * is];
            off[i] = g * gs + (q + s * R * pp) * is;
            pp_[i] = pp;
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < SL; i++) {
        if (off[i] >= 0) {
            dft<R>(v[i]);
            const int pp = pp_[i];
            if (pp) {
#pragma unroll
                for (int j = 1; j < R; j++) v[i][j] = cmul(v[i][j], __ldg(tw + j * pp * s));
            }
            V* dst = buf + off[i];
#pragma unroll
            for (int j = 0; j < R; j++) dst[j * s * is] = v[i][j];
        }
    }
    __syncthreads();
}

// All passes of `count` sub-transforms, in waves of P.G.  Caller must have
// synchronised the block after writing buf; returns synchronised.
template <typename V, int EMAX>
__device__ __forceinline__ void run_subffts(V* buf, const SubPlan& P, int count, int is, int gs) {
    const V* tw = (const V*)P.tw;
    for (int g0 = 0; g0 < count; g0 += P.G) {
        const int Gw = min(P.G, count - g0);
        V* b = buf + g0 * gs;
        int s = 1;
        for (int q = 0; q < P.np; q++) {
            const int r = P.radix[q];
            switch (r) {
                case 2: spass<V, EMAX, 2>(b, P.L, Gw, is, gs, s, tw); break;
                case 3: spass<V, EMAX, 3>(b, P.L, Gw, is, gs, s, tw); break;
                case 4: spass<V, EMAX, 4>(b, P.L, Gw, is, gs, s, tw); break;
                case 5: spass<V, EMAX, 5>(b, P.L, Gw, is, gs, s, tw); break;
                case 7: spass<V, EMAX, 7>(b, P.L, Gw, is, gs, s, tw); break;
                case 8: spass<V, EMAX, 8>(b, P.L, Gw, is, gs, s, tw); break;
                case 9: spass<V, EMAX, 9>(b, P.L, Gw, is, gs, s, tw); break;
                case 16: spass<V, EMAX, 16>(b, P.L, Gw, is, gs, s, tw); break;
                default: break;
            }
            s *= r;
        }
    }
}

// block-wide FP64 complex sum (result valid in every thread)
__device__ __forceinline__ double2 block_sum(double2 v, double2* scratch) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    double2 s = make_double2(0, 0);
    for (int i = 0; i < nw; i++) { s.x += scratch[i].x; s.y += scratch[i].y; }
    __syncthreads();
    return s;
}

// ---------------------------------------------------------------- ROWS mode
// smem: buf[V][PC] (+ for Rader: xs[V][XP]) + reduction scratch
template <typename V, int EMAX>
__device__ __forceinline__ void rows_body(const KParams& p, unsigned char* smem) {
    const int T = blockDim.x, tid = threadIdx.x;
    V* buf = (V*)smem;
    V* xs = buf + (size_t)p.V * p.PC;
    const int t0 = blockIdx.x * p.V;
    const int nrows = min(p.V, p.batch - t0);
    if (nrows <= 0) return;
    const V* in = (const V*)p.in + (long long)t0 * p.in_dist;
    V* out = (V*)p.out + (long long)t0 * p.out_dist;
    const int nx = p.nx, M = p.M;

    if (p.conv == CONV_NONE) {
        for (int idx = tid; idx < nrows * nx; idx += T) {
            const int r = idx / nx, i = idx - r * nx;
            buf[r * p.PC + i] = load_in(p, ldg_stream(in + (long long)r * p.in_dist + i));
        }
        __syncthreads();
        run_subffts<V, EMAX>(buf, p.pc, nrows, 1, p.PC);
        for (int idx = tid; idx < nrows * nx; idx += T) {
            const int r = idx / nx, i = idx - r * nx;
            stg_stream(out + (long long)r * p.out_dist + i, store_out(p, buf[r * p.PC + i]));
        }
        return;
    }

    if (p.conv == CONV_RADER) {
        for (int idx = tid; idx < nrows * nx; idx += T) {
            const int r = idx / nx, i = idx - r * nx;
            xs[r * p.XP + i] = load_in(p, ldg_stream(in + (long long)r * p.in_dist + i));
        }
        __syncthreads();
        const int L = nx - 1;
        for (int idx = tid; idx < nrows * M; idx += T) {
            const int r = idx / M, j = idx - r * M;
            buf[r * p.PC + j] = (j < L) ? xs[r * p.XP + __ldg(p.perm + j)] : zero<V>();
        }
    } else {
        for (int idx = tid; idx < nrows * M; idx += T) {
            const int r = idx / M, j = idx - r * M;
            V v = zero<V>();
            if (j < nx) {
                V x = load_in(p, ldg_stream(in + (long long)r * p.in_dist + j));
                v = fromd<V>(cmul(tod(x), __ldg(p.chirp + j)));
            }
            buf[r * p.PC + j] = v;
        }
    }
    __syncthreads();
    run_subffts<V, EMAX>(buf, p.pc, nrows, 1, p.PC);
    for (int idx = tid; idx < nrows * M; idx += T) {
        const int r = idx / M, k = idx - r * M;
        V* e = buf + r * p.PC + k;
        *e = conjv(fromd<V>(cmul(tod(*e), __ldg(p.spec + k))));
    }
    __syncthreads();
    run_subffts<V, EMAX>(buf, p.pc, nrows, 1, p.PC);

    if (p.conv == CONV_RADER) {
        const int L = nx - 1;
        // y[g^-j] = x0 + c[j]  (prime.jl:76-78), written into the staging rows
        for (int idx = tid; idx < nrows * L; idx += T) {
            const int r = idx / L, j = idx - r * L;
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
            const int r = idx / L, j = idx - r * L;
            xs[r * p.XP + __ldg(p.iperm + j)] = buf[r * p.PC + j];
        }
        __syncthreads();
        for (int idx = tid; idx < nrows * nx; idx += T) {
            const int r = idx / nx, i = idx - r * nx;
            stg_stream(out + (long long)r * p.out_dist + i, store_out(p, xs[r * p.XP + i]));
        }
    } else {
        for (int idx = tid; idx < nrows * nx; idx += T) {
            const int r = idx / nx, k = idx - r * nx;
            const V c = conjv(buf[r * p.PC + k]);
            const V y = fromd<V>(cmul(tod(c), __ldg(p.chirp + k)));
            stg_stream(out + (long long)r * p.out_dist + k, store_out(p, y));
        }
    }
}

// ---------------------------------------------------------------- FOUR mode
// Column layout (step A): (i1, j) at i1*PA + j, j < W = N2/C
// Row layout    (step C): (r, i2) at r*PC + i2, r < N1/C
template <typename V, int EMAX>
__device__ __forceinline__ void four_exchange_fwd(const KParams& p, V* buf, cg::cluster_group& cl, unsigned c) {
    // row (r, i2) <- column buffer of CTA i2/W at (k1, i2 % W), times w^(i2 k1)
    const int C = p.C, W = p.N2 / C, R1 = p.N1 / C;
    const int T = blockDim.x, tid = threadIdx.x;
    const int total = R1 * p.N2;
    V v[EMAX];
    cl.sync();
#pragma unroll
    for (int i = 0; i < EMAX; i++) {
        const int idx = tid + i * T;
        if (idx < total) {
            const int r = idx / p.N2, i2 = idx - r * p.N2;
            const int k1 = c * R1 + r, owner = i2 / W;
            const V* rb = cl.map_shared_rank(buf, owner);
            v[i] = apply_tw(rb[k1 * p.PA + (i2 - owner * W)], p.t4, (unsigned)(i2 * k1));
        }
    }
    cl.sync();
#pragma unroll
    for (int i = 0; i < EMAX; i++) {
        const int idx = tid + i * T;
        if (idx < total) {
            const int r = idx / p.N2, i2 = idx - r * p.N2;
            buf[r * p.PC + i2] = v[i];
        }
    }
    __syncthreads();
}

template <typename V, int EMAX>
__device__ __forceinline__ void four_exchange_inv(const KParams& p, V* buf, cg::cluster_group& cl, unsigned c) {
    // column (k1, j) <- row buffer of CTA k1/R1 at (k1 % R1, c*W + j), times w^(i2 k1)
    const int C = p.C, W = p.N2 / C, R1 = p.N1 / C;
    const int T = blockDim.x, tid = threadIdx.x;
    const int total = p.N1 * W;
    V v[EMAX];
    cl.sync();
#pragma unroll
    for (int i = 0; i < EMAX; i++) {
        const int idx = tid + i * T;
        if (idx < total) {
            const int k1 = idx / W, j = idx - k1 * W;
            const int owner = k1 / R1, i2 = c * W + j;
            const V* rb = cl.map_shared_rank(buf, owner);
            v[i] = apply_tw(rb[(k1 - owner * R1) * p.PC + i2], p.t4, (unsigned)(i2 * k1));
        }
    }
    cl.sync();
#pragma unroll
    for (int i = 0; i < EMAX; i++) {
        const int idx = tid + i * T;
        if (idx < total) {
            const int k1 = idx / W, j = idx - k1 * W;
            buf[k1 * p.PA + j] = v[i];
        }
    }
    __syncthreads();
}

// single-CTA four-step: twiddle in place (PA == PC, same layout)
template <typename V>
__device__ __forceinline__ void four_twiddle_local(const KParams& p, V* buf) {
    const int T = blockDim.x, tid = threadIdx.x;
    for (int idx = tid; idx < p.M; idx += T) {
        const int k1 = idx / p.N2, i2 = idx - k1 * p.N2;
        V* e = buf + k1 * p.PA + i2;
        *e = apply_tw(*e, p.t4, (unsigned)(i2 * k1));
    }
    __syncthreads();
}

template <typename V, int EMAX>
__device__ __forceinline__ void four_body(const KParams& p, unsigned char* smem) {
    cg::cluster_group cl = cg::this_cluster();
    const int C = p.C;
    const unsigned c = (C > 1) ? cl.block_rank() : 0;
    const int t = blockIdx.x / C;
    if (t >= p.batch) return;             // uniform across the cluster
    const int T = blockDim.x, tid = threadIdx.x;
    const int N1 = p.N1, N2 = p.N2, W = N2 / C, R1 = N1 / C, M = p.M, nx = p.nx;
    const int bufsz = max(N1 * p.PA, R1 * p.PC);
    V* buf = (V*)smem;
    V* xs = buf + bufsz;                  // Rader x chunk (XP elements)
    double2* red = after16(xs + p.XP);    // reduction scratch (32 + C entries)
    const V* in = (const V*)p.in + (long long)t * p.in_dist;
    V* out = (V*)p.out + (long long)t * p.out_dist;

    // ---- prologue: column layout of the (padded) input
    double2 xsum = make_double2(0, 0);
    V x0 = zero<V>();
    if (p.conv == CONV_NONE) {
        for (int idx = tid; idx < N1 * W; idx += T) {
            const int i1 = idx / W, j = idx - i1 * W;
            buf[i1 * p.PA + j] = load_in(p, ldg_stream(in + (long long)i1 * N2 + c * W + j));
        }
    } else if (p.conv == CONV_BLUE) {
        for (int idx = tid; idx < N1 * W; idx += T) {
            const int i1 = idx / W, j = idx - i1 * W;
            const int jj = i1 * N2 + c * W + j;
            V v = zero<V>();
            if (jj < nx) v = fromd<V>(cmul(tod(load_in(p, ldg_stream(in + jj))), __ldg(p.chirp + jj)));
            buf[i1 * p.PA + j] = v;
        }
    } else {
        // stage x in distributed chunks, sum x[1:], gather a[j] = x[g^j]
        const int XC = p.XP;
        double2 acc = make_double2(0, 0);
        for (int i = tid; i < XC; i += T) {
            const int gi = c * XC + i;
            V v = zero<V>();
            if (gi < nx) v = load_in(p, ldg_stream(in + gi));
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
        const int L = nx - 1;
        for (int idx = tid; idx < N1 * W; idx += T) {
            const int i1 = idx / W, j = idx - i1 * W;
            const int jj = i1 * N2 + c * W + j;
            V v = zero<V>();
            if (jj < L) {
                const int src = __ldg(p.perm + jj), owner = src / XC;
                const V* rx = (C > 1) ? cl.map_shared_rank(xs, owner) : xs;
                v = rx[src - owner * XC];
            }
            buf[i1 * p.PA + j] = v;
        }
    }
    __syncthreads();

    // ---- forward FFT_M: columns, twiddle + exchange, rows
    run_subffts<V, EMAX>(buf, p.pa, W, p.PA, 1);
    if (C > 1) four_exchange_fwd<V, EMAX>(p, buf, cl, c);
    else four_twiddle_local(p, buf);
    run_subffts<V, EMAX>(buf, p.pc, R1, 1, p.PC);

    if (p.conv == CONV_NONE) {
        // X[k1 + N1 k2] from row layout (r, k2), k1 = c*R1 + r
        for (int idx = tid; idx < R1 * N2; idx += T) {
            const int k2 = idx / R1, r = idx - k2 * R1;
            stg_stream(out + (long long)(c * R1 + r) + (long long)N1 * k2,
                       store_out(p, buf[r * p.PC + k2]));
        }
        return;
    }

    // ---- pointwise multiply by spectrum/M and conjugate (inverse via conj)
    for (int idx = tid; idx < R1 * N2; idx += T) {
        const int r = idx / N2, k2 = idx - r * N2;
        const int k = (c * R1 + r) + N1 * k2;
        V* e = buf + r * p.PC + k2;
        *e = conjv(fromd<V>(cmul(tod(*e), __ldg(p.spec + k))));
    }
    __syncthreads();
    // ---- second FFT_M in transposed order: rows, twiddle + exchange, columns
    run_subffts<V, EMAX>(buf, p.pc, R1, 1, p.PC);
    if (C > 1) four_exchange_inv<V, EMAX>(p, buf, cl, c);
    else four_twiddle_local(p, buf);
    run_subffts<V, EMAX>(buf, p.pa, W, p.PA, 1);
    // column layout now holds conj(c[j1*N2 + c*W + j])

    if (p.conv == CONV_BLUE) {
        for (int idx = tid; idx < N1 * W; idx += T) {
            const int j1 = idx / W, j = idx - j1 * W;
            const int jj = j1 * N2 + c * W + j;
            if (jj < nx) {
                const V cv = conjv(buf[j1 * p.PA + j]);
                stg_stream(out + jj, store_out(p, fromd<V>(cmul(tod(cv), __ldg(p.chirp + jj)))));
            }
        }
        return;
    }

    // Rader epilogue: y[g^-j] = x0 + c[j]; y[0] = x0 + sum(x[1:])
    const int XC = p.XP, L = nx - 1;
    if (C > 1) cl.sync(); else __syncthreads();   // everyone done reading xs
    for (int idx = tid; idx < N1 * W; idx += T) {
        const int j1 = idx / W, j = idx - j1 * W;
        const int jj = j1 * N2 + c * W + j;
        if (jj < L) {
            const V cv = conjv(buf[j1 * p.PA + j]);
            const int dst = __ldg(p.iperm + jj), owner = dst / XC;
            V* rx = (C > 1) ? cl.map_shared_rank(xs, owner) : xs;
            rx[dst - owner * XC] = mk<V>(x0.x + cv.x, x0.y + cv.y);
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
        if (gi < nx) stg_stream(out + gi, store_out(p, xs[i]));
    }
    if (C > 1) cl.sync();                          // keep smem alive for peers
}

// ------------------------------------------------------- COLPASS / ROWPASS
// COLPASS: tile of V adjacent columns c0..c0+V of the N1 x N2 view of one
// transform; column FFTs; store w^(i2 k1)-scaled result to scratch row-major.
template <typename V, int EMAX>
__device__ __forceinline__ void colpass_body(const KParams& p, unsigned char* smem) {
    const int T = blockDim.x, tid = threadIdx.x;
    const int tiles = p.N2 / p.V;
    const int t = blockIdx.x / tiles, c0 = (blockIdx.x - t * tiles) * p.V;
    if (t >= p.batch) return;
    V* buf = (V*)smem;
    const V* in = (const V*)p.in + (long long)t * p.in_dist;
    V* out = (V*)p.out + (long long)t * p.out_dist;
    const int N1 = p.N1, N2 = p.N2, Vw = p.V;
    for (int idx = tid; idx < N1 * Vw; idx += T) {
        const int i1 = idx / Vw, j = idx - i1 * Vw;
        const long long jj = (long long)i1 * N2 + c0 + j;
        V v;
        if (p.pre == PRE_CHIRP) {
            v = zero<V>();
            if (jj < p.nx) v = fromd<V>(cmul(tod(load_in(p, ldg_stream(in + jj))), __ldg(p.chirp + jj)));
        } else if (p.pre == PRE_SPEC) {
            v = conjv(fromd<V>(cmul(tod(ldg_stream(in + jj)), __ldg(p.spec + jj))));
        } else {
            v = load_in(p, ldg_stream(in + jj));
        }
        buf[i1 * p.PA + j] = v;
    }
    __syncthreads();
    run_subffts<V, EMAX>(buf, p.pa, Vw, p.PA, 1);
    for (int idx = tid; idx < N1 * Vw; idx += T) {
        const int k1 = idx / Vw, j = idx - k1 * Vw;
        const unsigned e = (unsigned)((unsigned long long)(c0 + j) * k1 % (unsigned long long)p.M);
        out[(long long)k1 * N2 + c0 + j] = apply_tw(buf[k1 * p.PA + j], p.t4, e);
    }
}

// ROWPASS: tile of V adjacent rows r0..r0+V of the scratch; row FFTs; store
// X[k1 + N1 k2] (natural order), optionally with the Bluestein epilogue.
template <typename V, int EMAX>
__device__ __forceinline__ void rowpass_body(const KParams& p, unsigned char* smem) {
    const int T = blockDim.x, tid = threadIdx.x;
    const int tiles = p.N1 / p.V;
    const int t = blockIdx.x / tiles, r0 = (blockIdx.x - t * tiles) * p.V;
    if (t >= p.batch) return;
    V* buf = (V*)smem;
    const V* in = (const V*)p.in + (long long)t * p.in_dist;
    V* out = (V*)p.out + (long long)t * p.out_dist;
    const int N1 = p.N1, N2 = p.N2, Vw = p.V;
    for (int idx = tid; idx < Vw * N2; idx += T) {
        const int r = idx / N2, i2 = idx - r * N2;
        buf[r * p.PC + i2] = in[(long long)(r0 + r) * N2 + i2];
    }
    __syncthreads();
    run_subffts<V, EMAX>(buf, p.pc, Vw, 1, p.PC);
    for (int idx = tid; idx < Vw * N2; idx += T) {
        const int k2 = idx / Vw, r = idx - k2 * Vw;
        const long long k = (long long)(r0 + r) + (long long)N1 * k2;
        V v = buf[r * p.PC + k2];
        if (p.post == POST_CHIRP) {
            if (k < p.nx)
                stg_stream(out + k, store_out(p, fromd<V>(cmul(tod(conjv(v)), __ldg(p.chirp + k)))));
        } else if (p.post == POST_RAW) {
            out[k] = v;                       // intermediate of a convolution
        } else {
            stg_stream(out + k, store_out(p, v));
        }
    }
}
