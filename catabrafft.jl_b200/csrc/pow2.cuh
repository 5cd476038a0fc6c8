// pow2.cuh -- power-of-two lengths n = N1 x 4096 (N1 = 2 .. 1024) as two
// register passes.
//
// With x[i + N1 c] (i < N1, c < 4096) and X[q + 4096 r] (q < 4096, r < N1):
//   X[q + 4096 r] = sum_i w_N1^(i r) [ w_n^(i q) sum_c x[i + N1 c] w_4096^(c q) ]
// Pass A (r4096_body<V, true>): for every i, the 4096-point DFT of the
//   stride-N1 subsequence, written as row i of an intermediate Z (N1 x 4096
//   per transform, sized to stay in L2).
// Pass B (this file): for every column q of Z, the four-step twiddle
//   w_n^(i q) and the N1-point DFT over i, written to X[q + 4096 r] -- row r
//   of the output viewed as N1 x 4096, so a tile of adjacent columns stores
//   contiguous segments.  A thread's twiddles for one column q and rows
//   i0 + d m are w_n^(q i0) (w_n^(q d))^m: two lookups of the FP64 two-level
//   table and an FP64 recurrence of at most 15 products (relative error a
//   few 1e-15), rounded once to the data type.
// The strided accesses are reads (pass A), which the L2 merges; every store
// to HBM is a contiguous segment.  The reference's pass structure for these
// lengths is the layered radix-8 Stockham sequence
// (src/radix_2_codelets.jl:279-447); here each pass keeps 16 elements per
// thread in registers.
//
// A column tile of pass B is VC = 4096 / N1 adjacent columns (4096 elements,
// 16 per thread, 256 threads).  Element k of thread tid is staged by cp.async
// in shared-memory slot tid + 256 k, which is tile position (row, col) =
// (slot / VC, slot % VC): each thread's copies land where it reads them, so
// the input needs no block barrier, and the next tile can stream in as soon
// as the buffer is free (persistent CTAs).  Once a tile is in shared memory
// its intermediate lines are dropped from L2 without a write-back.
//
// The column DFT of length N1 = 16^A * RL (RL in {1, 2, 4, 8}) runs as
// decimation-in-frequency Stockham stages: stage s of radix r splits every
// current sub-transform of length Ls = N1 / 16^s as t = t' + (Ls / r) m,
// does DFT_r over m, multiplies by w_Ls^(t' k) and leaves sub-transform
// K + 16^s k of length Ls / r.  Between stages, element (K, t) of column j
// sits at ((K Ls + t) VC + j): lanes run over adjacent columns, so every
// shared access of a quarter-warp is 8 consecutive 16-byte slots when VC >= 8
// (ComplexF64) and 16 consecutive 8-byte slots when VC >= 16 (ComplexF32).
// The output index of a column is K + 16^(S-1) k of the last stage.
#pragma once
#include "engine.cuh"

__host__ __device__ constexpr int p2_log16(int n) { return (n >= 16 && n % 16 == 0) ? 1 + p2_log16(n / 16) : 0; }
__host__ __device__ constexpr int p2_pow16(int a) { return a == 0 ? 1 : 16 * p2_pow16(a - 1); }
__host__ __device__ constexpr int p2_log2(int n) { return n <= 1 ? 0 : 1 + p2_log2(n / 2); }

template <int N1_> struct P2Col {
    static constexpr int N1 = N1_;
    static constexpr int LGN1 = p2_log2(N1);
    static constexpr int VC = 4096 / N1;                  // columns per tile
    static constexpr int LGVC = p2_log2(VC);
    static constexpr int A = p2_log16(N1);                // radix-16 stages
    static constexpr int RL = N1 / p2_pow16(A);           // last radix, 1 = none
    static constexpr int S = A + (RL > 1 ? 1 : 0);        // stages
    static constexpr int TPC = N1 >= 16 ? N1 / 16 : 1;    // threads per column
    static constexpr int CPT = N1 >= 16 ? 1 : 16 / N1;    // columns per thread (N1 < 16)
    static constexpr bool kExchange = S > 1;              // stages talk through shared memory
    static_assert(N1 >= 2 && N1 <= 1024 && (N1 & (N1 - 1)) == 0, "N1 is a power of two in [2, 1024]");
    static_assert(N1 >= 16 || A == 0, "");
};

// w_n^e from the FP64 two-level table
__device__ __forceinline__ double2 p2_wn(const double2* lo, const double2* hi, int bits, unsigned e) {
    return cmul(lo[e & ((1u << bits) - 1)], hi[e >> bits]);
}
// x w_N1^e from the single-level FP64 table (exactly rounded, once to V)
template <typename V>
__device__ __forceinline__ V p2_tw_stage(V v, const double2* tw, unsigned e) {
    return e ? cmul(v, fromd<V>(tw[e])) : v;
}
// L2 lines of the intermediate that no one reads again are dropped without a
// write-back to HBM (their contents become undefined)
__device__ __forceinline__ void l2_discard_line(const void* p) {
    asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
}

template <typename V, class PC>
__device__ __forceinline__ void p2col_prefetch(const KParams& p, V* buf, int tile, int tid) {
    // tile -> transform tile / N1, first column (tile % N1) VC
    const int tt = tile >> PC::LGN1;
    const int c0 = (tile & (PC::N1 - 1)) * PC::VC;
    const V* in = (const V*)p.in + (long long)tt * p.in_dist + c0;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        const int slot = tid + 256 * k;
        cp_async_elem(buf + slot, in + ((slot >> PC::LGVC) << 12) + (slot & (PC::VC - 1)));
    }
}

// discard the tile's intermediate lines once every thread's copies of them
// have landed (caller synchronised): thread tid owns slots tid + 256 k; when
// a tile row spans whole 128-byte lines, the first thread of each line drops it
template <typename V, class PC>
__device__ __forceinline__ void p2col_discard(const KParams& p, int tile, int tid) {
    constexpr int EPL = 128 / (int)sizeof(V);
    if constexpr (PC::VC >= EPL) {
        if ((tid & (EPL - 1)) == 0) {
            const int tt = tile >> PC::LGN1;
            const int c0 = (tile & (PC::N1 - 1)) * PC::VC;
            const V* in = (const V*)p.in + (long long)tt * p.in_dist + c0;
#pragma unroll
            for (int k = 0; k < 16; k++) {
                const int slot = tid + 256 * k;
                l2_discard_line(in + ((slot >> PC::LGVC) << 12) + (slot & (PC::VC - 1)));
            }
        }
    }
}
// an output of the last stage: X[q + 4096 r] = row r, column q
template <typename V>
__device__ __forceinline__ void p2col_store(const KParams& p, V* out, int col, int r, V v) {
    stg_stream(out + ((long long)r << 12) + col, store_out(p, v));
}

// radix-r DFT of v[g r .. g r + r)
template <int R, typename V> __device__ __forceinline__ void p2_dft_group(V* v) {
    dft<R>(*reinterpret_cast<V(*)[R]>(v));
}

// stage s >= 1 of a column of N1 >= 32 (an exchange through shared memory)
template <typename V, class PC, int s, bool PF = true>
__device__ __forceinline__ void p2col_stage(const KParams& p, V* buf, const double2* tw, int tile) {
    constexpr int r = (s < PC::A) ? 16 : PC::RL;
    constexpr int Ls = PC::N1 / p2_pow16(s);
    constexpr int nb = Ls / r;
    constexpr int G = 16 / r;
    constexpr int KR = p2_pow16(s);
    constexpr bool last = (s == PC::S - 1);
    const int tid = opaque_tid();
    const int j = tid & (PC::VC - 1), b = tid >> PC::LGVC;
    V v[16];
#pragma unroll
    for (int g = 0; g < G; g++) {
        const int beta = b + PC::TPC * g;
        const int tp = beta & (nb - 1), K = beta / nb;
#pragma unroll
        for (int m = 0; m < r; m++) v[g * r + m] = buf[((K * Ls + tp + nb * m) << PC::LGVC) + j];
    }
    __syncthreads();                            // every read of this stage before the writes
    if (last && PF) {
        // the buffer is free: the next tile streams in while this one finishes
        const int tn = tile + (int)gridDim.x;
        if (tn < p.batch) p2col_prefetch<V, PC>(p, buf, tn, tid);
        cp_async_commit();
    }
#pragma unroll
    for (int g = 0; g < G; g++) p2_dft_group<r>(v + g * r);
    if (last) {
        const int tt = tile >> PC::LGN1;
        const int c = (tile & (PC::N1 - 1)) * PC::VC + j;
        V* out = (V*)p.out + (long long)tt * p.out_dist;
#pragma unroll
        for (int g = 0; g < G; g++) {
            const int K = b + PC::TPC * g;      // nb == 1
#pragma unroll
            for (int k = 0; k < r; k++) p2col_store(p, out, c, K + KR * k, v[g * r + k]);
        }
    } else {
#pragma unroll
        for (int g = 0; g < G; g++) {
            const int beta = b + PC::TPC * g;
            const int tp = beta & (nb - 1), K = beta / nb;
#pragma unroll
            for (int k = 0; k < r; k++) {
                const V w = p2_tw_stage(v[g * r + k], tw, (unsigned)(tp * k * (PC::N1 / Ls)));
                buf[(((K + KR * k) * nb + tp) << PC::LGVC) + j] = w;
            }
        }
        __syncthreads();
    }
}
template <typename V, class PC, int s, bool PF = true>
__device__ __forceinline__ void p2col_stages(const KParams& p, V* buf, const double2* tw, int tile) {
    if constexpr (s < PC::S) {
        p2col_stage<V, PC, s, PF>(p, buf, tw, tile);
        p2col_stages<V, PC, s + 1, PF>(p, buf, tw, tile);
    }
}

// Pass B body: p.in = the intermediate (N1 x 4096 per transform, at
// in_dist), p.out = the output (at out_dist), p.batch = tiles (transforms x
// N1), p.twN1 = w_N1^e for e < N1 (staged in shared memory after the tile),
// p.t4n = the two-level table of w_n (staged after it when p.pre != 0).
// Pass A conjugated the input of the inverse directions; the stores here
// conjugate and scale.
// Pass A for ComplexF32 by tensor copies.  The 8-byte elements are narrower
// than a tensor copy's 16-byte minimum box row, so a CTA item is the pair of
// neighbouring subsequences (i, i + 1), i even, of one transform: 16 copies
// of a box of 256 columns x 16 bytes bring both, side by side (64 KB), onto
// an mbarrier.  Each subsequence then runs the 4096-point register FFT
// through the exchange buffer and is written, unscaled, as its row 2 b + h
// of the intermediate (row = transform x N1 + i, as in R4096_P2A).  The next
// pair's copies are issued as soon as every thread has read the second
// subsequence.  (Per-element cp.async of the strided input writes shared
// memory one sector at a time: most of the ComplexF32 pass's shared-memory
// traffic.)  KParams as for R4096_P2A: batch = rows (even), PA = log2 N1.
constexpr int kP2PairBytes = 4096 * 16;
__device__ __forceinline__ void p2row_pair_issue(const KParams& p, float4* pair, const CUtensorMap* tm,
                                                 uint64_t* bar, int pb) {
    const int sh = p.PA - 1;                    // pairs per transform: N1 / 2
    const int tt = pb >> sh, i = (pb & ((1 << sh) - 1)) << 1;
    mbar_expect_tx(bar, kP2PairBytes);
#pragma unroll
    for (int k = 0; k < 16; k++) tma_load_3d(pair + 256 * k, tm, bar, 2 * i, 256 * k, tt);
}
__device__ __forceinline__ void p2row_pair_body(const KParams& p, unsigned char* smem, const CUtensorMap* tm) {
    float4* pair = (float4*)smem;
    float2* buf = (float2*)(smem + kP2PairBytes);  // 16 planes of R4096_PL elements
    double2* tlo = after16(buf + 16 * R4096_PL);
    double2* thi = tlo + 64;
    uint64_t* bar = (uint64_t*)(thi + 65);
    const int npairs = p.batch >> 1;
    int b = block_id(p);
    if (b >= npairs) return;                    // uniform across the CTA
    {
        const int t = opaque_tid();
        if (t == 0) mbar_init(bar, 1);
        if (t < 64) tlo[t ^ (t >> 3)] = p.t4.lo[t];
        if (t < 65) thi[t] = p.t4.hi[t];
        __syncthreads();                        // the barrier is initialised, the tables staged
        if (t == 0) p2row_pair_issue(p, pair, tm, bar, b);
    }
    unsigned phase = 0;
    for (; b < npairs; b += gridDim.x) {
        {
            const bool ok = mbar_wait(bar, phase);  // the pair's tensor copies have landed
            phase ^= 1;
            // every thread leaves together when a copy timed out
            if (__syncthreads_or(!ok)) {
                if (opaque_tid() == 0) record_fault(kFaultTmaTimeout);
                return;
            }
        }
#pragma unroll 1
        for (int h = 0; h < 2; h++) {
            const int t = opaque_tid();
            float2 v[16];
#pragma unroll
            for (int k = 0; k < 16; k++) {
                const float4 q = pair[t + 256 * k];
                v[k] = load_in(p, h ? make_float2(q.z, q.w) : make_float2(q.x, q.y));
            }
            if (h == 1) {
                __syncthreads();                // both subsequences read: the pair buffer is free
                const int bn = b + (int)gridDim.x;
                if (t == 0 && bn < npairs) {
                    fence_proxy_async_smem();   // the reads above precede the copies' writes
                    p2row_pair_issue(p, pair, tm, bar, bn);
                }
            }
            fft4096_regs(v, buf, tlo, thi, t);
            float2* out = (float2*)p.out + (long long)(2 * b + h) * p.out_dist;
#pragma unroll
            for (int k3 = 0; k3 < 16; k3++) out[t + 256 * k3] = v[k3];
        }
    }
}

template <typename V, int N1>
__device__ __forceinline__ void p2col_body(const KParams& p, unsigned char* smem) {
    using PC = P2Col<N1>;
    V* buf = (V*)smem;                          // 4096 elements
    double2* tw = after16(buf + 4096);          // N1 entries
    int tile = block_id(p);
    if (tile >= p.batch) return;                // uniform across the CTA
    const int bits = p.t4n.bits;
    const double2 *lo = p.t4n.lo, *hi = p.t4n.hi;
    {
        const int tid = opaque_tid();
        p2col_prefetch<V, PC>(p, buf, tile, tid);
        cp_async_commit();
        for (int i = tid; i < N1; i += 256) tw[i] = p.twN1[i];
        if (p.pre) {
            double2* ts = tw + N1;
            const int nlo = 1 << bits, nhi = (p.t4n.N + nlo - 1) / nlo + 1;
            for (int i = tid; i < nlo + nhi; i += 256) ts[i] = (i < nlo) ? p.t4n.lo[i] : p.t4n.hi[i - nlo];
            lo = ts;
            hi = ts + nlo;
        }
        __syncthreads();
    }
    for (; tile < p.batch; tile += gridDim.x) {
        const int tid = opaque_tid();
        V v[16];
        cp_async_wait_all();                    // this thread's own slots
#pragma unroll
        for (int k = 0; k < 16; k++) v[k] = buf[tid + 256 * k];
        const int tt = tile >> PC::LGN1;
        const int c0 = (tile & (N1 - 1)) * PC::VC;
        V* out = (V*)p.out + (long long)tt * p.out_dist;
        if constexpr (N1 <= 16) {
            // no exchange: once the warp's copies have landed (a discarded
            // line spans lanes of one warp) the next tile is issued into
            // these slots right away
            __syncwarp();
            p2col_discard<V, PC>(p, tile, tid);
            const int tn = tile + (int)gridDim.x;
            if (tn < p.batch) p2col_prefetch<V, PC>(p, buf, tn, tid);
            cp_async_commit();
#pragma unroll
            for (int g = 0; g < PC::CPT; g++) {
                // column q, rows m < N1: twiddles (w_n^q)^m
                V u[N1];
                const unsigned q = (unsigned)(c0 + tid + 256 * g);
                const double2 st = p2_wn(lo, hi, bits, q);
                double2 w = st;
                u[0] = v[g];
#pragma unroll
                for (int m = 1; m < N1; m++) {
                    u[m] = cmul(v[g + PC::CPT * m], fromd<V>(w));
                    if (m + 1 < N1) w = cmul(w, st);
                }
                dft<N1>(u);
#pragma unroll
                for (int k = 0; k < N1; k++) p2col_store(p, out, (int)q, k, u[k]);
            }
        } else {
            const int j = tid & (PC::VC - 1), b = tid >> PC::LGVC;
            {
                // column q = c0 + j, rows b + TPC k: w_n^(q b) (w_n^(q TPC))^k
                const unsigned q = (unsigned)(c0 + j);
                double2 w = p2_wn(lo, hi, bits, q * (unsigned)b);
                const double2 st = p2_wn(lo, hi, bits, q * (unsigned)PC::TPC);
#pragma unroll
                for (int k = 0; k < 16; k++) {
                    v[k] = cmul(v[k], fromd<V>(w));
                    if (k < 15) w = cmul(w, st);
                }
            }
            dft<16>(v);
            // stage 0: twiddle w_N1^(b k), back into this thread's own
            // slots (row b + TPC k of the tile = sub-transform k, t = b)
#pragma unroll
            for (int k = 0; k < 16; k++) buf[tid + 256 * k] = p2_tw_stage(v[k], tw, (unsigned)(b * k));
            __syncthreads();                    // every copy of the tile has landed and been read
            p2col_discard<V, PC>(p, tile, tid);
            p2col_stages<V, PC, 1>(p, buf, tw, tile);
        }
    }
}

// ------------------------------------------------------------------------
// Single pass for n = C x 4096, C in {2, 4, 8, 16}: a cluster of C CTAs per
// transform.  CTA c loads the stride-C subsequence x[c + C t], t < 4096, into
// registers, transforms it with the register 4096-point FFT (fft4096_regs)
// and publishes F_c[k] in shared memory; after one cluster barrier the
// cluster's threads take k round robin and combine
//   X[k + 4096 q] = sum_c w_n^(c k) F_c[k] w_C^(c q)
// through distributed shared memory, storing whole segments for each q.  The
// data crosses HBM once (the two-pass form writes and reads an
// intermediate).  KParams: t4 = two-level table of w_4096 (staged), t4n =
// two-level table of w_n (read through L2), batch = transforms.
template <typename V, int C, bool TMA = false>
__device__ __forceinline__ void p2cl_body(const KParams& p, unsigned char* smem, const CUtensorMap* tm = nullptr) {
    cg::cluster_group cl = cg::this_cluster();
    const int c = (int)cl.block_rank();
    const int tr = block_id(p) / C;
    if (tr >= p.batch) return;                  // uniform across the cluster
    V* buf = (V*)smem;                          // 16 planes of R4096_PL elements
    double2* tlo = after16(buf + 16 * R4096_PL);
    double2* thi = tlo + 64;
    V v[16];
    if constexpr (TMA) {
        // ComplexF64: the stride-C subsequence by 16 tensor copies of 256
        // elements (tm maps the input as [transform][t < 4096][2 C doubles])
        // into buf[t], each thread then reading its own slots t + 256 k,
        // which the first exchange overwrites only from the same thread
        uint64_t* bar = (uint64_t*)(thi + 65);
        const int t = opaque_tid();
        if (t == 0) mbar_init(bar, 1);
        if (t < 64) tlo[t ^ (t >> 3)] = p.t4.lo[t];
        if (t < 65) thi[t] = p.t4.hi[t];
        __syncthreads();                        // barrier initialised, tables staged
        if (t == 0) {
            mbar_expect_tx(bar, 4096 * (unsigned)sizeof(V));
#pragma unroll 1
            for (int k = 0; k < 16; k++) tma_load_3d(buf + 256 * k, tm, bar, 2 * c, 256 * k, tr);
        }
        // a copy that timed out records the fault; the CTA still takes the
        // cluster barrier below
        if (!mbar_wait(bar, 0) && t == 0) record_fault(kFaultTmaTimeout);
#pragma unroll
        for (int k = 0; k < 16; k++) v[k] = load_in(p, buf[t + 256 * k]);
    } else {
        const int t = opaque_tid();
        if (t < 64) tlo[t ^ (t >> 3)] = p.t4.lo[t];
        if (t < 65) thi[t] = p.t4.hi[t];
        const V* x = (const V*)p.in + (long long)tr * p.in_dist + c + (long long)C * t;
#pragma unroll
        for (int k = 0; k < 16; k++) v[k] = load_in(p, __ldg(x + (long long)C * 256 * k));
        __syncthreads();                        // tables staged
    }
    fft4096_regs(v, buf, tlo, thi, opaque_tid());
    {
        const int t = opaque_tid();
#pragma unroll
        for (int k3 = 0; k3 < 16; k3++) buf[t + 256 * k3] = v[k3];
    }
    cl.sync();                                  // every F_c published
    {
        const int g = c * 256 + opaque_tid();
        V* out = (V*)p.out + (long long)tr * p.out_dist;
        const unsigned mask = (1u << p.t4n.bits) - 1;
#pragma unroll 1
        for (int k = g; k < 4096; k += C * 256) {
            V f[C];
#pragma unroll
            for (int q = 0; q < C; q++) f[q] = cl.map_shared_rank(buf, q)[k];
            // w_n^(q k) as FP64 powers of one table value, rounded once
            const double2 wk = cmul(__ldg(p.t4n.lo + (k & mask)), __ldg(p.t4n.hi + (k >> p.t4n.bits)));
            double2 w = wk;
#pragma unroll
            for (int q = 1; q < C; q++) {
                f[q] = cmul(f[q], fromd<V>(w));
                if (q + 1 < C) w = cmul(w, wk);
            }
            dft<C>(f);
#pragma unroll
            for (int q = 0; q < C; q++) stg_stream(out + k + 4096 * q, store_out(p, f[q]));
        }
    }
    cl.sync();                                  // no CTA leaves while a peer reads its F
}

// ------------------------------------------------------------------------
// Both passes in one persistent launch (dataflow).  Work items, claimed in
// order from a global ticket, are the pass-A rows (N1 per transform) and the
// pass-B column tiles (N1 per transform); slot s holds the rows of transform
// s and the tiles of transform s - lag.  A tile of transform t waits until
// all N1 rows of t are written; a row of transform t reuses ring slot
// t mod depth of the intermediate and waits until all tiles of t - depth
// have read it.  Items only wait on items claimed earlier, by CTAs that are
// running, so the launch needs no co-residency guarantee.  Producers publish
// with a fence and an atomic add after a block barrier; consumers acquire
// the counter, then a block barrier.  Every wait is bounded (about a second):
// on a timeout the item is skipped and the device fault word records it.
struct FlowCtl {
    int* ticket;                  // next item
    int* abort;                   // set by the first wait that times out: later waits give up at once
    int* cnt;                     // rows done per transform [nb], then tiles done [nb]
    void* ring;                   // depth intermediates of n elements
    int nb, lag, depth;           // transforms, slots between a row and its tiles, ring size
};
constexpr unsigned kFaultFlowTimeout = 2u;

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// thread 0 waits until *c >= target (bounded, about a second); the CTA
// learns the outcome.  The first wait of a launch that times out raises the
// launch's abort flag, so no later wait of that launch waits at all.
__device__ __forceinline__ bool flow_wait(const int* c, int target, int* flag, int* abort) {
    if (threadIdx.x == 0) {
        int ok = 0;
        for (int it = 0; it < (1 << 23); it++) {
            if (ld_acquire_gpu(c) >= target) { ok = 1; break; }
            if (ld_acquire_gpu(abort)) break;
            __nanosleep(128);
        }
        *flag = ok;
        if (!ok) {
            atomicExch(abort, 1);
            record_fault(kFaultFlowTimeout);
        }
    }
    __syncthreads();
    const bool ok = *flag != 0;
    __syncthreads();                            // the flag may be rewritten next
    return ok;
}
// every thread's stores of this item precede the count
__device__ __forceinline__ void flow_publish(int* c) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(c, 1);
}

// pa: pass A (in = the transforms at in_dist, PA = log2 N1, t4 = w_4096);
// pb: pass B (out = the output at out_dist, twN1, t4n staged when pre).
// Shared memory: 16 planes of R4096_PL elements (pass B uses the first 4096
// slots), the w_4096 table, the w_N1 table, the staged w_n table, two ints.
template <typename V, int N1>
__device__ __forceinline__ void p2flow_body(const KParams& pa, const KParams& pb, const FlowCtl& fc,
                                            unsigned char* smem) {
    using PC = P2Col<N1>;
    V* buf = (V*)smem;
    double2* tlo = after16(buf + 16 * R4096_PL);
    double2* thi = tlo + 64;
    double2* tw = thi + 65;                     // w_N1, N1 entries
    double2* ts = tw + N1;                      // staged w_n two-level table
    const int bits = pb.t4n.bits;
    const int nlo = 1 << bits, nhi = (pb.t4n.N + nlo - 1) / nlo + 1;
    int* sh = (int*)(ts + (pb.pre ? nlo + nhi : 0));
    const double2 *lo = pb.t4n.lo, *hi = pb.t4n.hi;
    {
        const int t = opaque_tid();
        if (t < 64) tlo[t ^ (t >> 3)] = pa.t4.lo[t];
        if (t < 65) thi[t] = pa.t4.hi[t];
        for (int i = t; i < N1; i += 256) tw[i] = pb.twN1[i];
        if (pb.pre) {
            for (int i = t; i < nlo + nhi; i += 256) ts[i] = (i < nlo) ? pb.t4n.lo[i] : pb.t4n.hi[i - nlo];
            lo = ts;
            hi = ts + nlo;
        }
    }
    const long long n = (long long)N1 * 4096;
    const int per = 2 * N1;
    const long long total = (long long)(fc.nb + fc.lag) * per;
    for (;;) {
        if (threadIdx.x == 0) sh[0] = atomicAdd(fc.ticket, 1);
        __syncthreads();                        // also: tables staged, buffer free
        const long long w = sh[0];
        __syncthreads();
        if (w >= total) break;
        const int s = (int)(w / per), r = (int)(w - (long long)s * per);
        if (r < N1) {
            // ---- pass A: row i of transform s
            const int tr = s, i = r;
            if (tr >= fc.nb) continue;
            if (tr >= fc.depth && !flow_wait(fc.cnt + fc.nb + (tr - fc.depth), N1, sh + 1, fc.abort)) continue;
            V v[16];
            {
                const int t = opaque_tid();
                const V* in = (const V*)pa.in + (long long)tr * pa.in_dist + i + (t << PC::LGN1);
#pragma unroll 1
                for (int k = 0; k < 16; k++, in += 256LL << PC::LGN1) cp_async_elem(buf + t + 256 * k, in);
                cp_async_commit();
                cp_async_wait_all();            // this thread's own slots
#pragma unroll
                for (int k = 0; k < 16; k++) v[k] = load_in(pa, buf[t + 256 * k]);
            }
            fft4096_regs(v, buf, tlo, thi, opaque_tid());
            {
                const int t = opaque_tid();
                V* row = (V*)fc.ring + (long long)(tr % fc.depth) * n + ((long long)i << 12);
#pragma unroll
                for (int k3 = 0; k3 < 16; k3++) row[t + 256 * k3] = v[k3];
            }
            flow_publish(fc.cnt + tr);
        } else {
            // ---- pass B: column tile of transform s - lag
            const int tr = s - fc.lag, tile_in_tr = r - N1;
            if (tr < 0 || tr >= fc.nb) continue;
            if (!flow_wait(fc.cnt + tr, N1, sh + 1, fc.abort)) continue;
            // the tile's view of the intermediate as a pass-B launch of one transform
            KParams q = pb;
            q.in = (const V*)fc.ring + (long long)(tr % fc.depth) * n;
            q.in_dist = n;
            q.out = (V*)pb.out + (long long)tr * pb.out_dist;
            const int tid = opaque_tid();
            p2col_prefetch<V, PC>(q, buf, tile_in_tr, tid);
            cp_async_commit();
            cp_async_wait_all();
            V v[16];
#pragma unroll
            for (int k = 0; k < 16; k++) v[k] = buf[tid + 256 * k];
            const int c0 = tile_in_tr * PC::VC;
            V* out = (V*)q.out;
            if constexpr (N1 <= 16) {
                __syncwarp();
                p2col_discard<V, PC>(q, tile_in_tr, tid);
#pragma unroll
                for (int g = 0; g < PC::CPT; g++) {
                    V u[N1];
                    const unsigned col = (unsigned)(c0 + tid + 256 * g);
                    const double2 st = p2_wn(lo, hi, bits, col);
                    double2 wv = st;
                    u[0] = v[g];
#pragma unroll
                    for (int m = 1; m < N1; m++) {
                        u[m] = cmul(v[g + PC::CPT * m], fromd<V>(wv));
                        if (m + 1 < N1) wv = cmul(wv, st);
                    }
                    dft<N1>(u);
#pragma unroll
                    for (int k = 0; k < N1; k++) p2col_store(q, out, (int)col, k, u[k]);
                }
            } else {
                const int j = tid & (PC::VC - 1), b = tid >> PC::LGVC;
                {
                    const unsigned col = (unsigned)(c0 + j);
                    double2 wv = p2_wn(lo, hi, bits, col * (unsigned)b);
                    const double2 st = p2_wn(lo, hi, bits, col * (unsigned)PC::TPC);
#pragma unroll
                    for (int k = 0; k < 16; k++) {
                        v[k] = cmul(v[k], fromd<V>(wv));
                        if (k < 15) wv = cmul(wv, st);
                    }
                }
                dft<16>(v);
#pragma unroll
                for (int k = 0; k < 16; k++) buf[tid + 256 * k] = p2_tw_stage(v[k], tw, (unsigned)(b * k));
                __syncthreads();
                p2col_discard<V, PC>(q, tile_in_tr, tid);
                p2col_stages<V, PC, 1, false>(q, buf, tw, tile_in_tr);
            }
            flow_publish(fc.cnt + fc.nb + tr);
        }
    }
}
