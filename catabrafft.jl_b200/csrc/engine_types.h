// engine_types.h -- parameter blocks shared by the kernels and the planner.
#pragma once
#include <vector_types.h>

#define CFFT_MAXP 24

// Radix passes run in this order: odd radices first, so that the first
// pass's stride-R writes never hit a multiple of 8 elements (which would
// put a quarter-warp of 16-byte stores on one bank group).
#define CFFT_EXEC_ORDER {9, 7, 5, 3, 16, 8, 4, 2}

struct SubPlan {
    int L;                        // sub-transform length
    int np;                       // number of radix passes
    int G;                        // sub-transforms per block-wide wave (fits EMAX regs/thread)
    int Gwarp;                    // sub-transforms per warp group (0: block mode)
    unsigned char radix[CFFT_MAXP];  // pass radices in execution order
    unsigned char cnt[8];         // multiplicities of 9, 7, 5, 3, 16, 8, 4, 2 (CFFT_EXEC_ORDER)
    int twlen;                    // entries of tw
    // per-pass twiddle blocks in execution order: pass p (stride s, n1 =
    // L/(s r)) owns (r-1)*n1 entries, tw[off + (j-1)*n1 + q] = w_L^(j*q*s),
    // so adjacent lanes (adjacent q) read adjacent entries
    const void* tw;
};

struct TwoLevel {                 // w_N^e = lo[e & mask] * hi[e >> bits]  (FP64)
    const double2* lo;
    const double2* hi;
    int bits;
    int N;
};

enum { MODE_ROWS = 0, MODE_FOUR = 1, MODE_COLPASS = 2, MODE_ROWPASS = 3, MODE_P2COL = 4, MODE_P2ROW = 5,
       MODE_CONVC = 6, MODE_MIXC = 7, MODE_P2CL = 8 };
// kernel selector only (KParams.mode stays MODE_FOUR): the generic four-step
// kernel instantiated with warp-synchronous sub-transforms
enum { MODE_FOUR_WARP = 16 };
enum { CONV_NONE = 0, CONV_RADER = 1, CONV_BLUE = 2 };
enum { PRE_NONE = 0, PRE_CHIRP = 1, PRE_SPEC = 2 };      // COLPASS prologue
enum { POST_OUT = 0, POST_RAW = 1, POST_CHIRP = 2 };     // ROWPASS epilogue

struct KParams {
    int mode, conv;
    int nx;                       // user transform length
    int M;                        // working FFT length (nx unless conv)
    int N1, N2, C;                // FOUR / pass split
    int V;                        // ROWS: transforms per CTA; passes: tile width
    int PA, PC;                   // smem pitches (column layout / row layout)
    int XP;                       // Rader x staging: row pitch (ROWS) or chunk (FOUR)
    int pre, post;                // pass prologue / epilogue
    SubPlan pa, pc;               // column (N1) / row (N2, or M in ROWS) plans
    TwoLevel t4;                  // four-step twiddles w_M^(i2 k1)
    const int* perm;              // Rader: g^j mod nx, j < nx-1
    const int* iperm;             // Rader: g^-j mod nx
    const double2* chirp;         // Bluestein: exp(-i pi j^2 / nx), j < nx
    const double2* spec;          // conv spectrum / M (FP64)
    const void* in;
    void* out;
    long long in_dist, out_dist;  // elements between consecutive transforms
    int batch;                    // transforms in this launch
    int units;                    // CTAs (ROWS/FOUR clusters) or tiles per transform
    int dir;                      // 0 forward, 1 inverse (scaled), 2 backward
    double scale;                 // 1/nx for dir 1, else 1
    // multiply-shift reciprocals (see fdiv) of the layout's divisors
    unsigned long long mW, mN2, mR1, mX, mM, mL, mV;
    int blk0;                     // first block of this parameter block in its launch
    unsigned char in_user, out_user;  // batched launches: in/out relative to the caller's buffers
    unsigned char in_fmt, out_fmt;    // IO_*: how in / out hold the caller's elements
    long long in_off, out_off;    // batched launches: element offsets added to the bases
    // power-of-two passes: the four-step table of w_n (row pass) and the
    // single-level table w_N1^e, e < N1 (column pass)
    TwoLevel t4n;
    const double2* twN1;
    // element strides of in / out (IO_STRIDED, IO_HALF; unused for IO_PLAIN)
    long long in_stride, out_stride;
};
// The caller's buffers as a plan's first and last stage address them:
// contiguous elements of the data type (IO_PLAIN), elements of the data type
// at a stride (IO_STRIDED), or ComplexF16 elements at a stride (IO_HALF, the
// arithmetic in ComplexF32).  Element i of transform t sits at
// t * dist + i * stride.
enum { IO_PLAIN = 0, IO_STRIDED = 1, IO_HALF = 2 };

// COLPASS / ROWPASS stage their sub-transform twiddle table in shared memory
// (ahead of the tile) when it is small; larger tables are read from L2.
// Host and device use this one rule to agree on the shared-memory size.
inline __host__ __device__ bool cfft_pass_tw_staged(int twlen, int elem_bytes) {
    return twlen > 0 && twlen * elem_bytes <= 16384;
}
inline __host__ __device__ int cfft_pass_tw_elems(int twlen, int elem_bytes) {
    return cfft_pass_tw_staged(twlen, elem_bytes) ? twlen : 0;
}
// COLPASS also stages the two-level four-step table (FP64 lo then hi, after
// the sub-transform table, 16-byte aligned) when it is at most 12 KB
inline __host__ __device__ int cfft_pass_t4_elems(int bits, int N) {
    const int nlo = 1 << bits, nhi = (N + nlo - 1) / nlo + 1;
    return (nlo + nhi) * 16 <= 12288 ? nlo + nhi : 0;
}
// shared memory of a COLPASS tile: sub-transform twiddles, four-step table, tile
inline __host__ __device__ size_t cfft_colpass_smem(int twlen, int bits, int N, int tile_elems, int elem_bytes) {
    const size_t a = ((size_t)cfft_pass_tw_elems(twlen, elem_bytes) * elem_bytes + 15) / 16 * 16;
    return a + (size_t)cfft_pass_t4_elems(bits, N) * 16 + (size_t)tile_elems * elem_bytes + 16;
}

// Tile widths of the two pass kernels for M = N1 x N2 (host side; the
// planner and the no-allocation entry point use the same rule).  A width is a
// divisor of the tile count of at most 64 whose tile fits the per-CTA budget
// (three ComplexF32 or two ComplexF64 CTAs per SM, staged tables included);
// a power of two whose V-element global segments span at least 128 bytes is
// preferred (it divides the block, so each thread keeps one column in the
// column pass's epilogue), else the widest that fits.
inline long long cfft_pick_tile(long long count, long long per, size_t limit, size_t e) {
    long long best = 1, best2 = 0;
    for (long long v = 1; v <= count && v <= 64; v++) {
        if (count % v || (size_t)(v * per) * e > limit) continue;
        best = v;
        if ((v & (v - 1)) == 0 && (size_t)v * e >= 128) best2 = v;
    }
    return best2 ? best2 : best;
}
// *Vc: columns per COLPASS tile; *Vr: rows per ROWPASS tile (row pitch PC)
inline void cfft_pass_tiles(long long N1, long long N2, long long PC, int twA, int twC, int bits, int M,
                            size_t e, long long* Vc, long long* Vr) {
    const size_t budget = (e == 8) ? 74 * 1024 : 112 * 1024;
    const size_t tile_lim = (e == 8) ? 72 * 1024 : 96 * 1024;
    const size_t tabc = cfft_colpass_smem(twA, bits, M, 0, (int)e);
    const size_t tabr = (size_t)cfft_pass_tw_elems(twC, (int)e) * e + 16;
    const size_t room_c = budget > tabc ? budget - tabc : 0, room_r = budget > tabr ? budget - tabr : 0;
    const size_t lim_c = room_c < tile_lim ? room_c : tile_lim, lim_r = room_r < tile_lim ? room_r : tile_lim;
    *Vc = cfft_pick_tile(N2, N1, lim_c, e);
    *Vr = cfft_pick_tile(N1, PC, lim_r, e);
}

// One launch of the batched executor: parameter blocks in device memory and,
// per block of the grid, the index of its parameter block.
struct BatchLaunch {
    const KParams* desc;
    const int* block_desc;
    const void* in_base;
    void* out_base;
    int dir;                      // direction of every block, or -1: each block's own
    int pad_;
};


// The batched form's single persistent launch: CTAs claim work items in
// ticket order; an item is one block of a parameter block (a whole
// single-CTA transform, or one tile of a two-pass stage).  An item may wait
// for a counter to reach `need` (the previous stage of its transform, or the
// release of the scratch half its chunk reuses) and adds one to counter
// `done` when finished.  Every wait is on items with smaller tickets, so the
// queue drains whatever the residency.
enum { QK_ROWS = 0, QK_FOUR = 1, QK_FOUR_WARP = 2, QK_COLPASS = 3, QK_ROWPASS = 4 };
struct QItem {
    int desc;                     // parameter block
    int blk;                      // block within the parameter block
    int kind;                     // QK_*
    int wait, need;               // counter (-1: none) and the count to wait for
    int done;                     // counter to add one to (-1: none)
};
struct QueueLaunch {
    const KParams* desc;
    const QItem* items;
    const void* in_base;
    void* out_base;
    int* ctl;                     // [0] ticket, [1] abort flag, [2 ...] counters; zero before each launch
    int nitems;
    int dir;                      // direction of every item, or -1: each parameter block's own
};
