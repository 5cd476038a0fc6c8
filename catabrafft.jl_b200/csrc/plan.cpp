// plan.cpp -- planner, FP64 table generation, plan cache and the C ABI.
//
// Host-side counterpart of CatabraFFT.jl's dispatcher (src/kernel.jl:72-199),
// planner (src/radix_plan.jl) and plan object (src/spells.jl).  Strategy:
//   n 7-smooth          -> Stockham on the device (ROWS / FOUR / two HBM passes)
//   n prime             -> Rader (src/prime.jl): generator permutation, cyclic
//                          convolution of length n-1 through a zero-padded
//                          smooth FFT of length M >= 2n-3, inverse permutation
//   other n             -> Bluestein convolution of length M >= 2n-1 (the
//                          reference recurses through mixed radix + Rader,
//                          src/kernel.jl:84-86; both compute the same DFT)
// Tables are generated here in FP64 with exact integer angle reduction and
// rounded once to the data type.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <thread>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/catabra_b200.h"
#include "kernels.h"
#include "trace.h"

// thread-local error text in a fixed buffer (set without touching the heap)
static thread_local char g_err[512];
void cfft_set_last_error(const char* msg) { snprintf(g_err, sizeof g_err, "%s", msg ? msg : ""); }
static int fail(int code, const std::string& msg) {
    cfft_set_last_error(msg.c_str());
    return code;
}
// ------------------------------------------------- allocation accounting
// Every device and pinned-host allocation of the library goes through these
// wrappers: they count live allocations and, for tests of the failure paths,
// can make allocations fail as out of memory (cfft_debug_alloc_hook).
static std::atomic<int64_t> g_live_allocs{0};
static std::atomic<int64_t> g_alloc_seq{0};       // allocations since the hook was last set
static std::atomic<int64_t> g_alloc_fail_from{0}; // 0: off; else fail the nth and later
static bool alloc_injected_failure() {
    const int64_t from = g_alloc_fail_from.load();
    if (from <= 0) return false;
    return g_alloc_seq.fetch_add(1) + 1 >= from;
}
template <class T> static cudaError_t lib_malloc(T** p, size_t bytes) {
    if (alloc_injected_failure()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    cudaError_t e = cudaMalloc((void**)p, bytes);
    if (e == cudaSuccess) g_live_allocs.fetch_add(1);
    return e;
}
template <class T> static cudaError_t lib_host_alloc(T** p, size_t bytes, unsigned flags) {
    if (alloc_injected_failure()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    cudaError_t e = cudaHostAlloc((void**)p, bytes, flags);
    if (e == cudaSuccess) g_live_allocs.fetch_add(1);
    return e;
}
static cudaError_t lib_free(void* p) {
    if (!p) return cudaSuccess;
    g_live_allocs.fetch_sub(1);
    return cudaFree(p);
}
static cudaError_t lib_free_host(void* p) {
    if (!p) return cudaSuccess;
    g_live_allocs.fetch_sub(1);
    return cudaFreeHost(p);
}

#define CUDA_TRY(call)                                                                     \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail(e_ == cudaErrorMemoryAllocation ? CFFT_ERR_NOMEM : CFFT_ERR_CUDA,  \
                        std::string(#call) + ": " + cudaGetErrorString(e_));               \
    } while (0)

// ------------------------------------------------------------ integer helpers
static bool is_smooth7(int64_t n) {
    if (n < 1) return false;
    for (int p : {2, 3, 5, 7})
        while (n % p == 0) n /= p;
    return n == 1;
}
static bool is_prime64(int64_t n) {
    if (n < 2) return false;
    if (n % 2 == 0) return n == 2;
    for (int64_t d = 3; d * d <= n; d += 2)
        if (n % d == 0) return false;
    return true;
}
static int64_t smooth_ceil(int64_t n) {
    for (int64_t m = std::max<int64_t>(n, 1);; m++)
        if (is_smooth7(m)) return m;
}
static int64_t powmod(int64_t b, int64_t e, int64_t m) {
    __int128 r = 1, x = b % m;
    while (e > 0) {
        if (e & 1) r = (r * x) % m;
        x = (x * x) % m;
        e >>= 1;
    }
    return (int64_t)r;
}
// smallest primitive root (the generator search of src/prime.jl:9-28)
static int64_t primitive_root(int64_t p) {
    int64_t phi = p - 1;
    std::vector<int64_t> fac;
    int64_t f = phi;
    for (int64_t q = 2; q * q <= f; q++)
        if (f % q == 0) {
            fac.push_back(q);
            while (f % q == 0) f /= q;
        }
    if (f > 1) fac.push_back(f);
    for (int64_t g = 2; g < p; g++) {
        bool ok = true;
        for (int64_t q : fac)
            if (powmod(g, phi / q, p) == 1) { ok = false; break; }
        if (ok) return g;
    }
    return -1;
}

// greedy radix split, largest first (create_std_radix_plan, radix_plan.jl:100-138,
// over the codelet set of this build)
static const int kRadices[] = {16, 9, 8, 7, 5, 4, 3, 2};   // split preference
static const int kExec[] = CFFT_EXEC_ORDER;                  // execution order
static std::vector<int> radix_split(int64_t L, const int* order = kRadices, int nord = 8) {
    std::vector<int> r;
    while (L > 1) {
        int c = 0;
        for (int i = 0; i < nord; i++)
            if (L % order[i] == 0) { c = order[i]; break; }
        if (!c) return {};
        r.push_back(c);
        L /= c;
    }
    return r;
}
static unsigned long long magic(int64_t d) {
    // ceil(2^40 / d); exact floor(n/d) for n < 2^24, d <= 2^16 (see fdiv)
    if (d < 1) d = 1;
    return ((1ULL << 40) + (unsigned long long)d - 1) / (unsigned long long)d;
}
static void radix_counts(const std::vector<int>& rad, unsigned char* cnt) {
    for (int ci = 0; ci < 8; ci++) {
        int c = 0;
        for (int r : rad) c += (r == kExec[ci]);
        cnt[ci] = (unsigned char)c;
    }
}
// radices of a split in execution order
static std::vector<int> exec_order(const std::vector<int>& rad) {
    std::vector<int> out;
    for (int ci = 0; ci < 8; ci++)
        for (int r : rad)
            if (r == kExec[ci]) out.push_back(r);
    return out;
}
// entries of the per-pass twiddle table of a sub-transform
static int64_t twiddle_len(int64_t L, const std::vector<int>& rad) {
    int64_t s = 1, len = 0;
    for (int r : exec_order(rad)) {
        len += (int64_t)(r - 1) * (L / (s * r));
        s *= r;
    }
    return len;
}
static int wave_G(const std::vector<int>& rad, int64_t L, int T) {
    if (L <= 1) return 1 << 20;
    int64_t g = 1 << 20;
    for (int r : rad) g = std::min<int64_t>(g, (int64_t)T * (CFFT_EMAX / r) * r / L);
    return (int)g;
}

// ------------------------------------------------------------- FP64 tables
// exp(sign * 2 pi i m / N) with exact integer reduction, long double kernel
static double2 omega(int64_t m, int64_t N, int sign) {
    m %= N;
    if (m < 0) m += N;
    // quadrant: theta = (pi/2) (q + r/N)
    __int128 fm = (__int128)4 * m;
    int64_t q = (int64_t)(fm / N);
    int64_t r = (int64_t)(fm - (__int128)q * N);
    const long double HALF_PI = 1.570796326794896619231321691639751442L;
    long double c, s;
    if (2 * r <= N) {
        long double x = HALF_PI * ((long double)r / (long double)N);
        c = cosl(x);
        s = sinl(x);
    } else {
        long double x = HALF_PI * ((long double)(N - r) / (long double)N);
        c = sinl(x);
        s = cosl(x);
    }
    long double cc, ss;
    switch (q & 3) {
        case 0: cc = c; ss = s; break;
        case 1: cc = -s; ss = c; break;
        case 2: cc = -c; ss = -s; break;
        default: cc = s; ss = -c; break;
    }
    return make_double2((double)cc, (double)(sign * ss));
}
// Julia's robust complex inverse (Smith's algorithm) for |z| near 1
static double2 julia_inv(double2 z) {
    volatile double c = z.x, d = z.y;
    double p, q;
    if (std::fabs(c) >= std::fabs(d)) {
        volatile double r = d / c;
        volatile double den = c + d * r;
        volatile double t = 1.0 / den;
        p = t;
        q = -r * t;
    } else {
        volatile double cc = d, dd = c;
        volatile double r = dd / cc;
        volatile double den = cc + dd * r;
        volatile double t = 1.0 / den;
        p = r * t;
        q = -t;
    }
    return make_double2(p, q);
}
static double2 cmul_h(double2 a, double2 b) {
    volatile double re1 = a.x * b.x, re2 = a.y * b.y, im1 = a.x * b.y, im2 = a.y * b.x;
    return make_double2(re1 - re2, im1 + im2);
}
// power_by_squaring (Julia Base) -- the reference builds Rader twiddles with it
static double2 pow_by_squaring(double2 x, int64_t p) {
    if (p == 1) return x;
    if (p == 0) return make_double2(1, 0);
    if (p == 2) return cmul_h(x, x);
    int t = __builtin_ctzll((unsigned long long)p) + 1;
    p >>= t;
    while ((t -= 1) > 0) x = cmul_h(x, x);
    double2 y = x;
    while (p > 0) {
        t = __builtin_ctzll((unsigned long long)p) + 1;
        p >>= t;
        while ((t -= 1) >= 0) x = cmul_h(x, x);
        y = cmul_h(y, x);
    }
    return y;
}

// ---------------------------------------------------------------- plan state
struct Stage {
    KParams kp;
    const void* fn = nullptr;    // kernel entry (generic or statically shaped)
    unsigned grid;
    int threads;
    size_t smem;
    int cluster;
    int in_sel, out_sel;     // 0 user in, 1 user out, 2 scratch0, 3 scratch1
    int max_units = 0;       // persistent kernels: co-resident clusters (0 = one per unit)
    size_t smem_batched = 0; // shared memory of the descriptor-driven variant (0: smem)
    unsigned persist = 0;    // kernels that loop over the batch: CTAs to launch at most
    int launch = 0;          // 1 / 3: pass A by tensor copies (ComplexF64 / ComplexF32 pairs); 2: dataflow
                             // launch; 4 / 5: mixed-radix / power-of-two cluster kernel with tensor copies
    KParams kp2;             // dataflow launch: the pass-B parameters
    int flow_lag = 0, flow_depth = 0;
};

struct Shape {
    int mode = MODE_ROWS;    // ROWS, FOUR or GLOBAL(=MODE_COLPASS)
    int conv = CONV_NONE;
    int64_t M = 0;
    int N1 = 1, N2 = 1, C = 1, V = 1;
    std::vector<int> ra, rc; // radix passes for N1 / N2 (ROWS: rc for M)
    size_t smem = 0;
    size_t smem_dyn = 0;     // FOUR: the generic (two-buffer) kernels' shared memory
    double score = 0;
    int var = 0;             // power-of-two passes: 1 = pass A by tensor copies
};

// Reference-counted device buffer.  Tables that depend only on a length (sub-
// transform twiddles, four-step tables, convolution spectra) are shared
// through a process-wide cache; plans hold references, so dropping the cache
// (cfft_empty_cache) never frees a table a live plan still uses.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    ~DevBuf() {
        if (p) lib_free(p);
    }
};
using DevPtr = std::shared_ptr<DevBuf>;

struct cfft_plan_s {
    int64_t n = 0, batch = 0;
    int dtype = 0, flags = 0;
    Shape shape;
    std::string desc;
    std::vector<Stage> stages;
    int64_t chunk = 0;       // transforms per stage sequence (GLOBAL)
    void* scratch[2] = {nullptr, nullptr};
    size_t scratch_bytes = 0;
    std::vector<void*> allocs;
    std::vector<DevPtr> tables;  // shared, cached tables
    bool shared_scratch = false; // scratch provided by a batch (not allocated here)
    int device = 0;
    // host-buffer pipeline (created on first cfft_execute_host)
    std::mutex host_mu;
    bool host_ready = false;
    int64_t host_chunk = 0;
    void* host_buf[3] = {nullptr, nullptr, nullptr};
    cudaStream_t host_st[3] = {nullptr, nullptr, nullptr};   // in, compute, out
    cudaEvent_t ev_in[3] = {}, ev_comp[3] = {}, ev_out[3] = {};
    void* stage_in[3] = {nullptr, nullptr, nullptr};    // pinned staging for pageable callers
    void* stage_out[3] = {nullptr, nullptr, nullptr};
    // strided plans (cfft_plan_create_many): element i of transform b at
    // b * dist + i * stride; gathered into / scattered from strided_work
    bool strided = false;
    int64_t istride = 1, idist = 0, ostride = 1, odist = 0;
    void* strided_work = nullptr;
    // ComplexF16 plans: ComplexF16 in/out around the ComplexF32 path
    bool io_half = false;
    void* half_work = nullptr;   // batch * n ComplexF32 (unfused plans only)
    // fused ComplexF16 / strided plans: the first and last stage address the
    // caller's layout themselves (KParams in_fmt / out_fmt, IO_*), so the
    // plan runs its plain launches and no widening or gathering sweep
    bool io_fused = false;
    int in_fmt = IO_PLAIN, out_fmt = IO_PLAIN;
    void* half_dev = nullptr;    // host entry: device copy of the ComplexF16 data
    int* flow_ctr = nullptr;     // dataflow plans: ticket, abort flag, per-transform counters (2 + 2 batch ints)
};

static size_t elem_bytes(int dtype) { return dtype == CFFT_C128 ? 16 : 8; }
static const size_t kSmemMax = 220 * 1024;
// two CTAs fit an SM's 228 KB of shared memory with up to 113 KB each (1 KB
// per CTA is reserved), static shared memory included: 112 KB of dynamic
static const size_t kSmemTwoPerSM = 112 * 1024;

static std::vector<int> exec_order(const std::vector<int>& rad);
static std::string join(const std::vector<int>& v0) {
    const std::vector<int> v = exec_order(v0);
    std::string s;
    for (size_t i = 0; i < v.size(); i++) s += (i ? "," : "") + std::to_string(v[i]);
    return s;
}

// ------------------------------------------------------------ shape choice
static bool rows_shape(int64_t M, int64_t nx, int conv, int dtype, int64_t batch, Shape& sh) {
    if (M > 4096) return false;
    auto rc = radix_split(M);
    if (M > 1 && rc.empty()) return false;
    if (wave_G(rc, M, CFFT_THREADS) < 1) return false;
    size_t e = elem_bytes(dtype);
    int64_t PC = M + ((M % 2 == 0) ? 1 : 0);
    int64_t XP = (conv == CONV_RADER) ? nx : 0;
    size_t per_row = (size_t)(PC + XP) * e;
    // rows per CTA: ~48 KB of smem, but keep >= ~2 CTAs per SM busy
    int64_t V = std::max<int64_t>(1, (int64_t)(48 * 1024) / (int64_t)per_row);
    int64_t need = (batch + 295) / 296;
    V = std::max<int64_t>(1, std::min<int64_t>(V, need));
    sh.mode = MODE_ROWS;
    sh.M = M;
    sh.V = (int)V;
    sh.rc = rc;
    sh.smem = (size_t)V * per_row + 64 * sizeof(double2) + 16;
    return sh.smem <= kSmemMax;
}

// shared memory of a FOUR CTA: sub-transform twiddles, the two-level four-step
// twiddle table, the data buffer, the Rader x chunk and the FP64 reduction
// scratch (layout documented at four_body in engine.cuh)
static int twolevel_bits(int64_t N) {
    int bits = 0;
    while ((1LL << (2 * bits)) < N) bits++;
    return bits;
}
static size_t four_smem_bytes(int64_t M, int64_t twA, int64_t twC, int64_t bufsz, int64_t XP, size_t e) {
    const int bits = twolevel_bits(M);
    const int64_t nlo = 1LL << bits, nhi = (M + nlo - 1) / nlo + 1;
    size_t b = (size_t)(twA + twC) * e;
    b = (b + 15) & ~(size_t)15;
    b += (size_t)(nlo + nhi) * sizeof(double2);
    b += (size_t)(bufsz + XP) * e;
    b = (b + 15) & ~(size_t)15;
    b += 48 * sizeof(double2);
    return b;
}

static void four_candidates(int64_t M, int64_t nx, int conv, int dtype, std::vector<Shape>& out) {
    size_t e = elem_bytes(dtype);
    for (int64_t N1 = 2; N1 <= 4096; N1++) {
        if (M % N1) continue;
        int64_t N2 = M / N1;
        if (N2 < 2 || N2 > 4096) continue;
        auto ra = radix_split(N1), rc = radix_split(N2);
        if (ra.empty() || rc.empty()) continue;
        if (wave_G(ra, N1, CFFT_THREADS) < 1 || wave_G(rc, N2, CFFT_THREADS) < 1) continue;
        for (int C = 1; C <= 16; C++) {
            if (N1 % C || N2 % C) continue;
            int64_t W = N2 / C, R1 = N1 / C;
            int64_t PA, PC;
            if (C == 1) {
                PA = PC = N2 + ((N2 % 2 == 0) ? 1 : 0);
            } else {
                if (W < 2 || R1 < 2) continue;
                PA = W;
                PC = N2 + ((N2 % 2 == 0) ? 1 : 0);
            }
            int64_t XP = (conv == CONV_RADER) ? (nx + C - 1) / C : 0;
            int64_t bufsz = (C == 1) ? N1 * PA : N1 * PA + R1 * PC;
            const int64_t tA = twiddle_len(N1, ra), tC = twiddle_len(N2, rc);
            // the generic kernels (and the batched forms) need this much
            const size_t smem_dyn = four_smem_bytes(M, tA, tC, bufsz, XP, e);
            if (smem_dyn > kSmemMax) continue;
            // a statically shaped kernel for exactly this shape folds strides
            // and counts to constants (preferred); a single-buffer one keeps
            // one buffer for both layouts
            unsigned char ca[8], cc[8];
            radix_counts(ra, ca);
            radix_counts(rc, cc);
            int single = 0;
            const bool stat = cfft_static_four(dtype, (int)N1, (int)N2, C, ca, cc, &single) != nullptr;
            const size_t smem = (stat && single) ? four_smem_bytes(M, tA, tC, std::max(N1 * PA, R1 * PC), XP, e)
                                                 : smem_dyn;
            Shape sh;
            sh.mode = MODE_FOUR;
            sh.conv = conv;
            sh.M = M;
            sh.N1 = (int)N1;
            sh.N2 = (int)N2;
            sh.C = C;
            sh.ra = ra;
            sh.rc = rc;
            sh.smem = smem;
            sh.smem_dyn = smem_dyn;
            double bal = std::fabs(std::log2((double)N1 / (double)N2));
            // one CTA per SM costs FP64 kernels more than FP32 ones (measured
            // on B200, 4096 x 3^9 ComplexF32: 3 CTAs of 111 KB, two per SM,
            // 1.23 ms; one CTA of 162 KB 1.34 ms; 9 CTAs 1.72 ms)
            const double one_per_sm = (dtype == CFFT_C64) ? 3.0 : 8.0;
            sh.score = (smem > kSmemTwoPerSM ? one_per_sm : 0.0) + (C > 8 ? 3.0 : 0.0) + 0.6 * C +
                       0.5 * bal + 0.1 * (ra.size() + rc.size());
            if (stat) sh.score -= 6.0;
            out.push_back(sh);
        }
    }
    std::sort(out.begin(), out.end(), [](const Shape& a, const Shape& b) { return a.score < b.score; });
}

static bool global_shape(int64_t M, int dtype, Shape& sh) {
    size_t e = elem_bytes(dtype);
    int64_t best = -1;
    double bestb = 1e9;
    for (int64_t N1 = 2; N1 <= 4096; N1++) {
        if (M % N1) continue;
        int64_t N2 = M / N1;
        if (N2 < 2 || N2 > 4096) continue;
        auto ra = radix_split(N1), rc = radix_split(N2);
        if (ra.empty() || rc.empty()) continue;
        if (wave_G(ra, N1, CFFT_THREADS) < 1 || wave_G(rc, N2, CFFT_THREADS) < 1) continue;
        double b = std::fabs(std::log2((double)N1 / (double)N2));
        if (b < bestb) { bestb = b; best = N1; }
    }
    if (best < 0) return false;
    sh.mode = MODE_COLPASS;
    sh.M = M;
    sh.N1 = (int)best;
    sh.N2 = (int)(M / best);
    sh.ra = radix_split(sh.N1);
    sh.rc = radix_split(sh.N2);
    (void)e;
    return true;
}

// conv length for a non-smooth n
static void conv_kind(int64_t n, int& conv, int64_t& M) {
    if (is_smooth7(n)) { conv = CONV_NONE; M = n; return; }
    if (is_prime64(n)) { conv = CONV_RADER; M = smooth_ceil(2 * n - 3); return; }
    conv = CONV_BLUE;
    M = smooth_ceil(2 * n - 1);
}

// power-of-two n = N1 x 4096 (N1 = 2 .. 1024) as two register passes
// (pow2.cuh); V carries the CTAs per SM the kernels are built for
static void pow2_candidates(int64_t n, int dtype, std::vector<Shape>& out) {
    if (n < 8192 || n > (1 << 22) || (n & (n - 1))) return;
    // up to 2^16: one pass on a cluster of n / 4096 register 4096-point CTAs.
    // Measured on B200 (1 GiB batches, ComplexF64): 8192 0.64 ms and 16384
    // 0.82 ms against 0.99 / 1.00 for the two passes; at 32768 and 65536 the
    // 8- and 16-CTA clusters fit only 33 / 14 at a time and lose (1.15 / 1.62
    // against 0.92 / 0.93 ms), so there they follow the two-pass shapes
    std::vector<Shape> cl;
    if (n <= 65536) {
        // var 1: ComplexF64 with the subsequences by tensor copies (two CTAs
        // per SM), offered last: measured slower than the direct strided
        // loads into registers (8192: 0.747 against 0.573 ms per GiB; 16384:
        // 0.757 against 0.698), which overlap better with the compute
        for (int c = 0; c < 3; c++) {
            const int var = c == 2 ? 1 : 0, mb = c == 1 ? 3 : 2;
            if (var == 1 && dtype != CFFT_C128) continue;
            Shape s;
            s.mode = MODE_P2CL;
            s.conv = CONV_NONE;
            s.M = n;
            s.N1 = (int)(n / 4096);
            s.N2 = 4096;
            s.C = (int)(n / 4096);
            s.V = mb;
            s.var = var;
            s.rc = {16, 16, 16};
            cl.push_back(s);
        }
    }
    const bool cluster_first = n <= 16384;
    if (cluster_first) out.insert(out.end(), cl.begin(), cl.end());
    // V = CTAs per SM of pass A (the n = 4096 kernel over strided rows):
    // three like the n = 4096 plan, or two (no spills) for ComplexF64;
    // ComplexF64 pass A by tensor copies (var = 1) first from N1 = 8 (one
    // 16-byte element per box row pays off once rows are 128 bytes apart;
    // measured 3-5 % faster there, 2-8 % slower at N1 = 2, 4)
    const bool tma_first = n >= 8 * 4096;
    // both passes in one persistent dataflow launch (var = 2, N1 >= 8),
    // offered after the two-launch forms
    std::vector<Shape> flow;
    if (n >= 8 * 4096) {
        Shape s;
        s.mode = MODE_P2COL;
        s.conv = CONV_NONE;
        s.M = n;
        s.N1 = (int)(n / 4096);
        s.N2 = 4096;
        s.V = 2;
        s.var = 2;
        s.ra = radix_split(s.N1);
        s.rc = {16, 16, 16};
        flow.push_back(s);
    }
    // ComplexF64 pass A at two CTAs per SM first (no spills; measured on
    // B200 with tensor copies: 2^15 0.819 against 0.881 ms per GiB at three,
    // 2^16 0.830 against 0.919)
    for (int c = 0; c < 4; c++) {
        const int var = ((c < 2) == tma_first) ? 1 : 0, mb = (c % 2 == 0) ? 2 : 3;
        // ComplexF32: pass A by cp.async at three CTAs per SM, or by tensor
        // copies of subsequence pairs at two
        if (dtype != CFFT_C128 && mb != (var == 1 ? 2 : 3)) continue;
        Shape s;
        s.var = var;
        s.mode = MODE_P2COL;
        s.conv = CONV_NONE;
        s.M = n;
        s.N1 = (int)(n / 4096);
        s.N2 = 4096;
        s.V = mb;
        s.ra = radix_split(s.N1);
        s.rc = {16, 16, 16};
        out.push_back(s);
    }
    out.insert(out.end(), flow.begin(), flow.end());
    if (!cluster_first) out.insert(out.end(), cl.begin(), cl.end());
}

// primes above 4096: Rader's convolution on a cluster of C register
// 4096-point CTAs, M = 4096 C >= 2n - 3 (convc.cuh); V carries the CTAs per SM
static void convc_candidates(int64_t n, int dtype, std::vector<Shape>& out) {
    if (n <= 4096 || !is_prime64(n)) return;
    int C = 0;
    for (int c : {3, 4, 5, 7, 8})
        if (4096LL * c >= 2 * n - 3) { C = c; break; }
    if (!C) return;
    // ComplexF64 at two CTAs per SM (no spills) measured 0.498 ms against
    // 0.567 ms at three for 1024 x 10007 on B200
    for (int mb : {2, 3}) {
        if (mb == 2 && dtype != CFFT_C128) continue;
        Shape s;
        s.mode = MODE_CONVC;
        s.conv = CONV_RADER;
        s.M = 4096LL * C;
        s.N1 = C;
        s.N2 = 4096;
        s.C = C;
        s.V = mb;
        s.rc = {16, 16, 16};
        out.push_back(s);
    }
}

// mixed-radix lengths with a cluster kernel of register L-point CTAs
// (mixc.cuh): n = C x L
static void mixc_candidates(int64_t n, int dtype, std::vector<Shape>& out) {
    // measured on B200 (1024 x 30240, ComplexF64): the strided input by
    // tensor copies 0.422 ms (9 x 3360, variant 5) and 0.447 ms (7 x 4320,
    // variant 4) against 0.471 / 0.477 ms by cp.async at two CTAs per SM and
    // 0.499 / 0.547 at three; ComplexF32 (no tensor copies: its 8-byte
    // elements are below a box row) 0.464 ms at three CTAs per SM (variant
    // 1) against 0.586 at two
    static const int order128[] = {5, 4, 3, 0, 2, 1}, order64[] = {1, 0, 2, 3};
    const int* order = dtype == CFFT_C128 ? order128 : order64;
    const int count = dtype == CFFT_C128 ? 6 : 4;
    for (int i = 0; i < count; i++) {
        const int var = order[i];
        const void* fn = nullptr;
        int C = 0, L = 0, T = 0;
        if (!cfft_mixc_lookup(n, dtype == CFFT_C128 ? CFFT_DT_C128 : CFFT_DT_C64, var, &fn, &C, &L, &T)) continue;
        Shape s;
        s.mode = MODE_MIXC;
        s.conv = CONV_NONE;
        s.M = n;
        s.N1 = C;
        s.N2 = L;
        s.C = C;
        s.V = T;
        s.var = var;
        out.push_back(s);
    }
}

// two HBM passes (COLPASS then ROWPASS; a convolution runs two of each);
// Rader here becomes Bluestein, and a convolution may use any 7-smooth
// length >= its minimum: take the first that splits into two factors of at
// most 4096
static bool twopass_shape(int64_t n, int conv, int64_t M, int dtype, Shape& g) {
    int c2 = conv;
    int64_t M2 = M;
    if (conv == CONV_RADER) { c2 = CONV_BLUE; M2 = smooth_ceil(2 * n - 1); }
    for (int tries = 0; tries < 256; tries++) {
        if (global_shape(M2, dtype, g)) {
            g.conv = c2;
            return true;
        }
        if (c2 == CONV_NONE) return false;
        M2 = smooth_ceil(M2 + 1);
    }
    return false;
}

static std::vector<Shape> candidate_shapes(int64_t n, int dtype, int64_t batch) {
    std::vector<Shape> v;
    int conv;
    int64_t M;
    conv_kind(n, conv, M);
    Shape sh;
    if (rows_shape(M, n, conv, dtype, batch, sh)) {
        sh.conv = conv;
        v.push_back(sh);
    }
    if (M > 64) four_candidates(M, n, conv, dtype, v);
    Shape g;
    if ((v.empty() || M >= 16384) && twopass_shape(n, conv, M, dtype, g)) {
        // beyond a cluster (or as the timed planners' alternative to one).
        // Measured on B200: from 2^15 points the two passes beat a cluster
        // for ComplexF32 transforms (1.3-1.5x at 2^16-2^17) and for
        // power-of-two ComplexF64 ones (1.3x at 2^15, 1.7x at 2^16);
        // otherwise second in line, so the heuristic keeps a single-kernel
        // shape and MEASURE/ENCHANT time both
        const bool pow2 = (M & (M - 1)) == 0;
        const bool first = (dtype == CFFT_C64 || pow2) && conv == CONV_NONE && M >= 32768;
        v.insert(v.begin() + (first ? 0 : std::min<size_t>(v.size(), 1)), g);
    }
    // the register kernels lead for the lengths they cover
    std::vector<Shape> reg;
    pow2_candidates(n, dtype, reg);
    convc_candidates(n, dtype, reg);
    mixc_candidates(n, dtype, reg);
    v.insert(v.begin(), reg.begin(), reg.end());
    return v;
}

static std::string shape_desc(const Shape& s, int64_t n) {
    std::string c = s.conv == CONV_RADER ? "rader" : s.conv == CONV_BLUE ? "bluestein" : "";
    std::string pre = c.empty() ? "" : c + "(n=" + std::to_string(n) + ",M=" + std::to_string(s.M) + ")+";
    if (s.mode == MODE_ROWS)
        return pre + "rows(V=" + std::to_string(s.V) + ")[" + join(s.rc) + "]";
    if (s.mode == MODE_P2CL)
        return "pow2cluster(C=" + std::to_string(s.C) + ",4096 per CTA,ctas_per_sm=" + std::to_string(s.V) +
               (s.var == 1 ? ",tma" : "") + ")";
    if (s.mode == MODE_MIXC)
        return "cluster(C=" + std::to_string(s.C) + ",L=" + std::to_string(s.N2) + " per CTA,threads=" +
               std::to_string(s.V) + (s.var == 1 || s.var == 2 ? ",ctas_per_sm=3" : "") + (s.var >= 4 ? ",tma" : "") +
               ")";
    if (s.mode == MODE_CONVC)
        return pre + "cluster(C=" + std::to_string(s.C) + ",4096 per CTA,ctas_per_sm=" + std::to_string(s.V) + ")";
    if (s.mode == MODE_P2COL)
        return "pow2(N1=" + std::to_string(s.N1) + ",N2=4096,ctas_per_sm=" + std::to_string(s.V) +
               (s.var == 1 ? ",tma" : s.var == 2 ? ",dataflow" : "") + ")";
    if (s.mode == MODE_FOUR)
        return pre + "four(C=" + std::to_string(s.C) + ",N1=" + std::to_string(s.N1) +
               ",N2=" + std::to_string(s.N2) + ")[" + join(s.ra) + "|" + join(s.rc) + "]";
    return pre + "twopass(N1=" + std::to_string(s.N1) + ",N2=" + std::to_string(s.N2) + ")[" +
           join(s.ra) + "|" + join(s.rc) + "]";
}

// ---------------------------------------------------------- device tables
static int dev_upload(cfft_plan_s* P, const void* h, size_t bytes, void** d) {
    CUDA_TRY(lib_malloc(d, bytes));
    P->allocs.push_back(*d);
    CUDA_TRY(cudaMemcpy(*d, h, bytes, cudaMemcpyHostToDevice));
    return CFFT_OK;
}
static std::mutex g_tab_mu;
static std::map<std::string, DevPtr> g_tables;

static int dev_alloc(size_t bytes, DevPtr* out) {
    auto b = std::make_shared<DevBuf>();
    cudaError_t e = lib_malloc(&b->p, bytes);
    if (e != cudaSuccess) {
        b->p = nullptr;
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? CFFT_ERR_NOMEM : CFFT_ERR_CUDA,
                    std::string("table allocation: ") + cudaGetErrorString(e));
    }
    b->bytes = bytes;
    *out = b;
    return CFFT_OK;
}
// cached table: look `key` up (per device); on a miss build the host image
// with `make` and upload it
template <class F>
static int cached_table(cfft_plan_s* P, const std::string& key0, F make, const void** out) {
    const std::string key = std::to_string(P->device) + "/" + key0;
    {
        std::lock_guard<std::mutex> lk(g_tab_mu);
        auto it = g_tables.find(key);
        if (it != g_tables.end()) {
            P->tables.push_back(it->second);
            *out = it->second->p;
            return CFFT_OK;
        }
    }
    std::vector<unsigned char> img;
    make(img);
    DevPtr b;
    int rc = dev_alloc(img.size(), &b);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpy(b->p, img.data(), img.size(), cudaMemcpyHostToDevice));
    {
        std::lock_guard<std::mutex> lk(g_tab_mu);
        auto it = g_tables.find(key);
        if (it != g_tables.end()) b = it->second;   // another thread won the race
        else g_tables[key] = b;
    }
    P->tables.push_back(b);
    *out = b->p;
    return CFFT_OK;
}
template <class T> static void put(std::vector<unsigned char>& img, const std::vector<T>& v) {
    img.resize(v.size() * sizeof(T));
    memcpy(img.data(), v.data(), img.size());
}

// prefer_block: keep the block-wide team whenever its lanes span at least
// 128 bytes of adjacent sub-transforms (conflict-free shared-memory access in
// both the column layout, sub-transforms adjacent, and the row layout, odd
// pitch); warp-owned sub-transforms walk one sub-transform with a stride and
// collide on the banks when that stride is an even multiple of 128 bytes
static int make_subplan(cfft_plan_s* P, int64_t L, const std::vector<int>& rad, int64_t count,
                        SubPlan& sp, bool prefer_block = false) {
    memset(&sp, 0, sizeof sp);
    sp.L = (int)L;
    sp.np = (int)rad.size();
    if (sp.np > CFFT_MAXP) return fail(CFFT_ERR_UNSUPPORTED, "too many radix passes");
    // the device runs passes in CFFT_EXEC_ORDER (odd radices first)
    radix_counts(rad, sp.cnt);
    {
        auto ex = exec_order(rad);
        if ((int)ex.size() != sp.np) return fail(CFFT_ERR_UNSUPPORTED, "radix outside the codelet set");
        for (int i = 0; i < sp.np; i++) sp.radix[i] = (unsigned char)ex[i];
    }
    sp.G = std::max(1, wave_G(rad, L, CFFT_THREADS));
    // warp-synchronous mode when a warp can own whole sub-transforms and
    // there are enough of them to occupy every warp of the block
    int gw = wave_G(rad, L, 32);
    if (gw > 1 << 16) gw = 1 << 16;
    sp.Gwarp = 0;
    if (gw >= 1 && count >= (int64_t)(CFFT_THREADS / 32) * gw / 2) sp.Gwarp = gw;
    if (prefer_block && std::min<int64_t>(sp.G, count) * (int64_t)elem_bytes(P->dtype) >= 128) sp.Gwarp = 0;
    if (L <= 1) { sp.tw = nullptr; sp.twlen = 0; return CFFT_OK; }
    // per-pass blocks: pass (r, s), n1 = L/(s r): tw[off + (j-1) n1 + q] = w_L^(j q s)
    sp.twlen = (int)twiddle_len(L, rad);
    if (sp.twlen == 0) { sp.tw = nullptr; return CFFT_OK; }
    std::string key = "tw/" + std::to_string(P->dtype) + "/" + std::to_string(L) + "/" + join(rad);
    const int np = sp.np;
    unsigned char radix[CFFT_MAXP];
    memcpy(radix, sp.radix, sizeof radix);
    const int dtype = P->dtype;
    return cached_table(P, key, [&](std::vector<unsigned char>& img) {
        std::vector<double2> w;
        int64_t s = 1;
        for (int i = 0; i < np; i++) {
            const int r = radix[i];
            const int64_t n1 = L / (s * r);
            for (int j = 1; j < r; j++)
                for (int64_t q = 0; q < n1; q++) w.push_back(omega((int64_t)j * q * s, L, -1));
            s *= r;
        }
        if (dtype == CFFT_C128) {
            put(img, w);
        } else {
            std::vector<float2> t(w.size());
            for (size_t m = 0; m < w.size(); m++) t[m] = make_float2((float)w[m].x, (float)w[m].y);
            put(img, t);
        }
    }, &sp.tw);
}
static int make_twolevel(cfft_plan_s* P, int64_t N, TwoLevel& t) {
    const int bits = twolevel_bits(N);
    const int64_t lo_n = 1LL << bits, hi_n = (N + lo_n - 1) / lo_n + 1;
    const void* d = nullptr;
    int rc = cached_table(P, "tl/" + std::to_string(N), [&](std::vector<unsigned char>& img) {
        std::vector<double2> v(lo_n + hi_n);
        for (int64_t a = 0; a < lo_n; a++) v[a] = omega(a, N, -1);
        for (int64_t b = 0; b < hi_n; b++) v[lo_n + b] = omega(b * lo_n, N, -1);
        put(img, v);
    }, &d);
    if (rc) return rc;
    t.lo = (const double2*)d;
    t.hi = (const double2*)d + lo_n;
    t.bits = bits;
    t.N = (int)N;
    return CFFT_OK;
}

static int plan_build(cfft_plan_s* P, const Shape& sh);
static int plan_execute(cfft_plan_s* P, const void* in, void* out, int dir, cudaStream_t st,
                        int64_t nbatch = -1, int64_t in_dist = -1, int64_t out_dist = -1);
static void plan_free(cfft_plan_s* P);

static int plan_create_impl(cfft_plan_s** out, int64_t n, int64_t batch, int dtype, int flags);

// cached table built on the device by `build(dptr)` on a miss
template <class F>
static int cached_dev_table(cfft_plan_s* P, const std::string& key0, size_t bytes, F build,
                            const void** out) {
    const std::string key = std::to_string(P->device) + "/" + key0;
    {
        std::lock_guard<std::mutex> lk(g_tab_mu);
        auto it = g_tables.find(key);
        if (it != g_tables.end()) {
            P->tables.push_back(it->second);
            *out = it->second->p;
            return CFFT_OK;
        }
    }
    DevPtr b;
    int rc = dev_alloc(bytes, &b);
    if (rc) return rc;
    rc = build(b->p);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(0));
    {
        std::lock_guard<std::mutex> lk(g_tab_mu);
        auto it = g_tables.find(key);
        if (it != g_tables.end()) b = it->second;
        else g_tables[key] = b;
    }
    P->tables.push_back(b);
    *out = b->p;
    return CFFT_OK;
}

// smooth FP64 plans (batch 1) that transform convolution kernel vectors,
// cached per (device, M)
static std::mutex g_spec_mu;
static std::map<std::pair<int, int64_t>, cfft_plan_s*> g_spec_plans;
static int spectrum_plan(int dev, int64_t M, cfft_plan_s** out) {
    std::lock_guard<std::mutex> lk(g_spec_mu);
    auto it = g_spec_plans.find({dev, M});
    if (it != g_spec_plans.end()) { *out = it->second; return CFFT_OK; }
    cfft_plan_s* S = nullptr;
    int rc = plan_create_impl(&S, M, 1, CFFT_C128, CFFT_NO_FLAG);
    if (rc) return rc;
    g_spec_plans[{dev, M}] = S;
    *out = S;
    return CFFT_OK;
}
// spectrum = FFT_M(b') / M in FP64, b' generated in place by `gen`
template <class G>
static int conv_spectrum(cfft_plan_s* P, const std::string& key, int64_t M, G gen, const double2** out) {
    cfft_plan_s* S = nullptr;
    int rc = spectrum_plan(P->device, M, &S);
    if (rc) return rc;
    const void* d = nullptr;
    rc = cached_dev_table(P, key, (size_t)M * sizeof(double2), [&](void* dp) -> int {
        double2* v = (double2*)dp;
        CUDA_TRY(gen(v));
        int r = plan_execute(S, v, v, CFFT_FORWARD, 0);
        if (r) return r;
        CUDA_TRY(cfft_scale(v, M, 1.0 / (double)M, 0));
        return CFFT_OK;
    }, &d);
    *out = (const double2*)d;
    return rc;
}

static int make_conv_tables(cfft_plan_s* P, const Shape& sh, KParams& kp, std::string* spec_key) {
    const int64_t n = P->n, M = sh.M;
    const std::string tag = std::to_string(n) + "/" + std::to_string(M);
    if (sh.conv == CONV_RADER) {
        const int64_t L = n - 1;
        const void* dperm = nullptr;
        // perm[j] = g^j mod n and iperm[j] = g^-j mod n (prime.jl:9-33), one buffer
        int rc = cached_table(P, "pm/" + std::to_string(n), [&](std::vector<unsigned char>& img) {
            const int64_t g = primitive_root(n), ginv = powmod(g, n - 2, n);
            std::vector<int> v(2 * L);
            int64_t a = 1, c = 1;
            for (int64_t i = 0; i < L; i++) {
                v[i] = (int)a;
                v[L + i] = (int)c;
                a = (int64_t)(((__int128)a * g) % n);
                c = (int64_t)(((__int128)c * ginv) % n);
            }
            put(img, v);
        }, &dperm);
        if (rc) return rc;
        kp.perm = (const int*)dperm;
        kp.iperm = (const int*)dperm + L;
        // W[m] = w^(-g^-m): the reference's recurrence (prime.jl:36-37) or exact
        const int exact = (P->flags & CFFT_EXACT_TWIDDLES) ? 1 : 0;
        double2 winv = make_double2(1, 0);
        if (!exact) {
            // cispi(T(2/n)) at the rounded argument 2/n, then Julia's inv
            const double arg = 2.0 / (double)n;
            const long double x = 3.141592653589793238462643383279502884L * (long double)arg;
            winv = julia_inv(make_double2((double)cosl(x), (double)sinl(x)));
        }
        const int* iperm = kp.iperm;
        *spec_key = "sr/" + tag + "/" + std::to_string(exact);
        return conv_spectrum(P, *spec_key, M, [&](double2* v) {
            return cfft_gen_rader_b(v, iperm, n, M, exact, winv, 0);
        }, &kp.spec);
    }
    // Bluestein: chirp[j] = exp(-i pi j^2 / n); b'[m] = conj(chirp[|m|])
    const void* dch = nullptr;
    int rc = cached_dev_table(P, "ch/" + std::to_string(n), (size_t)n * sizeof(double2), [&](void* dp) -> int {
        CUDA_TRY(cfft_gen_chirp((double2*)dp, n, 0));
        return CFFT_OK;
    }, &dch);
    if (rc) return rc;
    kp.chirp = (const double2*)dch;
    const double2* ch = kp.chirp;
    *spec_key = "sb/" + tag;
    return conv_spectrum(P, *spec_key, M, [&](double2* v) {
        return cfft_gen_bluestein_b(v, ch, n, M, 0);
    }, &kp.spec);
}

// bytes of intermediate one chunk of a two-pass plan may use: 64 MB for the
// generic passes (the intermediate then stays in the 126 MB L2) and 512 MB
// for the power-of-two register passes (measured on B200 at 1 GiB batches:
// fewer, longer persistent launches beat L2 residency by 7-20 %);
// CFFT_SCRATCH_MB overrides both (read at plan creation)
static int64_t scratch_budget(bool pow2 = false) {
    const char* v = getenv("CFFT_SCRATCH_MB");
    const long long mb = v ? atoll(v) : 0;
    if (mb > 0 && mb <= (1LL << 20)) return (int64_t)mb << 20;
    return (int64_t)(pow2 ? 512 : 64) << 20;
}

static int plan_build(cfft_plan_s* P, const Shape& sh) {
    P->shape = sh;
    P->stages.clear();
    P->desc = shape_desc(sh, P->n);
    const size_t e = elem_bytes(P->dtype);
    KParams kp;
    memset(&kp, 0, sizeof kp);
    kp.conv = sh.conv;
    kp.nx = (int)P->n;
    kp.M = (int)sh.M;
    int rc;
    if (sh.conv != CONV_NONE) {
        std::string spec_key;
        rc = make_conv_tables(P, sh, kp, &spec_key);
        if (rc) return rc;
        if (sh.mode == MODE_FOUR && sh.conv == CONV_RADER) {
            // the cluster kernels read the permutations in their own order:
            // entry c*N1*W + i1*W + j for position jj = i1*N2 + c*W + j holds
            // (owner << 24 | offset) of g^(+-jj) within the C x chunks of
            // ceil(n/C) elements, or -1 for the zero padding jj >= n - 1
            const int64_t n = P->n, L = n - 1, N1 = sh.N1, N2 = sh.N2, C = sh.C, W = N2 / C;
            const int64_t XC = (n + C - 1) / C;
            const void* d = nullptr;
            rc = cached_table(P, "pmc/" + std::to_string(n) + "/" + std::to_string(N1) + "/" + std::to_string(N2) +
                                     "/" + std::to_string(C),
                              [&](std::vector<unsigned char>& img) {
                const int64_t g = primitive_root(n), ginv = powmod(g, n - 2, n);
                std::vector<int> fw(L), bw(L);
                int64_t a = 1, b = 1;
                for (int64_t i = 0; i < L; i++) {
                    fw[i] = (int)a;
                    bw[i] = (int)b;
                    a = (int64_t)(((__int128)a * g) % n);
                    b = (int64_t)(((__int128)b * ginv) % n);
                }
                std::vector<int> v(2 * (size_t)N1 * N2);
                for (int64_t c = 0; c < C; c++)
                    for (int64_t i1 = 0; i1 < N1; i1++)
                        for (int64_t j = 0; j < W; j++) {
                            const int64_t jj = i1 * N2 + c * W + j, at = c * N1 * W + i1 * W + j;
                            auto code = [&](int64_t s) { return (int)(((s / XC) << 24) | (s % XC)); };
                            v[at] = jj < L ? code(fw[jj]) : -1;
                            v[N1 * N2 + at] = jj < L ? code(bw[jj]) : -1;
                        }
                put(img, v);
            }, &d);
            if (rc) return rc;
            kp.perm = (const int*)d;
            kp.iperm = (const int*)d + N1 * N2;
        }
        if (sh.mode == MODE_FOUR) {
            // the cluster kernels read the spectrum in row-major (k1, k2) order
            const double2* nat = kp.spec;
            const void* d = nullptr;
            const int64_t N1 = sh.N1, N2 = sh.N2;
            rc = cached_dev_table(P, spec_key + "/rm" + std::to_string(N1), (size_t)sh.M * sizeof(double2),
                                  [&](void* dp) -> int {
                                      CUDA_TRY(cfft_spec_rowmajor((double2*)dp, nat, N1, N2, 0));
                                      return CFFT_OK;
                                  }, &d);
            if (rc) return rc;
            kp.spec = (const double2*)d;
        }
    }
    if (sh.mode == MODE_P2CL) {
        // power-of-two n = C x 4096 in one pass on clusters of C CTAs
        kp.mode = MODE_P2CL;
        kp.C = sh.C;
        rc = make_twolevel(P, 4096, kp.t4);
        if (rc) return rc;
        rc = make_twolevel(P, P->n, kp.t4n);
        if (rc) return rc;
        Stage s;
        s.kp = kp;
        s.threads = CFFT_THREADS;
        s.smem = cfft_r4096_smem(e);
        s.cluster = sh.C;
        s.grid = 0;
        s.in_sel = 0;
        s.out_sel = 1;
        s.fn = sh.var == 1 ? cfft_p2cl_tma_kernel(sh.C) : cfft_p2cl_kernel(P->dtype, sh.C, sh.V);
        s.launch = sh.var == 1 ? 5 : 0;
        if (!s.fn) return fail(CFFT_ERR_UNSUPPORTED, "no power-of-two cluster kernel for C=" + std::to_string(sh.C));
        CUDA_TRY(cfft_prepare_fn(s.fn, s.smem, sh.C));
        int nclusters = 0;
        cudaError_t ce = cfft_max_active_clusters_fn(s.fn, CFFT_THREADS, s.smem, sh.C, &nclusters);
        if (ce != cudaSuccess || nclusters < 1) {
            cudaGetLastError();
            return fail(CFFT_ERR_UNSUPPORTED, "cluster configuration not schedulable: C=" + std::to_string(sh.C));
        }
        s.max_units = nclusters;
        P->stages.push_back(s);
        P->chunk = P->batch;
        return CFFT_OK;
    }
    if (sh.mode == MODE_MIXC) {
        // n = C x L on a cluster of C register L-point CTAs
        const void* fn = nullptr;
        int C = 0, L = 0, T = 0;
        if (!cfft_mixc_lookup(P->n, P->dtype == CFFT_C128 ? CFFT_DT_C128 : CFFT_DT_C64, sh.var, &fn, &C, &L, &T))
            return fail(CFFT_ERR_UNSUPPORTED, "no cluster kernel for n=" + std::to_string(P->n));
        kp.mode = MODE_MIXC;
        kp.C = C;
        kp.N1 = C;
        kp.N2 = L;
        rc = make_twolevel(P, L, kp.t4);
        if (rc) return rc;
        rc = make_twolevel(P, P->n, kp.t4n);
        if (rc) return rc;
        const int nlo = 1 << kp.t4.bits, nhi = (L + nlo - 1) / nlo + 1;
        const int mlo = 1 << kp.t4n.bits, mhi = (int)((P->n + mlo - 1) / mlo + 1);
        Stage s;
        s.kp = kp;
        s.threads = T;
        s.smem = (((size_t)L * e + 15) & ~(size_t)15) +
                 (size_t)(nlo + nhi + (sh.var == 1 ? 0 : mlo + mhi)) * sizeof(double2) +
                 (sh.var >= 4 ? 16 : 0);      // the tensor copies' mbarrier
        s.launch = sh.var >= 4 ? 4 : 0;
        s.cluster = C;
        s.grid = 0;
        s.in_sel = 0;
        s.out_sel = 1;
        s.fn = fn;
        CUDA_TRY(cfft_prepare_fn(s.fn, s.smem, C));
        int nclusters = 0;
        cudaError_t ce = cfft_max_active_clusters_fn(s.fn, T, s.smem, C, &nclusters);
        if (ce != cudaSuccess || nclusters < 1) {
            cudaGetLastError();
            return fail(CFFT_ERR_UNSUPPORTED, "cluster configuration not schedulable: C=" + std::to_string(C));
        }
        s.max_units = nclusters;
        P->stages.push_back(s);
        P->chunk = P->batch;
        return CFFT_OK;
    }
    if (sh.mode == MODE_CONVC) {
        // Rader on C register 4096-point CTAs: permutations in the kernel's
        // order (CTA c, slot i <-> convolution index c + C i)
        const int64_t n = P->n, L = n - 1, C = sh.C;
        const void* d = nullptr;
        rc = cached_table(P, "pc/" + std::to_string(n) + "/" + std::to_string(C), [&](std::vector<unsigned char>& img) {
            const int64_t g = primitive_root(n), ginv = powmod(g, n - 2, n);
            std::vector<int> fw(L), bw(L);
            int64_t a = 1, b = 1;
            for (int64_t i = 0; i < L; i++) {
                fw[i] = (int)a;
                bw[i] = (int)b;
                a = (int64_t)(((__int128)a * g) % n);
                b = (int64_t)(((__int128)b * ginv) % n);
            }
            std::vector<int> v(2 * (size_t)sh.M);
            for (int64_t c = 0; c < C; c++)
                for (int64_t i = 0; i < 4096; i++) {
                    const int64_t j = c + C * i;
                    v[c * 4096 + i] = j < L ? fw[j] : -1;
                    v[sh.M + c * 4096 + i] = j < L ? bw[j] : -1;
                }
            put(img, v);
        }, &d);
        if (rc) return rc;
        kp.mode = MODE_CONVC;
        kp.C = (int)C;
        kp.perm = (const int*)d;
        kp.iperm = (const int*)d + sh.M;
        rc = make_twolevel(P, 4096, kp.t4);
        if (rc) return rc;
        rc = make_twolevel(P, sh.M, kp.t4n);
        if (rc) return rc;
        Stage s;
        s.kp = kp;
        s.threads = CFFT_THREADS;
        s.smem = cfft_convc_smem(e);
        s.cluster = (int)C;
        s.grid = 0;
        s.in_sel = 0;
        s.out_sel = 1;
        s.fn = cfft_convc_kernel(P->dtype, (int)C, sh.V);
        if (!s.fn) return fail(CFFT_ERR_UNSUPPORTED, "no cluster Rader kernel for C=" + std::to_string(C));
        CUDA_TRY(cfft_prepare_fn(s.fn, s.smem, (int)C));
        int nclusters = 0;
        cudaError_t ce = cfft_max_active_clusters_fn(s.fn, CFFT_THREADS, s.smem, (int)C, &nclusters);
        if (ce != cudaSuccess || nclusters < 1) {
            cudaGetLastError();
            return fail(CFFT_ERR_UNSUPPORTED, "cluster configuration not schedulable: C=" + std::to_string(C));
        }
        s.max_units = nclusters;
        P->stages.push_back(s);
        P->chunk = P->batch;
        return CFFT_OK;
    }
    if (sh.mode == MODE_ROWS) {
        kp.mode = MODE_ROWS;
        kp.V = sh.V;
        kp.PC = (int)(sh.M + ((sh.M % 2 == 0) ? 1 : 0));
        kp.XP = (sh.conv == CONV_RADER) ? (int)P->n : 0;
        kp.mX = magic(P->n);
        kp.mM = magic(sh.M);
        kp.mL = magic(std::max<int64_t>(1, P->n - 1));
        rc = make_subplan(P, sh.M, sh.rc, sh.V, kp.pc);
        if (rc) return rc;
        Stage s;
        s.kp = kp;
        s.threads = CFFT_THREADS;
        s.smem = sh.smem;
        s.cluster = 1;
        s.grid = 0;  // set per execution from batch
        s.in_sel = 0;
        s.out_sel = 1;
        s.fn = cfft_kernel_for(MODE_ROWS, P->dtype);
        if (sh.conv == CONV_NONE && sh.M == 4096 && sh.V == 1) {
            // the register kernel; descriptor-driven launches keep the
            // generic rows kernel and its shared memory
            rc = make_twolevel(P, 4096, s.kp.t4);
            if (rc) return rc;
            s.fn = cfft_r4096_kernel(P->dtype);
            s.smem_batched = sh.smem;
            s.smem = cfft_r4096_smem(elem_bytes(P->dtype));
            P->desc += "+r4096";
        }
        CUDA_TRY(cfft_prepare_fn(s.fn, s.smem, 1));
        if (s.fn == cfft_r4096_kernel(P->dtype)) {
            // persistent: as many CTAs as are co-resident
            int nsm = 0, occ = 0;
            CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, P->device));
            CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, s.fn, CFFT_THREADS, s.smem));
            s.persist = (unsigned)(std::max(1, occ) * std::max(1, nsm));
        }
        P->stages.push_back(s);
        P->chunk = P->batch;
        return CFFT_OK;
    }
    if (sh.mode == MODE_FOUR) {
        kp.mode = MODE_FOUR;
        kp.N1 = sh.N1;
        kp.N2 = sh.N2;
        kp.C = sh.C;
        if (sh.C == 1) {
            kp.PA = kp.PC = sh.N2 + ((sh.N2 % 2 == 0) ? 1 : 0);
        } else {
            kp.PA = sh.N2 / sh.C;
            kp.PC = sh.N2 + ((sh.N2 % 2 == 0) ? 1 : 0);
        }
        kp.XP = (sh.conv == CONV_RADER) ? (int)((P->n + sh.C - 1) / sh.C) : 0;
        kp.mW = magic(sh.N2 / sh.C);
        kp.mN2 = magic(sh.N2);
        kp.mR1 = magic(sh.N1 / sh.C);
        kp.mX = magic(std::max(kp.XP, 1));
        rc = make_subplan(P, sh.N1, sh.ra, sh.N2 / sh.C, kp.pa, P->dtype == CFFT_C64);
        if (rc) return rc;
        rc = make_subplan(P, sh.N2, sh.rc, sh.N1 / sh.C, kp.pc, P->dtype == CFFT_C64);
        if (rc) return rc;
        rc = make_twolevel(P, sh.M, kp.t4);
        if (rc) return rc;
        Stage s;
        s.kp = kp;
        s.threads = CFFT_THREADS;
        s.smem = sh.smem;
        s.smem_batched = sh.smem_dyn;
        s.cluster = sh.C;
        s.grid = 0;
        s.in_sel = 0;
        s.out_sel = 1;
        s.fn = cfft_static_four(P->dtype, sh.N1, sh.N2, sh.C, kp.pa.cnt, kp.pc.cnt);
        if (s.fn) {
            P->desc += "+static";
        } else if (kp.pa.Gwarp > 0 && kp.pc.Gwarp > 0) {
            s.fn = cfft_kernel_for(MODE_FOUR_WARP, P->dtype);
            P->desc += "+warp";
        } else {
            // one team kind per kernel: both sub-plans block-wide
            s.fn = cfft_kernel_for(MODE_FOUR, P->dtype);
            s.kp.pa.Gwarp = 0;
            s.kp.pc.Gwarp = 0;
        }
        CUDA_TRY(cfft_prepare_fn(s.fn, s.smem, sh.C));
        {
            int nclusters = 0;
            cudaError_t ce = cfft_max_active_clusters_fn(s.fn, CFFT_THREADS, s.smem, sh.C, &nclusters);
            if (ce != cudaSuccess || nclusters < 1) {
                cudaGetLastError();
                return fail(CFFT_ERR_UNSUPPORTED, "cluster configuration not schedulable: C=" +
                                                      std::to_string(sh.C));
            }
            s.max_units = nclusters;
        }
        P->stages.push_back(s);
        P->chunk = P->batch;
        return CFFT_OK;
    }
    if (sh.mode == MODE_P2COL) {
        // power-of-two n = N1 x 4096 (pow2.cuh): pass A = the n = 4096
        // kernel over the N1 stride-N1 subsequences, into an L2-sized
        // intermediate; pass B = the N1-point column DFTs into the output
        const int64_t n = P->n, N1 = sh.N1;
        const int mb = sh.V;
        TwoLevel tn, t4096;
        rc = make_twolevel(P, n, tn);
        if (rc) return rc;
        rc = make_twolevel(P, 4096, t4096);
        if (rc) return rc;
        const void* w1 = nullptr;
        rc = cached_table(P, "w1/" + std::to_string(N1), [&](std::vector<unsigned char>& img) {
            std::vector<double2> v(N1);
            for (int64_t a = 0; a < N1; a++) v[a] = omega(a, N1, -1);
            put(img, v);
        }, &w1);
        if (rc) return rc;
        if (sh.var == 2) {
            // one persistent launch for the whole batch: a ring of `depth`
            // intermediates (in L2 where it fits) and the item counters
            const void* fn = cfft_p2flow_kernel(P->dtype, (int)N1);
            if (!fn) return fail(CFFT_ERR_UNSUPPORTED, "no dataflow kernel for N1=" + std::to_string(N1));
            const int nlo = 1 << tn.bits, nhi = (int)((n + nlo - 1) / nlo + 1);
            const size_t base = cfft_p2flow_smem(e, (int)N1, 0), tab = (size_t)(nlo + nhi) * sizeof(double2);
            const bool staged = base + tab <= (size_t)112 * 1024;
            Stage st;
            st.kp = kp;
            st.kp.mode = MODE_P2ROW;
            st.kp.N1 = (int)N1;
            st.kp.N2 = 4096;
            int lgN1 = 0;
            while ((1LL << lgN1) < N1) lgN1++;
            st.kp.PA = lgN1;
            st.kp.t4 = t4096;
            st.kp2 = kp;
            st.kp2.mode = MODE_P2COL;
            st.kp2.N1 = (int)N1;
            st.kp2.N2 = 4096;
            st.kp2.twN1 = (const double2*)w1;
            st.kp2.t4n = tn;
            st.kp2.pre = staged ? 1 : 0;
            st.threads = CFFT_THREADS;
            st.smem = cfft_p2flow_smem(e, (int)N1, staged ? nlo + nhi : 0);
            st.cluster = 1;
            st.in_sel = 0;
            st.out_sel = 1;
            st.fn = fn;
            st.launch = 2;
            CUDA_TRY(cfft_prepare_fn(st.fn, st.smem, 1));
            int nsm = 0, occ = 0;
            CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, P->device));
            CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, st.fn, CFFT_THREADS, st.smem));
            const int resident = std::max(1, occ) * std::max(1, nsm);
            st.persist = (unsigned)resident;
            // a transform's tiles are claimed about twice the resident CTAs
            // after its rows; the ring holds the transforms in between
            st.flow_lag = (int)std::max<int64_t>(1, (resident + 2 * N1 - 1) / (2 * N1));
            st.flow_depth = 2 * st.flow_lag + 1;
            P->chunk = P->batch;
            P->scratch_bytes = (size_t)st.flow_depth * n * e;
            if (!P->shared_scratch) {
                CUDA_TRY(lib_malloc(&P->scratch[0], P->scratch_bytes));
                P->allocs.push_back(P->scratch[0]);
            }
            CUDA_TRY(lib_malloc(&P->flow_ctr, (size_t)(2 + 2 * P->batch) * sizeof(int)));
            P->allocs.push_back(P->flow_ctr);
            P->stages.push_back(st);
            return CFFT_OK;
        }
        int64_t chunk = std::max<int64_t>(1, scratch_budget(true) / (int64_t)(n * e));
        chunk = std::min<int64_t>(chunk, P->batch);
        P->chunk = chunk;
        P->scratch_bytes = (size_t)chunk * n * e;
        if (!P->shared_scratch) {
            CUDA_TRY(lib_malloc(&P->scratch[0], P->scratch_bytes));
            P->allocs.push_back(P->scratch[0]);
        }
        int lg = 0;
        while ((1LL << lg) < N1) lg++;
        // pass B: two CTAs per SM for ComplexF64 (no spills), three for
        // ComplexF32; the w_n table rides in its shared memory when it fits
        const int mbB = (P->dtype == CFFT_C128) ? 2 : 3;
        const int nlo = 1 << tn.bits, nhi = (int)((n + nlo - 1) / nlo + 1);
        const size_t baseB = cfft_p2col_smem(e, (int)N1), tab = (size_t)(nlo + nhi) * sizeof(double2);
        const bool staged = baseB + tab <= (mbB == 2 ? (size_t)112 * 1024 : (size_t)74 * 1024);
        Stage a;
        a.kp = kp;
        a.kp.mode = MODE_P2ROW;
        a.kp.N1 = (int)N1;
        a.kp.N2 = 4096;
        a.kp.PA = lg;
        a.kp.t4 = t4096;
        a.threads = CFFT_THREADS;
        a.smem = cfft_r4096_smem(e);
        a.cluster = 1;
        a.in_sel = 0;
        a.out_sel = 2;
        a.fn = sh.var == 1 ? cfft_p2row_tma_kernel(mb) : cfft_p2row_kernel(P->dtype, mb);
        a.launch = sh.var == 1 ? 1 : 0;
        if (sh.var == 1 && P->dtype != CFFT_C128) {
            // ComplexF32: subsequence pairs per tensor-copy item
            a.fn = cfft_p2row_tma2_kernel();
            a.smem = cfft_p2row_tma2_smem();
            a.launch = 3;
        }
        Stage b;
        b.kp = kp;
        b.kp.mode = MODE_P2COL;
        b.kp.N1 = (int)N1;
        b.kp.N2 = 4096;
        b.kp.twN1 = (const double2*)w1;
        b.kp.t4n = tn;
        b.kp.pre = staged ? 1 : 0;
        b.threads = CFFT_THREADS;
        b.smem = baseB + (staged ? tab : 0);
        b.cluster = 1;
        b.in_sel = 2;
        b.out_sel = 1;
        b.fn = cfft_p2col_kernel(P->dtype, (int)N1, mbB);
        int nsm = 0;
        CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, P->device));
        for (Stage* st : {&a, &b}) {
            if (!st->fn) return fail(CFFT_ERR_UNSUPPORTED, "no power-of-two kernel for N1=" + std::to_string(N1));
            CUDA_TRY(cfft_prepare_fn(st->fn, st->smem, 1));
            int occ = 0;
            CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, st->fn, CFFT_THREADS, st->smem));
            st->persist = (unsigned)(std::max(1, occ) * std::max(1, nsm));
        }
        P->stages.push_back(a);
        P->stages.push_back(b);
        return CFFT_OK;
    }
    // two HBM passes per FFT_M (and two FFT_M for a convolution)
    const int64_t N1 = sh.N1, N2 = sh.N2, M = sh.M;
    const int64_t PC = N2 + ((N2 % 2 == 0) ? 1 : 0);
    int64_t Vc = 1, Vr = 1;
    {
        long long vc = 1, vr = 1;
        cfft_pass_tiles(N1, N2, PC, (int)twiddle_len(N1, sh.ra), (int)twiddle_len(N2, sh.rc), twolevel_bits(M),
                        (int)M, e, &vc, &vr);
        Vc = vc;
        Vr = vr;
    }
    SubPlan pa, pc;
    rc = make_subplan(P, N1, sh.ra, Vc, pa, true);
    if (rc) return rc;
    rc = make_subplan(P, N2, sh.rc, Vr, pc, true);
    if (rc) return rc;
    TwoLevel t4;
    rc = make_twolevel(P, M, t4);
    if (rc) return rc;
    // chunk the batch so the scratch of one chunk stays within ~64 MB (L2 sized)
    const int nscr = (sh.conv == CONV_NONE) ? 1 : 2;
    int64_t chunk = std::max<int64_t>(1, scratch_budget() / (int64_t)(M * e * nscr));
    chunk = std::min<int64_t>(chunk, P->batch);
    P->chunk = chunk;
    P->scratch_bytes = (size_t)chunk * M * e;
    if (!P->shared_scratch) {
        for (int i = 0; i < nscr; i++) {
            CUDA_TRY(lib_malloc(&P->scratch[i], P->scratch_bytes));
            P->allocs.push_back(P->scratch[i]);
        }
    }
    auto col = [&](int pre, int in_sel, int out_sel) {
        Stage s;
        s.kp = kp;
        s.kp.mode = MODE_COLPASS;
        s.kp.N1 = (int)N1;
        s.kp.N2 = (int)N2;
        s.kp.V = (int)Vc;
        s.kp.PA = (int)Vc;
        s.kp.mV = magic(Vc);
        s.kp.pa = pa;
        s.kp.t4 = t4;
        s.kp.pre = pre;
        s.threads = CFFT_THREADS;
        s.smem = cfft_colpass_smem(pa.twlen, t4.bits, t4.N, (int)(N1 * Vc), (int)e);
        s.cluster = 1;
        s.in_sel = in_sel;
        s.out_sel = out_sel;
        return s;
    };
    auto row = [&](int post, int in_sel, int out_sel) {
        Stage s;
        s.kp = kp;
        s.kp.mode = MODE_ROWPASS;
        s.kp.N1 = (int)N1;
        s.kp.N2 = (int)N2;
        s.kp.V = (int)Vr;
        s.kp.PC = (int)PC;
        s.kp.mV = magic(Vr);
        s.kp.mN2 = magic(N2);
        s.kp.pc = pc;
        s.kp.post = post;
        s.threads = CFFT_THREADS;
        s.smem = (size_t)(cfft_pass_tw_elems(pc.twlen, (int)e) + Vr * PC) * e + 16;
        s.cluster = 1;
        s.in_sel = in_sel;
        s.out_sel = out_sel;
        return s;
    };
    if (sh.conv == CONV_NONE) {
        P->stages.push_back(col(PRE_NONE, 0, 2));
        P->stages.push_back(row(POST_OUT, 2, 1));
    } else {
        P->stages.push_back(col(PRE_CHIRP, 0, 2));
        P->stages.push_back(row(POST_RAW, 2, 3));
        P->stages.push_back(col(PRE_SPEC, 3, 2));
        P->stages.push_back(row(POST_CHIRP, 2, 1));
    }
    for (auto& s : P->stages) {
        s.fn = cfft_kernel_for(s.kp.mode, P->dtype);
        CUDA_TRY(cfft_prepare_fn(s.fn, s.smem, 1));
    }
    return CFFT_OK;
}

// the host entry's pipeline (device chunk buffers, streams, events, pinned
// staging), whatever part of it exists
static void host_release(cfft_plan_s* P) {
    for (int i = 0; i < 3; i++) {
        lib_free(P->host_buf[i]);
        P->host_buf[i] = nullptr;
        if (P->host_st[i]) cudaStreamDestroy(P->host_st[i]);
        if (P->ev_in[i]) cudaEventDestroy(P->ev_in[i]);
        if (P->ev_comp[i]) cudaEventDestroy(P->ev_comp[i]);
        if (P->ev_out[i]) cudaEventDestroy(P->ev_out[i]);
        P->host_st[i] = nullptr;
        P->ev_in[i] = P->ev_comp[i] = P->ev_out[i] = nullptr;
        lib_free_host(P->stage_in[i]);
        lib_free_host(P->stage_out[i]);
        P->stage_in[i] = P->stage_out[i] = nullptr;
    }
    P->host_ready = false;
}

static void plan_free(cfft_plan_s* P) {
    host_release(P);
    for (void* p : P->allocs) lib_free(p);
    P->allocs.clear();
    P->tables.clear();
    P->stages.clear();
    P->scratch[0] = P->scratch[1] = nullptr;
    P->flow_ctr = nullptr;
}

// in_dist / out_dist: elements between consecutive transforms of the caller's
// input and output (default n)
static int plan_execute(cfft_plan_s* P, const void* in, void* out, int dir, cudaStream_t st,
                        int64_t nbatch, int64_t in_dist, int64_t out_dist) {
    if (dir < 0 || dir > 2) return fail(CFFT_ERR_INVALID, "direction must be 0, 1 or 2");
    const size_t e = elem_bytes(P->dtype);
    const int64_t n = P->n;
    const int64_t total = (nbatch < 0) ? P->batch : std::min(nbatch, P->batch);
    const int64_t idist = in_dist < 0 ? n : in_dist, odist = out_dist < 0 ? n : out_dist;
    // the caller's element sizes (ComplexF16 in fused plans)
    const size_t ei = P->in_fmt == IO_HALF ? 4 : e, eo = P->out_fmt == IO_HALF ? 4 : e;
    if (((uintptr_t)in % ei) != 0 || ((uintptr_t)out % eo) != 0)
        return fail(CFFT_ERR_INVALID, "buffers must be aligned to the element size");
    for (int64_t b0 = 0; b0 < total; b0 += P->chunk) {
        const int64_t nb = std::min(P->chunk, total - b0);
        for (auto& s : P->stages) {
            KParams kp = s.kp;
            kp.dir = dir;
            kp.scale = (dir == CFFT_INVERSE) ? 1.0 / (double)n : 1.0;
            kp.batch = (int)nb;
            const bool p2 = kp.mode == MODE_P2COL || kp.mode == MODE_P2ROW;
            if (p2) kp.batch = (int)(nb * kp.N1);     // column tiles / rows
            const char* user_in = (const char*)in + (size_t)b0 * idist * ei;
            char* user_out = (char*)out + (size_t)b0 * odist * eo;
            auto sel = [&](int w) -> void* {
                return w == 0 ? (void*)user_in : w == 1 ? (void*)user_out : P->scratch[w - 2];
            };
            kp.in = sel(s.in_sel);
            kp.out = sel(s.out_sel);
            auto dist = [&](int sel) -> int64_t { return sel >= 2 ? P->shape.M : sel == 0 ? idist : odist; };
            kp.in_dist = dist(s.in_sel);
            kp.out_dist = dist(s.out_sel);
            if (kp.mode == MODE_P2ROW) kp.out_dist = 4096;  // rows of the intermediate
            if (s.in_sel == 0 && P->in_fmt != IO_PLAIN) {
                kp.in_fmt = (unsigned char)P->in_fmt;
                kp.in_stride = P->strided ? P->istride : 1;
            }
            if (s.out_sel == 1 && P->out_fmt != IO_PLAIN) {
                kp.out_fmt = (unsigned char)P->out_fmt;
                kp.out_stride = P->strided ? P->ostride : 1;
            }
            unsigned grid;
            if (p2) grid = (unsigned)kp.batch;
            else if (kp.mode == MODE_ROWS) grid = (unsigned)((nb + kp.V - 1) / kp.V);
            else if (kp.mode == MODE_FOUR || kp.mode == MODE_CONVC || kp.mode == MODE_MIXC || kp.mode == MODE_P2CL)
                grid = (unsigned)(nb * kp.C);
            else if (kp.mode == MODE_COLPASS) grid = (unsigned)(nb * (kp.N2 / kp.V));
            else grid = (unsigned)(nb * (kp.N1 / kp.V));
            if (s.persist && grid > s.persist) grid = s.persist;
            cudaError_t ce;
            if (s.launch == 2) {
                // pass A reads the caller's input, pass B writes the caller's output
                KParams kb = s.kp2;
                kb.dir = kp.dir;
                kb.scale = kp.scale;
                kb.batch = (int)nb;
                kb.out = kp.out;
                kb.out_dist = odist;
                kp.batch = (int)nb;
                ce = cudaMemsetAsync(P->flow_ctr, 0, (size_t)(2 + 2 * nb) * sizeof(int), st);
                if (ce == cudaSuccess)
                    ce = cfft_launch_p2flow(s.fn, kp, kb, P->flow_ctr, P->scratch[0], (int)nb, s.flow_lag,
                                            s.flow_depth, s.persist, s.smem, st);
            } else if (s.launch == 1) {
                ce = cfft_launch_p2row_tma(s.fn, kp, grid, s.smem, st);
            } else if (s.launch == 3) {
                ce = cfft_launch_p2row_tma2(s.fn, kp, grid, s.smem, st);
            } else if (s.launch == 4) {
                ce = cfft_launch_mixc_tma(s.fn, kp, grid, s.threads, s.smem, s.cluster, st);
            } else if (s.launch == 5) {
                ce = cfft_launch_p2cl_tma(s.fn, kp, grid, s.smem, s.cluster, st);
            } else {
                ce = cfft_launch_fn(s.fn, kp, grid, s.threads, s.smem, s.cluster, st);
            }
            if (ce != cudaSuccess)
                return fail(CFFT_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(ce));
        }
    }
    return CFFT_OK;
}

// ------------------------------------------------------- autotune (MEASURE)
static float time_plan(cfft_plan_s* P, void* buf) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    plan_execute(P, buf, buf, 0, 0);
    cudaEventRecord(a, 0);
    const int reps = 3;
    for (int i = 0; i < reps; i++) plan_execute(P, buf, buf, 0, 0);
    cudaEventRecord(b, 0);
    cudaError_t ce = cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (ce != cudaSuccess) { cudaGetLastError(); return 1e30f; }
    return ms / reps;
}

// ------------------------------------------------------------------ wisdom
// Shapes chosen by MEASURE / ENCHANT, keyed by (n, batch, dtype, flags), so
// a later process can skip the timing: the reference's intent for its
// serialisable Spell (src/spells.jl:180-375, left unfinished there).  An
// entry names a shape by its signature; on use it must still be one of the
// planner's candidates for that key, else the planner times as usual.
struct WisdomKey {
    int64_t n, batch;
    int dtype, flags;
    bool operator<(const WisdomKey& o) const {
        return std::tie(n, batch, dtype, flags) < std::tie(o.n, o.batch, o.dtype, o.flags);
    }
};
static std::mutex g_wis_mu;
static std::map<WisdomKey, std::string> g_wisdom;

static std::string shape_signature(const Shape& s) {
    std::string r = std::to_string(s.mode) + " " + std::to_string(s.conv) + " " + std::to_string(s.M) + " " +
                    std::to_string(s.N1) + " " + std::to_string(s.N2) + " " + std::to_string(s.C) + " " +
                    std::to_string(s.V) + " a";
    for (int x : s.ra) r += " " + std::to_string(x);
    r += " c";
    for (int x : s.rc) r += " " + std::to_string(x);
    if (s.var) r += " v" + std::to_string(s.var);
    return r;
}
static bool wisdom_lookup(const WisdomKey& k, std::string& sig) {
    std::lock_guard<std::mutex> lk(g_wis_mu);
    auto it = g_wisdom.find(k);
    if (it == g_wisdom.end()) return false;
    sig = it->second;
    return true;
}
static void wisdom_store(const WisdomKey& k, const std::string& sig) {
    std::lock_guard<std::mutex> lk(g_wis_mu);
    g_wisdom[k] = sig;
}

// a plan whose every stage is a generic kernel (rows, four-step, column or
// row pass: the bodies that address the caller's layout through KParams
// in_fmt / out_fmt) can read ComplexF16 or strided input and write it back
// in its own first and last kernel.  The register kernels keep contiguous
// data of the plan's type: their ComplexF16 and strided plans widen / gather
// in a sweep of their own (measured faster there: 4096 x 2^16 ComplexF32
// runs 1.76 ms on the register passes, 3.49 ms as generic two-pass).
static bool io_fusable(const cfft_plan_s* P) {
    for (const auto& st : P->stages) {
        const int m = st.kp.mode;
        if (m != MODE_ROWS && m != MODE_FOUR && m != MODE_COLPASS && m != MODE_ROWPASS) return false;
        if (st.launch != 0 || st.fn == cfft_r4096_kernel(P->dtype == CFFT_C128 ? CFFT_DT_C128 : CFFT_DT_C64))
            return false;
    }
    return !P->stages.empty();
}

static int plan_create_impl(cfft_plan_s** out, int64_t n, int64_t batch, int dtype, int flags) {
    if (!out) return fail(CFFT_ERR_INVALID, "plan pointer is null");
    if (dtype == CFFT_C32) {
        // ComplexF16 data, ComplexF32 arithmetic: a ComplexF32 plan plus one
        // working buffer the data is widened into and narrowed out of
        if (n < 1 || batch < 1) return fail(CFFT_ERR_INVALID, "n and batch must be >= 1");
        int rc = plan_create_impl(out, n, batch, CFFT_C64, flags);
        if (rc) return rc;
        cfft_plan_s* P = *out;
        P->io_half = true;
        if (io_fusable(P)) {
            // the first kernel widens as it loads, the last narrows as it stores
            P->io_fused = true;
            P->in_fmt = P->out_fmt = IO_HALF;
            P->desc = "f16+" + P->desc;
            return CFFT_OK;
        }
        P->desc = "f16io+" + P->desc;
        if (lib_malloc(&P->half_work, (size_t)n * batch * sizeof(float2)) != cudaSuccess) {
            cudaGetLastError();
            plan_free(P);
            delete P;
            *out = nullptr;
            return fail(CFFT_ERR_NOMEM, "ComplexF16 working buffer allocation failed");
        }
        P->allocs.push_back(P->half_work);
        return CFFT_OK;
    }
    if (n < 1 || batch < 1) return fail(CFFT_ERR_INVALID, "n and batch must be >= 1");
    if (dtype != CFFT_C128 && dtype != CFFT_C64)
        return fail(CFFT_ERR_INVALID, "dtype must be CFFT_C128, CFFT_C64 or CFFT_C32");
    if (n > (1LL << 26)) return fail(CFFT_ERR_UNSUPPORTED, "n above 2^26 is not supported");
    int level = flags & 3;
    if (level > 2) return fail(CFFT_ERR_INVALID, "flag must be NO_FLAG, MEASURE or ENCHANT");
    auto cands = candidate_shapes(n, dtype, batch);
    if (cands.empty()) return fail(CFFT_ERR_UNSUPPORTED, "no execution shape for n=" + std::to_string(n));
    cfft_plan_s* P = new cfft_plan_s();
    P->n = n;
    P->batch = batch;
    P->dtype = dtype;
    P->flags = flags;
    cudaGetDevice(&P->device);
    int rc = CFFT_ERR_UNSUPPORTED;
    if (level == CFFT_NO_FLAG) {
        int nomem = 0;
        std::string nomem_err;
        for (auto& c : cands) {
            rc = plan_build(P, c);
            if (rc == CFFT_OK) break;
            if (rc == CFFT_ERR_NOMEM && !nomem) {
                nomem = 1;
                nomem_err = g_err;
            }
            plan_free(P);
        }
        // an out-of-memory failure outranks a later shape the device rejects
        if (rc != CFFT_OK && nomem) rc = fail(CFFT_ERR_NOMEM, nomem_err);
    } else {
        const WisdomKey wk{n, batch, dtype, flags};
        std::string sig;
        if (wisdom_lookup(wk, sig)) {
            for (auto& c : cands) {
                if (shape_signature(c) != sig) continue;
                rc = plan_build(P, c);
                if (rc == CFFT_OK) {
                    *out = P;
                    return CFFT_OK;
                }
                plan_free(P);
                break;
            }
        }
        // MEASURE: the best few heuristic candidates; ENCHANT: all of them
        size_t limit = (level == CFFT_MEASURE) ? std::min<size_t>(cands.size(), 4) : cands.size();
        limit = std::min<size_t>(limit, 24);
        const size_t e = elem_bytes(dtype);
        void* buf = nullptr;
        if (lib_malloc(&buf, (size_t)n * batch * e) != cudaSuccess) {
            delete P;
            return fail(CFFT_ERR_NOMEM, "autotune buffer allocation failed");
        }
        cudaMemset(buf, 0, (size_t)n * batch * e);
        float best = 1e30f;
        int best_i = -1, cand_rc = CFFT_ERR_UNSUPPORTED;
        const char* logenv = getenv("CFFT_TUNE_LOG");      // diagnostics: one line per candidate
        const bool log = logenv && logenv[0] == '1';
        std::string cand_err;
        for (size_t i = 0; i < limit; i++) {
            const int brc = plan_build(P, cands[i]);
            if (brc == CFFT_OK) {
                float t = time_plan(P, buf);
                if (log)
                    fprintf(stderr, "cfft-tune n=%lld batch=%lld %s smem=%zu co-resident=%d %.4f ms\n",
                            (long long)n, (long long)batch, P->desc.c_str(), P->stages[0].smem,
                            P->stages[0].max_units, t);
                if (t < best) { best = t; best_i = (int)i; }
            } else {
                // an out-of-memory failure outranks a shape the device rejects
                if (cand_rc != CFFT_ERR_NOMEM) {
                    cand_rc = brc;
                    cand_err = g_err;
                }
                if (log) fprintf(stderr, "cfft-tune n=%lld candidate %zu failed: %s\n", (long long)n, i, g_err);
            }
            plan_free(P);
        }
        lib_free(buf);
        if (best_i < 0) {
            delete P;
            return fail(cand_rc, "no candidate plan ran: " + cand_err);
        }
        rc = plan_build(P, cands[best_i]);
        if (rc == CFFT_OK) wisdom_store(wk, shape_signature(cands[best_i]));
    }
    if (rc != CFFT_OK) {
        std::string keep = g_err;
        plan_free(P);
        delete P;
        cfft_set_last_error(keep.c_str());
        return rc;
    }
    *out = P;
    return CFFT_OK;
}


// ------------------------------------------------------------ batched form
// Many transforms of mixed lengths packed back to back, captured once into a
// CUDA graph per (input, output, direction).  Two schedules:
//  * work queue (default): every transform is planned as a single-CTA
//    kernel (rows, or a one-CTA four-step) that fits the queue kernel's
//    shared-memory budget, or else as two HBM passes; the work items (whole
//    single-CTA transforms and pass tiles) run in one launch whose CTAs each
//    claim the next item by ticket (kq_batch, QItem): two-pass transforms
//    largest first in chunks that
//    take turns on a ring of scratch slots (a chunk's first pass waits for
//    the chunk that last used its slot to finish), each stage's tiles waiting for
//    the previous stage of their transform, then the single-CTA transforms
//    largest first to fill the tail;
//  * grouped (CFFT_BATCH_GROUPED): transforms whose plan is a single kernel
//    (rows or cluster four-step) are grouped by kernel variant, cluster size
//    and shared-memory class, each group one launch whose blocks look up
//    their parameter block; two-pass transforms run pass by pass on a shared
//    scratch; groups largest first (longest-processing-time order).
struct cfft_batch_s {
    int dtype = 0, flags = 0, device = 0;
    int64_t count = 0, total = 0;
    std::vector<int64_t> len, off;
    std::map<int64_t, cfft_plan_s*> plans;
    struct Group {
        const void* fn = nullptr;
        int cluster = 1;
        size_t smem = 0;
        unsigned grid = 0;
        KParams* d_desc = nullptr;
        int* d_map = nullptr;
        int ndesc = 0;
        double cost = 0;
    };
    std::vector<Group> groups;   // grouped form: single-kernel transforms
    std::vector<Group> passes;   // grouped form: two-pass transforms, chunk by chunk, pass by pass
    // queue form (the default): one launch over every work item
    bool queue = false;
    const void* qfn = nullptr;
    KParams* q_desc = nullptr;
    QItem* q_items = nullptr;
    int* q_ctl = nullptr;
    int q_nitems = 0, q_nctl = 0;
    unsigned q_grid = 0;
    size_t q_smem = 0;
    void* scratch[2] = {nullptr, nullptr};
    std::vector<void*> allocs;
    cudaStream_t cap = nullptr;
    cudaGraphExec_t gexec = nullptr;
    const void* g_in = nullptr;
    void* g_out = nullptr;
    int g_dir = -1;
    int launches = 0;
    std::mutex mu;
};

static void batch_free(cfft_batch_s* B) {
    if (B->gexec) cudaGraphExecDestroy(B->gexec);
    B->gexec = nullptr;
    if (B->cap) cudaStreamDestroy(B->cap);
    B->cap = nullptr;
    for (auto& kv : B->plans) {
        plan_free(kv.second);
        delete kv.second;
    }
    B->plans.clear();
    for (void* q : B->allocs) lib_free(q);
    B->allocs.clear();
}

// a batch-1 plan whose two-pass scratch is supplied by its caller (batched
// and serving forms)
static int build_shared_plan(int64_t n, int dtype, int flags, int device, cfft_plan_s** out) {
    if (n > (1LL << 26)) return fail(CFFT_ERR_UNSUPPORTED, "length above 2^26");
    auto cands = candidate_shapes(n, dtype, 1);
    cfft_plan_s* P = new cfft_plan_s();
    P->n = n;
    P->batch = 1;
    P->dtype = dtype;
    P->flags = flags;
    P->device = device;
    P->shared_scratch = true;
    int rc = fail(CFFT_ERR_UNSUPPORTED, "no execution shape for n=" + std::to_string(n));
    for (auto& c : cands) {
        // not descriptor driven: the batched and served forms skip these
        if (c.mode == MODE_P2COL || c.mode == MODE_CONVC || c.mode == MODE_MIXC || c.mode == MODE_P2CL) continue;
        rc = plan_build(P, c);
        if (rc == CFFT_OK) break;
        plan_free(P);
    }
    if (rc) {
        delete P;
        return rc;
    }
    *out = P;
    return CFFT_OK;
}
// batch-1 plan for the work queue: a single-CTA shape (rows or a
// one-CTA four-step) whose descriptor-driven variant fits `cap` bytes of
// shared memory, else two HBM passes
static size_t batched_smem(const Stage& st);
static bool single_kernel(const cfft_plan_s* P);
static int build_queue_plan(int64_t n, int dtype, int flags, int device, size_t cap, cfft_plan_s** out) {
    if (n > (1LL << 26)) return fail(CFFT_ERR_UNSUPPORTED, "length above 2^26");
    std::vector<Shape> v;
    for (auto& c : candidate_shapes(n, dtype, 1))
        if ((c.mode == MODE_ROWS || c.mode == MODE_FOUR) && c.C == 1) v.push_back(c);
    int conv;
    int64_t M;
    conv_kind(n, conv, M);
    Shape g;
    if (twopass_shape(n, conv, M, dtype, g)) v.push_back(g);
    cfft_plan_s* P = new cfft_plan_s();
    P->n = n;
    P->batch = 1;
    P->dtype = dtype;
    P->flags = flags;
    P->device = device;
    P->shared_scratch = true;
    int rc = fail(CFFT_ERR_UNSUPPORTED, "no queue shape for n=" + std::to_string(n));
    for (auto& c : v) {
        rc = plan_build(P, c);
        if (rc == CFFT_OK) {
            bool ok = true;
            if (single_kernel(P)) {
                ok = P->stages[0].cluster <= 1 && batched_smem(P->stages[0]) <= cap;
            } else {
                for (auto& st : P->stages)
                    ok = ok && (st.kp.mode == MODE_COLPASS || st.kp.mode == MODE_ROWPASS) && st.smem <= cap;
            }
            if (ok) break;
            rc = fail(CFFT_ERR_UNSUPPORTED, "no queue shape within the shared-memory budget for n=" +
                                                std::to_string(n));
        }
        plan_free(P);
    }
    if (rc) {
        delete P;
        return rc;
    }
    *out = P;
    return CFFT_OK;
}
// shared memory of a stage's descriptor-driven (generic) kernel
static size_t batched_smem(const Stage& st) { return st.smem_batched ? st.smem_batched : st.smem; }
static bool single_kernel(const cfft_plan_s* P) {
    return P->stages.size() == 1 &&
           (P->stages[0].kp.mode == MODE_ROWS || P->stages[0].kp.mode == MODE_FOUR);
}
// CTAs one parameter block occupies in a batched launch
static int blocks_for(const KParams& kp) {
    if (kp.mode == MODE_FOUR) return kp.C;
    if (kp.mode == MODE_COLPASS) return kp.N2 / kp.V;
    if (kp.mode == MODE_ROWPASS) return kp.N1 / kp.V;
    return 1;
}
// single-kernel stage -> its batched kernel variant (and the parameter fix-up
// that variant needs)
static const void* batched_variant(KParams& kp, int dtype) {
    int kmode = kp.mode;
    if (kp.mode == MODE_FOUR) {
        if (kp.pa.Gwarp > 0 && kp.pc.Gwarp > 0) kmode = MODE_FOUR_WARP;
        else kp.pa.Gwarp = kp.pc.Gwarp = 0;
    }
    return cfft_batch_kernel_for(kmode, dtype);
}

// launches are grouped by how many CTAs fit an SM (two below ~113 KB of
// shared memory, one above); a group runs with its largest member's size
static int smem_class(size_t smem) { return smem <= (size_t)112 * 1024 ? 0 : 1; }
// one launch: parameter blocks (largest first) and the block -> block map
template <class ItemT>
static int make_group(cfft_batch_s* B, const void* fn, int cluster, std::vector<ItemT>& items,
                      cfft_batch_s::Group& g) {
    std::stable_sort(items.begin(), items.end(), [](const ItemT& a, const ItemT& b) { return a.cost > b.cost; });
    g.fn = fn;
    g.cluster = cluster;
    g.smem = 0;
    for (auto& it : items) g.smem = std::max(g.smem, it.smem);
    std::vector<KParams> desc;
    std::vector<int> map;
    for (auto& it : items) {
        KParams kp = it.kp;
        kp.blk0 = (int)map.size();
        const int nb = blocks_for(kp);
        for (int b = 0; b < nb; b++) map.push_back((int)desc.size());
        desc.push_back(kp);
        g.cost += it.cost;
    }
    g.ndesc = (int)desc.size();
    g.grid = (unsigned)map.size();
    void *dd = nullptr, *dm = nullptr;
    CUDA_TRY(lib_malloc(&dd, desc.size() * sizeof(KParams)));
    B->allocs.push_back(dd);
    CUDA_TRY(lib_malloc(&dm, map.size() * sizeof(int)));
    B->allocs.push_back(dm);
    CUDA_TRY(cudaMemcpy(dd, desc.data(), desc.size() * sizeof(KParams), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(dm, map.data(), map.size() * sizeof(int), cudaMemcpyHostToDevice));
    g.d_desc = (KParams*)dd;
    g.d_map = (int*)dm;
    CUDA_TRY(cfft_prepare_fn(g.fn, g.smem, g.cluster));
    return CFFT_OK;
}

// work-queue schedule (see the batched form's header): plans,
// parameter blocks, work items and counters, uploaded once
static int batch_create_queue(cfft_batch_s* B) {
    const int dtype = B->dtype;
    const size_t e = elem_bytes(dtype);
    const int dt = dtype == CFFT_C128 ? CFFT_DT_C128 : CFFT_DT_C64;
    // ComplexF64 at two CTAs per SM, ComplexF32 at three (the pass kernels'
    // residency); the shared-memory budget per CTA follows
    const int mb = dtype == CFFT_C128 ? 2 : 3;
    const size_t cap = mb == 3 ? (size_t)74 * 1024 : (size_t)112 * 1024;
    for (int64_t n : B->len) {
        if (B->plans.count(n)) continue;
        cfft_plan_s* P = nullptr;
        int rc = build_queue_plan(n, dtype, B->flags, B->device, cap, &P);
        if (rc) return rc;
        B->plans[n] = P;
    }
    std::vector<KParams> desc;
    std::vector<QItem> items;
    int nctr = 0;
    size_t smax = 0;
    std::vector<int64_t> twopass, singles;
    for (int64_t i = 0; i < B->count; i++) (single_kernel(B->plans[B->len[i]]) ? singles : twopass).push_back(i);
    auto by_len = [&](int64_t a, int64_t b) { return B->len[a] > B->len[b]; };
    std::stable_sort(twopass.begin(), twopass.end(), by_len);
    std::stable_sort(singles.begin(), singles.end(), by_len);
    for (int64_t i : twopass)
        for (auto& st : B->plans[B->len[i]]->stages) smax = std::max(smax, st.smem);
    for (int64_t i : singles) smax = std::max(smax, batched_smem(B->plans[B->len[i]]->stages[0]));
    const void* fn = cfft_queue_kernel(dt, mb);
    CUDA_TRY(cfft_prepare_fn(fn, smax, 1));
    int per_sm = 0, nsm = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, CFFT_THREADS, smax));
    CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, B->device));
    if (per_sm < 1) return fail(CFFT_ERR_UNSUPPORTED, "the batch's queue kernel does not fit an SM");
    const int resident = per_sm * nsm;

    // Two-pass transforms, largest first, in slabs: consecutive transforms
    // whose scratch fits one slot of a ring, closed once a stage holds at
    // least two waves of tiles.  The items run as a software pipeline of
    // steps: step t holds stage 3 of slab t-3, stage 2 of slab t-2, stage 1
    // of slab t-1 and stage 0 of slab t, so an item's dependency (the
    // previous stage of its transform) was handed out a step earlier, and
    // the intermediate it reads was written recently (L2).  A slab first
    // waits for the slab that last used its slot; single-CTA transforms are
    // spread over the steps (no dependencies: they fill the waits).
    auto scratch_need = [&](int64_t i) {
        cfft_plan_s* P = B->plans[B->len[i]];
        return (size_t)P->shape.M * e * (P->stages.size() > 2 ? 2 : 1);
    };
    auto stage_tiles = [&](int64_t i, int s) { return blocks_for(B->plans[B->len[i]]->stages[s].kp); };
    std::vector<std::vector<int64_t>> slabs;
    size_t slot = 0;
    int nslots = 1;
    if (!twopass.empty()) {
        size_t total = 0, need_max = 0;
        for (int64_t i : twopass) {
            total += scratch_need(i);
            need_max = std::max(need_max, scratch_need(i));
        }
        slot = std::max(need_max, (size_t)scratch_budget());
        size_t used = 0;
        int64_t tiles = 0;
        slabs.emplace_back();
        for (int64_t i : twopass) {
            if (!slabs.back().empty() && (used + scratch_need(i) > slot || tiles >= 2 * resident)) {
                slabs.emplace_back();
                used = 0;
                tiles = 0;
            }
            slabs.back().push_back(i);
            used += scratch_need(i);
            tiles += stage_tiles(i, 0);
        }
        size_t freeb = 0, totb = 0;
        cudaMemGetInfo(&freeb, &totb);
        // the pipeline keeps four slabs in flight: six slots (or as many as
        // the slabs, or as a quarter of free memory holds, at least four)
        nslots = (int)std::min<size_t>(slabs.size(), std::max<size_t>(4, std::min<size_t>(6, freeb / 4 / slot)));
        if (slabs.size() == 1) slot = total;
        CUDA_TRY(lib_malloc(&B->scratch[0], slot * nslots));
        B->allocs.push_back(B->scratch[0]);
    }
    const int nslabs = (int)slabs.size();
    const int nsteps = nslabs ? nslabs + 3 : 1;
    std::vector<int> slab_ctr(nslabs), slab_need(nslabs, 0);
    for (int k = 0; k < nslabs; k++) slab_ctr[k] = nctr++;
    std::map<int64_t, std::pair<int64_t, int64_t>> so;   // scratch offsets (elements) in the slab's slot
    std::map<int64_t, std::vector<int>> sctr;            // stage counters per transform
    for (int k = 0; k < nslabs; k++) {
        int64_t cur = 0;
        for (int64_t i : slabs[k]) {
            cfft_plan_s* P = B->plans[B->len[i]];
            const int64_t M = P->shape.M;
            so[i] = {cur, P->stages.size() > 2 ? cur + M : -1};
            cur += M * (P->stages.size() > 2 ? 2 : 1);
        }
    }
    auto emit_stage = [&](int k, int64_t i, int pass) {
        cfft_plan_s* P = B->plans[B->len[i]];
        const int ns = (int)P->stages.size();
        const Stage& st = P->stages[pass];
        char* base = (char*)B->scratch[0] + (size_t)(k % nslots) * slot;
        KParams kp = st.kp;
        kp.batch = 1;
        kp.scale = 1.0 / (double)B->len[i];
        auto where = [&](int sel, const void** ptr, long long* off, unsigned char* user, long long* dist) {
            if (sel <= 1) {
                *ptr = nullptr;
                *off = B->off[i];
                *user = 1;
                *dist = B->len[i];
            } else {
                const int64_t o = (sel == 2) ? so[i].first : so[i].second;
                *ptr = base + (size_t)o * e;
                *off = 0;
                *user = 0;
                *dist = P->shape.M;
            }
        };
        const void *ip, *op;
        where(st.in_sel, &ip, &kp.in_off, &kp.in_user, &kp.in_dist);
        where(st.out_sel, &op, &kp.out_off, &kp.out_user, &kp.out_dist);
        kp.in = ip;
        kp.out = (void*)op;
        const int tiles = blocks_for(kp);
        int wait = -1, need = 0;
        if (pass == 0) {
            if (k >= nslots) {
                wait = slab_ctr[k - nslots];
                need = slab_need[k - nslots];
            }
        } else {
            wait = sctr[i][pass - 1];
            need = stage_tiles(i, pass - 1);
        }
        int done;
        if (pass == ns - 1) {
            done = slab_ctr[k];
            slab_need[k] += tiles;
        } else {
            done = nctr++;
            sctr[i].push_back(done);
        }
        const int kind = kp.mode == MODE_COLPASS ? QK_COLPASS : QK_ROWPASS;
        const int d = (int)desc.size();
        desc.push_back(kp);
        for (int b = 0; b < tiles; b++) items.push_back({d, b, kind, wait, need, done});
    };
    auto emit_single = [&](int64_t i) {
        cfft_plan_s* P = B->plans[B->len[i]];
        KParams kp = P->stages[0].kp;
        const void* vf = batched_variant(kp, dtype);
        const int kind = kp.mode == MODE_ROWS ? QK_ROWS
                         : vf == cfft_batch_kernel_for(MODE_FOUR_WARP, dt) ? QK_FOUR_WARP : QK_FOUR;
        kp.batch = 1;
        kp.in_off = kp.out_off = B->off[i];
        kp.in_user = kp.out_user = 1;
        kp.in_dist = kp.out_dist = B->len[i];
        kp.scale = 1.0 / (double)B->len[i];
        const int d = (int)desc.size();
        desc.push_back(kp);
        const int nb = blocks_for(kp);
        for (int b = 0; b < nb; b++) items.push_back({d, b, kind, -1, 0, -1});
    };
    size_t next_single = 0;
    for (int t = 0; t < nsteps; t++) {
        for (int s = 3; s >= 0; s--) {
            const int k = t - s;
            if (k < 0 || k >= nslabs) continue;
            for (int64_t i : slabs[k])
                if (s < (int)B->plans[B->len[i]]->stages.size()) emit_stage(k, i, s);
        }
        // this step's share of the single-CTA transforms
        const size_t upto = singles.size() * (size_t)(t + 1) / (size_t)nsteps;
        for (; next_single < upto; next_single++) emit_single(singles[next_single]);
    }
    B->qfn = fn;
    void *dd = nullptr, *di = nullptr, *dc = nullptr;
    CUDA_TRY(lib_malloc(&dd, desc.size() * sizeof(KParams)));
    B->allocs.push_back(dd);
    CUDA_TRY(lib_malloc(&di, items.size() * sizeof(QItem)));
    B->allocs.push_back(di);
    CUDA_TRY(lib_malloc(&dc, (size_t)(2 + nctr) * sizeof(int)));
    B->allocs.push_back(dc);
    CUDA_TRY(cudaMemcpy(dd, desc.data(), desc.size() * sizeof(KParams), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(di, items.data(), items.size() * sizeof(QItem), cudaMemcpyHostToDevice));
    B->queue = true;
    B->q_desc = (KParams*)dd;
    B->q_items = (QItem*)di;
    B->q_ctl = (int*)dc;
    B->q_nitems = (int)items.size();
    B->q_nctl = 2 + nctr;
    B->q_smem = smax;
    B->q_grid = (unsigned)B->q_nitems;              // one CTA per work item
    CUDA_TRY(cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking));
    return CFFT_OK;
}

static int batch_create_impl(cfft_batch_s* B, int64_t count, const int64_t* lengths, int dtype, int flags) {
    const size_t e = elem_bytes(dtype);
    B->dtype = dtype;
    B->flags = flags & CFFT_EXACT_TWIDDLES;
    B->count = count;
    cudaGetDevice(&B->device);
    B->len.assign(lengths, lengths + count);
    B->off.resize(count);
    int64_t acc = 0;
    for (int64_t i = 0; i < count; i++) {
        if (lengths[i] < 1) return fail(CFFT_ERR_INVALID, "every length must be >= 1");
        B->off[i] = acc;
        acc += lengths[i];
    }
    B->total = acc;
    if (!(flags & CFFT_BATCH_GROUPED)) return batch_create_queue(B);
    // one plan per distinct length (batch 1, scratch shared by the batch)
    for (int64_t n : B->len) {
        if (B->plans.count(n)) continue;
        cfft_plan_s* P = nullptr;
        int rc = build_shared_plan(n, dtype, B->flags, B->device, &P);
        if (rc) return rc;
        B->plans[n] = P;
    }
    // group single-kernel transforms; collect the two-pass ones
    struct Item { int64_t idx; KParams kp; double cost; size_t smem; };
    std::map<std::tuple<const void*, int, int>, std::vector<Item>> bins;
    std::vector<int64_t> twopass;
    for (int64_t i = 0; i < count; i++) {
        cfft_plan_s* P = B->plans[B->len[i]];
        const double cost = (double)P->shape.M * std::log2((double)std::max<int64_t>(2, P->shape.M));
        if (single_kernel(P)) {
            KParams kp = P->stages[0].kp;
            const void* fn = batched_variant(kp, dtype);
            kp.batch = 1;
            kp.in_off = kp.out_off = B->off[i];
            kp.in_user = kp.out_user = 1;
            kp.in_dist = kp.out_dist = B->len[i];
            kp.scale = 1.0 / (double)B->len[i];
            const size_t sm = batched_smem(P->stages[0]);
            bins[std::make_tuple(fn, P->stages[0].cluster, smem_class(sm))].push_back({i, kp, cost, sm});
        } else {
            twopass.push_back(i);
        }
    }
    for (auto& kv : bins) {
        cfft_batch_s::Group g;
        int rc = make_group(B, std::get<0>(kv.first), std::get<1>(kv.first), kv.second, g);
        if (rc) return rc;
        B->groups.push_back(g);
    }
    // costliest groups first
    std::stable_sort(B->groups.begin(), B->groups.end(),
                     [](const cfft_batch_s::Group& a, const cfft_batch_s::Group& b) { return a.cost > b.cost; });

    // two-pass transforms: chunks that fit a shared scratch; per chunk, pass k
    // of every transform runs as one launch per shared-memory class
    if (!twopass.empty()) {
        std::stable_sort(twopass.begin(), twopass.end(), [&](int64_t a, int64_t b) { return B->len[a] > B->len[b]; });
        size_t freeb = 0, totb = 0;
        cudaMemGetInfo(&freeb, &totb);
        size_t budget = std::min<size_t>((size_t)4 << 30, freeb / 4);
        size_t need_max = 0;
        for (int64_t i : twopass) {
            cfft_plan_s* P = B->plans[B->len[i]];
            need_max = std::max(need_max, (size_t)P->shape.M * e * (P->stages.size() > 2 ? 2 : 1));
        }
        budget = std::max(budget, need_max);
        CUDA_TRY(lib_malloc(&B->scratch[0], budget));
        B->allocs.push_back(B->scratch[0]);
        size_t used = 0;
        std::vector<int64_t> chunk;
        auto flush = [&]() -> int {
            if (chunk.empty()) return CFFT_OK;
            // scratch offsets (elements) per transform: S1, S2
            std::map<int64_t, std::pair<int64_t, int64_t>> so;
            int64_t cur = 0;
            for (int64_t i : chunk) {
                cfft_plan_s* P = B->plans[B->len[i]];
                const int64_t M = P->shape.M;
                so[i] = {cur, P->stages.size() > 2 ? cur + M : -1};
                cur += M * (P->stages.size() > 2 ? 2 : 1);
            }
            for (int pass = 0; pass < 4; pass++) {
                std::map<std::tuple<const void*, int, int>, std::vector<Item>> pb;
                for (int64_t i : chunk) {
                    cfft_plan_s* P = B->plans[B->len[i]];
                    if (pass >= (int)P->stages.size()) continue;
                    const Stage& st = P->stages[pass];
                    KParams kp = st.kp;
                    kp.batch = 1;
                    kp.scale = 1.0 / (double)B->len[i];
                    auto where = [&](int sel, const void** ptr, long long* off, unsigned char* user, long long* dist) {
                        if (sel <= 1) { *ptr = nullptr; *off = B->off[i]; *user = 1; *dist = B->len[i]; }
                        else {
                            const int64_t o = (sel == 2) ? so[i].first : so[i].second;
                            *ptr = (const char*)B->scratch[0] + (size_t)o * e;
                            *off = 0; *user = 0; *dist = P->shape.M;
                        }
                    };
                    const void* ip; const void* op;
                    where(st.in_sel, &ip, &kp.in_off, &kp.in_user, &kp.in_dist);
                    where(st.out_sel, &op, &kp.out_off, &kp.out_user, &kp.out_dist);
                    kp.in = ip;
                    kp.out = (void*)op;
                    const double cost = (double)P->shape.M;
                    pb[std::make_tuple(cfft_batch_kernel_for(kp.mode, dtype), 1, smem_class(st.smem))]
                        .push_back({i, kp, cost, st.smem});
                }
                for (auto& kv : pb) {
                    cfft_batch_s::Group g;
                    int rc = make_group(B, std::get<0>(kv.first), 1, kv.second, g);
                    if (rc) return rc;
                    B->passes.push_back(g);
                }
            }
            chunk.clear();
            used = 0;
            return CFFT_OK;
        };
        for (int64_t i : twopass) {
            cfft_plan_s* P = B->plans[B->len[i]];
            const size_t need = (size_t)P->shape.M * e * (P->stages.size() > 2 ? 2 : 1);
            if (used + need > budget) {
                int rc = flush();
                if (rc) return rc;
            }
            chunk.push_back(i);
            used += need;
        }
        int rc = flush();
        if (rc) return rc;
    }
    (void)e;
    CUDA_TRY(cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking));
    return CFFT_OK;
}

static int batch_enqueue(cfft_batch_s* B, const void* in, void* out, int dir, cudaStream_t st) {
    if (B->queue) {
        CUDA_TRY(cudaMemsetAsync(B->q_ctl, 0, (size_t)B->q_nctl * sizeof(int), st));
        QueueLaunch L;
        L.desc = B->q_desc;
        L.items = B->q_items;
        L.in_base = in;
        L.out_base = out;
        L.ctl = B->q_ctl;
        L.nitems = B->q_nitems;
        L.dir = dir;
        cudaError_t ce = cfft_launch_queue(B->qfn, L, B->q_grid, B->q_smem, st);
        if (ce != cudaSuccess) return fail(CFFT_ERR_CUDA, std::string("batched launch: ") + cudaGetErrorString(ce));
        B->launches = 1;
        return CFFT_OK;
    }
    int launches = 0;
    for (auto* list : {&B->groups, &B->passes}) {
        for (auto& g : *list) {
            BatchLaunch L;
            L.desc = g.d_desc;
            L.block_desc = g.d_map;
            L.in_base = in;
            L.out_base = out;
            L.dir = dir;
            L.pad_ = 0;
            cudaError_t ce = cfft_launch_batch(g.fn, L, g.grid, g.smem, g.cluster, st);
            if (ce != cudaSuccess)
                return fail(CFFT_ERR_CUDA, std::string("batched launch: ") + cudaGetErrorString(ce));
            launches++;
        }
    }
    B->launches = launches;
    return CFFT_OK;
}

// ------------------------------------------------------------ serving form
// Requests (n, device input, device output, direction) arrive one at a time
// from any host thread.  Batched mode: a worker thread forms a micro-batch
// from everything queued whenever one of its launch slots is idle
// (continuous batching: the next batch forms while earlier ones run),
// admitting requests in arrival order while the bytes in flight (input +
// output + two-pass scratch) stay under the cap, and runs the batch as
// grouped descriptor launches on the slot's stream, each request's
// direction in its own parameter block.  Direct mode: every request is
// launched on arrival through its own cached plan (the per-request
// baseline).  The worker observes completion by polling events; a request's
// latency is its completion time minus its submission time on the host's
// steady clock.
static double now_us() {
    return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

struct ServeReq {
    int64_t n = 0;
    const void* in = nullptr;
    void* out = nullptr;
    int dir = 0;
    double t_sub = 0, t_done = 0;
    std::atomic<int> state{0};    // 0 queued, 1 launched, 2 done, < 0 failed (-status)
};

struct ServeSlot {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    char* h_desc = nullptr;       // pinned staging of parameter blocks and block maps
    char* d_desc = nullptr;
    size_t desc_cap = 0;
    void* scratch = nullptr;
    size_t scratch_cap = 0;
    std::vector<int64_t> reqs;
    size_t bytes = 0;
    bool busy = false;
};

struct cfft_server_s {
    int dtype = 0, device = 0, mode = 0;
    size_t cap = 0;
    int64_t capacity = 0;
    std::unique_ptr<ServeReq[]> req;
    std::atomic<int64_t> next{0};
    std::mutex qmu;                           // queue, direct-mode launches
    std::condition_variable qcv;
    std::deque<int64_t> queue;
    std::deque<std::pair<int64_t, cudaEvent_t>> dpending;
    std::vector<cudaEvent_t> evpool;
    std::mutex dmu;                           // completion notification
    std::condition_variable dcv;
    std::mutex pmu;                           // plan caches
    std::map<int64_t, cfft_plan_s*> plans;    // caller-scratch plans (batched mode)
    std::map<int64_t, cfft_plan_s*> dplans;   // direct-mode plans (scratch: dscratch)
    void* dscratch = nullptr;                 // direct mode: one stream, one scratch
    size_t dscratch_cap = 0;
    std::vector<ServeSlot> slots;
    size_t inflight = 0;                      // worker only
    std::atomic<bool> stop{false};
    std::thread worker;
    cudaStream_t dstream = nullptr;
    std::atomic<int64_t> batches{0}, launches{0}, done{0};
    std::mutex emu;
    std::string errmsg;
};

static const size_t kServeAlign = 256;
static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

static int serve_plan(cfft_server_s* S, int64_t n, bool direct, cfft_plan_s** out) {
    std::lock_guard<std::mutex> lk(S->pmu);
    auto& m = direct ? S->dplans : S->plans;
    auto it = m.find(n);
    if (it != m.end()) {
        *out = it->second;
        return CFFT_OK;
    }
    cfft_plan_s* P = nullptr;
    int rc = build_shared_plan(n, S->dtype, 0, S->device, &P);
    if (rc) return rc;
    m[n] = P;
    *out = P;
    return CFFT_OK;
}
static size_t serve_scratch(const cfft_plan_s* P) {
    if (single_kernel(P)) return 0;
    const size_t one = align_up((size_t)P->shape.M * elem_bytes(P->dtype), kServeAlign);
    return P->stages.size() > 2 ? 2 * one : one;
}
static void serve_error(cfft_server_s* S, const std::string& msg) {
    std::lock_guard<std::mutex> lk(S->emu);
    S->errmsg = msg;
}
static void serve_finish(cfft_server_s* S, const std::vector<int64_t>& reqs, int state) {
    const double t = now_us();
    {
        std::lock_guard<std::mutex> lk(S->dmu);
        for (int64_t r : reqs) {
            S->req[r].t_done = t;
            S->req[r].state.store(state);
        }
    }
    S->done += (int64_t)reqs.size();
    S->dcv.notify_all();
}

// one micro-batch on an idle slot: grouped launches, then the slot's event
static int serve_launch(cfft_server_s* S, ServeSlot& sl) {
    cfft_trace::Range tr("serve_batch requests=%lld", (long long)sl.reqs.size(), 0);
    struct It { KParams kp; double cost; size_t smem; };
    std::map<std::tuple<const void*, int, int>, std::vector<It>> singles;
    std::map<std::tuple<const void*, int>, std::vector<It>> pass[4];
    size_t scur = 0;
    for (int64_t t : sl.reqs) {
        ServeReq& r = S->req[t];
        cfft_plan_s* P = nullptr;
        int rc = serve_plan(S, r.n, false, &P);
        if (rc) return rc;
        const double scale = (r.dir == CFFT_INVERSE) ? 1.0 / (double)r.n : 1.0;
        const double cost = (double)P->shape.M;
        if (single_kernel(P)) {
            KParams kp = P->stages[0].kp;
            const void* fn = batched_variant(kp, S->dtype);
            kp.batch = 1;
            kp.in = r.in;
            kp.out = r.out;
            kp.in_user = kp.out_user = 0;
            kp.in_off = kp.out_off = 0;
            kp.in_dist = kp.out_dist = r.n;
            kp.dir = r.dir;
            kp.scale = scale;
            const size_t sm = batched_smem(P->stages[0]);
            singles[std::make_tuple(fn, P->stages[0].cluster, smem_class(sm))].push_back({kp, cost, sm});
            continue;
        }
        const size_t one = align_up((size_t)P->shape.M * elem_bytes(S->dtype), kServeAlign);
        char* s1 = (char*)sl.scratch + scur;
        char* s2 = s1 + one;
        scur += serve_scratch(P);
        for (size_t k = 0; k < P->stages.size() && k < 4; k++) {
            const Stage& st = P->stages[k];
            KParams kp = st.kp;
            auto where = [&](int sel) -> void* {
                return sel == 0 ? (void*)r.in : sel == 1 ? r.out : sel == 2 ? (void*)s1 : (void*)s2;
            };
            kp.batch = 1;
            kp.in = where(st.in_sel);
            kp.out = where(st.out_sel);
            kp.in_dist = (st.in_sel >= 2) ? P->shape.M : r.n;
            kp.out_dist = (st.out_sel >= 2) ? P->shape.M : r.n;
            kp.in_user = kp.out_user = 0;
            kp.in_off = kp.out_off = 0;
            kp.dir = r.dir;
            kp.scale = scale;
            pass[k][std::make_tuple(cfft_batch_kernel_for(kp.mode, S->dtype), smem_class(st.smem))]
                .push_back({kp, cost, st.smem});
        }
    }
    // pack every group's parameter blocks and block map into one upload
    struct G { const void* fn; int cluster; size_t smem; size_t doff, moff; unsigned grid; };
    std::vector<G> gs;
    std::vector<char> host;
    auto add = [&](const void* fn, int cluster, std::vector<It>& items) {
        std::stable_sort(items.begin(), items.end(), [](const It& a, const It& b) { return a.cost > b.cost; });
        G g{fn, cluster, 0, 0, 0, 0};
        std::vector<int> map;
        std::vector<KParams> desc;
        for (auto& it : items) {
            KParams kp = it.kp;
            kp.blk0 = (int)map.size();
            for (int b = 0; b < blocks_for(kp); b++) map.push_back((int)desc.size());
            desc.push_back(kp);
            g.smem = std::max(g.smem, it.smem);
        }
        g.grid = (unsigned)map.size();
        g.doff = align_up(host.size(), 16);
        host.resize(g.doff + desc.size() * sizeof(KParams));
        memcpy(host.data() + g.doff, desc.data(), desc.size() * sizeof(KParams));
        g.moff = align_up(host.size(), 16);
        host.resize(g.moff + map.size() * sizeof(int));
        memcpy(host.data() + g.moff, map.data(), map.size() * sizeof(int));
        gs.push_back(g);
    };
    for (auto& kv : singles) add(std::get<0>(kv.first), std::get<1>(kv.first), kv.second);
    std::stable_sort(gs.begin(), gs.end(), [](const G& a, const G& b) { return a.grid > b.grid; });
    for (int k = 0; k < 4; k++)
        for (auto& kv : pass[k]) add(std::get<0>(kv.first), 1, kv.second);
    if (host.size() > sl.desc_cap) {
        if (sl.h_desc) lib_free_host(sl.h_desc);
        if (sl.d_desc) lib_free(sl.d_desc);
        sl.h_desc = sl.d_desc = nullptr;
        sl.desc_cap = 0;
        const size_t capb = align_up(host.size() * 2, 1 << 16);
        CUDA_TRY(lib_host_alloc((void**)&sl.h_desc, capb, cudaHostAllocDefault));
        CUDA_TRY(lib_malloc((void**)&sl.d_desc, capb));
        sl.desc_cap = capb;
    }
    memcpy(sl.h_desc, host.data(), host.size());
    CUDA_TRY(cudaMemcpyAsync(sl.d_desc, sl.h_desc, host.size(), cudaMemcpyHostToDevice, sl.st));
    for (auto& g : gs) {
        CUDA_TRY(cfft_prepare_fn(g.fn, g.smem, g.cluster));
        BatchLaunch L;
        L.desc = (const KParams*)(sl.d_desc + g.doff);
        L.block_desc = (const int*)(sl.d_desc + g.moff);
        L.in_base = nullptr;
        L.out_base = nullptr;
        L.dir = -1;
        L.pad_ = 0;
        cudaError_t ce = cfft_launch_batch(g.fn, L, g.grid, g.smem, g.cluster, sl.st);
        if (ce != cudaSuccess) return fail(CFFT_ERR_CUDA, std::string("serve launch: ") + cudaGetErrorString(ce));
    }
    CUDA_TRY(cudaEventRecord(sl.ev, sl.st));
    S->batches++;
    S->launches += (int64_t)gs.size();
    return CFFT_OK;
}

static void serve_worker(cfft_server_s* S) {
    cudaSetDevice(S->device);
    const size_t e = elem_bytes(S->dtype);
    std::vector<int64_t> done;
    while (true) {
        bool progressed = false;
        bool busy = false;
        for (auto& sl : S->slots) {
            if (!sl.busy) continue;
            const cudaError_t q = cudaEventQuery(sl.ev);
            if (q == cudaErrorNotReady) { busy = true; continue; }
            if (q != cudaSuccess) serve_error(S, std::string("serve batch: ") + cudaGetErrorString(q));
            serve_finish(S, sl.reqs, q == cudaSuccess ? 2 : -CFFT_ERR_CUDA);
            S->inflight -= sl.bytes;
            sl.reqs.clear();
            sl.bytes = 0;
            sl.busy = false;
            progressed = true;
        }
        if (S->mode == CFFT_SERVE_DIRECT) {   // completions in launch order
            std::unique_lock<std::mutex> lk(S->qmu);
            while (!S->dpending.empty()) {
                const cudaError_t q = cudaEventQuery(S->dpending.front().second);
                if (q == cudaErrorNotReady) { busy = true; break; }
                done.assign(1, S->dpending.front().first);
                S->evpool.push_back(S->dpending.front().second);
                S->dpending.pop_front();
                lk.unlock();
                if (q != cudaSuccess) serve_error(S, std::string("serve request: ") + cudaGetErrorString(q));
                serve_finish(S, done, q == cudaSuccess ? 2 : -CFFT_ERR_CUDA);
                progressed = true;
                lk.lock();
            }
        }
        ServeSlot* idle = nullptr;
        for (auto& sl : S->slots)
            if (!sl.busy) { idle = &sl; break; }
        if (S->mode == CFFT_SERVE_BATCHED && idle) {
            // admit in arrival order under the cap (a request alone always runs)
            size_t scr = 0;
            for (;;) {
                int64_t t;
                {
                    std::lock_guard<std::mutex> lk(S->qmu);
                    if (S->queue.empty()) break;
                    t = S->queue.front();
                    S->queue.pop_front();
                }
                ServeReq& r = S->req[t];
                cfft_plan_s* P = nullptr;
                int rc = serve_plan(S, r.n, false, &P);
                if (rc) {
                    serve_error(S, cfft_last_error());
                    serve_finish(S, std::vector<int64_t>(1, t), -rc);
                    continue;
                }
                const size_t sneed = serve_scratch(P);
                const size_t need = 2 * (size_t)r.n * e + sneed;
                const bool alone = idle->reqs.empty() && S->inflight == 0;
                if (!alone && (S->inflight + idle->bytes + need > S->cap || scr + sneed > idle->scratch_cap)) {
                    std::lock_guard<std::mutex> lk(S->qmu);
                    S->queue.push_front(t);
                    break;
                }
                if (scr + sneed > idle->scratch_cap) {
                    // grow (only when this request alone does not fit; the slot is idle)
                    if (idle->scratch) lib_free(idle->scratch);
                    idle->scratch = nullptr;
                    idle->scratch_cap = 0;
                    if (lib_malloc(&idle->scratch, scr + sneed) != cudaSuccess) {
                        cudaGetLastError();
                        serve_error(S, "serve: scratch allocation failed");
                        serve_finish(S, std::vector<int64_t>(1, t), -CFFT_ERR_NOMEM);
                        continue;
                    }
                    idle->scratch_cap = scr + sneed;
                }
                scr += sneed;
                idle->reqs.push_back(t);
                idle->bytes += need;
                r.state.store(1);
            }
            if (!idle->reqs.empty()) {
                int rc = serve_launch(S, *idle);
                if (rc) {
                    serve_error(S, cfft_last_error());
                    cudaStreamSynchronize(idle->st);
                    serve_finish(S, idle->reqs, -rc);
                    idle->reqs.clear();
                    idle->bytes = 0;
                } else {
                    S->inflight += idle->bytes;
                    idle->busy = true;
                    busy = true;
                }
                progressed = true;
            }
        }
        if (progressed) continue;
        bool queued;
        {
            std::lock_guard<std::mutex> lk(S->qmu);
            queued = !S->queue.empty() || !S->dpending.empty();
        }
        if (S->stop.load() && !busy && !queued) break;
        if (busy || queued) {
            std::this_thread::yield();
        } else {
            std::unique_lock<std::mutex> lk(S->qmu);
            S->qcv.wait_for(lk, std::chrono::milliseconds(2),
                            [&] { return !S->queue.empty() || !S->dpending.empty() || S->stop.load(); });
        }
    }
}

static void serve_free(cfft_server_s* S) {
    if (S->worker.joinable()) {
        S->stop.store(true);
        S->qcv.notify_all();
        S->worker.join();
    }
    for (auto& sl : S->slots) {
        if (sl.st) cudaStreamSynchronize(sl.st);
        if (sl.st) cudaStreamDestroy(sl.st);
        if (sl.ev) cudaEventDestroy(sl.ev);
        if (sl.h_desc) lib_free_host(sl.h_desc);
        if (sl.d_desc) lib_free(sl.d_desc);
        if (sl.scratch) lib_free(sl.scratch);
    }
    S->slots.clear();
    if (S->dstream) {
        cudaStreamSynchronize(S->dstream);
        cudaStreamDestroy(S->dstream);
    }
    if (S->dscratch) lib_free(S->dscratch);
    for (auto& pe : S->dpending) cudaEventDestroy(pe.second);
    for (cudaEvent_t ev : S->evpool) cudaEventDestroy(ev);
    for (auto* m : {&S->plans, &S->dplans})
        for (auto& kv : *m) {
            plan_free(kv.second);
            delete kv.second;
        }
}

static int serve_create_impl(cfft_server_s* S, int dtype, int64_t max_inflight_bytes, int64_t max_requests,
                             int mode) {
    if (dtype != CFFT_C128 && dtype != CFFT_C64) return fail(CFFT_ERR_INVALID, "dtype must be CFFT_C128 or CFFT_C64");
    if (mode != CFFT_SERVE_BATCHED && mode != CFFT_SERVE_DIRECT)
        return fail(CFFT_ERR_INVALID, "mode must be CFFT_SERVE_BATCHED or CFFT_SERVE_DIRECT");
    if (max_inflight_bytes < 0 || max_requests < 0) return fail(CFFT_ERR_INVALID, "negative limit");
    S->dtype = dtype;
    S->mode = mode;
    cudaGetDevice(&S->device);
    S->cap = max_inflight_bytes ? (size_t)max_inflight_bytes : ((size_t)64 << 30);
    S->capacity = max_requests ? max_requests : (1 << 18);
    S->req.reset(new ServeReq[(size_t)S->capacity]);
    if (mode == CFFT_SERVE_BATCHED) {
        S->slots.resize(3);
        for (auto& sl : S->slots) {
            CUDA_TRY(cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking));
            CUDA_TRY(cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming));
            sl.scratch_cap = std::min<size_t>(S->cap / 4, (size_t)1 << 30);
            CUDA_TRY(lib_malloc(&sl.scratch, sl.scratch_cap));
        }
    } else {
        CUDA_TRY(cudaStreamCreateWithFlags(&S->dstream, cudaStreamNonBlocking));
    }
    S->worker = std::thread(serve_worker, S);
    return CFFT_OK;
}

// ------------------------------------------------------------------- C ABI
static std::mutex g_cache_mu;
static std::map<std::tuple<int, int64_t, int64_t, int, int>, cfft_plan_s*> g_cache;

extern "C" {

int cfft_version(void) { return 100; }

const char* cfft_last_error(void) { return g_err; }

int cfft_device_faults(int clear) {
    unsigned w = 0;
    cudaError_t e = cfft_device_fault_word(&w, clear);
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(CFFT_ERR_CUDA, std::string("device fault word: ") + cudaGetErrorString(e));
        return -1;
    }
    return (int)w;
}

int cfft_debug_wait_timeout(int polls) {
    if (polls < 1 || polls > (1 << 20)) return fail(CFFT_ERR_INVALID, "polls must be in [1, 2^20]");
    CUDA_TRY(cfft_wait_probe(polls));
    return CFFT_OK;
}

int64_t cfft_debug_alloc_hook(int64_t nth) {
    g_alloc_seq.store(0);
    g_alloc_fail_from.store(nth > 0 ? nth : 0);
    return g_live_allocs.load();
}

int cfft_plan_create(cfft_plan* plan, int64_t n, int64_t batch, int dtype, int flags) {
    cfft_trace::Range tr("plan_create n=%lld batch=%lld dtype=%lld flags=%lld", n, batch, dtype, flags);
    g_err[0] = 0;
    return plan_create_impl(plan, n, batch, dtype, flags);
}

static int execute_half(cfft_plan_s* P, const void* d_in, void* d_out, int direction, cudaStream_t st) {
    if (direction < 0 || direction > 2) return fail(CFFT_ERR_INVALID, "direction must be 0, 1 or 2");
    if (((uintptr_t)d_in % 4) != 0 || ((uintptr_t)d_out % 4) != 0)
        return fail(CFFT_ERR_INVALID, "ComplexF16 buffers must be 4-byte aligned");
    if (P->io_fused) return plan_execute(P, d_in, d_out, direction, st);
    const long long count = (long long)P->n * P->batch;
    CUDA_TRY(cfft_half_to_float(d_in, P->half_work, count, st));
    int rc = plan_execute(P, P->half_work, P->half_work, direction, st);
    if (rc) return rc;
    CUDA_TRY(cfft_float_to_half(P->half_work, d_out, count, st));
    return CFFT_OK;
}

static int execute_strided(cfft_plan_s* P, const void* d_in, void* d_out, int direction, cudaStream_t st) {
    if (direction < 0 || direction > 2) return fail(CFFT_ERR_INVALID, "direction must be 0, 1 or 2");
    const size_t e = elem_bytes(P->dtype);
    if (((uintptr_t)d_in % e) != 0 || ((uintptr_t)d_out % e) != 0)
        return fail(CFFT_ERR_INVALID, "buffers must be aligned to the element size");
    if (P->io_fused) return plan_execute(P, d_in, d_out, direction, st, -1, P->idist, P->odist);
    CUDA_TRY(cfft_gather(d_in, P->strided_work, P->n, P->batch, P->istride, P->idist, P->dtype, st));
    int rc = plan_execute(P, P->strided_work, P->strided_work, direction, st);
    if (rc) return rc;
    CUDA_TRY(cfft_scatter(P->strided_work, d_out, P->n, P->batch, P->ostride, P->odist, P->dtype, st));
    return CFFT_OK;
}

int cfft_plan_create_many(cfft_plan* plan, int64_t n, int64_t batch, int dtype, int flags, int64_t istride,
                          int64_t idist, int64_t ostride, int64_t odist) {
    cfft_trace::Range tr("plan_create_many n=%lld batch=%lld istride=%lld ostride=%lld", n, batch, istride, ostride);
    g_err[0] = 0;
    if (!plan) return fail(CFFT_ERR_INVALID, "plan pointer is null");
    if (istride < 1 || ostride < 1 || idist < 0 || odist < 0)
        return fail(CFFT_ERR_INVALID, "strides must be >= 1 and distances >= 0");
    if (dtype != CFFT_C128 && dtype != CFFT_C64)
        return fail(CFFT_ERR_INVALID, "strided plans take CFFT_C128 or CFFT_C64");
    int rc = plan_create_impl(plan, n, batch, dtype, flags);
    if (rc) return rc;
    cfft_plan_s* P = *plan;
    if (istride == 1 && ostride == 1 && (idist == n || batch == 1) && (odist == n || batch == 1)) return CFFT_OK;
    P->strided = true;
    P->istride = istride;
    P->idist = idist;
    P->ostride = ostride;
    P->odist = odist;
    if (io_fusable(P)) {
        // the first kernel gathers as it loads, the last scatters as it stores
        P->io_fused = true;
        P->in_fmt = P->out_fmt = IO_STRIDED;
        P->desc = "strided(fused)+" + P->desc;
        return CFFT_OK;
    }
    if (lib_malloc(&P->strided_work, (size_t)n * batch * elem_bytes(dtype)) != cudaSuccess) {
        cudaGetLastError();
        plan_free(P);
        delete P;
        *plan = nullptr;
        return fail(CFFT_ERR_NOMEM, "strided working buffer allocation failed");
    }
    P->allocs.push_back(P->strided_work);
    P->desc = "strided+" + P->desc;
    return CFFT_OK;
}

int cfft_execute(cfft_plan plan, const void* d_in, void* d_out, int direction, void* stream) {
    cfft_trace::Range tr(plan ? plan->desc.c_str() : "execute");
    if (!plan || !d_in || !d_out) return fail(CFFT_ERR_INVALID, "null plan or buffer");
    if (plan->io_half) return execute_half(plan, d_in, d_out, direction, (cudaStream_t)stream);
    if (plan->strided) return execute_strided(plan, d_in, d_out, direction, (cudaStream_t)stream);
    return plan_execute(plan, d_in, d_out, direction, (cudaStream_t)stream);
}

// page-locked (or otherwise DMA-able) host memory?
static bool host_pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeManaged;
}
// memcpy split over a few threads (pageable <-> pinned staging)
static void par_memcpy(void* dst, const void* src, size_t bytes) {
    const size_t kMin = (size_t)4 << 20;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned nt = (unsigned)std::min<size_t>(std::min(8u, hw), std::max<size_t>(1, bytes / kMin));
    if (nt <= 1) {
        memcpy(dst, src, bytes);
        return;
    }
    std::vector<std::thread> th;
    const size_t step = (bytes + nt - 1) / nt;
    for (unsigned t = 0; t < nt; t++) {
        const size_t a = t * step, b = std::min(bytes, a + step);
        if (a < b) th.emplace_back([=] { memcpy((char*)dst + a, (const char*)src + a, b - a); });
    }
    for (auto& x : th) x.join();
}
// Pageable host buffers (a Julia Vector, a numpy array): the chunks pass
// through pinned staging buffers; the CPU copies chunk i in (and chunk i-3
// out) while the GPU moves and transforms the chunks in between.
static int execute_host_staged(cfft_plan_s* P, const void* h_in, void* h_out, int direction, size_t tbytes) {
    cudaStream_t sin = P->host_st[0], scomp = P->host_st[1], sout = P->host_st[2];
    const size_t cap = (size_t)P->host_chunk * tbytes;
    for (int k = 0; k < 3; k++) {
        if (!P->stage_in[k]) CUDA_TRY(lib_host_alloc(&P->stage_in[k], cap, cudaHostAllocDefault));
        if (!P->stage_out[k]) CUDA_TRY(lib_host_alloc(&P->stage_out[k], cap, cudaHostAllocDefault));
    }
    const int64_t nch = (P->batch + P->host_chunk - 1) / P->host_chunk;
    auto span = [&](int64_t i, size_t* off, size_t* bytes) {
        const int64_t b0 = i * P->host_chunk, nb = std::min(P->host_chunk, P->batch - b0);
        *off = (size_t)b0 * tbytes;
        *bytes = (size_t)nb * tbytes;
    };
    auto drain = [&](int64_t i) -> int {          // chunk i's result to the caller
        const int k = (int)(i % 3);
        size_t off, bytes;
        span(i, &off, &bytes);
        CUDA_TRY(cudaEventSynchronize(P->ev_out[k]));
        par_memcpy((char*)h_out + off, P->stage_out[k], bytes);
        return CFFT_OK;
    };
    for (int64_t i = 0; i < nch; i++) {
        const int k = (int)(i % 3);
        size_t off, bytes;
        span(i, &off, &bytes);
        if (i >= 3) {
            int rc = drain(i - 3);                 // frees stage_in/out[k] and host_buf[k]
            if (rc) return rc;
        }
        par_memcpy(P->stage_in[k], (const char*)h_in + off, bytes);
        CUDA_TRY(cudaMemcpyAsync(P->host_buf[k], P->stage_in[k], bytes, cudaMemcpyHostToDevice, sin));
        CUDA_TRY(cudaEventRecord(P->ev_in[k], sin));
        CUDA_TRY(cudaStreamWaitEvent(scomp, P->ev_in[k], 0));
        int rc = plan_execute(P, P->host_buf[k], P->host_buf[k], direction, scomp, (int64_t)(bytes / tbytes));
        if (rc) { cudaStreamSynchronize(scomp); return rc; }
        CUDA_TRY(cudaEventRecord(P->ev_comp[k], scomp));
        CUDA_TRY(cudaStreamWaitEvent(sout, P->ev_comp[k], 0));
        CUDA_TRY(cudaMemcpyAsync(P->stage_out[k], P->host_buf[k], bytes, cudaMemcpyDeviceToHost, sout));
        CUDA_TRY(cudaEventRecord(P->ev_out[k], sout));
    }
    for (int64_t i = std::max<int64_t>(0, nch - 3); i < nch; i++) {
        int rc = drain(i);
        if (rc) return rc;
    }
    CUDA_TRY(cudaStreamSynchronize(scomp));
    return CFFT_OK;
}

int cfft_execute_host(cfft_plan plan, const void* h_in, void* h_out, int direction) {
    cfft_trace::Range tr("execute_host n=%lld batch=%lld", plan ? plan->n : 0, plan ? plan->batch : 0);
    if (!plan || !h_in || !h_out) return fail(CFFT_ERR_INVALID, "null plan or buffer");
    if (direction < 0 || direction > 2) return fail(CFFT_ERR_INVALID, "direction must be 0, 1 or 2");
    cfft_plan_s* P = plan;
    if (P->strided) return fail(CFFT_ERR_UNSUPPORTED, "strided plans take device buffers (cfft_execute)");
    std::lock_guard<std::mutex> lk(P->host_mu);
    if (P->io_half) {
        const size_t bytes = (size_t)P->n * P->batch * 4;
        if (!P->half_dev) {
            CUDA_TRY(lib_malloc(&P->half_dev, bytes));
            P->allocs.push_back(P->half_dev);
        }
        CUDA_TRY(cudaMemcpy(P->half_dev, h_in, bytes, cudaMemcpyHostToDevice));
        int rc = execute_half(P, P->half_dev, P->half_dev, direction, nullptr);
        if (rc) return rc;
        CUDA_TRY(cudaMemcpy(h_out, P->half_dev, bytes, cudaMemcpyDeviceToHost));
        return CFFT_OK;
    }
    const size_t e = elem_bytes(P->dtype);
    const size_t tbytes = (size_t)P->n * e;
    if (!P->host_ready) {
        // ~32 MB chunks, a multiple of the plan's own chunk when it has scratch
        int64_t c = std::max<int64_t>(1, (int64_t)(32LL << 20) / (int64_t)tbytes);
        c = std::min<int64_t>(c, P->batch);
        if (P->chunk > 0 && P->chunk < P->batch) c = std::max<int64_t>(P->chunk, (c / P->chunk) * P->chunk);
        P->host_chunk = std::min<int64_t>(c, P->batch);
        auto setup = [&]() -> int {
            for (int i = 0; i < 3; i++) {
                CUDA_TRY(lib_malloc(&P->host_buf[i], (size_t)P->host_chunk * tbytes));
                CUDA_TRY(cudaStreamCreateWithFlags(&P->host_st[i], cudaStreamNonBlocking));
                CUDA_TRY(cudaEventCreateWithFlags(&P->ev_in[i], cudaEventDisableTiming));
                CUDA_TRY(cudaEventCreateWithFlags(&P->ev_comp[i], cudaEventDisableTiming));
                CUDA_TRY(cudaEventCreateWithFlags(&P->ev_out[i], cudaEventDisableTiming));
            }
            return CFFT_OK;
        };
        const int rc = setup();
        if (rc) {
            host_release(P);        // nothing half-built survives a failed set-up
            return rc;
        }
        P->host_ready = true;
    }
    // three-stage pipeline: H2D (stream 0) -> transform (stream 1) -> D2H
    // (stream 2) over a ring of three device chunk buffers
    cudaStream_t sin = P->host_st[0], scomp = P->host_st[1], sout = P->host_st[2];
    if (!host_pinned(h_in) || !host_pinned(h_out)) return execute_host_staged(P, h_in, h_out, direction, tbytes);
    int64_t i = 0;
    for (int64_t b0 = 0; b0 < P->batch; b0 += P->host_chunk, i++) {
        const int64_t nb = std::min(P->host_chunk, P->batch - b0);
        const int k = (int)(i % 3);
        const size_t off = (size_t)b0 * tbytes, bytes = (size_t)nb * tbytes;
        if (i >= 3) CUDA_TRY(cudaStreamWaitEvent(sin, P->ev_out[k], 0));
        CUDA_TRY(cudaMemcpyAsync(P->host_buf[k], (const char*)h_in + off, bytes, cudaMemcpyHostToDevice, sin));
        CUDA_TRY(cudaEventRecord(P->ev_in[k], sin));
        CUDA_TRY(cudaStreamWaitEvent(scomp, P->ev_in[k], 0));
        int rc = plan_execute(P, P->host_buf[k], P->host_buf[k], direction, scomp, nb);
        if (rc) { cudaStreamSynchronize(scomp); return rc; }
        CUDA_TRY(cudaEventRecord(P->ev_comp[k], scomp));
        CUDA_TRY(cudaStreamWaitEvent(sout, P->ev_comp[k], 0));
        CUDA_TRY(cudaMemcpyAsync((char*)h_out + off, P->host_buf[k], bytes, cudaMemcpyDeviceToHost, sout));
        CUDA_TRY(cudaEventRecord(P->ev_out[k], sout));
    }
    CUDA_TRY(cudaStreamSynchronize(sout));
    CUDA_TRY(cudaStreamSynchronize(scomp));
    return CFFT_OK;
}

int cfft_plan_destroy(cfft_plan plan) {
    if (!plan) return fail(CFFT_ERR_INVALID, "null plan");
    plan_free(plan);
    delete plan;
    return CFFT_OK;
}

int cfft_fft(int64_t n, int64_t batch, int dtype, int flags, const void* d_in, void* d_out,
             int direction, void* stream) {
    cfft_trace::Range tr("fft n=%lld batch=%lld dtype=%lld flags=%lld", n, batch, dtype, flags);
    int dev = 0;
    cudaGetDevice(&dev);
    cfft_plan_s* P = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        auto key = std::make_tuple(dev, n, batch, dtype, flags);
        auto it = g_cache.find(key);
        if (it != g_cache.end()) {
            P = it->second;
        } else {
            int rc = plan_create_impl(&P, n, batch, dtype, flags);
            if (rc) return rc;
            g_cache[key] = P;
        }
    }
    return cfft_execute(P, d_in, d_out, direction, stream);
}

int cfft_empty_cache(void) {
    cfft_trace::Range tr("empty_cache");
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        for (auto& kv : g_cache) {
            plan_free(kv.second);
            delete kv.second;
        }
        g_cache.clear();
    }
    {
        std::lock_guard<std::mutex> lk(g_spec_mu);
        for (auto& kv : g_spec_plans) {
            plan_free(kv.second);
            delete kv.second;
        }
        g_spec_plans.clear();
    }
    std::lock_guard<std::mutex> lk(g_tab_mu);
    g_tables.clear();   // live plans keep their own references
    return CFFT_OK;
}

int cfft_plan_describe(cfft_plan plan, char* buf, int len) {
    if (!plan || !buf || len < 1) return fail(CFFT_ERR_INVALID, "bad describe arguments");
    snprintf(buf, (size_t)len, "%s", plan->desc.c_str());
    return CFFT_OK;
}

int cfft_describe_strategy(int64_t n, int dtype, char* buf, int len) {
    if (n < 1 || !buf || len < 1) return fail(CFFT_ERR_INVALID, "bad describe arguments");
    auto c = candidate_shapes(n, dtype, 1);
    if (c.empty()) return fail(CFFT_ERR_UNSUPPORTED, "no shape");
    snprintf(buf, (size_t)len, "%s", shape_desc(c[0], n).c_str());
    return CFFT_OK;
}

int64_t cfft_plan_workspace_bytes(cfft_plan plan) {
    if (!plan) return -1;
    return (int64_t)plan->scratch_bytes * ((plan->scratch[1] != nullptr) ? 2 : (plan->scratch[0] ? 1 : 0));
}


int cfft_batch_create(cfft_batch* batch, int64_t count, const int64_t* lengths, int dtype, int flags) {
    cfft_trace::Range tr("batch_create count=%lld dtype=%lld", count, dtype);
    g_err[0] = 0;
    if (!batch || !lengths || count < 1) return fail(CFFT_ERR_INVALID, "batch, lengths and count >= 1 required");
    if (dtype != CFFT_C128 && dtype != CFFT_C64) return fail(CFFT_ERR_INVALID, "dtype must be CFFT_C128 or CFFT_C64");
    cfft_batch_s* B = new cfft_batch_s();
    int rc = batch_create_impl(B, count, lengths, dtype, flags);
    if (rc) {
        std::string keep = g_err;
        batch_free(B);
        delete B;
        cfft_set_last_error(keep.c_str());
        return rc;
    }
    *batch = B;
    return CFFT_OK;
}

int cfft_batch_execute(cfft_batch batch, const void* d_in, void* d_out, int direction, void* stream) {
    cfft_trace::Range tr("batch_execute count=%lld dir=%lld", batch ? batch->count : 0, direction);
    if (!batch || !d_in || !d_out) return fail(CFFT_ERR_INVALID, "null batch or buffer");
    if (direction < 0 || direction > 2) return fail(CFFT_ERR_INVALID, "direction must be 0, 1 or 2");
    cfft_batch_s* B = batch;
    const size_t e = elem_bytes(B->dtype);
    if (((uintptr_t)d_in % e) || ((uintptr_t)d_out % e))
        return fail(CFFT_ERR_INVALID, "buffers must be aligned to the element size");
    std::lock_guard<std::mutex> lk(B->mu);
    if (!B->gexec || B->g_in != d_in || B->g_out != d_out || B->g_dir != direction) {
        if (B->gexec) cudaGraphExecDestroy(B->gexec);
        B->gexec = nullptr;
        cudaGraph_t g = nullptr;
        CUDA_TRY(cudaStreamBeginCapture(B->cap, cudaStreamCaptureModeThreadLocal));
        int rc = batch_enqueue(B, d_in, d_out, direction, B->cap);
        cudaError_t ce = cudaStreamEndCapture(B->cap, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ce != cudaSuccess) return fail(CFFT_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(&B->gexec, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) {
            B->gexec = nullptr;
            return fail(CFFT_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
        }
        B->g_in = d_in;
        B->g_out = d_out;
        B->g_dir = direction;
    }
    CUDA_TRY(cudaGraphLaunch(B->gexec, (cudaStream_t)stream));
    return CFFT_OK;
}

int cfft_batch_destroy(cfft_batch batch) {
    if (!batch) return fail(CFFT_ERR_INVALID, "null batch");
    batch_free(batch);
    delete batch;
    return CFFT_OK;
}

int64_t cfft_batch_elements(cfft_batch batch) { return batch ? batch->total : -1; }

int cfft_batch_launches(cfft_batch batch) {
    if (!batch) return -1;
    return batch->queue ? 1 : (int)(batch->groups.size() + batch->passes.size());
}

int cfft_plan_launches(cfft_plan plan) {
    if (!plan) return -1;
    int64_t chunks = (plan->batch + plan->chunk - 1) / plan->chunk;
    // unfused ComplexF16 / strided plans add their widening and narrowing
    // (gathering and scattering) kernels
    const int extra = ((plan->io_half || plan->strided) && !plan->io_fused) ? 2 : 0;
    return (int)(chunks * (int64_t)plan->stages.size()) + extra;
}

}  // extern "C"

int cfft_serve_create(cfft_server* server, int dtype, int64_t max_inflight_bytes, int64_t max_requests,
                      int mode) {
    cfft_trace::Range tr("serve_create dtype=%lld cap=%lld", dtype, max_inflight_bytes);
    g_err[0] = 0;
    if (!server) return fail(CFFT_ERR_INVALID, "server pointer is null");
    *server = nullptr;
    cfft_server_s* S = new cfft_server_s();
    int rc = serve_create_impl(S, dtype, max_inflight_bytes, max_requests, mode);
    if (rc) {
        serve_free(S);
        delete S;
        return rc;
    }
    *server = S;
    return CFFT_OK;
}

int cfft_serve_prepare(cfft_server server, int64_t count, const int64_t* lengths) {
    if (!server || (count > 0 && !lengths)) return fail(CFFT_ERR_INVALID, "null server or lengths");
    for (int64_t i = 0; i < count; i++) {
        if (lengths[i] < 1) return fail(CFFT_ERR_INVALID, "every length must be >= 1");
        cfft_plan_s* P = nullptr;
        int rc = serve_plan(server, lengths[i], server->mode == CFFT_SERVE_DIRECT, &P);
        if (rc) return rc;
    }
    return CFFT_OK;
}

int cfft_serve_submit(cfft_server server, int64_t n, const void* d_in, void* d_out, int direction,
                      int64_t* ticket) {
    if (!server || !d_in || !d_out || !ticket) return fail(CFFT_ERR_INVALID, "null server, buffer or ticket");
    if (n < 1) return fail(CFFT_ERR_INVALID, "n must be >= 1");
    if (direction < 0 || direction > 2) return fail(CFFT_ERR_INVALID, "direction must be 0, 1 or 2");
    const size_t e = elem_bytes(server->dtype);
    if (((uintptr_t)d_in % e) != 0 || ((uintptr_t)d_out % e) != 0)
        return fail(CFFT_ERR_INVALID, "buffers must be aligned to the element size");
    cfft_server_s* S = server;
    cfft_plan_s* P = nullptr;
    if (S->mode == CFFT_SERVE_DIRECT) {
        int rc = serve_plan(S, n, true, &P);
        if (rc) return rc;
    }
    const int64_t t = S->next.fetch_add(1);
    if (t >= S->capacity) {
        S->next.fetch_sub(1);
        return fail(CFFT_ERR_NOMEM, "request table full (max_requests)");
    }
    ServeReq& r = S->req[t];
    r.n = n;
    r.in = d_in;
    r.out = d_out;
    r.dir = direction;
    r.t_done = 0;
    r.state.store(0);
    r.t_sub = now_us();
    if (S->mode == CFFT_SERVE_DIRECT) {
        std::lock_guard<std::mutex> lk(S->qmu);
        const size_t need = serve_scratch(P);
        if (need > S->dscratch_cap) {
            if (S->dscratch) {
                cudaStreamSynchronize(S->dstream);
                lib_free(S->dscratch);
            }
            S->dscratch = nullptr;
            S->dscratch_cap = 0;
            CUDA_TRY(lib_malloc(&S->dscratch, need));
            S->dscratch_cap = need;
        }
        P->scratch[0] = S->dscratch;
        P->scratch[1] = (char*)S->dscratch + need / 2;
        int rc = plan_execute(P, d_in, d_out, direction, S->dstream, -1);
        if (rc) {
            r.state.store(-rc);
            S->done++;
            return rc;
        }
        cudaEvent_t ev;
        if (!S->evpool.empty()) {
            ev = S->evpool.back();
            S->evpool.pop_back();
        } else {
            CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        }
        CUDA_TRY(cudaEventRecord(ev, S->dstream));
        r.state.store(1);
        S->dpending.push_back({t, ev});
        S->launches += (int64_t)P->stages.size();
    } else {
        std::lock_guard<std::mutex> lk(S->qmu);
        S->queue.push_back(t);
    }
    S->qcv.notify_one();
    *ticket = t;
    return CFFT_OK;
}

static int serve_status(cfft_server_s* S, int64_t t, double* latency_us) {
    const int st = S->req[t].state.load();
    if (st < 0) {
        std::lock_guard<std::mutex> lk(S->emu);
        return fail(-st, S->errmsg.empty() ? "request failed" : S->errmsg);
    }
    if (latency_us) *latency_us = S->req[t].t_done - S->req[t].t_sub;
    return CFFT_OK;
}

int cfft_serve_query(cfft_server server, int64_t ticket, int* done, double* latency_us) {
    if (!server || !done) return fail(CFFT_ERR_INVALID, "null server or flag");
    if (ticket < 0 || ticket >= server->next.load()) return fail(CFFT_ERR_INVALID, "unknown ticket");
    const int st = server->req[ticket].state.load();
    *done = (st == 2 || st < 0) ? 1 : 0;
    if (!*done) return CFFT_OK;
    return serve_status(server, ticket, latency_us);
}

int cfft_serve_wait(cfft_server server, int64_t ticket, double* latency_us) {
    if (!server) return fail(CFFT_ERR_INVALID, "null server");
    if (ticket < 0 || ticket >= server->next.load()) return fail(CFFT_ERR_INVALID, "unknown ticket");
    {
        std::unique_lock<std::mutex> lk(server->dmu);
        server->dcv.wait(lk, [&] {
            const int st = server->req[ticket].state.load();
            return st == 2 || st < 0;
        });
    }
    return serve_status(server, ticket, latency_us);
}

int cfft_serve_drain(cfft_server server) {
    if (!server) return fail(CFFT_ERR_INVALID, "null server");
    const int64_t n = server->next.load();
    {
        std::unique_lock<std::mutex> lk(server->dmu);
        server->dcv.wait(lk, [&] { return server->done.load() >= n; });
    }
    for (int64_t t = 0; t < n; t++)
        if (server->req[t].state.load() < 0) return serve_status(server, t, nullptr);
    return CFFT_OK;
}

int cfft_serve_stats(cfft_server server, int64_t* requests, int64_t* batches, int64_t* launches) {
    if (!server) return fail(CFFT_ERR_INVALID, "null server");
    if (requests) *requests = server->next.load();
    if (batches) *batches = server->batches.load();
    if (launches) *launches = server->launches.load();
    return CFFT_OK;
}

int cfft_serve_destroy(cfft_server server) {
    if (!server) return fail(CFFT_ERR_INVALID, "null server");
    serve_free(server);
    delete server;
    return CFFT_OK;
}

// Wisdom file: a header line, then one line per entry:
//   n batch dtype flags | mode conv M N1 N2 C V a <radices> c <radices>
int cfft_wisdom_export(const char* path) {
    cfft_trace::Range tr("wisdom_export");
    if (!path) return fail(CFFT_ERR_INVALID, "null path");
    FILE* f = fopen(path, "w");
    if (!f) return fail(CFFT_ERR_INVALID, std::string("cannot write ") + path);
    std::lock_guard<std::mutex> lk(g_wis_mu);
    fprintf(f, "catabra-b200-wisdom 1\n");
    for (auto& kv : g_wisdom)
        fprintf(f, "%lld %lld %d %d | %s\n", (long long)kv.first.n, (long long)kv.first.batch, kv.first.dtype,
                kv.first.flags, kv.second.c_str());
    const bool bad = ferror(f) != 0;
    fclose(f);
    return bad ? fail(CFFT_ERR_INVALID, std::string("write failed: ") + path) : CFFT_OK;
}

int cfft_wisdom_import(const char* path) {
    cfft_trace::Range tr("wisdom_import");
    if (!path) return fail(CFFT_ERR_INVALID, "null path");
    FILE* f = fopen(path, "r");
    if (!f) return fail(CFFT_ERR_INVALID, std::string("cannot read ") + path);
    char line[1024];
    std::map<WisdomKey, std::string> got;
    int rc = CFFT_OK;
    if (!fgets(line, sizeof line, f) || strncmp(line, "catabra-b200-wisdom 1", 21) != 0) {
        rc = fail(CFFT_ERR_INVALID, "not a wisdom file (missing header)");
    } else {
        while (fgets(line, sizeof line, f)) {
            long long n = 0, b = 0;
            int dt = 0, fl = 0, used = 0;
            if (line[0] == '\n' || line[0] == '#') continue;
            if (sscanf(line, "%lld %lld %d %d | %n", &n, &b, &dt, &fl, &used) != 4 || used == 0 || n < 1 || b < 1 ||
                (dt != CFFT_C128 && dt != CFFT_C64)) {
                rc = fail(CFFT_ERR_INVALID, std::string("malformed wisdom line: ") + line);
                break;
            }
            std::string sig(line + used);
            while (!sig.empty() && (sig.back() == '\n' || sig.back() == '\r' || sig.back() == ' ')) sig.pop_back();
            got[WisdomKey{n, b, dt, fl}] = sig;
        }
    }
    fclose(f);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(g_wis_mu);
    for (auto& kv : got) g_wisdom[kv.first] = kv.second;
    return CFFT_OK;
}

int cfft_wisdom_forget(void) {
    std::lock_guard<std::mutex> lk(g_wis_mu);
    g_wisdom.clear();
    return CFFT_OK;
}

int64_t cfft_wisdom_entries(void) {
    std::lock_guard<std::mutex> lk(g_wis_mu);
    return (int64_t)g_wisdom.size();
}

// ------------------------------------------------------------ real input
// rfft / irfft / brfft (AbstractFFTs' plan_rfft / plan_brfft, stubs in the
// reference at src/CatabraFFT.jl:199-209).  Even n runs a complex FFT of n/2
// points on the reals read as complex pairs plus one post- (pre-) processing
// kernel; odd n goes through the complex path of n points on a scratch.
struct cfft_rplan_s {
    int64_t n = 0, batch = 0;
    int dtype = 0;
    cfft_plan_s* P = nullptr;
    void* scratch = nullptr;     // odd n: batch * n complex
    void* d_real = nullptr;      // host entry: device copies of the two sides
    void* d_cplx = nullptr;
    std::mutex mu;
};

int cfft_rfft_plan_create(cfft_rplan* plan, int64_t n, int64_t batch, int dtype, int flags) {
    cfft_trace::Range tr("rfft_plan_create n=%lld batch=%lld dtype=%lld flags=%lld", n, batch, dtype, flags);
    g_err[0] = 0;
    if (!plan) return fail(CFFT_ERR_INVALID, "plan pointer is null");
    *plan = nullptr;
    if (n < 1 || batch < 1) return fail(CFFT_ERR_INVALID, "n and batch must be >= 1");
    if (dtype != CFFT_C128 && dtype != CFFT_C64) return fail(CFFT_ERR_INVALID, "dtype must be CFFT_C128 or CFFT_C64");
    cfft_rplan_s* R = new cfft_rplan_s();
    R->n = n;
    R->batch = batch;
    R->dtype = dtype;
    const bool even = (n % 2 == 0);
    int rc = plan_create_impl(&R->P, even ? n / 2 : n, batch, dtype, flags);
    if (rc == CFFT_OK && !even) {
        if (lib_malloc(&R->scratch, (size_t)n * batch * elem_bytes(dtype)) != cudaSuccess) {
            cudaGetLastError();
            rc = fail(CFFT_ERR_NOMEM, "real-transform scratch allocation failed");
        }
    }
    if (rc) {
        std::string keep = g_err;
        if (R->P) {
            plan_free(R->P);
            delete R->P;
        }
        delete R;
        cfft_set_last_error(keep.c_str());
        return rc;
    }
    *plan = R;
    return CFFT_OK;
}

int cfft_rfft_execute(cfft_rplan plan, const void* d_real, void* d_complex, void* stream) {
    cfft_trace::Range tr("rfft_execute");
    if (!plan || !d_real || !d_complex) return fail(CFFT_ERR_INVALID, "null plan or buffer");
    cfft_rplan_s* R = plan;
    const size_t e = elem_bytes(R->dtype);
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t n = R->n, h = n / 2 + 1;
    if (n % 2 == 0) {
        if (((uintptr_t)d_real % e) != 0 || ((uintptr_t)d_complex % e) != 0)
            return fail(CFFT_ERR_INVALID, "buffers must be aligned to the complex element size");
        int rc = plan_execute(R->P, d_real, d_complex, CFFT_FORWARD, st, -1, n / 2, h);
        if (rc) return rc;
        CUDA_TRY(cfft_r2c_post(d_complex, n / 2, n, R->batch, h, R->dtype, st));
        return CFFT_OK;
    }
    CUDA_TRY(cfft_r2c_widen(d_real, R->scratch, n, R->batch, R->dtype, st));
    int rc = plan_execute(R->P, R->scratch, R->scratch, CFFT_FORWARD, st, -1);
    if (rc) return rc;
    CUDA_TRY(cfft_r2c_keep(R->scratch, d_complex, n, R->batch, R->dtype, st));
    return CFFT_OK;
}

int cfft_rfft_execute_inverse(cfft_rplan plan, const void* d_complex, void* d_real, int direction, void* stream) {
    cfft_trace::Range tr("rfft_execute_inverse");
    if (!plan || !d_real || !d_complex) return fail(CFFT_ERR_INVALID, "null plan or buffer");
    if (direction != CFFT_INVERSE && direction != CFFT_BACKWARD)
        return fail(CFFT_ERR_INVALID, "direction must be CFFT_INVERSE (irfft) or CFFT_BACKWARD (brfft)");
    cfft_rplan_s* R = plan;
    const size_t e = elem_bytes(R->dtype);
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t n = R->n, h = n / 2 + 1;
    const double scale = (direction == CFFT_INVERSE) ? 1.0 / (double)n : 1.0;
    if (n % 2 == 0) {
        if (((uintptr_t)d_real % e) != 0 || ((uintptr_t)d_complex % e) != 0)
            return fail(CFFT_ERR_INVALID, "buffers must be aligned to the complex element size");
        CUDA_TRY(cfft_c2r_pre(d_complex, d_real, n / 2, n, R->batch, h, scale, R->dtype, st));
        return plan_execute(R->P, d_real, d_real, CFFT_BACKWARD, st, -1);
    }
    CUDA_TRY(cfft_c2r_expand(d_complex, R->scratch, n, R->batch, scale, R->dtype, st));
    int rc = plan_execute(R->P, R->scratch, R->scratch, CFFT_BACKWARD, st, -1);
    if (rc) return rc;
    CUDA_TRY(cfft_c2r_real(R->scratch, d_real, n, R->batch, R->dtype, st));
    return CFFT_OK;
}

int cfft_rfft_execute_host(cfft_rplan plan, const void* h_in, void* h_out, int direction) {
    cfft_trace::Range tr("rfft_execute_host");
    if (!plan || !h_in || !h_out) return fail(CFFT_ERR_INVALID, "null plan or buffer");
    if (direction < 0 || direction > 2) return fail(CFFT_ERR_INVALID, "direction must be 0, 1 or 2");
    cfft_rplan_s* R = plan;
    std::lock_guard<std::mutex> lk(R->mu);
    const size_t e = elem_bytes(R->dtype);
    const size_t rbytes = (size_t)R->n * R->batch * (e / 2), cbytes = (size_t)(R->n / 2 + 1) * R->batch * e;
    if (!R->d_real) {
        CUDA_TRY(lib_malloc(&R->d_real, rbytes + e));
        CUDA_TRY(lib_malloc(&R->d_cplx, cbytes));
    }
    int rc;
    if (direction == CFFT_FORWARD) {
        CUDA_TRY(cudaMemcpy(R->d_real, h_in, rbytes, cudaMemcpyHostToDevice));
        rc = cfft_rfft_execute(R, R->d_real, R->d_cplx, nullptr);
        if (rc == CFFT_OK) CUDA_TRY(cudaMemcpy(h_out, R->d_cplx, cbytes, cudaMemcpyDeviceToHost));
    } else {
        CUDA_TRY(cudaMemcpy(R->d_cplx, h_in, cbytes, cudaMemcpyHostToDevice));
        rc = cfft_rfft_execute_inverse(R, R->d_cplx, R->d_real, direction, nullptr);
        if (rc == CFFT_OK) CUDA_TRY(cudaMemcpy(h_out, R->d_real, rbytes, cudaMemcpyDeviceToHost));
    }
    return rc;
}

int cfft_rfft_plan_destroy(cfft_rplan plan) {
    if (!plan) return fail(CFFT_ERR_INVALID, "null plan");
    if (plan->d_real) lib_free(plan->d_real);
    if (plan->d_cplx) lib_free(plan->d_cplx);
    if (plan->P) {
        plan_free(plan->P);
        delete plan->P;
    }
    if (plan->scratch) lib_free(plan->scratch);
    delete plan;
    return CFFT_OK;
}
