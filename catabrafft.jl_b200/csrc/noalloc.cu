// noalloc.cu -- cfft_fft_twopass_noalloc: the two-HBM-pass FFT with no
// device allocation.
//
// Some callers cannot allocate device memory at the moment they need a
// transform: code running inside a memory pool that forbids cudaMalloc, or
// inside a framework that owns every allocation through its own allocator
// and may not see the library allocate behind its back.  This entry point
// serves them: its scratch (the intermediate between the column pass and the
// row pass) and its twiddle tables live in one file-scope __device__ array of
// fixed size that every GPU loading the library holds until the process
// exits.  The caller passes the
// input and output; nothing else is allocated -- no cudaMalloc / cudaFree,
// no allocating library call, no host heap.
//
// Limits and behaviour:
//   * n must be 7-smooth and split as n = N1 * N2 with N1, N2 <= 4096, and
//     n <= kScratchBytes / element size (2^21 ComplexF64 or 2^22 ComplexF32
//     elements); larger or non-smooth n are rejected with CFFT_ERR_UNSUPPORTED.
//   * The batch is processed in chunks that fit the scratch.
//   * The first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) and sets kernel attributes, once per device,
//     with that device current; make that first call before any stream
//     capture begins.
//   * Every call shares the array, and each call overwrites the tables and
//     scratch it uses (nothing is assumed to start at zero): calls that
//     overlap on the GPU -- on different streams, or from different host
//     threads -- race and corrupt each other's results.  Serialise them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/catabra_b200.h"
#include "engine_types.h"
#include "kernels.h"

static constexpr size_t kScratchBytes = 32u << 20;   // intermediate between the passes
static constexpr size_t kTableBytes = 256u << 10;    // sub-transform + four-step twiddles
static constexpr int kMaxDevices = 64;

// the whole working set of the entry point, 256-byte aligned; in host code
// this name is a host-side stand-in, never a device address
static __device__ __align__(256) unsigned char g_noalloc_arena[kScratchBytes + kTableBytes];

namespace {

std::mutex g_setup_mu;
unsigned char* g_arena_ptr[kMaxDevices] = {};

// errors go to the library's thread-local cfft_last_error() text (a fixed
// buffer, no heap)
int noalloc_fail(int code, const char* what, cudaError_t e = cudaSuccess) {
    char msg[256];
    if (e != cudaSuccess)
        snprintf(msg, sizeof msg, "cfft_fft_twopass_noalloc: %s: %s", what, cudaGetErrorString(e));
    else
        snprintf(msg, sizeof msg, "cfft_fft_twopass_noalloc: %s", what);
    cfft_set_last_error(msg);
    return code;
}

// w_L^m = exp(-2 pi i m / L) in FP64 (sincospi), rounded once to the data type
template <typename V> __device__ V round_to(double c, double s);
template <> __device__ double2 round_to<double2>(double c, double s) { return make_double2(c, s); }
template <> __device__ float2 round_to<float2>(double c, double s) {
    return make_float2((float)c, (float)s);
}
__device__ double2 omega_dev(long long m, long long L) {
    m %= L;
    double s, c;
    sincospi(-2.0 * (double)m / (double)L, &s, &c);
    return make_double2(c, s);
}
// per-pass twiddle blocks of one sub-transform (layout of SubPlan.tw)
struct PassTable {
    int L, np, twlen;
    int r[CFFT_MAXP], s[CFFT_MAXP], off[CFFT_MAXP];
};
template <typename V>
__global__ void k_noalloc_tables(V* twA, PassTable A, V* twC, PassTable Cc, double2* lo, int nlo,
                                 double2* hi, int nhi, int M) {
    const int stride = gridDim.x * blockDim.x;
    const int total = max(max(A.twlen, Cc.twlen), max(nlo, nhi));
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        for (int w = 0; w < 2; w++) {
            const PassTable& T = w ? Cc : A;
            V* dst = w ? twC : twA;
            if (i >= T.twlen) continue;
            int p = 0;
            while (p + 1 < T.np && T.off[p + 1] <= i) p++;
            const int n1 = T.L / (T.s[p] * T.r[p]), k = i - T.off[p];
            const int j = k / n1 + 1, q = k - (j - 1) * n1;
            const double2 v = omega_dev((long long)j * q * T.s[p], T.L);
            dst[i] = round_to<V>(v.x, v.y);
        }
        if (i < nlo) lo[i] = omega_dev(i, M);
        if (i < nhi) hi[i] = omega_dev((long long)i * nlo, M);
    }
}

// greedy radix split (largest codelet first), passes stored in CFFT_EXEC_ORDER
const int kRad[8] = {16, 9, 8, 7, 5, 4, 3, 2};
const int kExec[8] = CFFT_EXEC_ORDER;
bool split_canonical(long long L, SubPlan& sp) {
    sp.L = (int)L;
    sp.np = 0;
    for (int i = 0; i < 8; i++) sp.cnt[i] = 0;
    long long rem = L;
    while (rem > 1) {
        int k = -1;
        for (int i = 0; i < 8; i++)
            if (rem % kRad[i] == 0) { k = i; break; }
        if (k < 0 || sp.np >= CFFT_MAXP) return false;
        for (int i = 0; i < 8; i++)
            if (kExec[i] == kRad[k]) sp.cnt[i]++;
        sp.np++;
        rem /= kRad[k];
    }
    int k = 0;
    for (int i = 0; i < 8; i++)
        for (int c = 0; c < sp.cnt[i]; c++) sp.radix[k++] = (unsigned char)kExec[i];
    // block-wide waves only: G sub-transforms per wave fit 256 threads x 16 elements
    long long g = 1 << 20;
    for (int i = 0; i < sp.np; i++) {
        const int r = sp.radix[i];
        g = std::min<long long>(g, (long long)CFFT_THREADS * (CFFT_EMAX / r) * r / sp.L);
    }
    sp.G = (int)std::max<long long>(1, std::min<long long>(g, 1 << 20));
    sp.Gwarp = 0;
    return sp.np == 0 || g >= 1;
}
void pass_table(const SubPlan& sp, PassTable& T) {
    T.L = sp.L;
    T.np = sp.np;
    long long s = 1, off = 0;
    for (int i = 0; i < sp.np; i++) {
        T.r[i] = sp.radix[i];
        T.s[i] = (int)s;
        T.off[i] = (int)off;
        off += (long long)(sp.radix[i] - 1) * (sp.L / (s * sp.radix[i]));
        s *= sp.radix[i];
    }
    T.twlen = (int)off;
}
unsigned long long magic(long long d) {
    return ((1ULL << 40) + (unsigned long long)d - 1) / (unsigned long long)d;
}
}  // namespace

extern "C" int cfft_fft_twopass_noalloc(int64_t n, int64_t batch, int dtype, const void* d_in,
                                        void* d_out, int direction, void* stream) {
    cfft_set_last_error("");
    if (n < 4 || batch < 1 || !d_in || !d_out || direction < 0 || direction > 2)
        return noalloc_fail(CFFT_ERR_INVALID, "bad argument (n >= 4, batch >= 1, buffers, direction)");
    if (dtype != CFFT_C128 && dtype != CFFT_C64)
        return noalloc_fail(CFFT_ERR_INVALID, "dtype must be CFFT_C128 or CFFT_C64");
    const size_t e = (dtype == CFFT_C128) ? 16 : 8;
    if ((size_t)n * e > kScratchBytes)
        return noalloc_fail(CFFT_ERR_UNSUPPORTED,
                            "n exceeds the fixed scratch (2^21 ComplexF64 / 2^22 ComplexF32 elements)");
    if (((uintptr_t)d_in % e) || ((uintptr_t)d_out % e))
        return noalloc_fail(CFFT_ERR_INVALID, "buffers must be aligned to the element size");
    // balanced split with both factors <= 4096 and 7-smooth
    long long N1 = -1;
    double best = 1e30;
    SubPlan pa, pc;
    for (long long a = 2; a <= 4096; a++) {
        if (n % a) continue;
        const long long b = n / a;
        if (b < 2 || b > 4096) continue;
        SubPlan ta, tc;
        if (!split_canonical(a, ta) || !split_canonical(b, tc)) continue;
        const double bal = std::fabs(std::log2((double)a / (double)b));
        if (bal < best) { best = bal; N1 = a; pa = ta; pc = tc; }
    }
    if (N1 < 0)
        return noalloc_fail(CFFT_ERR_UNSUPPORTED,
                            "n must be 7-smooth with a split n = N1*N2, N1, N2 <= 4096");
    const long long N2 = n / N1;

    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess) return noalloc_fail(CFFT_ERR_CUDA, "cudaGetDevice", ce);
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(CFFT_ERR_UNSUPPORTED, "device index");
    const void* fcol = cfft_kernel_for(MODE_COLPASS, dtype);
    const void* frow = cfft_kernel_for(MODE_ROWPASS, dtype);
    unsigned char* arena;
    {
        std::lock_guard<std::mutex> lk(g_setup_mu);
        if (!g_arena_ptr[dev]) {
            // host code must not use g_noalloc_arena's name as an address: ask
            // the runtime for this device's copy, with this device current
            void* ptr = nullptr;
            ce = cudaGetSymbolAddress(&ptr, g_noalloc_arena);
            if (ce != cudaSuccess || !ptr)
                return noalloc_fail(CFFT_ERR_CUDA, "cudaGetSymbolAddress", ce);
            // shared-memory attributes for both element types' pass kernels
            for (int dt = 0; dt < 2 && ce == cudaSuccess; dt++) {
                ce = cfft_prepare_fn(cfft_kernel_for(MODE_COLPASS, dt), 128 * 1024, 1);
                if (ce == cudaSuccess) ce = cfft_prepare_fn(cfft_kernel_for(MODE_ROWPASS, dt), 128 * 1024, 1);
            }
            if (ce != cudaSuccess) return noalloc_fail(CFFT_ERR_CUDA, "kernel attributes", ce);
            g_arena_ptr[dev] = (unsigned char*)ptr;
        }
        arena = g_arena_ptr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;

    // carve the table region: twA[N1] twC[N2] (data type), then FP64 lo/hi
    int bits = 0;
    while ((1LL << (2 * bits)) < n) bits++;
    const int nlo = 1 << bits, nhi = (int)((n + nlo - 1) / nlo + 1);
    unsigned char* tab = arena + kScratchBytes;
    PassTable TA, TC;
    pass_table(pa, TA);
    pass_table(pc, TC);
    pa.twlen = TA.twlen;
    pc.twlen = TC.twlen;
    void* twA = tab;
    void* twC = tab + (size_t)TA.twlen * e;
    size_t off = (size_t)((TA.twlen + TC.twlen) * e + 255) & ~(size_t)255;
    double2* lo = (double2*)(tab + off);
    double2* hi = lo + nlo;
    if (off + (size_t)(nlo + nhi) * sizeof(double2) > kTableBytes)
        return noalloc_fail(CFFT_ERR_UNSUPPORTED, "twiddle tables exceed the fixed table region");
    if (dtype == CFFT_C128)
        k_noalloc_tables<double2><<<32, 256, 0, st>>>((double2*)twA, TA, (double2*)twC, TC, lo, nlo, hi,
                                                        nhi, (int)n);
    else
        k_noalloc_tables<float2><<<32, 256, 0, st>>>((float2*)twA, TA, (float2*)twC, TC, lo, nlo, hi,
                                                       nhi, (int)n);
    ce = cudaGetLastError();
    if (ce != cudaSuccess) return noalloc_fail(CFFT_ERR_CUDA, "table kernel launch", ce);

    KParams kp;
    memset(&kp, 0, sizeof kp);
    kp.conv = CONV_NONE;
    kp.nx = (int)n;
    kp.M = (int)n;
    kp.N1 = (int)N1;
    kp.N2 = (int)N2;
    kp.C = 1;
    kp.dir = direction;
    kp.scale = (direction == CFFT_INVERSE) ? 1.0 / (double)n : 1.0;
    kp.t4.lo = lo;
    kp.t4.hi = hi;
    kp.t4.bits = bits;
    kp.t4.N = (int)n;
    pa.tw = twA;
    pc.tw = twC;
    const long long PC = N2 + ((N2 % 2 == 0) ? 1 : 0);
    // the planner's tile rule: widths within the per-CTA shared-memory budget
    // (staged tables included), power-of-two widths preferred
    long long Vc = 1, Vr = 1;
    cfft_pass_tiles(N1, N2, PC, pa.twlen, pc.twlen, bits, (int)n, e, &Vc, &Vr);
    KParams col = kp, row = kp;
    col.mode = MODE_COLPASS;
    col.V = (int)Vc;
    col.PA = (int)Vc;
    col.pa = pa;
    col.mV = magic(Vc);
    col.pre = PRE_NONE;
    row.mode = MODE_ROWPASS;
    row.V = (int)Vr;
    row.PC = (int)PC;
    row.pc = pc;
    row.mV = magic(Vr);
    row.mN2 = magic(N2);
    row.post = POST_OUT;
    const size_t smem_col = cfft_colpass_smem(pa.twlen, bits, (int)n, (int)(N1 * Vc), (int)e);
    const size_t smem_row = (size_t)(cfft_pass_tw_elems(pc.twlen, (int)e) + Vr * PC) * e + 16;

    const long long chunk = std::max<long long>(1, (long long)(kScratchBytes / ((size_t)n * e)));
    for (long long b0 = 0; b0 < batch; b0 += chunk) {
        const long long nb = std::min(chunk, batch - b0);
        col.batch = row.batch = (int)nb;
        col.in = (const char*)d_in + (size_t)b0 * n * e;
        col.out = arena;
        col.in_dist = n;
        col.out_dist = n;
        row.in = arena;
        row.out = (char*)d_out + (size_t)b0 * n * e;
        row.in_dist = n;
        row.out_dist = n;
        ce = cfft_launch_fn(fcol, col, (unsigned)(nb * (N2 / Vc)), CFFT_THREADS, smem_col, 1, st);
        if (ce == cudaSuccess)
            ce = cfft_launch_fn(frow, row, (unsigned)(nb * (N1 / Vr)), CFFT_THREADS, smem_row, 1, st);
        if (ce != cudaSuccess) return noalloc_fail(CFFT_ERR_CUDA, "kernel launch", ce);
    }
    return CFFT_OK;
}
