// kernels.cu -- sm_100a kernel entry points, the registry of statically
// shaped kernels, and the launcher.
#include <cudaTypedefs.h>

#include "convc.cuh"
#include "engine.cuh"
#include "mixc.cuh"
#include "kernels.h"
#include "pow2.cuh"

// 256 threads per CTA; FP64 data keeps 2 CTAs/SM resident (128 regs/thread),
// and so does FP32 data (the exchange staging needs the headroom).
template <typename V> struct MinBlocks { static constexpr int value = 2; };
template <> struct MinBlocks<double2> { static constexpr int value = 2; };

template <typename V, int EMAX>
__global__ void __launch_bounds__(CFFT_THREADS, MinBlocks<V>::value) k_rows(KParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    rows_body<V, EMAX>(p, smem);
}
template <typename V, int EMAX, class K>
__global__ void __launch_bounds__(CFFT_THREADS, MinBlocks<V>::value) k_four(KParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    four_body<V, EMAX, K>(p, smem);
}
// statically shaped variant with its own residency target: a smaller
// per-thread element budget (EMAX) and a single shared buffer let three
// ComplexF64 CTAs share an SM
template <typename V, int EMAX, class K, int MB>
__global__ void __launch_bounds__(CFFT_THREADS, MB) k_four_mb(KParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    four_body<V, EMAX, K>(p, smem);
}
// the pass kernels keep three ComplexF32 CTAs resident per SM (80 registers
// suffice for their radix-16 codelets)
template <typename V> struct PassBlocks { static constexpr int value = 3; };
template <> struct PassBlocks<double2> { static constexpr int value = 2; };

template <typename V, int EMAX>
__global__ void __launch_bounds__(CFFT_THREADS, PassBlocks<V>::value) k_colpass(KParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    colpass_body<V, EMAX>(p, smem);
}
template <typename V, int EMAX>
__global__ void __launch_bounds__(CFFT_THREADS, PassBlocks<V>::value) k_rowpass(KParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    rowpass_body<V, EMAX>(p, smem);
}

// ---- batched entry points: each block finds its parameter block, stages it
// in shared memory with the launch's base pointers and direction applied, and
// runs the same body as the single-plan kernels.
template <typename V>
__device__ __forceinline__ const KParams& stage_params(const BatchLaunch& L, KParams* sp) {
    if (threadIdx.x == 0) {
        KParams p = L.desc[L.block_desc[blockIdx.x]];
        if (p.in_user) p.in = (const V*)L.in_base + p.in_off;
        if (p.out_user) p.out = (V*)L.out_base + p.out_off;
        if (L.dir >= 0) {                 // one direction for the launch
            p.dir = L.dir;
            if (L.dir != 1) p.scale = 1.0;
        }                                 // else: per-block direction and scale
        *sp = p;
    }
    __syncthreads();
    return *sp;
}
template <typename V, int EMAX>
__global__ void __launch_bounds__(CFFT_THREADS, MinBlocks<V>::value) kb_rows(BatchLaunch L) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ KParams sp;
    rows_body<V, EMAX>(stage_params<V>(L, &sp), smem);
}
template <typename V, int EMAX, class K>
__global__ void __launch_bounds__(CFFT_THREADS, MinBlocks<V>::value) kb_four(BatchLaunch L) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ KParams sp;
    four_body<V, EMAX, K>(stage_params<V>(L, &sp), smem);
}

template <typename V, int EMAX>
__global__ void __launch_bounds__(CFFT_THREADS, PassBlocks<V>::value) kb_colpass(BatchLaunch L) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ KParams sp;
    colpass_body<V, EMAX>(stage_params<V>(L, &sp), smem);
}
template <typename V, int EMAX>
__global__ void __launch_bounds__(CFFT_THREADS, PassBlocks<V>::value) kb_rowpass(BatchLaunch L) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ KParams sp;
    rowpass_body<V, EMAX>(stage_params<V>(L, &sp), smem);
}

const void* cfft_batch_kernel_for(int mode, int dtype) {
    if (dtype == CFFT_DT_C128) {
        switch (mode) {
            case MODE_ROWS: return (const void*)kb_rows<double2, CFFT_EMAX>;
            case MODE_FOUR: return (const void*)kb_four<double2, CFFT_EMAX, DynK<0>>;
            case MODE_FOUR_WARP: return (const void*)kb_four<double2, CFFT_EMAX, DynK<1>>;
            case MODE_COLPASS: return (const void*)kb_colpass<double2, CFFT_EMAX>;
            case MODE_ROWPASS: return (const void*)kb_rowpass<double2, CFFT_EMAX>;
        }
    } else {
        switch (mode) {
            case MODE_ROWS: return (const void*)kb_rows<float2, CFFT_EMAX>;
            case MODE_FOUR: return (const void*)kb_four<float2, CFFT_EMAX, DynK<0>>;
            case MODE_FOUR_WARP: return (const void*)kb_four<float2, CFFT_EMAX, DynK<1>>;
            case MODE_COLPASS: return (const void*)kb_colpass<float2, CFFT_EMAX>;
            case MODE_ROWPASS: return (const void*)kb_rowpass<float2, CFFT_EMAX>;
        }
    }
    return nullptr;
}

cudaError_t cfft_launch_batch(const void* f, const BatchLaunch& L, unsigned grid, size_t smem,
                              int cluster, cudaStream_t stream) {
    if (!f) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid, 1, 1);
    cfg.blockDim = dim3(CFFT_THREADS, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    if (cluster > 1) {
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = cluster;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
    void* args[] = {(void*)&L};
    cudaError_t e = cudaLaunchKernelExC(&cfg, f, args);
    if (e != cudaSuccess) cudaGetLastError();
    return e;
}

// n = 4096: persistent CTAs, registers + two shared-memory exchanges.  Three
// CTAs per SM (80 registers; a few dozen bytes of spills) measured faster
// than two without spills: more transforms in flight hide the HBM latency.
template <typename V>
__global__ void __launch_bounds__(CFFT_THREADS, 3) k_r4096(KParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    r4096_body<V>(p, smem);
}
const void* cfft_r4096_kernel(int dtype) {
    return dtype == CFFT_DT_C128 ? (const void*)k_r4096<double2> : (const void*)k_r4096<float2>;
}
size_t cfft_r4096_smem(size_t elem_bytes) {
    // planes, w_4096 table (129 FP64 entries), one mbarrier (tensor-copy mode)
    return ((16 * R4096_PL * elem_bytes + 15) & ~(size_t)15) + 129 * sizeof(double2) + 16;
}

// power-of-two lengths n = N1 x 4096 (pow2.cuh): pass A is the n = 4096
// kernel over the stride-N1 subsequences (k_p2row), pass B the column DFTs
// (k_p2col, one kernel per N1); persistent, MB CTAs per SM (ComplexF64 at
// three has 80 registers and spills, at two none)
template <typename V, int N1, int MB>
__global__ void __launch_bounds__(CFFT_THREADS, MB) k_p2col(KParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    p2col_body<V, N1>(p, smem);
}
template <typename V, int MB>
__global__ void __launch_bounds__(CFFT_THREADS, MB) k_p2row(KParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    r4096_body<V, R4096_P2A>(p, smem);
}
// pass A with tensor copies (ComplexF64): tm maps the chunk's input as
// [transform][c < 4096][2 N1 doubles] (strides N1 x 16 B, in_dist x 16 B)
template <int MB>
__global__ void __launch_bounds__(CFFT_THREADS, MB) k_p2row_tma(const __grid_constant__ CUtensorMap tm, KParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    r4096_body<double2, R4096_P2A_TMA>(p, smem, &tm);
}
// pass A for ComplexF32 with tensor copies of subsequence pairs (two CTAs
// per SM: 64 KB of pair buffer + the exchange buffer): tm maps the chunk's
// input as [transform][c < 4096][2 N1 floats] (strides N1 x 8 B, in_dist x 8 B)
__global__ void __launch_bounds__(CFFT_THREADS, 2) k_p2row_tma2(const __grid_constant__ CUtensorMap tm, KParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    p2row_pair_body(p, smem, &tm);
}
template <typename V, int MB> static const void* p2col_for(int N1) {
    switch (N1) {
        case 2: return (const void*)k_p2col<V, 2, MB>;
        case 4: return (const void*)k_p2col<V, 4, MB>;
        case 8: return (const void*)k_p2col<V, 8, MB>;
        case 16: return (const void*)k_p2col<V, 16, MB>;
        case 32: return (const void*)k_p2col<V, 32, MB>;
        case 64: return (const void*)k_p2col<V, 64, MB>;
        case 128: return (const void*)k_p2col<V, 128, MB>;
        case 256: return (const void*)k_p2col<V, 256, MB>;
        case 512: return (const void*)k_p2col<V, 512, MB>;
        case 1024: return (const void*)k_p2col<V, 1024, MB>;
    }
    return nullptr;
}
const void* cfft_p2col_kernel(int dtype, int N1, int mb) {
    if (dtype == CFFT_DT_C128) return mb == 2 ? p2col_for<double2, 2>(N1) : p2col_for<double2, 3>(N1);
    return p2col_for<float2, 3>(N1);
}
// single-pass power-of-two n = C x 4096 on clusters of C CTAs (pow2.cuh)
template <typename V, int C, int MB>
__global__ void __launch_bounds__(CFFT_THREADS, MB) k_p2cl(KParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    p2cl_body<V, C>(p, smem);
}
// ComplexF64 with the stride-C subsequence by tensor copies (two CTAs per SM)
template <int C>
__global__ void __launch_bounds__(CFFT_THREADS, 2) k_p2cl_tma(const __grid_constant__ CUtensorMap tm, KParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    p2cl_body<double2, C, true>(p, smem, &tm);
}
const void* cfft_p2cl_tma_kernel(int C) {
    switch (C) {
        case 2: return (const void*)k_p2cl_tma<2>;
        case 4: return (const void*)k_p2cl_tma<4>;
        case 8: return (const void*)k_p2cl_tma<8>;
        case 16: return (const void*)k_p2cl_tma<16>;
    }
    return nullptr;
}
template <typename V, int MB> static const void* p2cl_for(int C) {
    switch (C) {
        case 2: return (const void*)k_p2cl<V, 2, MB>;
        case 4: return (const void*)k_p2cl<V, 4, MB>;
        case 8: return (const void*)k_p2cl<V, 8, MB>;
        case 16: return (const void*)k_p2cl<V, 16, MB>;
    }
    return nullptr;
}
const void* cfft_p2cl_kernel(int dtype, int C, int mb) {
    if (dtype == CFFT_DT_C128) return mb == 2 ? p2cl_for<double2, 2>(C) : p2cl_for<double2, 3>(C);
    return mb == 2 ? p2cl_for<float2, 2>(C) : p2cl_for<float2, 3>(C);
}
// both power-of-two passes in one persistent dataflow launch (pow2.cuh),
// two CTAs per SM
template <typename V, int N1>
__global__ void __launch_bounds__(CFFT_THREADS, 2) k_p2flow(KParams pa, KParams pb, FlowCtl fc) {
    extern __shared__ __align__(128) unsigned char smem[];
    p2flow_body<V, N1>(pa, pb, fc, smem);
}
template <typename V> static const void* p2flow_for(int N1) {
    switch (N1) {
        case 8: return (const void*)k_p2flow<V, 8>;
        case 16: return (const void*)k_p2flow<V, 16>;
        case 32: return (const void*)k_p2flow<V, 32>;
        case 64: return (const void*)k_p2flow<V, 64>;
        case 128: return (const void*)k_p2flow<V, 128>;
        case 256: return (const void*)k_p2flow<V, 256>;
        case 512: return (const void*)k_p2flow<V, 512>;
        case 1024: return (const void*)k_p2flow<V, 1024>;
    }
    return nullptr;
}
const void* cfft_p2flow_kernel(int dtype, int N1) {
    return dtype == CFFT_DT_C128 ? p2flow_for<double2>(N1) : p2flow_for<float2>(N1);
}
size_t cfft_p2flow_smem(size_t elem_bytes, int N1, int staged_entries) {
    return ((16 * R4096_PL * elem_bytes + 15) & ~(size_t)15) + (129 + (size_t)N1 + staged_entries) * sizeof(double2) +
           16;
}
cudaError_t cfft_launch_p2flow(const void* f, const KParams& pa, const KParams& pb, int* ctr, void* ring, int nb,
                               int lag, int depth, unsigned grid, size_t smem, cudaStream_t st) {
    if (!f) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid, 1, 1);
    cfg.blockDim = dim3(CFFT_THREADS, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    KParams a = pa, b = pb;
    FlowCtl fc = {ctr, ctr + 1, ctr + 2, ring, nb, lag, depth};
    void* args[] = {(void*)&a, (void*)&b, (void*)&fc};
    cudaError_t e = cudaLaunchKernelExC(&cfg, f, args);
    if (e != cudaSuccess) cudaGetLastError();
    return e;
}
const void* cfft_p2row_tma_kernel(int mb) {
    return mb == 2 ? (const void*)k_p2row_tma<2> : (const void*)k_p2row_tma<3>;
}
const void* cfft_p2row_tma2_kernel() { return (const void*)k_p2row_tma2; }
size_t cfft_p2row_tma2_smem() { return (size_t)kP2PairBytes + cfft_r4096_smem(sizeof(float2)); }
// the driver's tensor-map encoder, looked up once through the runtime
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return (PFN_cuTensorMapEncodeTiled_v12000)f;
    }();
    return fn;
}
cudaError_t cfft_launch_p2row_tma(const void* f, const KParams& p, unsigned grid, size_t smem, cudaStream_t st) {
    auto enc = tensor_map_encoder();
    if (!f || !enc) return cudaErrorNotSupported;
    const int N1 = 1 << p.PA;
    const long long nb = (long long)p.batch >> p.PA;
    if (nb < 1 || nb > 0x7fffffffLL || ((uintptr_t)p.in & 15)) return cudaErrorInvalidValue;
    CUtensorMap tm;
    const cuuint64_t dims[3] = {(cuuint64_t)(2 * N1), 4096, (cuuint64_t)nb};
    const cuuint64_t strides[2] = {(cuuint64_t)N1 * 16, (cuuint64_t)p.in_dist * 16};
    const cuuint32_t box[3] = {2, 256, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    // L2 promotion to 256 B: the neighbouring subsequences of the same
    // lines are read by the CTAs working on the next rows
    CUresult r = enc(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void*)p.in, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid, 1, 1);
    cfg.blockDim = dim3(CFFT_THREADS, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    KParams pc = p;
    void* args[] = {(void*)&tm, (void*)&pc};
    cudaError_t e = cudaLaunchKernelExC(&cfg, f, args);
    if (e != cudaSuccess) cudaGetLastError();
    return e;
}
cudaError_t cfft_launch_p2row_tma2(const void* f, const KParams& p, unsigned grid, size_t smem, cudaStream_t st) {
    auto enc = tensor_map_encoder();
    if (!f || !enc) return cudaErrorNotSupported;
    const int N1 = 1 << p.PA;
    const long long nb = (long long)p.batch >> p.PA;
    // pairs of subsequences: N1 even, rows a multiple of 2; 16-byte aligned
    // base and strides (N1 x 8 B, in_dist x 8 B)
    if (N1 < 2 || (p.batch & 1) || nb < 1 || nb > 0x7fffffffLL || ((uintptr_t)p.in & 15) || (p.in_dist & 1))
        return cudaErrorInvalidValue;
    CUtensorMap tm;
    const cuuint64_t dims[3] = {(cuuint64_t)(2 * N1), 4096, (cuuint64_t)nb};
    const cuuint64_t strides[2] = {(cuuint64_t)N1 * 8, (cuuint64_t)p.in_dist * 8};
    const cuuint32_t box[3] = {4, 256, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void*)p.in, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid, 1, 1);
    cfg.blockDim = dim3(CFFT_THREADS, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    KParams pc = p;
    void* args[] = {(void*)&tm, (void*)&pc};
    cudaError_t e = cudaLaunchKernelExC(&cfg, f, args);
    if (e != cudaSuccess) cudaGetLastError();
    return e;
}
// a cluster kernel whose CTA c reads the stride-C subsequence x[c + C t],
// t < L, of its transform by tensor copies of `rows` x 16 bytes: the map is
// [transform][t < L][2 C doubles] (strides C x 16 B, in_dist x 16 B)
static cudaError_t launch_subseq_tma(const void* f, const KParams& p, int C, int L, int rows, unsigned grid,
                                     int threads, size_t smem, int cluster, cudaStream_t st) {
    auto enc = tensor_map_encoder();
    if (!f || !enc) return cudaErrorNotSupported;
    if (C < 1 || L < 1 || rows < 1 || rows > 256 || L % rows || p.batch < 1 || ((uintptr_t)p.in & 15))
        return cudaErrorInvalidValue;
    CUtensorMap tm;
    const cuuint64_t dims[3] = {(cuuint64_t)(2 * C), (cuuint64_t)L, (cuuint64_t)p.batch};
    const cuuint64_t strides[2] = {(cuuint64_t)C * 16, (cuuint64_t)p.in_dist * 16};
    const cuuint32_t box[3] = {2, (cuuint32_t)rows, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(&tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void*)p.in, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid, 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    KParams pc = p;
    void* args[] = {(void*)&tm, (void*)&pc};
    cudaError_t e = cudaLaunchKernelExC(&cfg, f, args);
    if (e != cudaSuccess) cudaGetLastError();
    return e;
}
cudaError_t cfft_launch_mixc_tma(const void* f, const KParams& p, unsigned grid, int threads, size_t smem,
                                 int cluster, cudaStream_t st) {
    return launch_subseq_tma(f, p, p.C, p.N2, mix_box_rows(p.N2), grid, threads, smem, cluster, st);
}
cudaError_t cfft_launch_p2cl_tma(const void* f, const KParams& p, unsigned grid, size_t smem, int cluster,
                                 cudaStream_t st) {
    return launch_subseq_tma(f, p, p.C, 4096, 256, grid, CFFT_THREADS, smem, cluster, st);
}
// The timeout path of the bounded waits, exercised without a fault: one
// thread arms nothing and waits on a fresh mbarrier's phase 0, which no one
// completes; after `polls` polls the wait gives up and records the fault bit
// exactly as a kernel whose tensor copy never landed would.
__global__ void k_wait_probe(int polls) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        if (!mbar_wait(&bar, 0, polls)) record_fault(kFaultTmaTimeout);
    }
}
cudaError_t cfft_wait_probe(int polls) {
    k_wait_probe<<<1, 32>>>(polls);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return e;
}
// each translation unit with kernels that record faults has its own copy of
// the word: this one's, OR-ed with the queue kernel's (queue.cu)
cudaError_t cfft_device_fault_word(unsigned* out, int clear) {
    cudaError_t e = cudaMemcpyFromSymbol(out, g_cfft_fault, sizeof(unsigned));
    if (e == cudaSuccess && clear) {
        const unsigned z = 0;
        e = cudaMemcpyToSymbol(g_cfft_fault, &z, sizeof(unsigned));
    }
    unsigned q = 0;
    if (e == cudaSuccess) e = cfft_queue_fault_word(&q, clear);
    if (e == cudaSuccess) *out |= q;
    return e;
}
const void* cfft_p2row_kernel(int dtype, int mb) {
    if (dtype == CFFT_DT_C128) return mb == 2 ? (const void*)k_p2row<double2, 2> : (const void*)k_p2row<double2, 3>;
    return (const void*)k_p2row<float2, 3>;
}
size_t cfft_p2col_smem(size_t elem_bytes, int N1) {
    return ((4096 * elem_bytes + 15) & ~(size_t)15) + (size_t)N1 * sizeof(double2);
}

// Rader on a cluster of C register-FFT CTAs (convc.cuh), MB CTAs per SM
// (ComplexF64 at three: 80 registers and some spills; at two: none)
template <typename V, int C, int MB>
__global__ void __launch_bounds__(CFFT_THREADS, MB) k_convc(KParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    convc_rader_body<V, C>(p, smem);
}
template <typename V, int MB> static const void* convc_for(int C) {
    switch (C) {
        case 3: return (const void*)k_convc<V, 3, MB>;
        case 4: return (const void*)k_convc<V, 4, MB>;
        case 5: return (const void*)k_convc<V, 5, MB>;
        case 7: return (const void*)k_convc<V, 7, MB>;
        case 8: return (const void*)k_convc<V, 8, MB>;
    }
    return nullptr;
}
const void* cfft_convc_kernel(int dtype, int C, int mb) {
    if (dtype == CFFT_DT_C128) return mb == 2 ? convc_for<double2, 2>(C) : convc_for<double2, 3>(C);
    return convc_for<float2, 3>(C);
}
size_t cfft_convc_smem(size_t elem_bytes) {
    // planes, w_4096 table (129), partial sum (1), reduction scratch (32) and
    // the total for y[0] (1), FP64
    return ((16 * R4096_PL * elem_bytes + 15) & ~(size_t)15) + (129 + 1 + 33) * sizeof(double2);
}

// mixed-radix lengths n = C L on a cluster of C register L-point CTAs
// (mixc.cuh): two CTAs per SM with both tables staged, or three with the
// w_n table read through L2 (variant 1; ComplexF64 spills at that budget)
template <typename V, class S, int MB, bool GTAB>
__global__ void __launch_bounds__(S::T, MB) k_mixc(KParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    mixc_body<V, S, GTAB>(p, smem);
}
// ComplexF64 with the strided input by tensor copies (tm: see mixc_body)
template <class S, int MB>
__global__ void __launch_bounds__(S::T, MB) k_mixc_tma(const __grid_constant__ CUtensorMap tm, KParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    mixc_body<double2, S, false, true>(p, smem, &tm);
}
struct MixEntry {
    int n, C, L, threads;
    const void* fn[2];            // ComplexF64, ComplexF32 (nullptr: none)
};
// 30240 = 7 x 4320, 4320 = 16 x 18 x 15 on 288 threads (variants 0, 1), and
// 30240 = 9 x 3360, 3360 = 14 x 16 x 15 on 240 threads (variants 2 and 3:
// the stages keep 240 / 210 / 224 of 240 threads busy, 16 values per thread
// at most; three or two CTAs per SM)
using Mix30240 = MixShape<7, 16, 18, 15, 288>;
using Mix30240b = MixShape<9, 14, 16, 15, 240>;
// variants 4 and 5: ComplexF64 by tensor copies, both splits, two CTAs per SM
static const MixEntry kMix[][6] = {
    {{30240, 7, 4320, 288, {(const void*)k_mixc<double2, Mix30240, 2, false>, (const void*)k_mixc<float2, Mix30240, 2, false>}},
     {30240, 7, 4320, 288, {(const void*)k_mixc<double2, Mix30240, 3, true>, (const void*)k_mixc<float2, Mix30240, 3, true>}},
     {30240, 9, 3360, 240, {(const void*)k_mixc<double2, Mix30240b, 3, false>, (const void*)k_mixc<float2, Mix30240b, 3, false>}},
     {30240, 9, 3360, 240, {(const void*)k_mixc<double2, Mix30240b, 2, false>, (const void*)k_mixc<float2, Mix30240b, 2, false>}},
     {30240, 7, 4320, 288, {(const void*)k_mixc_tma<Mix30240, 2>, nullptr}},
     {30240, 9, 3360, 240, {(const void*)k_mixc_tma<Mix30240b, 2>, nullptr}}},
};
int cfft_mixc_lookup(long long n, int dtype, int variant, const void** fn, int* C, int* L, int* threads) {
    for (const auto& row : kMix) {
        if (row[0].n != n || variant < 0 || variant > 5) continue;
        const MixEntry& m = row[variant];
        if (!m.fn[dtype == CFFT_DT_C128 ? 0 : 1]) return 0;
        *fn = m.fn[dtype == CFFT_DT_C128 ? 0 : 1];
        *C = m.C;
        *L = m.L;
        *threads = m.threads;
        return 1;
    }
    return 0;
}

const void* cfft_kernel_for(int mode, int dtype) {
    if (dtype == CFFT_DT_C128) {
        switch (mode) {
            case MODE_ROWS: return (const void*)k_rows<double2, CFFT_EMAX>;
            case MODE_FOUR: return (const void*)k_four<double2, CFFT_EMAX, DynK<0>>;
            case MODE_FOUR_WARP: return (const void*)k_four<double2, CFFT_EMAX, DynK<1>>;
            case MODE_COLPASS: return (const void*)k_colpass<double2, CFFT_EMAX>;
            case MODE_ROWPASS: return (const void*)k_rowpass<double2, CFFT_EMAX>;
        }
    } else {
        switch (mode) {
            case MODE_ROWS: return (const void*)k_rows<float2, CFFT_EMAX>;
            case MODE_FOUR: return (const void*)k_four<float2, CFFT_EMAX, DynK<0>>;
            case MODE_FOUR_WARP: return (const void*)k_four<float2, CFFT_EMAX, DynK<1>>;
            case MODE_COLPASS: return (const void*)k_colpass<float2, CFFT_EMAX>;
            case MODE_ROWPASS: return (const void*)k_rowpass<float2, CFFT_EMAX>;
        }
    }
    return nullptr;
}

// ---- statically shaped FOUR kernels for the hot lengths
// radix multiplicities are listed in CFFT_EXEC_ORDER (9, 7, 5, 3, 16, 8, 4, 2)
// and each Seq<> names the passes in that order
struct StaticFour {
    int dtype, N1, N2, C;
    unsigned char ca[8], cc[8];
    const void* fn;
    int single;                   // one shared buffer for both layouts
};
// 30240 = 168 x 180 on a 12-CTA cluster (ComplexF64 mixed-radix batch)
using K_168x180_c12 = StatK<168, 180, 12, Seq<7, 3, 8>, true, 1, Seq<9, 5, 4>, true, 1>;
// Rader M = 20160 = 168 x 120 on an 8-CTA cluster (primes 10007 .. 10081)
using K_168x120_c8 = StatK<168, 120, 8, Seq<7, 3, 8>, true, 1, Seq<5, 3, 8>, true, 3>;
// 30240 on a 6-CTA cluster with one shared buffer per CTA (two CTAs/SM at
// twice the elements per CTA; 8 % faster than the 12-CTA kernel on B200),
// each warp transforming two columns at a time (another 10 %)
using K_168x180_c6s = StatK<168, 180, 6, Seq<7, 3, 8>, true, 2, Seq<9, 5, 4>, true, 1, true>;
// single-buffer 12- and 8-CTA shapes at three CTAs/SM (EMAX 10 / 9)
using K_168x180_c12s = StatK<168, 180, 12, Seq<7, 3, 8>, true, 1, Seq<9, 5, 4>, true, 1, true>;
using K_168x120_c8s = StatK<168, 120, 8, Seq<7, 3, 8>, true, 1, Seq<5, 3, 8>, true, 1, true>;
// 65536 = 256 x 256 on a 16-CTA cluster (ComplexF32 precision form)
using K_256x256_c16 = StatK<256, 256, 16, Seq<16, 16>, true, 2, Seq<16, 16>, true, 2>;

static const StaticFour kStatic[] = {
    //                        9  7  5  3 16  8  4  2
    {CFFT_DT_C128, 168, 180, 12, {0, 1, 0, 1, 0, 1, 0, 0}, {1, 0, 1, 0, 0, 0, 1, 0},
     (const void*)k_four_mb<double2, 10, K_168x180_c12s, 3>, 1},
    {CFFT_DT_C64, 168, 180, 12, {0, 1, 0, 1, 0, 1, 0, 0}, {1, 0, 1, 0, 0, 0, 1, 0},
     (const void*)k_four<float2, CFFT_EMAX, K_168x180_c12>, 0},
    {CFFT_DT_C128, 168, 120, 8, {0, 1, 0, 1, 0, 1, 0, 0}, {0, 0, 1, 1, 0, 1, 0, 0},
     (const void*)k_four_mb<double2, 9, K_168x120_c8s, 3>, 1},
    {CFFT_DT_C64, 168, 120, 8, {0, 1, 0, 1, 0, 1, 0, 0}, {0, 0, 1, 1, 0, 1, 0, 0},
     (const void*)k_four<float2, CFFT_EMAX, K_168x120_c8>, 0},
    {CFFT_DT_C128, 168, 180, 6, {0, 1, 0, 1, 0, 1, 0, 0}, {1, 0, 1, 0, 0, 0, 1, 0},
     (const void*)k_four<double2, CFFT_EMAX, K_168x180_c6s>, 1},
    {CFFT_DT_C64, 256, 256, 16, {0, 0, 0, 0, 2, 0, 0, 0}, {0, 0, 0, 0, 2, 0, 0, 0},
     (const void*)k_four<float2, CFFT_EMAX, K_256x256_c16>, 0},
};

const void* cfft_static_four(int dtype, int N1, int N2, int C, const unsigned char* ca,
                             const unsigned char* cc, int* single) {
    for (const auto& e : kStatic) {
        if (e.dtype != dtype || e.N1 != N1 || e.N2 != N2 || e.C != C) continue;
        bool same = true;
        for (int i = 0; i < 8; i++) same = same && e.ca[i] == ca[i] && e.cc[i] == cc[i];
        if (same) {
            if (single) *single = e.single;
            return e.fn;
        }
    }
    return nullptr;
}

cudaError_t cfft_prepare_fn(const void* f, size_t smem, int cluster) {
    if (!f) return cudaErrorInvalidValue;
    // always the device maximum: a smaller value set for one plan would break
    // another plan that shares the kernel and needs more
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, f);
    if (e != cudaSuccess) return e;
    const size_t cap = 232448 - fa.sharedSizeBytes;   // 227 KB per block minus static
    if (smem > cap) return cudaErrorInvalidValue;
    e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap);
    if (e != cudaSuccess) return e;
    if (cluster > 8) {
        e = cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t cfft_launch_fn(const void* f, const KParams& p, unsigned grid, int threads, size_t smem,
                           int cluster, cudaStream_t stream) {
    if (!f) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid, 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    if (cluster > 1) {
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = cluster;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
    void* args[] = {(void*)&p};
    cudaError_t e = cudaLaunchKernelExC(&cfg, f, args);
    if (e != cudaSuccess) cudaGetLastError();   // do not leave it for the caller's next check
    return e;
}

cudaError_t cfft_max_active_clusters_fn(const void* f, int threads, size_t smem, int cluster, int* out) {
    if (!f) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cluster, 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaOccupancyMaxActiveClusters(out, f, &cfg);
}
