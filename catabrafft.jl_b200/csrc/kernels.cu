// kernels.cu -- sm_100a kernel entry points and their launcher.
#include "engine.cuh"
#include "kernels.h"

// 256 threads per CTA; FP64 data keeps 2 CTAs/SM resident (128 regs/thread),
// FP32 data 3 CTAs/SM (85 regs/thread).
template <typename V> struct MinBlocks { static constexpr int value = 3; };
template <> struct MinBlocks<double2> { static constexpr int value = 2; };

template <typename V, int EMAX>
__global__ void __launch_bounds__(CFFT_THREADS, MinBlocks<V>::value) k_rows(KParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    rows_body<V, EMAX>(p, smem);
}
template <typename V, int EMAX>
__global__ void __launch_bounds__(CFFT_THREADS, MinBlocks<V>::value) k_four(KParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    four_body<V, EMAX>(p, smem);
}
template <typename V, int EMAX>
__global__ void __launch_bounds__(CFFT_THREADS, MinBlocks<V>::value) k_colpass(KParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    colpass_body<V, EMAX>(p, smem);
}
template <typename V, int EMAX>
__global__ void __launch_bounds__(CFFT_THREADS, MinBlocks<V>::value) k_rowpass(KParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    rowpass_body<V, EMAX>(p, smem);
}

static const void* kernel_for(int mode, int dtype) {
    if (dtype == CFFT_DT_C128) {
        switch (mode) {
            case MODE_ROWS: return (const void*)k_rows<double2, CFFT_EMAX>;
            case MODE_FOUR: return (const void*)k_four<double2, CFFT_EMAX>;
            case MODE_COLPASS: return (const void*)k_colpass<double2, CFFT_EMAX>;
            case MODE_ROWPASS: return (const void*)k_rowpass<double2, CFFT_EMAX>;
        }
    } else {
        switch (mode) {
            case MODE_ROWS: return (const void*)k_rows<float2, CFFT_EMAX>;
            case MODE_FOUR: return (const void*)k_four<float2, CFFT_EMAX>;
            case MODE_COLPASS: return (const void*)k_colpass<float2, CFFT_EMAX>;
            case MODE_ROWPASS: return (const void*)k_rowpass<float2, CFFT_EMAX>;
        }
    }
    return nullptr;
}

cudaError_t cfft_prepare_kernel(int mode, int dtype, size_t smem, int cluster) {
    const void* f = kernel_for(mode, dtype);
    if (!f) return cudaErrorInvalidValue;
    // always the device maximum: a smaller value set for one plan would break
    // another plan that shares the kernel and needs more
    if (smem > 232448) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, 232448);
    if (e != cudaSuccess) return e;
    if (cluster > 8) {
        e = cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t cfft_launch(const KParams& p, int dtype, unsigned grid, int threads, size_t smem,
                        int cluster, cudaStream_t stream) {
    const void* f = kernel_for(p.mode, dtype);
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
    return cudaLaunchKernelExC(&cfg, f, args);
}

cudaError_t cfft_max_active_clusters(int mode, int dtype, int threads, size_t smem, int cluster,
                                     int* out) {
    const void* f = kernel_for(mode, dtype);
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
