// kernels.h -- host-side view of the device engine (shared with plan.cpp).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>


#define CFFT_DT_C128 0
#define CFFT_DT_C64 1
#define CFFT_EMAX 16
#define CFFT_THREADS 256

#include "engine_types.h"

cudaError_t cfft_prepare_kernel(int mode, int dtype, size_t smem, int cluster);
cudaError_t cfft_launch(const KParams& p, int dtype, unsigned grid, int threads, size_t smem,
                        int cluster, cudaStream_t stream);
cudaError_t cfft_max_active_clusters(int mode, int dtype, int threads, size_t smem, int cluster,
                                     int* out);
