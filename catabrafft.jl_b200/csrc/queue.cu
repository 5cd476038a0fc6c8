// queue.cu -- the batched form's single launch over a queue of work items
// (QItem, engine_types.h).  Each CTA claims one ticket (atomic, so tickets
// are handed out in order whatever order the CTAs start in), waits (bounded)
// for its item's dependency, stages the item's parameter block with the
// launch's base pointers and direction, sets blk0 so that the body sees the
// item's block index, and runs the single-plan body of the item's kind.
// A CTA per item rather than a loop over items: every body keeps the
// register allocation it has as a kernel of its own (a loop around the
// bodies, or calls to non-inlined copies, spill kilobytes per thread).
// Every wait is on smaller tickets, whose CTAs are already running, so the
// launch drains for any residency.  A wait that runs out sets the abort
// flag and the fault word (kFaultFlowTimeout); later CTAs then skip their
// items.
#include "engine.cuh"
#include "kernels.h"
#include "pow2.cuh"

template <typename V, int MB>
__global__ void __launch_bounds__(CFFT_THREADS, MB) kq_batch(QueueLaunch L) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ KParams sp;
    __shared__ int s_item[2];
    int* const abort = L.ctl + 1;
    int* const ctr = L.ctl + 2;
    if (threadIdx.x == 0) {
        int i = atomicAdd(L.ctl, 1);
        if (i < L.nitems && ld_acquire_gpu(abort)) i = L.nitems;
        s_item[0] = i;
    }
    __syncthreads();
    const int i = s_item[0];
    if (i >= L.nitems) return;
    const QItem it = L.items[i];
    if (it.wait >= 0 && !flow_wait(ctr + it.wait, it.need, s_item + 1, abort)) return;
    if (threadIdx.x == 0) {
        KParams p = L.desc[it.desc];
        if (p.in_user) p.in = (const V*)L.in_base + p.in_off;
        if (p.out_user) p.out = (V*)L.out_base + p.out_off;
        if (L.dir >= 0) {
            p.dir = L.dir;
            if (L.dir != 1) p.scale = 1.0;
        }
        p.blk0 = (int)blockIdx.x - it.blk;
        sp = p;
    }
    __syncthreads();
    switch (it.kind) {
        case QK_ROWS: rows_body<V, CFFT_EMAX>(sp, smem); break;
        case QK_FOUR: four_body<V, CFFT_EMAX, DynK<0>>(sp, smem); break;
        case QK_FOUR_WARP: four_body<V, CFFT_EMAX, DynK<1>>(sp, smem); break;
        case QK_COLPASS: colpass_body<V, CFFT_EMAX>(sp, smem); break;
        default: rowpass_body<V, CFFT_EMAX>(sp, smem); break;
    }
    if (it.done >= 0) flow_publish(ctr + it.done);
}

// ComplexF64 at two CTAs per SM (128 registers); ComplexF32 at three (the
// pass kernels' residency, 80 registers) or two
const void* cfft_queue_kernel(int dtype, int mb) {
    if (dtype == CFFT_DT_C128) return (const void*)kq_batch<double2, 2>;
    return mb == 3 ? (const void*)kq_batch<float2, 3> : (const void*)kq_batch<float2, 2>;
}
cudaError_t cfft_launch_queue(const void* fn, const QueueLaunch& L, unsigned grid, size_t smem, cudaStream_t st) {
    void* args[] = {(void*)&L};
    cudaError_t e = cudaLaunchKernel(fn, dim3(grid), dim3(CFFT_THREADS), args, smem, st);
    if (e != cudaSuccess) cudaGetLastError();
    return e;
}
cudaError_t cfft_queue_fault_word(unsigned* out, int clear) {
    cudaError_t e = cudaMemcpyFromSymbol(out, g_cfft_fault, sizeof(unsigned));
    if (e == cudaSuccess && clear) {
        const unsigned z = 0;
        e = cudaMemcpyToSymbol(g_cfft_fault, &z, sizeof(unsigned));
    }
    return e;
}
