// tma.cuh -- Blackwell tile movement: tensor-memory-accelerator (TMA) copies
// completing on shared-memory mbarriers, with bounded waits.
//
// One elected thread arms an mbarrier with the bytes it expects and issues
// cp.async.bulk.tensor copies of boxes described by a CUtensorMap (encoded on
// the host, passed as a __grid_constant__ kernel parameter); the copies land
// in shared memory without passing through registers or the load/store
// queue.  Every other thread waits on the barrier's phase.  Only this GPU's
// own memory is ever a source, and no copy uses cluster multicast.
//
// Waits are bounded: a wait that has not completed after kWaitLimit polls
// records kFaultTmaTimeout in the device fault word (read and cleared by the
// host with cfft_device_faults) and the kernel leaves its loop, so a copy
// that never completes cannot hang the GPU.
#pragma once
#include <cuda.h>
#include <stdint.h>

// device fault word: bit 0 = an mbarrier wait on a tensor copy timed out
static __device__ unsigned int g_cfft_fault = 0;
constexpr unsigned kFaultTmaTimeout = 1u;
// polls of try_wait (each may suspend the thread for a short, hardware
// chosen time) before a wait gives up: seconds, far beyond any copy
constexpr int kWaitLimit = 1 << 24;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    // make the initialised barrier visible to the async (TMA) proxy
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
// true once the barrier's phase `parity` has completed; false after `limit`
// polls (kWaitLimit unless a caller asks for fewer)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int limit = kWaitLimit) {
    const uint32_t a = smem_addr(bar);
    for (int it = 0; it < limit; it++) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// order this thread's earlier generic-proxy shared-memory accesses (made
// visible to it by a barrier) before async-proxy writes it issues next
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// 3-D tiled tensor copy global -> shared, completing on `bar`
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
        "[%2];" ::"r"(smem_addr(dst)),
        "l"((uint64_t)map), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}
__device__ __forceinline__ void record_fault(unsigned bits) { atomicOr(&g_cfft_fault, bits); }
