// tcs_tma.cuh -- tensor-memory-accelerator (TMA) tile loads into shared
// memory for one thread block, with mbarrier completion, for sm_100a.
//
// Only plain tiled loads of this GPU's own memory are issued (one CTA, no
// cluster multicast).  Every wait on an mbarrier is bounded: a wait that runs
// out returns false, and the caller records the failure and leaves the kernel
// after bounded waits for its other copies in flight.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace tcs {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes the initialised barriers visible to the asynchronous (TMA) proxy.
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Orders this thread's earlier shared-memory accesses before later
// asynchronous-proxy accesses (a TMA write into a buffer the block has read).
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity to complete, at most `limit`
// polls (each try_wait itself suspends for a bounded time).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int limit)
{
    for (int it = 0; it < limit; it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// A 3-D tiled load of the box at (x, y, z) of the tensor map into dst
// (128-byte aligned shared memory); completion is counted on bar in bytes.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
                 ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
                 : "memory");
}

} // namespace tcs
