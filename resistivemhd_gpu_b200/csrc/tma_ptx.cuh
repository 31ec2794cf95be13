// tma_ptx.cuh -- the PTX with which the fused stage kernel stages its tile:
// mbarrier set-up and tries, the bulk tensor (TMA) loads of the tile and of
// the eta table, the async-proxy fence, and an L2 prefetch, one inline
// function each.
//
// A host build of the stage kernel (CPU tests) defines
// RMHD_HOST_EMULATION and supplies its own definitions of these
// functions; this header then only declares them.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace rmhd2d {

#if defined(RMHD_HOST_EMULATION)

void mbar_init_tile(uint64_t *bar);
bool mbar_try_wait(uint64_t *bar, uint32_t phase);
void fence_proxy_async();
void mbar_expect_tx(uint64_t *bar, uint32_t bytes);
void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z);
void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y);
void prefetch_l2(const void *p);

#else

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// One-arrival mbarrier for the tile's staging, made visible to the async proxy.
__device__ __forceinline__ void mbar_init_tile(uint64_t *bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One try of the wait for phase `phase` (suspending for at most 20 us).
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t phase)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(phase), "r"(20000u)
        : "memory");
    return ok != 0;
}

// Orders the CTA's earlier shared-memory accesses before an async copy.
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// The arrival of the staging thread, expecting `bytes` of async copies.
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// Box of `map` at (x, y, z) into shared memory at dst, completing on bar.
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)),
          "r"(x), "r"(y), "r"(z)
        : "memory");
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)),
          "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void prefetch_l2(const void *p)
{
    asm volatile("prefetch.global.L2 [%0];" ::"l"(__cvta_generic_to_global(p)));
}

#endif

}  // namespace rmhd2d
