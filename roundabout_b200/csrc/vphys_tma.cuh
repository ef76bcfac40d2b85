// vphys_tma.cuh -- the pieces shared by the TMA-staged column solves: bounded
// mbarrier waits and plain (non-multicast) tiled TMA loads of level blocks
// into shared memory.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>

#include "vphys_tiles.cuh"

namespace vphys {

// ---- mbarriers and TMA ------------------------------------------------------
constexpr long long TMA_WAIT_LIMIT = 1LL << 22;   // try_wait polls before a wait is declared lost

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mb_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mb_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mb_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
// bounded wait for the phase of parity `parity`; false when the limit ran out
__device__ __forceinline__ bool mb_wait(uint64_t *bar, uint32_t parity)
{
    const uint32_t a = smem_addr(bar);
    for (long long it = 0; it < TMA_WAIT_LIMIT; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}
// 2-D tiled load (x: the element index inside a level plane, y: the level)
// into shared memory, completing on `bar`; never multicast
__device__ __forceinline__ void tma_load_2d_f64(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar,
                                                uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1, {%2, %3}], [%4], %5;" ::"r"(smem_addr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar)), "l"(policy)
        : "memory");
}

}  // namespace vphys
