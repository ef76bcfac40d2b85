// vphys_tmem.cuh -- the tensor-memory row store of the column solves.
//
// A CTA holds all 512 columns of its SM's tensor memory (one CTA per SM; warp
// 0 allocates before the work and frees after it).  Warp w owns the 32 lanes
// of quarter w % 4 and a slot of 2*nzp 32-bit columns, (w / 4) * 2*nzp
// onwards, so three warps share a quarter at nz <= 85.  A level's two words
// go in with one tcgen05.st (32x32b.x2) and eight levels come back with one
// tcgen05.ld (32x32b.x16); the column solves keep their per-level rows there
// instead of in shared memory, which leaves the SM's L1 to the loads.
#pragma once

#include <cstdint>

namespace vphys {

__device__ __forceinline__ void tmem_alloc_all(uint32_t *slot)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(slot))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free_all(uint32_t base)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(base) : "memory");
}
__device__ __forceinline__ void tmem_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// taddr of warp `w`'s slot: lane quarter w % 4, columns (w / 4) * 2 nzp
__device__ __forceinline__ uint32_t tmem_warp_slot(uint32_t base, int w, int nzp)
{
    return base + ((uint32_t)(32 * (w & 3)) << 16) + (uint32_t)((w >> 2) * 2 * nzp);
}

// level k's two words at columns 2(k-1), 2(k-1)+1 of the slot
__device__ __forceinline__ void tmem_put2(uint32_t slot, int k, uint32_t a, uint32_t b)
{
    __syncwarp();
    asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(slot + 2u * (uint32_t)(k - 1)), "r"(a),
                 "r"(b)
                 : "memory");
}
__device__ __forceinline__ void tmem_store_done()
{
    __syncwarp();
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
// levels 8 kb + 1 .. 8 kb + 8: 16 words, two per level
__device__ __forceinline__ void tmem_get16(uint32_t slot, int kb, uint32_t (&r)[16])
{
    __syncwarp();
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(slot + 16u * (uint32_t)kb));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

}  // namespace vphys
