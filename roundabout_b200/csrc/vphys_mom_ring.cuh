// vphys_mom_ring.cuh -- the TMA-staged ring of the momentum face solves,
// shared by the exact (FP64) and the mixed-precision solver.
//
// A tile is MT_TW consecutive u (or v) faces in the flattened face index;
// u and v tiles alternate (mt_tile_of) so the cells' h and kv that both
// families read come from HBM once and hit L2 the second time.  One CTA per
// SM slot is persistent and walks tiles blockIdx.x, blockIdx.x + grid, ...:
//
//   * warp MT_WARPS, lane 0 (the producer) streams each tile's levels in
//     blocks of MT_U into an MT_S-stage shared-memory ring: one plain 2-D
//     cp.async.bulk.tensor per field and block (the cells either side of the
//     faces -- h and kv, one block for u tiles, the rows j-1 and j for v
//     tiles -- and the velocities), completing on the stage's mbarrier;
//   * warps 0..MT_WARPS-1 run one face each: the solver's forward sweep
//     reads the ring, a stage is released to the producer once every
//     consumer warp is done with it, and the back-substitution runs from the
//     solver's shared-memory rows while the producer already fills the ring
//     with the next tile.
//
// Tiles whose every face touches land and carries a zero velocity at every
// level are skipped (p.mom_tile_skip, set by k_mom_tile_flags).  Every
// mbarrier wait is bounded; on expiry the kernel records the failure in
// p.dev_err and the CTA stops, the producer first draining the copies it
// issued.  No copy is multicast and every tensor map covers this GPU's own
// buffers.
//
// The solver F provides, for one face (member state):
//   start(p, dt, fc, valid, uf, PF, rows, tid)  the face's set-up
//   first(hl, hr, uw)                           level 1's face thickness
//   row(m, hl, hr, kvl, kvr, uw)                row m (1..nz-1) with level m+1's data
//   last()                                      row nz
//   back()                                      the back-substitution and the store
// `rows` is the CTA's shared-memory row area, nz * MT_TW * 8 bytes.
#pragma once

#include "vphys_kernels.cuh"
#include "vphys_tiles.cuh"
#include "vphys_tma.cuh"

#ifndef VPHYS_MT_U
#define VPHYS_MT_U 2
#endif
#ifndef VPHYS_MT_S
#define VPHYS_MT_S 3
#endif

namespace vphys {

constexpr int MT_U = VPHYS_MT_U;               // levels per stage
constexpr int MT_S = VPHYS_MT_S;               // stages in the ring
constexpr int MT_THREADS = MT_TW + 32;         // + the producer warp

__host__ __device__ constexpr int mt_round128(int b) { return (b + 127) / 128 * 128; }
constexpr int MT_BLK_C = mt_round128(MT_U * MT_BW * 8);   // bytes of one cell block (h or kv, one row of cells)
constexpr int MT_BLK_W = mt_round128(MT_U * MT_TW * 8);   // bytes of the velocity block
// stage: hA, hB, kA, kB (cell blocks), w (velocities)
constexpr int MT_STAGE = 4 * MT_BLK_C + MT_BLK_W;
constexpr uint32_t MT_TX_U = (uint32_t)(2 * MT_U * MT_BW * 8 + MT_U * MT_TW * 8);   // bytes a u stage delivers
constexpr uint32_t MT_TX_V = (uint32_t)(4 * MT_U * MT_BW * 8 + MT_U * MT_TW * 8);   // bytes a v stage delivers

struct MomMaps {
    CUtensorMap h, kv, u, v;
};

// Tiles alternate between the families: tile 2k is u tile k, tile 2k+1 is v
// tile k.  Both cover nearly the same rows (k*128 faces into rows of nx+1 and
// nx faces).  A tile past its family's last face is skipped.
__host__ __device__ __forceinline__ void mt_tile_of(int t, bool &xf, long long &f0)
{
    xf = (t & 1) == 0;
    f0 = (long long)(t >> 1) * MT_TW;
}

// Dynamic shared memory of the ring kernel for nz levels.
__host__ __device__ constexpr size_t mt_smem_bytes(int nz)
{
    return 128 + (size_t)MT_S * MT_STAGE + 2 * MT_S * sizeof(unsigned long long) + 32 * sizeof(int) +
           (size_t)nz * MT_TW * 8;
}

// Host side (vphys_momentum_tma.cu): the tensor maps and the tile flags of a
// ring launch (false: the configuration or the buffers do not qualify), and
// the persistent grid of a ring kernel.
bool momentum_ring_prepare(const Params &p, MomMaps *maps, int *ntiles, cudaStream_t stream);
// the tensor map of a level-major FP64 field [planes][n], boxes {box_x, box_y}
bool tma_map_planes(CUtensorMap *m, const void *base, size_t n, int planes, int box_x, int box_y);
int momentum_ring_grid(const void *kernel, int ntiles, size_t smem);

template <class F>
__device__ __forceinline__ void momentum_ring_cta(const MomMaps &maps, const Params &p, double dt, int ntiles,
                                                  unsigned char *smem_raw)
{
    // the ring's blocks start on 128-byte boundaries (the size has 128 B of slack)
    unsigned char *ring = reinterpret_cast<unsigned char *>(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    uint64_t *full = reinterpret_cast<uint64_t *>(ring + (size_t)MT_S * MT_STAGE);
    uint64_t *empty = full + MT_S;
    int *abort_flag = reinterpret_cast<int *>(empty + MT_S);
    unsigned char *rows = reinterpret_cast<unsigned char *>(abort_flag + 32);   // the solver's [nz][MT_TW] rows

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nz = p.nz, nx = p.nx, ny = p.ny;
    const int nst = (nz + MT_U - 1) / MT_U;   // stages per tile
    volatile int *abort_v = abort_flag;

    if (threadIdx.x == 0) {
        for (int s = 0; s < MT_S; ++s) {
            mb_init(&full[s], 1);
            mb_init(&empty[s], MT_WARPS);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == MT_WARPS) {
        // ---- producer ----
        if (lane != 0) return;
        const uint64_t pol = l2_policy_evict_normal();
        long long it = 0;   // stages armed so far
        bool lost = false;
        for (int t = blockIdx.x; t < ntiles && !lost; t += gridDim.x) {
            if (p.mom_tile_skip[t]) continue;
            bool xf;
            long long f0;
            mt_tile_of(t, xf, f0);
            const FaceTile ft = face_tile(xf, f0, nx);
            const CUtensorMap *wmap = xf ? &maps.u : &maps.v;
            for (int s = 0; s < nst; ++s, ++it) {
                const int slot = (int)(it % MT_S);
                if (!mb_wait(&empty[slot], (uint32_t)(((it / MT_S) & 1) ^ 1)) || *abort_v) {
                    atomicOr(p.dev_err, 2u);
                    *abort_v = 1;
                    lost = true;
                    break;
                }
                unsigned char *st = ring + (size_t)slot * MT_STAGE;
                const int y = s * MT_U;
                mb_expect_tx(&full[slot], xf ? MT_TX_U : MT_TX_V);
                tma_load_2d_f64(st, &maps.h, (int)ft.xa, y, &full[slot], pol);
                tma_load_2d_f64(st + 2 * MT_BLK_C, &maps.kv, (int)ft.xa, y, &full[slot], pol);
                if (!xf) {
                    tma_load_2d_f64(st + MT_BLK_C, &maps.h, (int)ft.xb, y, &full[slot], pol);
                    tma_load_2d_f64(st + 3 * MT_BLK_C, &maps.kv, (int)ft.xb, y, &full[slot], pol);
                }
                tma_load_2d_f64(st + 4 * MT_BLK_C, wmap, (int)ft.xw, y, &full[slot], pol);
            }
        }
        if (lost) {
            // drain: every armed stage's bytes land before the CTA may exit
            const long long first = it > MT_S ? it - MT_S : 0;
            for (long long a = first; a < it; ++a)
                if (!mb_wait(&full[(int)(a % MT_S)], (uint32_t)((a / MT_S) & 1))) atomicOr(p.dev_err, 4u);
        }
        return;
    }

    // ---- consumers: one thread per face ----
    const int tid = threadIdx.x;
    constexpr int KOFF = 2 * (MT_BLK_C / 8);
    constexpr int WOFF = 4 * (MT_BLK_C / 8);
    long long it = 0;   // stages consumed so far
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        if (p.mom_tile_skip[t]) continue;
        bool xf;
        long long f0;
        mt_tile_of(t, xf, f0);
        const long long nf = xf ? (long long)(nx + 1) * ny : (long long)nx * (ny + 1);
        const FaceTile ft = face_tile(xf, f0, nx);
        const bool valid = f0 + tid < nf;
        const long long f = valid ? f0 + tid : nf - 1;
        const FaceCells fc = face_cells(xf, f, nx, ny, ft);
        const size_t PF = xf ? p.plane_u : p.plane_v;
        // offsets (doubles) of the two cells' h inside a stage; kv sits 2 blocks further
        const int lo = fc.bl * (MT_BLK_C / 8) + fc.ol;
        const int ro = fc.br * (MT_BLK_C / 8) + fc.orr;
        F face;
        face.start(p, dt, fc, valid, (xf ? p.u : p.v) + f, PF, rows, tid);
        for (int sg = 0; sg < nst; ++sg, ++it) {
            const int slot = (int)(it % MT_S);
            if (!mb_wait(&full[slot], (uint32_t)((it / MT_S) & 1)) || *abort_v) {
                if (lane == 0) atomicOr(p.dev_err, 1u);
                *abort_v = 1;
                return;
            }
            const double *st = reinterpret_cast<const double *>(ring + (size_t)slot * MT_STAGE);
#pragma unroll
            for (int q = 0; q < MT_U; ++q) {
                const int m = sg * MT_U + q;   // the level plane this slot holds (0-based)
                if (m >= nz) break;
                const double hl = st[lo + q * MT_BW], hr = st[ro + q * MT_BW];
                const double uw = st[WOFF + q * MT_TW + tid];
                if (m == 0)
                    face.first(hl, hr, uw);
                else
                    face.row(m, hl, hr, st[KOFF + lo + q * MT_BW], st[KOFF + ro + q * MT_BW], uw);
            }
            __syncwarp();
            if (lane == 0) mb_arrive(&empty[slot]);
        }
        face.last();
        face.back();
    }
}

}  // namespace vphys
