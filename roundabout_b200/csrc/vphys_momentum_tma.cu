// vphys_momentum_tma.cu -- the host side of the TMA-staged momentum ring
// (vphys_mom_ring.cuh: the tensor maps, the eligibility of a configuration,
// the persistent grid) and the tile flags it reads.
//
// The ring runs the mixed-precision face solve (vphys_mixed.cu, MixedFace).
// The exact solve stays on the register-prefetched k_momentum: measured on
// 1440x1080x75, the same arithmetic fed from the ring ran 4.72 ms against
// 4.69 ms (its forward sweep waits on dependent FP64 divisions, not on
// loads), and a branch-free proven-quotient form of it ran 5.01 ms.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "vphys_device.cuh"
#include "vphys_faces.cuh"
#include "vphys_kernels.cuh"
#include "vphys_mom_ring.cuh"

namespace vphys {

// One CTA per tile: the tile is skipped when every face in it touches land
// and has a zero velocity at every level (what the register-prefetched solve
// skips face by face), or lies past the last face.
__global__ void __launch_bounds__(MT_TW) k_mom_tile_flags(const Params p)
{
    const int t = blockIdx.x;
    bool xf;
    long long f0;
    mt_tile_of(t, xf, f0);
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const long long nf = xf ? (long long)(nx + 1) * ny : (long long)nx * (ny + 1);
    const long long f = f0 + threadIdx.x;
    int skip = 1;
    if (f < nf) {
        const FaceTile ft = face_tile(xf, f0, nx);
        const FaceCells fc = face_cells(xf, f, nx, ny, ft);
        skip = fmn(p.wet[fc.cl], p.wet[fc.cr]) == 0.0;
        if (skip) {
            const double *uf = (xf ? p.u : p.v) + f;
            const size_t PF = xf ? p.plane_u : p.plane_v;
            for (int k = 0; k < nz && skip; ++k) skip = (uf[PF * (size_t)k] == 0.0);
        }
    }
    skip = __syncthreads_and(skip);
    if (threadIdx.x == 0) p.mom_tile_skip[t] = (unsigned char)skip;
}

// ---- host side ---------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 mt_encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *q = nullptr;
        cudaDriverEntryPointQueryResult r;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &q, cudaEnableDefault, &r) == cudaSuccess &&
            r == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(q);
    });
    return fn;
}

// FP64 [planes][n] (n contiguous), boxes of {box_x, box_y}: the tensor map
// of a level-major field for the ring kernels
bool tma_map_planes(CUtensorMap *m, const void *base, size_t n, int planes, int box_x, int box_y)
{
    auto fn = mt_encode_fn();
    if (!fn || !base) return false;
    cuuint64_t dims[2] = {(cuuint64_t)n, (cuuint64_t)planes};
    cuuint64_t strides[1] = {(cuuint64_t)n * 8};
    cuuint32_t box[2] = {(cuuint32_t)box_x, (cuuint32_t)box_y};
    cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void *>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

size_t momentum_tma_smem(int nz) { return mt_smem_bytes(nz); }

int momentum_tma_tiles(const Params &p)
{
    const long long nfu = (long long)(p.nx + 1) * p.ny, nfv = (long long)p.nx * (p.ny + 1);
    const long long nt = (nfu > nfv ? nfu : nfv) + MT_TW - 1;
    return (int)(2 * (nt / MT_TW));
}

// The ring applies to the default momentum knobs without
// caller-set k_top/k_bot, on planes whose byte strides are multiples of 16
// (tensor-map strides) and 16-byte-aligned fields; false: use k_momentum.
bool momentum_tma_eligible(const Params &p)
{
    if (!is_default_face_knobs(p.cfg) || p.k_top_u || p.k_top_v || p.k_bot_u || p.k_bot_v) return false;
    if (!p.zcol || !p.mom_tile_skip || !p.dev_err) return false;
    if ((p.plane & 1) || (p.plane_u & 1) || (p.plane_v & 1)) return false;
    if ((((uintptr_t)p.h) | ((uintptr_t)p.kv) | ((uintptr_t)p.u) | ((uintptr_t)p.v)) & 15) return false;
    if (p.plane > 0x7fffffffull || p.plane_u > 0x7fffffffull || p.plane_v > 0x7fffffffull) return false;
    if (momentum_tma_smem(p.nz) > 227 * 1024) return false;
    return mt_encode_fn() != nullptr;
}

// The tensor maps of the ring kernels and the tile flags (launched on
// `stream`); false when the configuration or the buffers do not qualify.
bool momentum_ring_prepare(const Params &p, MomMaps *maps, int *ntiles, cudaStream_t stream)
{
    if (!momentum_tma_eligible(p)) return false;
    if (!tma_map_planes(&maps->h, p.h, p.plane, p.nz, MT_BW, MT_U) ||
        !tma_map_planes(&maps->kv, p.kv, p.plane, p.nz + 1, MT_BW, MT_U) ||
        !tma_map_planes(&maps->u, p.u, p.plane_u, p.nz, MT_TW, MT_U) ||
        !tma_map_planes(&maps->v, p.v, p.plane_v, p.nz, MT_TW, MT_U))
        return false;
    *ntiles = momentum_tma_tiles(p);
    k_mom_tile_flags<<<*ntiles, MT_TW, 0, stream>>>(p);
    return true;
}

// Persistent grid of a ring kernel: its resident CTAs on every SM, at most
// one per tile.
int momentum_ring_grid(const void *kernel, int ntiles, size_t smem)
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, MT_THREADS, smem);
    if (per_sm < 1) per_sm = 1;
    return ntiles < sms * per_sm ? ntiles : sms * per_sm;
}

}  // namespace vphys
