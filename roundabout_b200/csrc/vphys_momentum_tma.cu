// vphys_momentum_tma.cu -- the exact (FP64) momentum viscosity solve with its
// level blocks staged into shared memory by TMA
// (diffuse_velocity_columns_impl, rdb_ocean_vdiff.F90:1611-1925, the z_clear
// branch of vdiff_face_layer :1964-2056 and vdiff_interface_coupling
// :2058-2115 at the default momentum knobs).
//
// The register-prefetched solve (k_momentum) keeps only a few levels of each
// column in flight per thread, and its occupancy is capped by the c' rows in
// shared memory, so the HBM pipe idles while the threads wait on loads.  Here
// the loads are decoupled from the arithmetic:
//
//   * a tile is 128 consecutive u (or v) faces in the flattened face index;
//     u and v tiles alternate (mt_tile_of) and the CTA is persistent,
//     walking tiles blockIdx.x, blockIdx.x + grid, ...
//   * warp 4, lane 0 (the producer) streams the tile's levels in blocks of
//     MT_U levels into an MT_S-stage shared-memory ring: one plain 2-D
//     cp.async.bulk.tensor per field and block -- the cells either side of
//     the tiles' faces (h, kv; one block for u tiles, the rows j-1 and j for
//     v tiles) and the velocities -- completing on the stage's mbarrier;
//   * warps 0-3 (one thread per face) run the forward Thomas sweep from the
//     ring in the reference's operation order, c' into shared memory and d'
//     in place over the velocity (L2 evict_last), release each stage to the
//     producer, then back-substitute from c' and the L2-resident d' while the
//     producer already fills the ring with the next tile.
//
// Tiles whose every face touches land and carries a zero velocity at every
// level are skipped (k_mom_tile_flags): their solve would reproduce the zeros.
// Results are the register-prefetched solve's bit for bit (same arithmetic,
// same order, -fmad=false).  Every mbarrier wait is bounded; on expiry the
// kernel records the failure in p.dev_err and the CTA stops, the producer
// first draining the copies it issued.  No copy is multicast and every tensor
// map covers this GPU's own buffers.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "vphys_device.cuh"
#include "vphys_faces.cuh"
#include "vphys_kernels.cuh"
#include "vphys_mom_ring.cuh"

#ifndef VPHYS_MT_MB
#define VPHYS_MT_MB 8
#endif

namespace vphys {

constexpr int MT_MB = VPHYS_MT_MB;   // levels per load block of the back-substitution

// The column state carried from one level of a face's forward sweep to the
// next (the register variables of diffuse_velocity_columns_impl).
struct FaceSweep {
    double zacc, zcol_l, zcol_r, d_min, i_hbbl;
    double hv_p, zi_p, num_t, dz_t;
    double cp_prev, dp_prev, u_k;
};

// Iteration k of the forward sweep (rdb_ocean_vdiff.F90:1700-1880 at the
// default knobs: kb = kb_live = 1, ktop = nz, no stress, drag, glue or cuts).
// NEXT: level k+1 exists (k < nz) and its h, kv and velocity are given.
template <bool NEXT>
__device__ __forceinline__ void face_iteration(const vphys_config &c, FaceSweep &s, int k, int nz, double dt,
                                               double hl, double hr, double kvl, double kvr, double u_next,
                                               double &cp, double &dp)
{
    const double hv_0 = s.hv_p, zi_0 = s.zi_p;
    const double num_b = s.num_t, dz_b = s.dz_t;
    if (NEXT) {
        double u_kp1 = u_next;
        face_layer<double>(c, hl, hr, u_kp1, k + 1, 1, s.d_min, s.i_hbbl, s.zacc, s.zcol_l, s.zcol_r, s.hv_p, s.zi_p);
        bool cut;
        interface_coupling<double>(c, hv_0, s.hv_p, zi_0, dt, 0.0, c.hbbl_visc, kvl, kvr, s.num_t, s.dz_t, cut);
    }
    double a_k = 0.0, b_k = 1.0, c_k = 0.0;
    const double hf_k = fmx(hv_0, H_VANISHED);
    if (k == 1) {
        double alpha = 0.0;
        if (1 < nz) alpha = xdiv(s.num_t, hf_k * s.dz_t);
        c_k = -alpha;
        b_k = 1.0 + alpha;
    }
    if (k == nz && k > 1) {
        const double beta = xdiv(num_b, hf_k * dz_b);
        a_k = -beta;
        b_k = 1.0 + beta;
    }
    if (k > 1 && k < nz) {
        const double beta = xdiv(num_b, hf_k * dz_b);
        const double alpha = xdiv(s.num_t, hf_k * s.dz_t);
        a_k = -beta;
        c_k = -alpha;
        b_k = 1.0 + alpha + beta;
    }
    const double r_k = s.u_k;
    const Rcp denom = rcp_of((k == 1) ? b_k : b_k - a_k * s.cp_prev);
    cp = qdiv(c_k, denom);
    dp = qdiv((k == 1) ? r_k : r_k - a_k * s.dp_prev, denom);
    s.cp_prev = cp;
    s.dp_prev = dp;
    if (NEXT) s.u_k = u_next;
}

// One face of the exact solve, driven by momentum_ring_cta: c' in the
// shared-memory rows, d' in place over the velocity (L2 evict_last).
struct ExactFace {
    FaceSweep s;
    vphys_config c;
    const Params *pp;
    double dt;
    double *uf;
    size_t PF;
    double *cpp;
    int tid, nz;
    bool valid;
    unsigned long long pol_keep;

    __device__ __forceinline__ void start(const Params &p, double dt_, const FaceCells &fc, bool valid_, double *uf_,
                                          size_t PF_, unsigned char *rows, int tid_)
    {
        c = p.cfg;
        default_face_knobs(c);
        pp = &p;
        dt = dt_;
        uf = uf_;
        PF = PF_;
        cpp = reinterpret_cast<double *>(rows);
        tid = tid_;
        nz = p.nz;
        valid = valid_;
        pol_keep = l2_policy_evict_last();
        s.zacc = 0.0;
        s.zcol_l = p.zcol[fc.cl];
        s.zcol_r = p.zcol[fc.cr];
        s.d_min = fmn(-s.zcol_l, -s.zcol_r);
        s.i_hbbl = 1.0 / (c.hbbl_visc + EPS_HVEL);
        s.num_t = 0.0;
        s.dz_t = 1.0;
        s.cp_prev = 0.0;
        s.dp_prev = 0.0;
    }
    __device__ __forceinline__ void first(double hl, double hr, double uw)
    {
        s.u_k = uw;
        face_layer<double>(c, hl, hr, s.u_k, 1, 1, s.d_min, s.i_hbbl, s.zacc, s.zcol_l, s.zcol_r, s.hv_p, s.zi_p);
    }
    __device__ __forceinline__ void row(int m, double hl, double hr, double kvl, double kvr, double uw)
    {
        double cp, dp;
        face_iteration<true>(c, s, m, nz, dt, hl, hr, kvl, kvr, uw, cp, dp);
        cpp[(size_t)(m - 1) * MT_TW + tid] = cp;
        if (valid) st_hint(uf + PF * (size_t)(m - 1), dp, pol_keep);
    }
    __device__ __forceinline__ void last()
    {
        double cp, dp;
        face_iteration<false>(c, s, nz, nz, dt, 0.0, 0.0, 0.0, 0.0, 0.0, cp, dp);
        cpp[(size_t)(nz - 1) * MT_TW + tid] = cp;
    }
    // back-substitution: c' from shared memory, d' from the L2-resident velocity
    __device__ __forceinline__ void back()
    {
        double u_next = s.dp_prev;
        if (valid) uf[PF * (size_t)(nz - 1)] = u_next;
        for (int k0 = nz - 1; k0 >= 1; k0 -= MT_MB) {
            double dps[MT_MB];
#pragma unroll
            for (int q = 0; q < MT_MB; ++q) {
                const int k = k0 - q;
                dps[q] = (k >= 1 && valid) ? ld_hint(uf + PF * (size_t)(k - 1), pol_keep) : 0.0;
            }
#pragma unroll
            for (int q = 0; q < MT_MB; ++q) {
                const int k = k0 - q;
                if (k >= 1) {
                    const double cpk = cpp[(size_t)(k - 1) * MT_TW + tid];
                    u_next = dps[q] - cpk * u_next;
                    if (valid) uf[PF * (size_t)(k - 1)] = u_next;
                }
            }
        }
    }
};

__global__ void __launch_bounds__(MT_THREADS, 2)
    k_momentum_tma(const __grid_constant__ MomMaps maps, const Params p, double dt, int ntiles)
{
    extern __shared__ __align__(128) unsigned char mt_smem[];
    momentum_ring_cta<ExactFace>(maps, p, dt, ntiles, mt_smem);
}

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

// FP64 [planes][n] (n contiguous), boxes of {box_x, MT_U}
static bool mt_map(CUtensorMap *m, const void *base, size_t n, int planes, int box_x)
{
    auto fn = mt_encode_fn();
    if (!fn || !base) return false;
    cuuint64_t dims[2] = {(cuuint64_t)n, (cuuint64_t)planes};
    cuuint64_t strides[1] = {(cuuint64_t)n * 8};
    cuuint32_t box[2] = {(cuuint32_t)box_x, (cuuint32_t)MT_U};
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

// The TMA-staged solve applies to the default momentum knobs without
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
    if (!mt_map(&maps->h, p.h, p.plane, p.nz, MT_BW) || !mt_map(&maps->kv, p.kv, p.plane, p.nz + 1, MT_BW) ||
        !mt_map(&maps->u, p.u, p.plane_u, p.nz, MT_TW) || !mt_map(&maps->v, p.v, p.plane_v, p.nz, MT_TW))
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

bool launch_momentum_tma(const Params &p, double dt, cudaStream_t stream)
{
    MomMaps maps;
    int ntiles = 0;
    if (!momentum_ring_prepare(p, &maps, &ntiles, stream)) return false;
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_momentum_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr_set = true;
    }
    const size_t smem = momentum_tma_smem(p.nz);
    const int grid = momentum_ring_grid((const void *)k_momentum_tma, ntiles, smem);
    k_momentum_tma<<<grid, MT_THREADS, smem, stream>>>(maps, p, dt, ntiles);
    return true;
}

}  // namespace vphys
