// vphys_gemm.cu -- BF16 x BF16 -> FP32 GEMM on the 5th-generation tensor
// cores (tcgen05), the building block of the learned KPP surrogate's forward
// and backward passes.
//
//   C[M, N] = alpha * A[M, K] . B[N, K]^T      (both operands K-contiguous, "TN")
//
// followed by a fused epilogue: + bias[N], optional multiplication by
// GELU'(z) of a saved pre-activation (the backward of a GELU layer), storing
// FP32 (pre-activation or plain), BF16 of GELU(v) or v, and/or a transposed
// BF16 copy (the operand layout the weight-gradient GEMMs read).
//
// Persistent kernel, one CTA per SM, looping over 128-row tiles (each against
// all N <= 256 output columns), warp-specialised:
//   * warp 0 lane 0 streams K in 64-element steps with TMA
//     (cp.async.bulk.tensor, 128-byte swizzle) into a 4-stage ring,
//   * warp 1 lane 0 issues tcgen05.mma (M=128, N, K=16) from the shared-memory
//     descriptors into one of two FP32 accumulators in tensor memory (all 512
//     columns), releasing each stage with tcgen05.commit,
//   * warps 2-9 drain the other accumulator with tcgen05.ld (two warps per
//     32-lane quarter, alternate 16-column chunks), so the epilogue of tile i
//     overlaps the loads and MMAs of tile i+1.
// Every mbarrier wait is bounded: on expiry the CTA records an error code in
// *err and skips the rest of its work.  Before the teardown it drains what it
// already issued -- the producer waits (bounded) for the bytes of every stage
// it armed, the MMA issuer for its last commit, i.e. for every MMA issued --
// so no TMA write or tensor-core access is in flight when the CTA frees its
// tensor memory and exits.
// No load is multicast; the kernel runs on the calling GPU's memory only.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <mutex>

#include "../../include/vphys.h"
#include "vphys_kernels.cuh"

namespace vphys {

constexpr int GM = 128;        // rows per CTA (tcgen05 M)
constexpr int GK = 64;         // K per stage: one 128-byte swizzle row of BF16
constexpr int GSTAGES = 4;
constexpr int GN_MAX = 256;    // N per CTA (tcgen05 N <= 256)
constexpr int GEMM_THREADS = 320;   // producer, MMA, 8 epilogue warps
constexpr int EPI_WARPS = 8;
constexpr uint32_t TMEM_COLS = 512;  // two 256-column accumulators
constexpr size_t GEMM_SMEM = (size_t)GSTAGES * (GM + GN_MAX) * GK * 2 + 1024 /* barriers */ + 1024 /* align */;
constexpr long long WAIT_LIMIT = 1LL << 24;   // try_wait polls before a wait is declared lost

struct GemmEpi {
    int M, N, K;
    float alpha;
    const float *bias;      // [N] or null
    const float *zin;       // [M, ld_z] pre-activation: multiply by GELU'(z), or null
    int ld_z;
    int act;                // 1: the BF16 outputs hold GELU(v), 0: v
    float *out_f32;         // [M, ld_f32] v (before the activation), or null
    int ld_f32;
    __nv_bfloat16 *out_bf16;    // [M, ld_bf16], or null
    int ld_bf16;
    __nv_bfloat16 *out_bf16_t;  // [N, ld_t] transposed, or null
    int ld_t;
    int vec;                // row-major outputs 16-byte aligned with ld % 8 == 0: vector stores
    int *err;
};

// ---- small PTX wrappers ----------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// bounded wait for the phase of parity `parity` to complete; false on expiry
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    const uint32_t a = smem_u32(bar);
    for (long long it = 0; it < WAIT_LIMIT; ++it) {
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
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 B apart (SBO), descriptor version 1 (sm_100)
__device__ __forceinline__ uint64_t smem_desc_sw128(const void *p)
{
    const uint64_t addr = smem_u32(p);
    uint64_t d = 0;
    d |= (addr >> 4) & 0x3FFFull;            // start address, bits [0,14)
    d |= (uint64_t)(16 >> 4) << 16;          // leading byte offset (unused with this swizzle), bits [16,30)
    d |= (uint64_t)(1024 >> 4) << 32;        // stride byte offset, bits [32,46)
    d |= (uint64_t)1 << 46;                  // version, bits [46,48)
    d |= (uint64_t)2 << 61;                  // layout: 128-byte swizzle, bits [61,64)
    return d;
}
// instruction descriptor, kind::f16: BF16 A and B, FP32 D, both K-major
__device__ __forceinline__ uint32_t idesc_bf16(int m, int n)
{
    uint32_t d = 0;
    d |= 1u << 4;                        // D format: F32
    d |= 1u << 7;                        // A format: BF16
    d |= 1u << 10;                       // B format: BF16
    d |= (uint32_t)(n >> 3) << 17;       // N / 8
    d |= (uint32_t)(m >> 4) << 24;       // M / 16
    return d;
}

// hardware tanh (MUFU, relative error about 2^-11: below the BF16 rounding
// every activation then goes through)
__device__ __forceinline__ float tanh_hw(float x)
{
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
// GELU, tanh form (Hendrycks & Gimpel 2016): 0.5 x (1 + tanh(c (x + 0.044715 x^3))),
// c = sqrt(2/pi), with the argument as x (c + c 0.044715 x^2) and the result as
// hx + hx t (hx = x / 2): three multiply-adds around the hardware tanh
constexpr float GELU_C0 = 0.7978845608028654f;
constexpr float GELU_C1 = 0.7978845608028654f * 0.044715f;
__device__ __forceinline__ float gelu_arg(float x) { return x * fmaf(GELU_C1, x * x, GELU_C0); }
__device__ __forceinline__ float gelu_tanh(float x)
{
    const float t = tanh_hw(gelu_arg(x));
    const float hx = 0.5f * x;
    return fmaf(hx, t, hx);
}
__device__ __forceinline__ float gelu_tanh_grad(float x)
{
    const float t = tanh_hw(gelu_arg(x));
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * GELU_C0 * (1.0f + 3.0f * 0.044715f * x * x);
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
    tmem_ld16_async(taddr, r);
    tmem_ld_wait();
}

// The inference epilogues (vphys_kpp's in-step forward: alpha = 1, a bias,
// no gradient input, row-major 16-byte-aligned outputs only), without the
// general epilogue's per-element option tests.  EP 1: a hidden layer, BF16 of
// GELU(v + bias); EP 2: the output layer, FP32 v + bias.
template <int EP>
__device__ __forceinline__ void epilogue16_inf(const GemmEpi &g, int row, int c0, const uint32_t (&r)[16])
{
    float b[16];
    const float4 *b4 = reinterpret_cast<const float4 *>(g.bias + c0);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float4 v = __ldg(b4 + q);
        b[4 * q] = v.x, b[4 * q + 1] = v.y, b[4 * q + 2] = v.z, b[4 * q + 3] = v.w;
    }
    if (EP == 1) {
        __nv_bfloat162 pk[8];
#pragma unroll
        for (int q = 0; q < 8; ++q)
            pk[q] = __floats2bfloat162_rn(gelu_tanh(__uint_as_float(r[2 * q]) + b[2 * q]),
                                          gelu_tanh(__uint_as_float(r[2 * q + 1]) + b[2 * q + 1]));
        uint4 *o4 = reinterpret_cast<uint4 *>(g.out_bf16 + (size_t)row * g.ld_bf16 + c0);
        o4[0] = *reinterpret_cast<uint4 *>(&pk[0]);
        o4[1] = *reinterpret_cast<uint4 *>(&pk[4]);
    } else {
        float4 *o4 = reinterpret_cast<float4 *>(g.out_f32 + (size_t)row * g.ld_f32 + c0);
#pragma unroll
        for (int q = 0; q < 4; ++q)
            o4[q] = make_float4(__uint_as_float(r[4 * q]) + b[4 * q], __uint_as_float(r[4 * q + 1]) + b[4 * q + 1],
                                __uint_as_float(r[4 * q + 2]) + b[4 * q + 2],
                                __uint_as_float(r[4 * q + 3]) + b[4 * q + 3]);
    }
}

// epilogue of one 16-column chunk of one row (v[] = accumulator values)
__device__ __forceinline__ void epilogue16(const GemmEpi &g, int row, int c0, const uint32_t (&r)[16])
{
    float v[16], a[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int col = c0 + q;
        float x = g.alpha * __uint_as_float(r[q]);
        if (g.bias) x += __ldg(g.bias + col);
        if (g.zin) x *= gelu_tanh_grad(__ldg(g.zin + (size_t)row * g.ld_z + col));
        v[q] = x;
        a[q] = g.act ? gelu_tanh(x) : x;
    }
    if (g.out_f32) {
        float *o = g.out_f32 + (size_t)row * g.ld_f32 + c0;
        if (g.vec) {
#pragma unroll
            for (int q = 0; q < 16; q += 4) *reinterpret_cast<float4 *>(o + q) = make_float4(v[q], v[q + 1], v[q + 2], v[q + 3]);
        } else {
#pragma unroll
            for (int q = 0; q < 16; ++q) o[q] = v[q];
        }
    }
    if (g.out_bf16 || g.out_bf16_t) {
        __nv_bfloat162 pk[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) pk[q] = __floats2bfloat162_rn(a[2 * q], a[2 * q + 1]);
        if (g.out_bf16) {
            __nv_bfloat16 *o = g.out_bf16 + (size_t)row * g.ld_bf16 + c0;
            if (g.vec) {
                uint4 *o4 = reinterpret_cast<uint4 *>(o);
                o4[0] = *reinterpret_cast<uint4 *>(&pk[0]);
                o4[1] = *reinterpret_cast<uint4 *>(&pk[4]);
            } else {
#pragma unroll
                for (int q = 0; q < 8; ++q) *reinterpret_cast<__nv_bfloat162 *>(o + 2 * q) = pk[q];
            }
        }
        if (g.out_bf16_t) {
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                g.out_bf16_t[(size_t)(c0 + 2 * q) * g.ld_t + row] = pk[q].x;
                g.out_bf16_t[(size_t)(c0 + 2 * q + 1) * g.ld_t + row] = pk[q].y;
            }
        }
    }
}

// EP: 0 the general epilogue (training), 1 / 2 the inference epilogues
template <int EP>
__global__ void __launch_bounds__(GEMM_THREADS, 1)
    k_gemm_tn(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, const GemmEpi g)
{
    extern __shared__ uint8_t smraw[];
    uint8_t *sm = reinterpret_cast<uint8_t *>(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    __nv_bfloat16 *sa = reinterpret_cast<__nv_bfloat16 *>(sm);
    __nv_bfloat16 *sb = sa + (size_t)GSTAGES * GM * GK;
    uint64_t *full = reinterpret_cast<uint64_t *>(sb + (size_t)GSTAGES * GN_MAX * GK);
    uint64_t *empty = full + GSTAGES;
    uint64_t *acc_full = empty + GSTAGES;     // [2] MMA -> epilogue
    uint64_t *acc_empty = acc_full + 2;       // [2] epilogue -> MMA
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(acc_empty + 2);
    int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int N = g.N;
    const int nk = (g.K + GK - 1) / GK;
    const int tiles = (g.M + GM - 1) / GM;
    const int my_tiles = (tiles > (int)blockIdx.x) ? (tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < GSTAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&acc_full[a], 1);
            mbar_init(&acc_empty[a], EPI_WARPS);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    volatile int *abort_v = abort_flag;

    if (warp == 0) {
        if (lane == 0) {
            // ---- TMA producer ----
            const uint32_t bytes = (uint32_t)(GM + N) * GK * 2;
            long long it = 0;   // stages armed so far
            for (int t = 0; t < my_tiles && !*abort_v; ++t) {
                const int m0 = ((int)blockIdx.x + t * (int)gridDim.x) * GM;
                for (int kt = 0; kt < nk; ++kt) {
                    const int s = (int)(it % GSTAGES);
                    const uint32_t round = (uint32_t)(it / GSTAGES);
                    if (!mbar_wait(&empty[s], (round & 1) ^ 1)) {
                        atomicExch(g.err, 1);
                        *abort_v = 1;
                        break;
                    }
                    mbar_expect_tx(&full[s], bytes);
                    tma_load_2d(sa + (size_t)s * GM * GK, &tmA, kt * GK, m0, &full[s]);
                    tma_load_2d(sb + (size_t)s * GN_MAX * GK, &tmB, kt * GK, 0, &full[s]);
                    ++it;
                }
            }
            if (*abort_v) {
                // Drain: the loads of the last GSTAGES armed stages may still be
                // writing shared memory.  Each stage's latest armed phase
                // completes when its bytes have landed (whether or not the MMA
                // warp consumed it), and no stage is re-armed after this point,
                // so waiting on that phase's parity is unambiguous.
                const long long first = it > GSTAGES ? it - GSTAGES : 0;
                for (long long a = first; a < it; ++a)
                    if (!mbar_wait(&full[(int)(a % GSTAGES)], (uint32_t)((a / GSTAGES) & 1))) atomicExch(g.err, 5);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer ----
            const uint32_t idesc = idesc_bf16(GM, N);
            long long it = 0;
            int last_commit = -1;   // the tile of the last acc_full commit
            for (int t = 0; t < my_tiles && !*abort_v; ++t) {
                const int a = t & 1;
                if (!mbar_wait(&acc_empty[a], ((t >> 1) & 1) ^ 1)) {
                    atomicExch(g.err, 4);
                    *abort_v = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = tmem + (uint32_t)(a * GN_MAX);
                bool ok = true;
                for (int kt = 0; kt < nk; ++kt, ++it) {
                    const int s = (int)(it % GSTAGES);
                    const uint32_t round = (uint32_t)(it / GSTAGES);
                    if (!mbar_wait(&full[s], round & 1)) {
                        atomicExch(g.err, 2);
                        *abort_v = 1;
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const __nv_bfloat16 *as = sa + (size_t)s * GM * GK;
                    const __nv_bfloat16 *bs = sb + (size_t)s * GN_MAX * GK;
#pragma unroll
                    for (int kk = 0; kk < GK / 16; ++kk) {
                        const uint64_t ad = smem_desc_sw128(as + kk * 16);
                        const uint64_t bd = smem_desc_sw128(bs + kk * 16);
                        const uint32_t acc = (kt > 0 || kk > 0) ? 1u : 0u;
                        asm volatile(
                            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
                            "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                            : "memory");
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     smem_u32(&empty[s]))
                                 : "memory");
                }
                // the accumulator is ready (or, after an abort, every MMA issued has finished)
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&acc_full[a]))
                             : "memory");
                last_commit = t;
                if (!ok) break;
            }
            if (*abort_v && last_commit >= 0) {
                // Drain: the commit arrives on acc_full once every MMA issued
                // before it has retired (its shared-memory reads and its tensor-
                // memory writes), so the teardown below frees nothing in use.
                if (!mbar_wait(&acc_full[last_commit & 1], (uint32_t)((last_commit >> 1) & 1))) atomicExch(g.err, 6);
            }
        }
    } else {
        // ---- epilogue warps 2..9: quarter (warp % 4) of the lanes, alternate chunks ----
        const int quarter = warp & 3;
        const int half = (warp - 2) >> 2;
        for (int t = 0; t < my_tiles; ++t) {
            const int a = t & 1;
            const bool ok = mbar_wait(&acc_full[a], (t >> 1) & 1);
            if (!ok) {
                if (lane == 0) atomicExch(g.err, 3);
                *abort_v = 1;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (!ok || *abort_v) break;
            const int row = ((int)blockIdx.x + t * (int)gridDim.x) * GM + quarter * 32 + lane;
            const uint32_t tl = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(a * GN_MAX);
            if (EP == 0) {
                for (int c0 = half * 16; c0 < N; c0 += 32) {
                    uint32_t r[16];
                    tmem_ld16(tl + (uint32_t)c0, r);
                    if (row < g.M) epilogue16(g, row, c0, r);
                }
            } else {
                // two chunks per wait: the second load overlaps the first's latency
                for (int c0 = half * 16; c0 < N; c0 += 64) {
                    uint32_t r0[16], r1[16];
                    const bool two = c0 + 32 < N;
                    tmem_ld16_async(tl + (uint32_t)c0, r0);
                    if (two) tmem_ld16_async(tl + (uint32_t)(c0 + 32), r1);
                    tmem_ld_wait();
                    if (row < g.M) {
                        epilogue16_inf<EP>(g, row, c0, r0);
                        if (two) epilogue16_inf<EP>(g, row, c0 + 32, r1);
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[a]);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// ---- the three layers of the KPP surrogate in one kernel -----------------------
// Y = (GELU(GELU(X W1^T + b1) W2^T + b2)) W3^T + b3 for 128-row tiles, the
// hidden activations never leaving the SM: the epilogue warps write GELU(H)
// as BF16 straight into shared memory in the layout a TMA load with 128-byte
// swizzle produces (the A operand of the next layer's MMAs), so the layers
// make no HBM round trip.  Per tile the products and their order are those
// of three k_gemm_tn<1/1/2> launches (K slices in order, K = 16 per MMA), so
// Y is theirs bit for bit.  Roles as in k_gemm_tn: warp 0 lane 0 streams the
// X tile and the weights' 64-wide K slices (W1: 3, W2: 4, W3: 4 per tile)
// through an ML_STAGES ring, warp 1 lane 0 issues the MMAs, warps 2-9 drain
// the accumulator.  Barriers: x_full / x_empty (the X tile), w_full / w_empty
// (the weight ring), acc_full (a layer's accumulator is complete: three
// phases per tile), h_full (the hidden tile in shared memory is written and
// the accumulator read: two phases per tile).  Every wait is bounded.
constexpr int ML_STAGES = 3;
constexpr int ML_XCH = 3;                        // 64-wide K slices of X (160 -> 192, zero-filled)
constexpr int ML_HCH = 4;                        // 64-wide K slices of a hidden tile (256)
constexpr int ML_CHUNK_X = GM * GK * 2;          // bytes of one [128 x 64] BF16 slice
constexpr int ML_WSTAGE = GN_MAX * GK * 2;       // bytes of one [256 x 64] weight slice
constexpr int ML_NBIAS = 2 * GN_MAX + LK_OUTP;   // b1, b2, b3, staged in shared memory
constexpr size_t ML_SMEM = (size_t)ML_XCH * ML_CHUNK_X + (size_t)ML_HCH * ML_CHUNK_X + (size_t)ML_STAGES * ML_WSTAGE +
                           (size_t)ML_NBIAS * 4 + 1024 /* barriers */ + 1024 /* align */;
constexpr int ML_ACC3 = 256;                     // tensor-memory column of the output layer's accumulator
// 16 epilogue warps (four per lane quarter, each a quarter of the columns):
// the epilogue is the kernel's bound, and it cannot overlap the next tile's
// MMAs here as it does in k_gemm_tn
constexpr int ML_EPI = 16;
constexpr int ML_THREADS = 64 + 32 * ML_EPI;

struct MlpArgs {
    int M;
    const float *b1, *b2, *b3;
    float *Y;   // [M, LK_OUTP]
    int *err;
};

// GELU(v + bias) of 16 accumulator columns of row r into the hidden tile
// (row r, columns c0..c0+15: two 16-byte units of the 128-byte-swizzled slice)
__device__ __forceinline__ void mlp_hidden16(uint8_t *hs, int r, int c0, const float *bias, const uint32_t (&v)[16])
{
    float b[16];   // the layer's bias, staged in shared memory
    const float4 *b4 = reinterpret_cast<const float4 *>(bias + c0);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float4 t = b4[q];
        b[4 * q] = t.x, b[4 * q + 1] = t.y, b[4 * q + 2] = t.z, b[4 * q + 3] = t.w;
    }
    __nv_bfloat162 pk[8];
#pragma unroll
    for (int q = 0; q < 8; ++q)
        pk[q] = __floats2bfloat162_rn(gelu_tanh(__uint_as_float(v[2 * q]) + b[2 * q]),
                                      gelu_tanh(__uint_as_float(v[2 * q + 1]) + b[2 * q + 1]));
    const int kt = c0 >> 6, ch = (c0 & 63) >> 3;   // slice, first 16-byte unit of the 128-byte row
    uint8_t *row = hs + (size_t)kt * ML_CHUNK_X + (size_t)r * 128;
    *reinterpret_cast<uint4 *>(row + (((ch) ^ (r & 7)) << 4)) = *reinterpret_cast<uint4 *>(&pk[0]);
    *reinterpret_cast<uint4 *>(row + (((ch + 1) ^ (r & 7)) << 4)) = *reinterpret_cast<uint4 *>(&pk[4]);
}

__global__ void __launch_bounds__(ML_THREADS, 1)
    k_mlp3(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmW1,
           const __grid_constant__ CUtensorMap tmW2, const __grid_constant__ CUtensorMap tmW3, const MlpArgs g)
{
    extern __shared__ uint8_t smraw[];
    uint8_t *sm = reinterpret_cast<uint8_t *>(((uintptr_t)smraw + 1023) & ~(uintptr_t)1023);
    uint8_t *sx = sm;                                           // X tile: ML_XCH slices
    uint8_t *sh = sx + (size_t)ML_XCH * ML_CHUNK_X;             // hidden tile: ML_HCH slices
    uint8_t *sw = sh + (size_t)ML_HCH * ML_CHUNK_X;             // weight ring
    float *sb = reinterpret_cast<float *>(sw + (size_t)ML_STAGES * ML_WSTAGE);   // b1 | b2 | b3
    uint64_t *x_full = reinterpret_cast<uint64_t *>(sb + ML_NBIAS);
    uint64_t *x_empty = x_full + 1;
    uint64_t *w_full = x_empty + 1;                             // [ML_STAGES]
    uint64_t *w_empty = w_full + ML_STAGES;                     // [ML_STAGES]
    uint64_t *acc_full = w_empty + ML_STAGES;
    uint64_t *h_full = acc_full + 1;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(h_full + 1);
    int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles = (g.M + GM - 1) / GM;
    const int my_tiles = (tiles > (int)blockIdx.x) ? (tiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;

    if (threadIdx.x == 0) {
        mbar_init(x_full, 1);
        mbar_init(x_empty, 1);
        for (int s = 0; s < ML_STAGES; ++s) {
            mbar_init(&w_full[s], 1);
            mbar_init(&w_empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(h_full, ML_EPI);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = threadIdx.x; i < ML_NBIAS; i += blockDim.x)
        sb[i] = i < GN_MAX ? g.b1[i] : (i < 2 * GN_MAX ? g.b2[i - GN_MAX] : g.b3[i - 2 * GN_MAX]);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    volatile int *abort_v = abort_flag;
    // the weight slices of one tile, in the order the MMA warp takes them
    constexpr int NW = ML_XCH + 2 * ML_HCH;

    if (warp == 0) {
        if (lane == 0) {
            // ---- TMA producer ----
            long long it = 0;   // weight slices armed so far
            int xt = 0;         // X tiles armed so far
            bool lost = false;
            for (int t = 0; t < my_tiles && !lost; ++t) {
                const int m0 = ((int)blockIdx.x + t * (int)gridDim.x) * GM;
                if (!mbar_wait(x_empty, (uint32_t)((t & 1) ^ 1)) || *abort_v) {
                    atomicExch(g.err, 1);
                    *abort_v = 1;
                    break;
                }
                mbar_expect_tx(x_full, (uint32_t)(ML_XCH * ML_CHUNK_X));
                for (int c = 0; c < ML_XCH; ++c) tma_load_2d(sx + (size_t)c * ML_CHUNK_X, &tmX, c * GK, m0, x_full);
                ++xt;
                for (int w = 0; w < NW; ++w, ++it) {
                    const int s = (int)(it % ML_STAGES);
                    if (!mbar_wait(&w_empty[s], (uint32_t)(((it / ML_STAGES) & 1) ^ 1)) || *abort_v) {
                        atomicExch(g.err, 1);
                        *abort_v = 1;
                        lost = true;
                        break;
                    }
                    uint8_t *dst = sw + (size_t)s * ML_WSTAGE;
                    if (w < ML_XCH) {
                        mbar_expect_tx(&w_full[s], (uint32_t)(GN_MAX * GK * 2));
                        tma_load_2d(dst, &tmW1, w * GK, 0, &w_full[s]);
                    } else if (w < ML_XCH + ML_HCH) {
                        mbar_expect_tx(&w_full[s], (uint32_t)(GN_MAX * GK * 2));
                        tma_load_2d(dst, &tmW2, (w - ML_XCH) * GK, 0, &w_full[s]);
                    } else {
                        mbar_expect_tx(&w_full[s], (uint32_t)(LK_OUTP * GK * 2));
                        tma_load_2d(dst, &tmW3, (w - ML_XCH - ML_HCH) * GK, 0, &w_full[s]);
                    }
                }
            }
            if (*abort_v) {
                // drain: the bytes of every armed slice and X tile land before the CTA exits
                const long long first = it > ML_STAGES ? it - ML_STAGES : 0;
                for (long long a = first; a < it; ++a)
                    if (!mbar_wait(&w_full[(int)(a % ML_STAGES)], (uint32_t)((a / ML_STAGES) & 1))) atomicExch(g.err, 5);
                if (xt > 0 && !mbar_wait(x_full, (uint32_t)((xt - 1) & 1))) atomicExch(g.err, 5);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer ----
            long long it = 0;
            long long commits = 0;   // acc_full commits so far
            bool ok = true;
            for (int t = 0; t < my_tiles && ok && !*abort_v; ++t) {
                if (!mbar_wait(x_full, (uint32_t)(t & 1))) {
                    atomicExch(g.err, 2);
                    *abort_v = 1;
                    break;
                }
                for (int layer = 0; layer < 3 && ok; ++layer) {
                    if (layer > 0 && !mbar_wait(h_full, (uint32_t)((2 * t + layer - 1) & 1))) {
                        atomicExch(g.err, 4);
                        *abort_v = 1;
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const int nch = layer == 0 ? ML_XCH : ML_HCH;
                    const int N = layer == 2 ? LK_OUTP : GN_MAX;
                    const uint32_t idesc = idesc_bf16(GM, N);
                    const uint32_t d = tmem + (uint32_t)(layer == 2 ? ML_ACC3 : 0);
                    const uint8_t *abase = layer == 0 ? sx : sh;
                    for (int c = 0; c < nch; ++c, ++it) {
                        const int s = (int)(it % ML_STAGES);
                        if (!mbar_wait(&w_full[s], (uint32_t)((it / ML_STAGES) & 1))) {
                            atomicExch(g.err, 2);
                            *abort_v = 1;
                            ok = false;
                            break;
                        }
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                        const uint8_t *as = abase + (size_t)c * ML_CHUNK_X;
                        const uint8_t *bs = sw + (size_t)s * ML_WSTAGE;
#pragma unroll
                        for (int kk = 0; kk < GK / 16; ++kk) {
                            const uint64_t ad = smem_desc_sw128(as + kk * 32);
                            const uint64_t bd = smem_desc_sw128(bs + kk * 32);
                            const uint32_t acc = (c > 0 || kk > 0) ? 1u : 0u;
                            asm volatile(
                                "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                                " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
                                "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                                : "memory");
                        }
                        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                         smem_u32(&w_empty[s]))
                                     : "memory");
                    }
                    if (layer == 0)   // the X tile is read once the first layer's MMAs retire
                        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                         smem_u32(x_empty))
                                     : "memory");
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     smem_u32(acc_full))
                                 : "memory");
                    ++commits;
                }
            }
            if (*abort_v && commits > 0) {
                // drain: the last commit arrives once every MMA issued before it has retired
                if (!mbar_wait(acc_full, (uint32_t)((commits - 1) & 1))) atomicExch(g.err, 6);
            }
        }
    } else {
        // ---- epilogue warps 2..17: lanes of quarter warp % 4; group (warp - 2) / 4 takes
        //      the 16-column chunks group, group + 4, ... ----
        const int quarter = warp & 3;
        const int grp = (warp - 2) >> 2;
        const int r = quarter * 32 + lane;   // row of the tile
        const uint32_t tl = tmem + ((uint32_t)(quarter * 32) << 16);
        bool ok = true;
        for (int t = 0; t < my_tiles && ok; ++t) {
            const int row = ((int)blockIdx.x + t * (int)gridDim.x) * GM + r;
            for (int layer = 0; layer < 3; ++layer) {
                if (!mbar_wait(acc_full, (uint32_t)((3 * t + layer) & 1))) {
                    if (lane == 0) atomicExch(g.err, 3);
                    *abort_v = 1;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                if (*abort_v) {
                    ok = false;
                    break;
                }
                if (layer < 2) {
                    const float *bias = sb + (layer == 0 ? 0 : GN_MAX);
                    for (int c0 = grp * 16; c0 < GN_MAX; c0 += 128) {
                        uint32_t v0[16], v1[16];
                        tmem_ld16_async(tl + (uint32_t)c0, v0);
                        tmem_ld16_async(tl + (uint32_t)(c0 + 64), v1);
                        tmem_ld_wait();
                        mlp_hidden16(sh, r, c0, bias, v0);
                        mlp_hidden16(sh, r, c0 + 64, bias, v1);
                    }
                    // the hidden tile is visible to the tensor cores' reads, the accumulator read
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    __syncwarp();
                    if (lane == 0) mbar_arrive(h_full);
                } else {
                    for (int c0 = grp * 16; c0 < LK_OUTP; c0 += 64) {
                        uint32_t v[16];
                        tmem_ld16(tl + (uint32_t)(ML_ACC3 + c0), v);
                        if (row < g.M) {
                            float4 *o4 = reinterpret_cast<float4 *>(g.Y + (size_t)row * LK_OUTP + c0);
                            const float4 *b4 = reinterpret_cast<const float4 *>(sb + 2 * GN_MAX + c0);
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                const float4 b = b4[q];
                                o4[q] = make_float4(__uint_as_float(v[4 * q]) + b.x, __uint_as_float(v[4 * q + 1]) + b.y,
                                                    __uint_as_float(v[4 * q + 2]) + b.z,
                                                    __uint_as_float(v[4 * q + 3]) + b.w);
                            }
                        }
                    }
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// ---- host side ---------------------------------------------------------------
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// 2-D BF16 row-major [rows, cols] (cols contiguous, rows `ld` elements
// apart) tiled {64, box_rows}, 128-byte swizzle
static bool make_map(CUtensorMap *m, const void *base, int rows, int cols, long long ld, int box_rows)
{
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    cuuint32_t box[2] = {(cuuint32_t)GK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int gemm_tn_bf16(const void *A, long long lda, const void *B, long long ldb, int M, int N, int K, float alpha,
                 const float *bias, const float *zin, int ld_z, int act, float *out_f32, int ld_f32, void *out_bf16,
                 int ld_bf16, void *out_bf16_t, int ld_t, int *err, cudaStream_t stream)
{
    if (M <= 0 || N < 16 || N > GN_MAX || (N % 16) != 0 || K <= 0 || (K % 8) != 0)
        return report_error(VPHYS_ERR_BAD_SHAPE, "vphys_gemm_tn_bf16: need M > 0, 16 <= N <= 256 with N % 16 == 0, "
                                                 "K > 0 with K % 8 == 0");
    if (lda < K || ldb < K || (lda % 8) != 0 || (ldb % 8) != 0)
        return report_error(VPHYS_ERR_BAD_SHAPE, "vphys_gemm_tn_bf16: lda, ldb must be >= K and multiples of 8");
    if (((uintptr_t)A | (uintptr_t)B) & 15)
        return report_error(VPHYS_ERR_BAD_SHAPE, "vphys_gemm_tn_bf16: A and B must be 16-byte aligned");
    CUtensorMap ma, mb;
    if (!make_map(&ma, A, M, K, lda, GM) || !make_map(&mb, B, N, K, ldb, N))
        return report_error(VPHYS_ERR_CUDA, "vphys_gemm_tn_bf16: cuTensorMapEncodeTiled failed");
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_gemm_tn<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GEMM_SMEM);
        cudaFuncSetAttribute(k_gemm_tn<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GEMM_SMEM);
        cudaFuncSetAttribute(k_gemm_tn<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GEMM_SMEM);
        attr_set = true;
    }
    GemmEpi g{};
    g.M = M;
    g.N = N;
    g.K = K;
    g.alpha = alpha;
    g.bias = bias;
    g.zin = zin;
    g.ld_z = ld_z;
    g.act = act;
    g.out_f32 = out_f32;
    g.ld_f32 = ld_f32;
    g.out_bf16 = reinterpret_cast<__nv_bfloat16 *>(out_bf16);
    g.ld_bf16 = ld_bf16;
    g.out_bf16_t = reinterpret_cast<__nv_bfloat16 *>(out_bf16_t);
    g.ld_t = ld_t;
    g.err = err;
    const bool f32_vec = !out_f32 || ((((uintptr_t)out_f32) & 15) == 0 && (ld_f32 % 4) == 0);
    const bool b16_vec = !out_bf16 || ((((uintptr_t)out_bf16) & 15) == 0 && (ld_bf16 % 8) == 0);
    g.vec = (f32_vec && b16_vec) ? 1 : 0;
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    const int tiles = (M + GM - 1) / GM;
    const int grid = tiles < sms ? tiles : sms;
    // the inference forms: alpha 1, a 16-byte-aligned bias, no gradient
    // input, one row-major vector output
    const bool inf = alpha == 1.0f && bias && ((((uintptr_t)bias) & 15) == 0) && !zin && !out_bf16_t && g.vec;
    if (inf && act && out_bf16 && !out_f32)
        k_gemm_tn<1><<<grid, GEMM_THREADS, GEMM_SMEM, stream>>>(ma, mb, g);
    else if (inf && !act && out_f32 && !out_bf16)
        k_gemm_tn<2><<<grid, GEMM_THREADS, GEMM_SMEM, stream>>>(ma, mb, g);
    else
        k_gemm_tn<0><<<grid, GEMM_THREADS, GEMM_SMEM, stream>>>(ma, mb, g);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return report_error(VPHYS_ERR_CUDA, cudaGetErrorString(e));
    return VPHYS_OK;
}

// The surrogate's forward pass in one launch: X [M, LK_INP] BF16 (the padded
// inputs zero), W1 [LK_HID, LK_INP], W2 [LK_HID, LK_HID], W3 [LK_OUTP, LK_HID]
// BF16 K-contiguous, biases FP32, Y [M, LK_OUTP] FP32; every pointer 16-byte
// aligned.
int mlp3_bf16(const void *X, int M, const void *W1, const float *b1, const void *W2, const float *b2, const void *W3,
              const float *b3, float *Y, int *err, cudaStream_t stream)
{
    if (M <= 0) return VPHYS_OK;
    if ((((uintptr_t)X) | ((uintptr_t)W1) | ((uintptr_t)W2) | ((uintptr_t)W3) | ((uintptr_t)b1) | ((uintptr_t)b2) |
         ((uintptr_t)b3) | ((uintptr_t)Y)) &
        15)
        return report_error(VPHYS_ERR_BAD_SHAPE, "vphys_mlp3_bf16: every operand must be 16-byte aligned");
    CUtensorMap mx, m1, m2, m3;
    if (!make_map(&mx, X, M, LK_INP, LK_INP, GM) || !make_map(&m1, W1, LK_HID, LK_INP, LK_INP, LK_HID) ||
        !make_map(&m2, W2, LK_HID, LK_HID, LK_HID, LK_HID) || !make_map(&m3, W3, LK_OUTP, LK_HID, LK_HID, LK_OUTP))
        return report_error(VPHYS_ERR_CUDA, "vphys_mlp3_bf16: cuTensorMapEncodeTiled failed");
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_mlp3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ML_SMEM);
        attr_set = true;
    }
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    MlpArgs a{M, b1, b2, b3, Y, err};
    const int tiles = (M + GM - 1) / GM;
    k_mlp3<<<tiles < sms ? tiles : sms, ML_THREADS, ML_SMEM, stream>>>(mx, m1, m2, m3, a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return report_error(VPHYS_ERR_CUDA, cudaGetErrorString(e));
    return VPHYS_OK;
}

}  // namespace vphys

extern "C" int vphys_mlp3_bf16(const void *X, int M, const void *W1, const float *b1, const void *W2, const float *b2,
                               const void *W3, const float *b3, float *Y, int *err, void *stream)
{
    return vphys::mlp3_bf16(X, M, W1, b1, W2, b2, W3, b3, Y, err, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int vphys_gemm_tn_bf16(const void *A, long long lda, const void *B, long long ldb, int M, int N, int K,
                                  float alpha, const float *bias, const float *zin, int ld_z, int act, float *out_f32,
                                  int ld_f32, void *out_bf16, int ld_bf16, void *out_bf16_t, int ld_t, int *err,
                                  void *stream)
{
    return vphys::gemm_tn_bf16(A, lda, B, ldb, M, N, K, alpha, bias, zin, ld_z, act, out_f32, ld_f32, out_bf16,
                               ld_bf16, out_bf16_t, ld_t, err, reinterpret_cast<cudaStream_t>(stream));
}
