// vphys_learned.cu -- the learned KPP surrogate: features, targets, training
// helpers and the in-step application with its range gate and sampled check.
//
// The reference's KPP pass 1 (vmix_kpp_overlay_impl, rdb_ocean_vmix.F90:1288-1426)
// walks each column down from the surface accumulating the bulk Richardson
// number until it crosses ri_crit.  The surrogate is an MLP
//     154 features -> 256 GELU -> 256 GELU -> 77 outputs        (BF16, FP32 accumulation)
// whose inputs are the quantities that walk looks at, per column:
//     u* = sqrt(|tau| / rho0), B0 (the surface buoyancy flux of pass 1), f, the
//     column depth H, and for the 75 layers below the surface layer the bulk
//     N^2 = db/dd and bulk shear^2 = |dV|^2/dd^2 relative to the surface layer
// (signed log1p(|x|/1e-6) of those two), each standardised with the training
// set's mean and standard deviation.  Outputs: log(h_b / 10 m), log(h_b w_s)
// and the shape G(sigma) * 27/4 at the 75 interfaces below the surface, each
// standardised the same way.  Training's GEMMs are vphys_gemm_tn_bf16 (tcgen05).
//
// In a step with cfg.learned_kpp: k_kpp_roll -> k_kpp_features -> k_mlp3 (the
// three layers in one launch, vphys_gemm.cu) -> k_kpp_apply, then the
// assembly takes h_b from the network for every column
// except (a) those whose standardised features leave [-gate, gate] (range
// gate), (b) a hashed `check_fraction` of the columns, which run the plain
// pass 1 and count a failure when the network's h_b differs from it by more
// than `check_tolerance` (relative), and (c) every column of a step that
// follows one whose failed fraction exceeded `fail_fraction` (fallback).
// Pass 2 (the K profile, rdb_ocean_vmix.F90:1429-1515) is the reference's,
// driven by whichever h_b the column got.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "vphys_device.cuh"
#include "vphys_kernels.cuh"

namespace vphys {

// ---- features ----------------------------------------------------------------
struct FeatOut {
    float *raw;             // [ncols, LK_IN] unstandardised, or null
    __nv_bfloat16 *X;       // [ncols, LK_INP] standardised, or null
    __nv_bfloat16 *XT;      // [LK_INP, ld_t] standardised, transposed, or null
    long long ld_t;
    const float *mean, *istd;   // [LK_INP]; null: raw values
    float limit;
};

// signed log1p(|x| / 1e-6) with the fast hardware logarithm: the feature is
// rounded to BF16 (8 significant bits) after standardisation, far above the
// fast form's error
__device__ __forceinline__ float slog6(float x) { return copysignf(__logf(1.0f + fabsf(x) * 1.0e6f), x); }

constexpr int FEAT_THREADS = 128;
constexpr int FEAT_LD = LK_INP + 2;   // shared row stride (BF16): odd word stride, no bank conflicts

// feature m of this thread's column: raw (training), standardised BF16 into the
// block's shared rows (copied out coalesced) and/or transposed (coalesced as is)
__device__ __forceinline__ void emit(const FeatOut &o, __nv_bfloat16 *srow, size_t col, int m, float x, bool &oor)
{
    if (o.raw) o.raw[col * LK_IN + m] = x;
    const float v = o.mean ? (x - o.mean[m]) * o.istd[m] : x;
    oor = oor || !(fabsf(v) <= o.limit);
    const __nv_bfloat16 b = __float2bfloat16_rn(v);
    srow[m] = b;
    if (o.XT) o.XT[(size_t)m * o.ld_t + col] = b;
}

__global__ void __launch_bounds__(FEAT_THREADS) k_kpp_features(const Params p, const FeatOut o, unsigned char *gate,
                                                               float *colH)
{
    __shared__ __nv_bfloat16 tile[FEAT_THREADS * FEAT_LD];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    __nv_bfloat16 *srow = tile + threadIdx.x * FEAT_LD;
    const int i0 = blockIdx.x * blockDim.x;
    const int rows = min((int)blockDim.x, p.nx - i0);   // columns of this block (consecutive in memory)
    if (i < p.nx) {
    const vphys_config &c = p.cfg;
    const int nx = p.nx, nz = p.nz;
    const size_t P = p.plane, PU = p.plane_u, PV = p.plane_v;
    const size_t col = (size_t)i + (size_t)nx * j;
    const double *__restrict__ hp = p.h + col;
    const double *__restrict__ rp = p.rho + col;
    const double *__restrict__ up = p.u + (size_t)i + (size_t)(nx + 1) * j;
    const double *__restrict__ vp = p.v + (size_t)i + (size_t)nx * j;
    auto HH = [&](int k) { return __ldg(hp + P * (size_t)(k - 1)); };
    auto UC = [&](int k) { return 0.5 * (__ldg(up + PU * (size_t)(k - 1)) + __ldg(up + PU * (size_t)(k - 1) + 1)); };
    auto VC = [&](int k) { return 0.5 * (__ldg(vp + PV * (size_t)(k - 1)) + __ldg(vp + PV * (size_t)(k - 1) + nx)); };
    const double rho0 = c.rho0;

    // surface layer and column depth, as KPP pass 1 (rdb_vl_first_live)
    int k_sfc = nz;
    bool all_zero = true;
    for (int k = nz; k >= 1; --k) {
        const double hk = HH(k);
        if (hk > H_VANISHED) {
            k_sfc = k;
            all_zero = false;
            break;
        }
        all_zero = all_zero && (hk == 0.0);
    }

    const double u_star = sqrt(xdiv(p.stress_mag[col], rho0));
    // the B0 of KPP pass 1: with shortwave, the part passing the lagged h_b is not charged
    const double q_T_kin = kpp_q_t_kin(c, p.q_heat[col], p.sw_src + col, p.sw_kappa, col, p.plane, p.bl_depth[col], HH(k_sfc));
    const double q_S_kin = xdiv(p.q_salt[col], rho0);
    double T_sfc = 0.0, S_sfc = 0.0;
    if (c.buoyancy_coeffs) {   // the same surface (T, S) the assembly's B0 will use
        T_sfc = p.tr[c.idx_temperature][col + P * (size_t)(k_sfc - 1)];
        S_sfc = p.tr[c.idx_salinity][col + P * (size_t)(k_sfc - 1)];
    }
    const double B_0 = kpp_surface_b0(c, q_T_kin, q_S_kin, HH(k_sfc), T_sfc, S_sfc);
    const double f = p.coriolis ? p.coriolis[col] : 0.0;
    bool oor = false;
    emit(o, srow, col, 0, (float)(u_star * 100.0), oor);
    emit(o, srow, col, 1, (float)(B_0 * 1.0e8), oor);
    emit(o, srow, col, 2, (float)(f * 1.0e4), oor);

    double u_ref = 0, v_ref = 0, b_ref = 0, d_ref = 0, d_c = 0, h_above = 0;
    if (!all_zero) {
        u_ref = UC(k_sfc);
        v_ref = VC(k_sfc);
        b_ref = -(GRAVITY * __ldg(rp + P * (size_t)(k_sfc - 1)) / rho0);
        h_above = HH(k_sfc);
        d_ref = 0.5 * h_above;
        d_c = d_ref;
    }
    // the walk down from the surface layer, loads FEAT_U levels at a time;
    // the column depth H (the surface layer, the walked layers, then any
    // below them) is summed on the way, so h is read once.  (Loading the next
    // block during the current one measured slower here: 156 registers
    // against 100 leave 12 warps per SM instead of 20.)
    double H = all_zero ? 0.0 : h_above;
#ifndef VPHYS_FEAT_U
#define VPHYS_FEAT_U 4
#endif
    constexpr int FEAT_U = VPHYS_FEAT_U;
    for (int m0 = 0; m0 < LK_LEV; m0 += FEAT_U) {
        double hk[FEAT_U], rk[FEAT_U], ua[FEAT_U], ub[FEAT_U], va[FEAT_U], vb[FEAT_U];
#pragma unroll
        for (int q = 0; q < FEAT_U; ++q) {
            const int k = k_sfc - 1 - (m0 + q);
            const bool in = !all_zero && k >= 1 && m0 + q < LK_LEV;
            const size_t o = P * (size_t)(k - 1), ou = PU * (size_t)(k - 1), ov = PV * (size_t)(k - 1);
            hk[q] = in ? __ldg(hp + o) : 0.0;
            rk[q] = in ? __ldg(rp + o) : 0.0;
            ua[q] = in ? __ldg(up + ou) : 0.0;
            ub[q] = in ? __ldg(up + ou + 1) : 0.0;
            va[q] = in ? __ldg(vp + ov) : 0.0;
            vb[q] = in ? __ldg(vp + ov + nx) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < FEAT_U; ++q) {
            const int m = m0 + q;
            if (m >= LK_LEV) break;
            const int k = k_sfc - 1 - m;
            float n2 = 0.0f, s2 = 0.0f;
            if (!all_zero && k >= 1) {
                d_c = d_c + 0.5 * (h_above + hk[q]);
                const double dd = d_c - d_ref;
                const double db = b_ref - (-(GRAVITY * rk[q] / rho0));
                const double du = 0.5 * (ua[q] + ub[q]) - u_ref, dv = 0.5 * (va[q] + vb[q]) - v_ref;
                if (dd > 0.0) {
                    // the differences in FP64 (a density step of 1e-3 on 1027 keeps
                    // only 3 digits in FP32), the quotients in FP32 (BF16 features)
                    const float rdd = __frcp_rn((float)dd);
                    n2 = (float)db * rdd;
                    s2 = (float)(du * du + dv * dv) * (rdd * rdd);
                }
                h_above = hk[q];
                H += hk[q];
            }
            emit(o, srow, col, 4 + m, slog6(n2), oor);
            emit(o, srow, col, 4 + LK_LEV + m, slog6(s2), oor);
        }
    }
    for (int k = k_sfc - 1 - LK_LEV; k >= 1 && !all_zero; --k) H += HH(k);
    emit(o, srow, col, 3, (float)(H * 1.0e-3), oor);
    for (int m = LK_IN; m < LK_INP; ++m) {   // K padding
        srow[m] = __float2bfloat16_rn(0.0f);
        if (o.XT) o.XT[(size_t)m * o.ld_t + col] = __float2bfloat16_rn(0.0f);
    }
    if (gate) gate[col] = oor ? 1 : 0;
    if (colH) colH[col] = all_zero ? -1.0f : (float)H;
    }
    __syncthreads();
    if (o.X && rows > 0) {
        // the block's rows are consecutive columns: one contiguous run of
        // rows * 160 BF16, written as 4-byte words by consecutive threads
        const size_t col0 = (size_t)i0 + (size_t)p.nx * j;
        uint32_t *dst = reinterpret_cast<uint32_t *>(o.X + col0 * LK_INP);
        const int words = rows * (LK_INP / 2);
        for (int w = threadIdx.x; w < words; w += blockDim.x) {
            const int r = w / (LK_INP / 2), c2 = w % (LK_INP / 2);
            const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162 *>(tile + r * FEAT_LD + 2 * c2);
            dst[w] = *reinterpret_cast<const uint32_t *>(&v);
        }
    }
}

// ---- training targets from the plain KPP's state ------------------------------
__global__ void k_kpp_targets(const Params p, float *T)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= p.nx) return;
    const vphys_config &c = p.cfg;
    const int nx = p.nx, nz = p.nz;
    const size_t P = p.plane;
    const size_t col = (size_t)i + (size_t)nx * j;
    const double *__restrict__ hp = p.h + col;
    int k_sfc = nz;
    for (int k = nz; k >= 1; --k)
        if (__ldg(hp + P * (size_t)(k - 1)) > H_VANISHED) {
            k_sfc = k;
            break;
        }
    const double rho0 = c.rho0;
    const double h_b = p.bl_depth[col];
    const double u_star = sqrt(xdiv(p.stress_mag[col], rho0));
    const double q_T_kin = xdiv(p.q_heat[col], rho0 * c.cp);
    const double q_S_kin = xdiv(p.q_salt[col], rho0);
    // with "eos" coefficients or shortwave, the B0 of the assembly that set this h_b
    const double B_0 = (c.buoyancy_coeffs || c.sw_pen_frac != 0.0)
                           ? p.b0[col]
                           : (GRAVITY / rho0) * (c.alpha_T * q_T_kin - c.beta_S * q_S_kin);
    const double w_star = sm_cbrt(fmx(0.0, -B_0) * h_b);
    const double w_s = sqrt(u_star * u_star + w_star * w_star);
    float *t = T + col * LK_OUTP;
    t[0] = logf(fmaxf((float)h_b, 0.1f) / 10.0f);
    t[1] = logf(fmaxf((float)(h_b * w_s), 1.0e-9f));
    double d = 0.0;
    for (int m = 0; m < LK_LEV; ++m) {
        const int q = k_sfc - m;
        float g = 0.0f;
        if (q >= 1) {
            d += __ldg(hp + P * (size_t)(q - 1));
            if (q > 1 && h_b > 0.0 && d < h_b) {
                const double s = d / h_b;
                g = (float)(6.75 * s * (1.0 - s) * (1.0 - s));
            }
        }
        t[2 + m] = g;
    }
    for (int m = LK_OUT; m < LK_OUTP; ++m) t[m] = 0.0f;
}

// ---- training helpers ----------------------------------------------------------
// dY = scale * w[c] * (Y - T) (FP32, BF16, BF16 transposed); loss += sum w (Y - T)^2
__global__ void k_mse_grad(const float *__restrict__ Y, const float *__restrict__ T, const float *__restrict__ w,
                           int rows, int cols, float scale, float *dY32, __nv_bfloat16 *dY, __nv_bfloat16 *dYT,
                           float *loss)
{
    const long long n = (long long)rows * cols;
    float acc = 0.0f;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(idx / cols), cc = (int)(idx % cols);
        const float e = Y[idx] - T[idx];
        const float g = scale * w[cc] * e;
        acc += w[cc] * e * e;
        if (dY32) dY32[idx] = g;
        const __nv_bfloat16 gb = __float2bfloat16_rn(g);
        if (dY) dY[idx] = gb;
        if (dYT) dYT[(size_t)cc * rows + r] = gb;
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && loss) atomicAdd(loss, acc);
}

// out[c] += sum over rows of G[r, c] (G row-major, ld)
__global__ void k_colsum(const float *__restrict__ G, int rows, int cols, int ld, float *out)
{
    __shared__ float part[8][33];
    const int c = blockIdx.x * 32 + threadIdx.x;
    float acc = 0.0f;
    if (c < cols)
        for (int r = blockIdx.y * 8 + threadIdx.y; r < rows; r += gridDim.y * 8) acc += G[(size_t)r * ld + c];
    part[threadIdx.y][threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.y == 0 && c < cols) {
        float s = 0.0f;
        for (int y = 0; y < 8; ++y) s += part[y][threadIdx.x];
        atomicAdd(out + c, s);
    }
}

// sum and sum of squares of each column (FP64 accumulation)
__global__ void k_colstats(const float *__restrict__ X, long long rows, int cols, int ld, double *sum, double *sumsq)
{
    __shared__ double ps[8][33], pq[8][33];
    const int c = blockIdx.x * 32 + threadIdx.x;
    double a = 0.0, b = 0.0;
    if (c < cols)
        for (long long r = blockIdx.y * 8 + threadIdx.y; r < rows; r += (long long)gridDim.y * 8) {
            const double x = X[r * ld + c];
            a += x;
            b += x * x;
        }
    ps[threadIdx.y][threadIdx.x] = a;
    pq[threadIdx.y][threadIdx.x] = b;
    __syncthreads();
    if (threadIdx.y == 0 && c < cols) {
        double s = 0.0, q = 0.0;
        for (int y = 0; y < 8; ++y) {
            s += ps[y][threadIdx.x];
            q += pq[y][threadIdx.x];
        }
        atomicAdd(sum + c, s);
        atomicAdd(sumsq + c, q);
    }
}

// (raw[r, c] - mean[c]) * istd[c] for c < cols_in, 0 for cols_in <= c < cols_out
__global__ void k_standardize(const float *__restrict__ raw, long long rows, int cols_in, int ld_in,
                              const float *mean, const float *istd, int cols_out, __nv_bfloat16 *X,
                              __nv_bfloat16 *XT, long long ld_t, float *out32)
{
    const long long n = rows * cols_out;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long r = idx / cols_out;
        const int c = (int)(idx % cols_out);
        const float v = (c < cols_in) ? (raw[r * ld_in + c] - mean[c]) * istd[c] : 0.0f;
        if (out32) out32[idx] = v;
        const __nv_bfloat16 b = __float2bfloat16_rn(v);
        if (X) X[idx] = b;
        if (XT) XT[(size_t)c * ld_t + r] = b;
    }
}

// Adam (Kingma & Ba 2015) on an FP32 master [rows, cols]; refreshes its BF16
// copy [rows, cols] and transposed copy [cols, rows] (either may be null)
__global__ void k_adam(float *w, float *m, float *v, const float *__restrict__ g, int rows, int cols, float lr,
                       float b1, float b2, float eps, float bc1, float bc2, __nv_bfloat16 *wb, __nv_bfloat16 *wbt)
{
    const long long n = (long long)rows * cols;
    for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const float gi = g[idx];
        const float mi = b1 * m[idx] + (1.0f - b1) * gi;
        const float vi = b2 * v[idx] + (1.0f - b2) * gi * gi;
        m[idx] = mi;
        v[idx] = vi;
        const float wi = w[idx] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        w[idx] = wi;
        const __nv_bfloat16 b = __float2bfloat16_rn(wi);
        if (wb) wb[idx] = b;
        if (wbt) wbt[(size_t)(idx % cols) * rows + idx / cols] = b;
    }
}

// ---- in-step application ----------------------------------------------------------
// kpp_stats: [0] checked this step, [1] failed, [2] fallback flag of the running
// step, [3] gated this step, [4] total checked, [5] total failed, [6] fallback
// steps, [7] total gated, [8] sum of squared relative errors * 1e6, [9] steps
__global__ void k_kpp_roll(unsigned long long *st, float fail_fraction)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const bool fb = st[0] > 0 && (double)st[1] > (double)fail_fraction * (double)st[0];
    st[2] = fb ? 1ull : 0ull;
    st[4] += st[0];
    st[5] += st[1];
    st[6] += fb ? 1ull : 0ull;
    st[7] += st[3];
    st[9] += 1;
    st[0] = st[1] = st[3] = 0;
}

__device__ __forceinline__ unsigned hash_col(unsigned long long col, unsigned gen)
{
    unsigned long long z = col * 0x9e3779b97f4a7c15ull + (unsigned long long)gen * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 30)) * 0x94d049bb133111ebull;
    return (unsigned)((z ^ (z >> 31)) & 0xffffffffu);
}

__global__ void k_kpp_apply(size_t ncols, const float *__restrict__ Y, float tmean0, float tstd0,
                            const unsigned char *__restrict__ gate, const float *__restrict__ colH, float *pred,
                            float *check, unsigned long long *st, unsigned gen, float check_fraction)
{
    const size_t col = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (col >= ncols) return;
    const float H = colH[col];
    if (H < 0.0f) {   // no live layer: pass 1 gives 0 without a walk
        pred[col] = 0.0f;
        check[col] = -1.0f;
        return;
    }
    float hb = 10.0f * expf(Y[col * LK_OUTP] * tstd0 + tmean0);
    hb = fminf(fmaxf(hb, 0.0f), H);
    const bool gated = gate[col] != 0;
    if (gated) atomicAdd(st + 3, 1ull);
    const bool fallback = st[2] != 0;
    const bool sampled = (float)hash_col(col, gen) < check_fraction * 4294967296.0f;
    if (fallback || gated || !(hb == hb)) {
        pred[col] = -1.0f;
        check[col] = -1.0f;
    } else if (sampled) {
        pred[col] = -1.0f;
        check[col] = hb;
    } else {
        pred[col] = hb;
        check[col] = -1.0f;
    }
}

// ---- launchers ---------------------------------------------------------------------
void launch_kpp_features(const Params &p, float *raw, void *X, void *XT, long long ld_t, const float *mean,
                         const float *istd, float limit, unsigned char *gate, float *colH, cudaStream_t s)
{
    FeatOut o{raw, reinterpret_cast<__nv_bfloat16 *>(X), reinterpret_cast<__nv_bfloat16 *>(XT), ld_t, mean, istd,
              limit};
    k_kpp_features<<<dim3((p.nx + FEAT_THREADS - 1) / FEAT_THREADS, p.ny), FEAT_THREADS, 0, s>>>(p, o, gate, colH);
}

void launch_kpp_targets(const Params &p, float *T, cudaStream_t s)
{
    k_kpp_targets<<<dim3((p.nx + 127) / 128, p.ny), 128, 0, s>>>(p, T);
}

void launch_kpp_roll(unsigned long long *st, float fail_fraction, cudaStream_t s)
{
    k_kpp_roll<<<1, 32, 0, s>>>(st, fail_fraction);
}

void launch_kpp_apply(size_t ncols, const float *Y, float tmean0, float tstd0, const unsigned char *gate,
                      const float *colH, float *pred, float *check, unsigned long long *st, unsigned gen,
                      float check_fraction, cudaStream_t s)
{
    k_kpp_apply<<<(unsigned)((ncols + 255) / 256), 256, 0, s>>>(ncols, Y, tmean0, tstd0, gate, colH, pred, check, st,
                                                               gen, check_fraction);
}

static int grid_for(long long n)
{
    long long b = (n + 255) / 256;
    return (int)(b < 148 * 32 ? (b > 0 ? b : 1) : 148 * 32);
}

}  // namespace vphys

extern "C" {

int vphys_mlp_loss(const float *Y, const float *T, const float *w, int rows, int cols, float scale, float *dY32,
                   void *dY, void *dYT, float *loss, void *stream)
{
    vphys::k_mse_grad<<<vphys::grid_for((long long)rows * cols), 256, 0, (cudaStream_t)stream>>>(
        Y, T, w, rows, cols, scale, dY32, reinterpret_cast<__nv_bfloat16 *>(dY), reinterpret_cast<__nv_bfloat16 *>(dYT),
        loss);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VPHYS_OK : vphys::report_error(VPHYS_ERR_CUDA, cudaGetErrorString(e));
}

int vphys_mlp_colsum(const float *G, int rows, int cols, int ld, float *out, void *stream)
{
    dim3 grid((cols + 31) / 32, (unsigned)(rows / 64 + 1 < 256 ? rows / 64 + 1 : 256));
    vphys::k_colsum<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(G, rows, cols, ld, out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VPHYS_OK : vphys::report_error(VPHYS_ERR_CUDA, cudaGetErrorString(e));
}

int vphys_mlp_colstats(const float *X, long long rows, int cols, int ld, double *sum, double *sumsq, void *stream)
{
    dim3 grid((cols + 31) / 32, (unsigned)(rows / 64 + 1 < 512 ? rows / 64 + 1 : 512));
    vphys::k_colstats<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(X, rows, cols, ld, sum, sumsq);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VPHYS_OK : vphys::report_error(VPHYS_ERR_CUDA, cudaGetErrorString(e));
}

int vphys_mlp_standardize(const float *raw, long long rows, int cols_in, int ld_in, const float *mean,
                          const float *istd, int cols_out, void *X, void *XT, long long ld_t, float *out32,
                          void *stream)
{
    vphys::k_standardize<<<vphys::grid_for(rows * cols_out), 256, 0, (cudaStream_t)stream>>>(
        raw, rows, cols_in, ld_in, mean, istd, cols_out, reinterpret_cast<__nv_bfloat16 *>(X),
        reinterpret_cast<__nv_bfloat16 *>(XT), ld_t, out32);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VPHYS_OK : vphys::report_error(VPHYS_ERR_CUDA, cudaGetErrorString(e));
}

int vphys_mlp_adam(float *w, float *m, float *v, const float *g, int rows, int cols, float lr, float b1, float b2,
                   float eps, int step, void *wb, void *wbt, void *stream)
{
    if (step < 1) return vphys::report_error(VPHYS_ERR_CONFIG, "vphys_mlp_adam: step counts from 1");
    const float bc1 = 1.0f - powf(b1, (float)step), bc2 = 1.0f - powf(b2, (float)step);
    vphys::k_adam<<<vphys::grid_for((long long)rows * cols), 256, 0, (cudaStream_t)stream>>>(
        w, m, v, g, rows, cols, lr, b1, b2, eps, bc1, bc2, reinterpret_cast<__nv_bfloat16 *>(wb),
        reinterpret_cast<__nv_bfloat16 *>(wbt));
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? VPHYS_OK : vphys::report_error(VPHYS_ERR_CUDA, cudaGetErrorString(e));
}

}  // extern "C"
