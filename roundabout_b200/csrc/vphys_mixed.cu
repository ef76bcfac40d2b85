// vphys_mixed.cu -- the mixed-precision form of the implicit solves: FP32
// factorisation and sweeps, FP64 residual and FP64 forward accumulation.
//
// Each column solves A x = d (A = I + dt * vertical diffusion operator:
// rdb_ocean_vdiff.F90:1248-1349 for tracers, 1611-1925 for momentum) for the
// INCREMENT x = d + delta.  Row k scaled by its thickness H_k is the
// conservative form
//     (H_k + E_k + F_k + F_{k+1}) x_k - F_k x_{k-1} - F_{k+1} x_{k+1} = H_k rhs_k
// with F_k = dt K_k / dz_k the coupling of interface k (alpha_k = F_{k+1}/H_k,
// beta_k = F_k/H_k in the reference's rows) and E_k a diagonal extra (bottom
// drag, BBL glue).  The increment solves the same matrix with the FP64
// residual b = H rhs - (H + E + G) d, i.e. b_k = F_k (d_{k-1} - d_k) +
// F_{k+1} (d_{k+1} - d_k) - E_k d_k (+ the wind stress), built from the SAME
// FP32 couplings the factorisation uses, so the telescoping sum of the
// internal fluxes cancels exactly and FP32 rounding only perturbs delta.
//
// The factorisation keeps, per row, the pivot p_k = s_k + F_{k+1}, its excess
//     s_k = H_k + E_k + F_k q_{k-1}         (a sum of positive terms)
// and BOTH complementary ratios u_k = F_{k+1}/p_k and q_k = s_k/p_k
// (u + q = 1): across a stiff interface (F >> s: a 1 mm layer under KPP
// mixing) u rounds to 1 in FP32 and only q carries the information, across a
// weak one (F << s) it is the other way round, so each multiplication by
// u_k is done as (1 - q_k)*z = z - q_k z when q_k < 1/2 and as u_k z
// otherwise (t_k below: -q_k or u_k).  Then
//     forward (FP64):  w_k = b_k + u_{k-1} w_{k-1},   v_k = w_k / p_k
//     backward (FP32): delta_k = v_k + u_k delta_{k+1},   x_k = d_k + delta_k (FP64)
//
// Tracers: one warp per block, 32 columns (the lanes) x one tracer; the grid
// runs the tracers of a column group back to back (adjacent blocks), so
// h and K, read by each of them, come from L2 after the first.  Each warp
// factorises in its own upward pass (FP32 arithmetic is cheap next to the
// loads; no warp waits for another), keeps t and v (8 B per level and lane)
// in shared memory, and reads d again from L2 in the back-substitution.  All
// loads of a pass are issued MP_TR_U levels ahead of the arithmetic.
//
// Momentum: one thread per u or v face column; t and v in shared memory, the
// velocity read again from L2 (evict_last) by the back-substitution.
#include <cuda_runtime.h>

#include <cstdlib>

#include "vphys_device.cuh"
#include "vphys_faces.cuh"
#include "vphys_kernels.cuh"
#include "vphys_mom_ring.cuh"
#include "vphys_tmem.cuh"

namespace vphys {

constexpr int MP_TR_COLS = 32;      // columns (lanes) per tracer block
#ifndef VPHYS_MP_TR_U
#define VPHYS_MP_TR_U 4
#endif
#ifndef VPHYS_MP_MOM_THREADS
#define VPHYS_MP_MOM_THREADS 32
#endif
#ifndef VPHYS_MP_MOM_U
// levels per load block of the register face solve, whose loads of the next
// block are in flight during the current one (1440x1080x75: 2.57 ms with 4,
// 2.65 with 6, 3.31 with 8 -- registers; before the pipelining 2.87 with 6)
#define VPHYS_MP_MOM_U 4
#endif
#ifndef VPHYS_MP_MOM_UB
// levels per load block of the ring face solve's back-substitution
// (1440x1080x75: 2.84 ms with 4, 2.75 with 6, 2.69 with 8)
#define VPHYS_MP_MOM_UB 8
#endif
constexpr int MP_TR_U = VPHYS_MP_TR_U;                // levels per tracer load block
#ifndef VPHYS_MP_TR_UF
#define VPHYS_MP_TR_UF 6   // 1440x1080x75 step: 8.955 ms with 4, 8.898 with 6, 9.40 with 8
#endif
constexpr int MP_TR_UF = VPHYS_MP_TR_UF;   // levels per load block of the back-substitution with the non-local deposit
constexpr int MP_MOM_THREADS = VPHYS_MP_MOM_THREADS;  // face columns per momentum block
constexpr int MP_MOM_U = VPHYS_MP_MOM_U;              // levels per momentum load block
constexpr int MP_MOM_UB = VPHYS_MP_MOM_UB;            // levels per load block of the ring solve's back-substitution
// Largest tracer increment (in the tracer's units) a mixed solve keeps.  The
// FP32 couplings and the FP32 back-substitution leave an error of about
// 3 eps_32 |delta| (eps_32 = 6e-8): 2 units keep it under 4e-7.  A column
// group with a larger increment in one step -- a 1 mm top layer taking a
// surface heat flux warms by tens of kelvin -- is re-solved in FP64.
constexpr float MP_DELTA_MAX = 2.0f;

// Hardware reciprocal (MUFU, within 1 ulp): the FP32 factors carry no
// bitwise contract, and their rounding is a consistent perturbation of the
// couplings that the FP64 residual then sees.
__device__ __forceinline__ float rcp_approx(float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// One row of the factorisation: the pivot's reciprocal and the signed
// multiplier t (-q when q < 1/2, else u) from the excess s and the coupling
// above; q = 1, t = 0 exactly for a row not coupled upward.
__device__ __forceinline__ void pivot_row(float s, float f_up, float &ip, float &t, float &q)
{
    ip = rcp_approx(s + f_up);
    const float qq = s * ip;
    q = (f_up == 0.0f) ? 1.0f : qq;
    t = (f_up == 0.0f) ? 0.0f : ((qq < 0.5f) ? -qq : f_up * ip);
}
// u * z from the signed multiplier
__device__ __forceinline__ double mul_u(float t, double z) { return (t < 0.0f) ? z + (double)t * z : (double)t * z; }
__device__ __forceinline__ float mul_u(float t, float z) { return (t < 0.0f) ? z + t * z : t * z; }

// Live span of every column: the first live layer from the bed and from the
// surface (rdb_vl_first_live's test h > H_VANISHED), packed lo | hi << 16,
// 0 for a column without one.  Loads go MP_TR_U levels at a time, so a column
// with many fillers under its bathymetry costs a few load latencies, not one
// per filler.
__global__ void k_spans(const Params p)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= p.nx) return;
    const size_t col = (size_t)i + (size_t)p.nx * j;
    const double *__restrict__ hp = p.h + col;
    const size_t P = p.plane;
    const int nz = p.nz;
    int lo = 0, hi = 0;
    for (int k0 = 1; k0 <= nz && lo == 0; k0 += MP_TR_U) {
        double hv[MP_TR_U];
#pragma unroll
        for (int u = 0; u < MP_TR_U; ++u) hv[u] = (k0 + u <= nz) ? __ldg(hp + P * (size_t)(k0 + u - 1)) : 0.0;
#pragma unroll
        for (int u = MP_TR_U - 1; u >= 0; --u)
            if (hv[u] > H_VANISHED) lo = k0 + u;
    }
    if (lo > 0) {
        for (int k0 = nz; k0 >= lo && hi == 0; k0 -= MP_TR_U) {
            double hv[MP_TR_U];
#pragma unroll
            for (int u = 0; u < MP_TR_U; ++u) hv[u] = (k0 - u >= lo) ? __ldg(hp + P * (size_t)(k0 - u - 1)) : 0.0;
#pragma unroll
            for (int u = MP_TR_U - 1; u >= 0; --u)
                if (hv[u] > H_VANISHED) hi = k0 - u;
        }
    }
    p.span[col] = lo | (hi << 16);
    if (col == 0) {
        if (p.mp_redo) p.mp_redo[0] = 0;     // the re-solve list of the tracer kernel that follows
        if (p.work_ctr) p.work_ctr[0] = 0;   // and its work counter
    }
}

// Back-substitution of one tracer column from the t and v rows; with FULL the
// heat/salt budgets and the KPP non-local deposit (nonlocal_face_flux,
// rdb_ocean_vmix.F90:1605-1714) ride along.
template <bool FULL, bool CI = false>
__device__ __forceinline__ void tracer_back(const Params &p, double dt, double *__restrict__ trc,
                                            const double *__restrict__ hp, const float *tu, const float *vv, int w_lo,
                                            int w_hi, int lo, int hi, double *bud, bool nl_t, bool nl, double h_b,
                                            double q_kin, unsigned long long pol, double *c_new = nullptr,
                                            double *e_new = nullptr)
{
    const size_t P = p.plane;
    const int nz = p.nz;
    float delta = 0.0f;
    double g_above = 0.0, d_run = 0.0, h_a = 0.0;
    double h_c = (FULL && lo <= hi) ? __ldg(hp + P * (size_t)(hi - 1)) : 0.0;
    const double r_hb = (FULL && nl) ? rcp_nr(h_b) : 0.0;   // sigma = d_run / h_b as a product
    constexpr int BU = FULL ? MP_TR_UF : MP_TR_U;   // the deposit's registers leave room for fewer loads
    // a block's old values and, with the deposit, the thicknesses one level
    // down, loaded while the block above is computed
    auto load_down = [&](int k0, double (&db_)[BU], double (&hb_)[BU]) {
#pragma unroll
        for (int u = 0; u < BU; ++u) {
            const int k = k0 - u;
            db_[u] = (k >= lo && k <= hi) ? ld_hint(trc + P * (size_t)(k - 1), pol) : 0.0;
            if (FULL) hb_[u] = (k > 1 && k >= lo && k <= hi) ? __ldg(hp + P * (size_t)(k - 2)) : 0.0;
        }
    };
    double dk[BU], hb[BU];
    load_down(w_hi, dk, hb);
    for (int k0 = w_hi; k0 >= w_lo; k0 -= BU) {
        double dx[BU], hx[BU];
        load_down(k0 - BU, dx, hx);
#pragma unroll
        for (int u = 0; u < BU; ++u) {
            const int k = k0 - u;
            if (k < w_lo) break;
            const size_t s = (size_t)(k - 1) * MP_TR_COLS;
            delta = vv[s] + mul_u(tu[s], delta);   // rows outside the span: v = t = 0
            if (k < lo || k > hi) continue;
            const size_t off = P * (size_t)(k - 1);
            const double d_k = dk[u];
            double x = d_k + (double)delta;
            if (FULL) {
                if (bud) bud[off] = bud[off] + (h_c * x - h_c * d_k);
                const double h_bl = hb[u];
                if (nl_t) {
                    double gk = 0.0;
                    if (nl) {
                        d_run = d_run + h_c;
                        if (k > 1 && d_run < h_b) {
                            const double sigma = d_run * r_hb;
                            gk = p.cfg.cs_nonlocal * (sigma * (1.0 - sigma) * (1.0 - sigma)) * q_kin;
                        }
                    }
                    double f_up = 0.0, f_dn = 0.0;
                    if (k < nz) f_up = nonlocal_face_flux(g_above, h_c, h_a);
                    if (k > 1) f_dn = nonlocal_face_flux(gk, h_bl, h_c);
                    const double src = dt * (f_up - f_dn);
                    if (src != 0.0) x = conc_add_source_mp(x, h_c, src, rcp_nr(h_c + H_DIV_EPS));
                    g_above = gk;
                }
                if (CI) neumaier_add(*c_new, *e_new, h_c * x);
                h_a = h_c;
                h_c = h_bl;
            }
            trc[off] = x;
        }
#pragma unroll
        for (int u = 0; u < BU; ++u) {
            dk[u] = dx[u];
            if (FULL) hb[u] = hx[u];
        }
    }
}

// The non-local column scalars of a live column (FP64, as KPP pass 2): the
// boundary-layer depth h_b and the kinematic heat and salt fluxes; true when
// the column takes the deposit (h_b > 0, w_s > 0, B_0 < 0).
__device__ __forceinline__ bool nonlocal_column(const Params &p, const vphys_config &c, size_t col,
                                                const double *__restrict__ hp, int hi, double &h_b, double &q_T_kin,
                                                double &q_S_kin)
{
    const double rho0 = c.rho0;
    h_b = p.bl_depth[col];
    const double u_star = sqrt(xdiv(p.stress_mag[col], rho0));
    // the heat flux pass 2 charged (shortwave: what passes h_b, or the
    // surface layer hi)
    q_T_kin = kpp_q_t_kin(c, p.q_heat[col], p.sw_src + col, p.sw_kappa, col, p.plane, h_b,
                          __ldg(hp + p.plane * (size_t)(hi - 1)));
    q_S_kin = xdiv(p.q_salt[col], rho0);
    // with "eos" coefficients or shortwave B0 is the assembly's (pass 2
    // stored it before the solve changed the surface T and S); otherwise
    // the same number recomputed
    const double B_0 = (c.buoyancy_coeffs || c.sw_pen_frac != 0.0)
                           ? p.b0[col]
                           : (GRAVITY / rho0) * (c.alpha_T * q_T_kin - c.beta_S * q_S_kin);
    const double wstar3 = fmx(0.0, -B_0) * h_b;
    const double w_star = sm_cbrt(wstar3);
    const double w_s = sqrt(u_star * u_star + w_star * w_star);
    return h_b > 0.0 && w_s > 0.0 && B_0 < 0.0;
}

// tracer_back<true> for the TPW tracers of a group in one downward pass: the
// thicknesses, the running depth and the shape of the non-local profile are
// loaded and computed once for the group, each tracer keeping its own
// increment, budget and deposit (dep[q]: the tracer takes the KPP deposit
// with kinematic flux q_kin[q]; nl: the column is convective).  Per tracer
// the arithmetic is tracer_back<true>'s.
template <int TPW>
__device__ __forceinline__ void tracer_back_group(const Params &p, double dt, double *const (&trc)[TPW], int nt,
                                                  const double *__restrict__ hp, const float *tu, const float *vv,
                                                  size_t NB, int w_lo, int w_hi, int lo, int hi,
                                                  double *const (&bud)[TPW], const bool (&dep)[TPW], bool nl,
                                                  double h_b, const double (&q_kin)[TPW], unsigned long long pol)
{
    const size_t P = p.plane;
    const int nz = p.nz;
    float delta[TPW];
    double g_above[TPW];
#pragma unroll
    for (int q = 0; q < TPW; ++q) delta[q] = 0.0f, g_above[q] = 0.0;
    double d_run = 0.0, h_a = 0.0;
    double h_c = (lo <= hi) ? __ldg(hp + P * (size_t)(hi - 1)) : 0.0;
    const double r_hb = nl ? rcp_nr(h_b) : 0.0;   // sigma = d_run / h_b as a product
    bool any_dep = false;
#pragma unroll
    for (int q = 0; q < TPW; ++q) any_dep = any_dep || dep[q];
    constexpr int BU = MP_TR_U;
    auto load_down = [&](int k0, double (&db_)[BU][TPW], double (&hb_)[BU]) {
#pragma unroll
        for (int u = 0; u < BU; ++u) {
            const int k = k0 - u;
            const bool in = k >= lo && k <= hi;
#pragma unroll
            for (int q = 0; q < TPW; ++q) db_[u][q] = (in && q < nt) ? ld_hint(trc[q] + P * (size_t)(k - 1), pol) : 0.0;
            hb_[u] = (in && k > 1) ? __ldg(hp + P * (size_t)(k - 2)) : 0.0;
        }
    };
    double dk[BU][TPW], hb[BU];
    load_down(w_hi, dk, hb);
    for (int k0 = w_hi; k0 >= w_lo; k0 -= BU) {
        double dx[BU][TPW], hx[BU];
        load_down(k0 - BU, dx, hx);
#pragma unroll
        for (int u = 0; u < BU; ++u) {
            const int k = k0 - u;
            if (k < w_lo) break;
            const size_t s = (size_t)(k - 1) * MP_TR_COLS;
            const float tk = tu[s];
#pragma unroll
            for (int q = 0; q < TPW; ++q) delta[q] = vv[(size_t)q * NB + s] + mul_u(tk, delta[q]);
            if (k < lo || k > hi) continue;
            const size_t off = P * (size_t)(k - 1);
            const double h_bl = hb[u];
            double shape = 0.0;   // cs_nonlocal * sigma (1 - sigma)^2 inside the boundary layer
            bool in_bl = false;
            if (nl) {
                d_run = d_run + h_c;
                if (k > 1 && d_run < h_b) {
                    const double sigma = d_run * r_hb;
                    shape = p.cfg.cs_nonlocal * (sigma * (1.0 - sigma) * (1.0 - sigma));
                    in_bl = true;
                }
            }
            // one reciprocal of the layer for every tracer's deposit
            const double r_h = any_dep ? rcp_nr(h_c + H_DIV_EPS) : 0.0;
#pragma unroll
            for (int q = 0; q < TPW; ++q) {
                if (q >= nt) break;
                const double d_k = dk[u][q];
                double x = d_k + (double)delta[q];
                if (bud[q]) bud[q][off] = bud[q][off] + (h_c * x - h_c * d_k);
                if (dep[q]) {
                    const double gk = in_bl ? shape * q_kin[q] : 0.0;
                    double f_up = 0.0, f_dn = 0.0;
                    if (k < nz) f_up = nonlocal_face_flux(g_above[q], h_c, h_a);
                    if (k > 1) f_dn = nonlocal_face_flux(gk, h_bl, h_c);
                    x = conc_add_source_mp(x, h_c, dt * (f_up - f_dn), r_h);
                    g_above[q] = gk;
                }
                trc[q][off] = x;
            }
            h_a = h_c;
            h_c = h_bl;
        }
#pragma unroll
        for (int u = 0; u < BU; ++u) {
            hb[u] = hx[u];
#pragma unroll
            for (int q = 0; q < TPW; ++q) dk[u][q] = dx[u][q];
        }
    }
}

// Tracer groups of a launch: the first `single` groups hold one tracer each
// (one tracer per warp: every tracer; otherwise none), the rest up to TPW
// tracers in the order of `perm`.
struct TracerGroups {
    int single, ngroups;
    signed char perm[NTR_MAX];
};

// TPW tracers per warp share one factorisation and one t array (TWO, a
// separate ks, keeps one tracer per warp); their forward chains interleave.
// CI (one tracer per warp): the compensated column content before the solve
// (terms bottom-up, from the FP64 old values of the upward pass) and after it
// (top-down, the FP64 new values of the downward pass) into p.content_old /
// p.content_new; a group re-solved in FP64 gets them from the re-solve.
template <bool TWO, int TPW, bool DEF, bool CI = false>
__global__ void __launch_bounds__(MP_TR_COLS) k_tracers_mp(const Params p, double dt, int nonlocal, int ngx,
                                                           const TracerGroups tg)
{
    const int ngroups = tg.ngroups;
    constexpr int U = (TPW >= 4) ? 4 : MP_TR_U;   // levels per load block
    extern __shared__ __align__(16) float smf[];
    const int lane = threadIdx.x;
    const int grp = blockIdx.x % ngroups;          // the tracer groups of a column group are adjacent blocks
    const unsigned g = blockIdx.x / ngroups;
    const int gi = g % ngx, j = g / ngx;
    const int i = gi * MP_TR_COLS + lane;
    vphys_config cd = p.cfg;   // DEF: the default knobs folded in (is_default_tracer_knobs)
    if (DEF) default_tracer_knobs(cd);
    const vphys_config &c = cd;
    const int nx = p.nx, nz = p.nz;
    const size_t P = p.plane;
    const bool in_grid = i < nx;
    const size_t col = (size_t)(in_grid ? i : 0) + (size_t)nx * j;
    const double *__restrict__ hp = p.h + col;
    const int iT = c.idx_temperature, iS = c.idx_salinity, iPS = c.idx_pseudo_salt;
    const size_t NB = (size_t)nz * MP_TR_COLS;
    int nt, tix[TPW];   // tracers of this group
    if (grp < tg.single) {
        nt = 1;
        tix[0] = tg.perm[grp];
    } else {
        const int base = tg.single + (grp - tg.single) * TPW;
        nt = min(TPW, p.ntr - base);
#pragma unroll
        for (int q = 0; q < TPW; ++q) tix[q] = tg.perm[base + (q < nt ? q : 0)];
    }
    if (grp >= tg.single) {
#pragma unroll
        for (int q = 1; q < TPW; ++q)
            if (q >= nt) tix[q] = tix[0];
    } else {
#pragma unroll
        for (int q = 1; q < TPW; ++q) tix[q] = tix[0];
    }
    float *tu = smf + lane;                        // t per level, this lane's column
    float *vv = tu + NB;                           // v per level and tracer (stride NB)
    const float HV = (float)H_VANISHED;

    // ---- this column's live span (k_spans); rows outside it are identity rows ----
    const int sp = in_grid ? p.span[col] : 0;
    const bool live = (sp & 0xffff) > 0;
    const int lo = live ? (sp & 0xffff) : nz + 1, hi = live ? (sp >> 16) : 0;
    const int w_lo = __reduce_min_sync(0xffffffffu, live ? lo : 0x7fffffff);
    const int w_hi = __reduce_max_sync(0xffffffffu, hi);
    if (w_hi == 0) {
        if (CI && in_grid) p.content_old[col + P * (size_t)tix[0]] = p.content_new[col + P * (size_t)tix[0]] = 0.0;
        return;
    }
    double c_old = 0.0, e_old = 0.0, c_new = 0.0, e_new = 0.0;   // CI: Neumaier sums and compensations

    const double *__restrict__ Kp = ((TWO && tix[0] != iT) ? p.ks : p.kt) + col;
    double *trc[TPW];
#pragma unroll
    for (int q = 0; q < TPW; ++q) trc[q] = p.tr[tix[q]] + col;
    const unsigned long long pol_keep = l2_policy_evict_last();
    const float dtf = (float)dt;

    float vsum = 0.0f;   // sum of |v| over rows and tracers: a bound on every |delta| below
    // ---- upward: factorisation (FP32, once for the group) + FP64 residual and
    //      accumulation of every tracer.  Branch-free rows: outside [lo, hi]
    //      nothing is loaded, h = 0 gates both couplings off and the row
    //      solves to an increment of 0 ----
    {
        const bool first = (w_lo == lo);   // the lane's span starts at the warp's first row
        double h_c = first ? __ldg(hp + P * (size_t)(w_lo - 1)) : 0.0;
        double d_c[TPW], d_m[TPW], w[TPW];
#pragma unroll
        for (int q = 0; q < TPW; ++q) {
            d_c[q] = (first && q < nt) ? ld_hint(trc[q] + P * (size_t)(w_lo - 1), pol_keep) : 0.0;
            d_m[q] = 0.0;
            w[q] = 0.0;
        }
        float f_dn = 0.0f, q_prev = 1.0f, t_prev = 0.0f;
        // row k reads h, K and d one level up; the loads of block k0 + U are
        // issued before block k0 is computed (two register buffers), so the
        // first row of a block does not wait on its own loads
        auto load_block = [&](int k0, double (&hb_)[U], double (&kb_)[U], double (&db_)[U][TPW]) {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int k = k0 + u;
                const bool need = k + 1 >= lo && k + 1 <= hi;
                const size_t o = P * (size_t)k;
                hb_[u] = need ? __ldg(hp + o) : 0.0;
                kb_[u] = need ? __ldg(Kp + o) : 0.0;
#pragma unroll
                for (int q = 0; q < TPW; ++q) db_[u][q] = (need && q < nt) ? ld_hint(trc[q] + o, pol_keep) : 0.0;
            }
        };
        double hn[U], kn[U], dn[U][TPW];
        load_block(w_lo, hn, kn, dn);
        for (int k0 = w_lo; k0 <= w_hi; k0 += U) {
            double hx[U], kx[U], dx[U][TPW];
            load_block(k0 + U, hx, kx, dx);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int k = k0 + u;
                if (k > w_hi) break;
                // row k (build_factorize_tracer_matrix: rdb_ocean_vdiff.F90:1285-1341;
                // gates on the raw FP64 thicknesses)
                const float H = fmx((float)h_c, HV);
                const float Hp = fmx((float)hn[u], HV);
                const bool coupled = h_c > H_VANISHED && hn[u] > H_VANISHED;
                const float f_up = coupled ? __fdividef(dtf * (float)kn[u], face_thick(H, Hp, c.use_harmonic)) : 0.0f;
                float ip, t, qq;
                pivot_row(H + f_dn * q_prev, f_up, ip, t, qq);
                const size_t s = (size_t)(k - 1) * MP_TR_COLS;
                const double fd = (double)f_dn, fu = (double)f_up, ipd = (double)ip;
                if (CI) neumaier_add(c_old, e_old, h_c * d_c[0]);   // rows off the span: 0 * 0
#pragma unroll
                for (int q = 0; q < TPW; ++q) {
                    const double b = fd * (d_m[q] - d_c[q]) + fu * (dn[u][q] - d_c[q]);
                    w[q] = b + mul_u(t_prev, w[q]);
                    const float vq = (float)(w[q] * ipd);
                    vv[(size_t)q * NB + s] = vq;
                    vsum += fabsf(vq);
                    d_m[q] = d_c[q];
                    d_c[q] = dn[u][q];
                }
                tu[s] = t;
                t_prev = t;
                q_prev = qq;
                f_dn = f_up;
                h_c = hn[u];
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                hn[u] = hx[u];
                kn[u] = kx[u];
#pragma unroll
                for (int q = 0; q < TPW; ++q) dn[u][q] = dx[u][q];
            }
        }
    }

    // ---- a group whose increment reaches MP_DELTA_MAX goes to the FP64 re-solve ----
    // delta_k = v_k + u_k delta_{k+1} with 0 <= u_k <= 1, so max |delta| <= sum |v|;
    // only when that bound is exceeded does the warp run the exact recurrence
    // (shared memory only) for max |delta|.  A listed group writes nothing.
    if (p.mp_redo && __any_sync(0xffffffffu, vsum > MP_DELTA_MAX)) {
        float dmax = 0.0f;
        for (int q = 0; q < nt; ++q) {
            const float *vq = vv + (size_t)q * NB;
            float delta = 0.0f;
            for (int k = w_hi; k >= w_lo; --k) {
                const size_t s = (size_t)(k - 1) * MP_TR_COLS;
                delta = vq[s] + mul_u(tu[s], delta);
                dmax = fmaxf(dmax, fabsf(delta));
            }
        }
        if (__any_sync(0xffffffffu, dmax > MP_DELTA_MAX)) {
            if (lane == 0) {
                const unsigned base = atomicAdd(p.mp_redo, (unsigned)nt);
                for (int q = 0; q < nt; ++q) p.mp_redo[1 + base + q] = (g << 5) | (unsigned)tix[q];
            }
            return;
        }
    }

    // ---- back-substitution ----
    const unsigned long long pol_once = l2_policy_evict_first();
    bool any_full = false;
#pragma unroll
    for (int q = 0; q < TPW; ++q) {
        const int tr = tix[q];
        if (q < nt && (((nonlocal && c.use_kpp) && (tr == iT || tr == iS || tr == iPS)) ||
                       (c.budgets && (tr == iT || tr == iS))))
            any_full = true;
    }
    if (!any_full) {
        // every tracer of the group is a plain diffusion: one fused downward pass
        float delta[TPW];
#pragma unroll
        for (int q = 0; q < TPW; ++q) delta[q] = 0.0f;
        // old values (and CI: thicknesses) of block k0 - U loaded while block k0 is computed
        auto load_down = [&](int k0, double (&db_)[U][TPW], double (&hb_)[U]) {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int k = k0 - u;
#pragma unroll
                for (int q = 0; q < TPW; ++q)
                    db_[u][q] = (k >= lo && k <= hi && q < nt) ? ld_hint(trc[q] + P * (size_t)(k - 1), pol_once) : 0.0;
                if (CI) hb_[u] = (k >= lo && k <= hi) ? __ldg(hp + P * (size_t)(k - 1)) : 0.0;
            }
        };
        double dk[U][TPW], hk[U];
        load_down(w_hi, dk, hk);
        for (int k0 = w_hi; k0 >= w_lo; k0 -= U) {
            double dx[U][TPW], hx[U];
            load_down(k0 - U, dx, hx);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int k = k0 - u;
                if (k < w_lo) break;
                const size_t s = (size_t)(k - 1) * MP_TR_COLS;
                const float tk = tu[s];
#pragma unroll
                for (int q = 0; q < TPW; ++q) delta[q] = vv[(size_t)q * NB + s] + mul_u(tk, delta[q]);
                if (k < lo || k > hi) continue;
                const size_t off = P * (size_t)(k - 1);
                if (CI) neumaier_add(c_new, e_new, hk[u] * (dk[u][0] + (double)delta[0]));
#pragma unroll
                for (int q = 0; q < TPW; ++q)
                    if (q < nt) trc[q][off] = dk[u][q] + (double)delta[q];
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                hk[u] = hx[u];
#pragma unroll
                for (int q = 0; q < TPW; ++q) dk[u][q] = dx[u][q];
            }
        }
        if (CI && in_grid) {
            p.content_old[col + P * (size_t)tix[0]] = c_old + e_old;
            p.content_new[col + P * (size_t)tix[0]] = c_new + e_new;
        }
        return;
    }
    if constexpr (TPW > 1) {
        // a group with a deposit or a budget: one fused downward pass
        double *bud[TPW], q_kin[TPW];
        bool dep[TPW], any_dep = false;
#pragma unroll
        for (int q = 0; q < TPW; ++q) {
            const int tr = tix[q];
            dep[q] = q < nt && nonlocal && c.use_kpp && (tr == iT || tr == iS || tr == iPS);
            any_dep = any_dep || dep[q];
            bud[q] = nullptr;
            if (q < nt && c.budgets && tr == iT) bud[q] = p.heat_budget + col;
            if (q < nt && c.budgets && tr == iS) bud[q] = p.salt_budget + col;
        }
        bool nl = false;
        double h_b = 0.0, q_T_kin = 0.0, q_S_kin = 0.0;
        if (any_dep && live) nl = nonlocal_column(p, c, col, hp, hi, h_b, q_T_kin, q_S_kin);
#pragma unroll
        for (int q = 0; q < TPW; ++q) q_kin[q] = (tix[q] == iT) ? q_T_kin : q_S_kin;
        tracer_back_group<TPW>(p, dt, trc, nt, hp, tu, vv, NB, w_lo, w_hi, lo, hi, bud, dep, nl, h_b, q_kin,
                               pol_once);
        return;
    } else {
        for (int q = 0; q < nt; ++q) {
            const int tr = tix[q];
            // ---- non-local column scalars (FP64, as KPP pass 2) ----
            const bool nl_t = nonlocal && c.use_kpp && (tr == iT || tr == iS || tr == iPS);
            bool nl = nl_t && live;
            double h_b = 0.0, q_kin = 0.0;
            if (nl) {
                double q_T_kin, q_S_kin;
                nl = nonlocal_column(p, c, col, hp, hi, h_b, q_T_kin, q_S_kin);
                q_kin = (tr == iT) ? q_T_kin : q_S_kin;
            }
            double *bud = nullptr;
            if (c.budgets && tr == iT) bud = p.heat_budget + col;
            if (c.budgets && tr == iS) bud = p.salt_budget + col;
            double *t_ptr = p.tr[tr] + col;
            const float *vq = vv + (size_t)q * NB;
            if (CI) {
                tracer_back<true, true>(p, dt, t_ptr, hp, tu, vq, w_lo, w_hi, lo, hi, bud, nl_t, nl, h_b, q_kin,
                                        pol_once, &c_new, &e_new);
                if (in_grid) {
                    p.content_old[col + P * (size_t)tr] = c_old + e_old;
                    p.content_new[col + P * (size_t)tr] = c_new + e_new;
                }
            } else if (nl_t || bud)
                tracer_back<true>(p, dt, t_ptr, hp, tu, vq, w_lo, w_hi, lo, hi, bud, nl_t, nl, h_b, q_kin, pol_once);
            else
                tracer_back<false>(p, dt, t_ptr, hp, tu, vq, w_lo, w_hi, lo, hi, nullptr, false, false, 0.0, 0.0,
                                   pol_once);
        }
    }
}

// ---------------------------------------------------------------------------
// Tracers with the solver rows in tensor memory.
//
// k_tracers_mp holds the t and v rows of a warp's 32 columns in shared
// memory: 8 B per level and column, 19.2 KB per warp at nz = 75, which caps
// it at ~11 warps per SM, and its per-level chains run at the pace of the
// warps in flight (halving them doubled its time).  The 256 KB of tensor
// memory of an SM are free on this path, so k_tracers_mp_tm keeps one
// persistent CTA per SM whose first warps store their rows in tensor memory
// (tcgen05.st of each level's (t, v) pair into the warp's 32 lanes, read
// back eight levels at a time with tcgen05.ld; up to three warps per lane
// quarter, 2 * nzp columns each); the kernel can give further warps rows in
// shared memory, which the launcher does not use (they squeeze the L1 the
// tracers of a column group share).  The arithmetic is
// k_tracers_mp<false, 1, true>'s, level for level (the default knobs, one
// factorisation, one tracer per warp); work items are (32-column group,
// tracer), tracer fastest, strided over all warps of the grid.
// ---------------------------------------------------------------------------
// rows of one warp in shared memory: level k at tu[(k-1)*32], vv[(k-1)*32]
struct SRows {
    float *tu, *vv;
    int nz;   // rows above nz do not exist (the last block of a column may be partial)
    __device__ __forceinline__ void put(int k, float t, float v)
    {
        tu[(size_t)(k - 1) * MP_TR_COLS] = t;
        vv[(size_t)(k - 1) * MP_TR_COLS] = v;
    }
    __device__ __forceinline__ void done_writing() {}
    // levels 8 kb + 1 .. 8 kb + 8
    __device__ __forceinline__ void load8(int kb, float (&t)[8], float (&v)[8]) const
    {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int k = 8 * kb + q + 1;
            t[q] = (k <= nz) ? tu[(size_t)(k - 1) * MP_TR_COLS] : 0.0f;
            v[q] = (k <= nz) ? vv[(size_t)(k - 1) * MP_TR_COLS] : 0.0f;
        }
    }
};

// rows of one warp in tensor memory: level k's (t, v) at columns
// col0 + 2(k-1), 2(k-1)+1 of the warp's 32 lanes (taddr: lane << 16 | column)
struct TRows {
    uint32_t base;
    __device__ __forceinline__ void put(int k, float t, float v) { tmem_put2(base, k, __float_as_uint(t), __float_as_uint(v)); }
    __device__ __forceinline__ void done_writing() { tmem_store_done(); }
    __device__ __forceinline__ void load8(int kb, float (&t)[8], float (&v)[8]) const
    {
        uint32_t r[16];
        tmem_get16(base, kb, r);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            t[q] = __uint_as_float(r[2 * q]);
            v[q] = __uint_as_float(r[2 * q + 1]);
        }
    }
};

// The back-substitution of one tracer column from the rows (tracer_back's
// arithmetic, its levels taken in aligned blocks of eight so that a row
// block is one tensor-memory load); FULL adds the KPP non-local deposit.
template <bool FULL, class Rows>
__device__ __forceinline__ void tracer_back_rows(const Params &p, double dt, double *__restrict__ trc,
                                                 const double *__restrict__ hp, const Rows &rows, int w_lo, int w_hi,
                                                 int lo, int hi, bool nl, double h_b, double q_kin,
                                                 unsigned long long pol)
{
    const size_t P = p.plane;
    const int nz = p.nz;
    float delta = 0.0f;
    double g_above = 0.0, d_run = 0.0, h_a = 0.0;
    double h_c = (FULL && lo <= hi) ? __ldg(hp + P * (size_t)(hi - 1)) : 0.0;
    const double r_hb = (FULL && nl) ? rcp_nr(h_b) : 0.0;   // sigma = d_run / h_b as a product
    // old values and (deposit) the thicknesses one level down of row block
    // kb - 1, loaded while block kb is computed
    auto load_down = [&](int kb, double (&db_)[8], double (&hb_)[8]) {
#pragma unroll
        for (int q = 7; q >= 0; --q) {
            const int k = 8 * kb + q + 1;
            db_[q] = (k >= lo && k <= hi) ? ld_hint(trc + P * (size_t)(k - 1), pol) : 0.0;
            if (FULL) hb_[q] = (k > 1 && k >= lo && k <= hi) ? __ldg(hp + P * (size_t)(k - 2)) : 0.0;
        }
    };
    double dk[8], hb[8];
    load_down((w_hi - 1) >> 3, dk, hb);
    for (int kb = (w_hi - 1) >> 3; kb >= ((w_lo - 1) >> 3); --kb) {
        float t8[8], v8[8];
        rows.load8(kb, t8, v8);
        double dx[8], hx[8];
        load_down(kb - 1, dx, hx);
#pragma unroll
        for (int q = 7; q >= 0; --q) {
            const int k = 8 * kb + q + 1;
            if (k > w_hi || k < w_lo) continue;
            delta = v8[q] + mul_u(t8[q], delta);   // rows outside the span: v = t = 0
            if (k < lo || k > hi) continue;
            const size_t off = P * (size_t)(k - 1);
            double x = dk[q] + (double)delta;
            if (FULL) {
                const double h_bl = hb[q];
                double gk = 0.0;
                if (nl) {
                    d_run = d_run + h_c;
                    if (k > 1 && d_run < h_b) {
                        const double sigma = d_run * r_hb;
                        gk = p.cfg.cs_nonlocal * (sigma * (1.0 - sigma) * (1.0 - sigma)) * q_kin;
                    }
                }
                double f_up = 0.0, f_dn = 0.0;
                if (k < nz) f_up = nonlocal_face_flux(g_above, h_c, h_a);
                if (k > 1) f_dn = nonlocal_face_flux(gk, h_bl, h_c);
                const double src = dt * (f_up - f_dn);
                if (src != 0.0) x = conc_add_source_mp(x, h_c, src, rcp_nr(h_c + H_DIV_EPS));
                g_above = gk;
                h_a = h_c;
                h_c = h_bl;
            }
            trc[off] = x;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            dk[q] = dx[q];
            if (FULL) hb[q] = hx[q];
        }
    }
}

// One work item (32-column group g, tracer tr) of k_tracers_mp_tm.
template <class Rows>
__device__ __forceinline__ void tracer_item_tm(const Params &p, const vphys_config &c, double dt, int nonlocal,
                                               int ngx, int item, Rows &rows, int lane)
{
    const int ntr = p.ntr, nx = p.nx, nz = p.nz;
    const int tr = item % ntr;
    const unsigned g = (unsigned)(item / ntr);
    const int gi = (int)(g % (unsigned)ngx), j = (int)(g / (unsigned)ngx);
    const int i = gi * MP_TR_COLS + lane;
    const size_t P = p.plane;
    const bool in_grid = i < nx;
    const size_t col = (size_t)(in_grid ? i : 0) + (size_t)nx * j;
    const double *__restrict__ hp = p.h + col;
    const float HV = (float)H_VANISHED;
    constexpr int U = MP_TR_U;

    const int sp = in_grid ? p.span[col] : 0;
    const bool live = (sp & 0xffff) > 0;
    const int lo = live ? (sp & 0xffff) : nz + 1, hi = live ? (sp >> 16) : 0;
    const int w_lo = __reduce_min_sync(0xffffffffu, live ? lo : 0x7fffffff);
    const int w_hi = __reduce_max_sync(0xffffffffu, hi);
    if (w_hi == 0) return;

    const double *__restrict__ Kp = p.kt + col;
    double *trc = p.tr[tr] + col;
    const unsigned long long pol_keep = l2_policy_evict_last();
    const float dtf = (float)dt;
    float vsum = 0.0f;
    {
        const bool first = (w_lo == lo);
        double h_c = first ? __ldg(hp + P * (size_t)(w_lo - 1)) : 0.0;
        double d_c = first ? ld_hint(trc + P * (size_t)(w_lo - 1), pol_keep) : 0.0;
        double d_m = 0.0, w = 0.0;
        float f_dn = 0.0f, q_prev = 1.0f, t_prev = 0.0f;
        // the loads of block k0 + U are issued before block k0 is computed
        auto load_block = [&](int k0, double (&hb_)[U], double (&kb_)[U], double (&db_)[U]) {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int k = k0 + u;
                const bool need = k + 1 >= lo && k + 1 <= hi;
                const size_t o = P * (size_t)k;
                hb_[u] = need ? __ldg(hp + o) : 0.0;
                kb_[u] = need ? __ldg(Kp + o) : 0.0;
                db_[u] = need ? ld_hint(trc + o, pol_keep) : 0.0;
            }
        };
        double hn[U], kn[U], dn[U];
        load_block(w_lo, hn, kn, dn);
        for (int k0 = w_lo; k0 <= w_hi; k0 += U) {
            double hx[U], kx[U], dx[U];
            load_block(k0 + U, hx, kx, dx);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int k = k0 + u;
                if (k > w_hi) break;
                const float H = fmx((float)h_c, HV);
                const float Hp = fmx((float)hn[u], HV);
                const bool coupled = h_c > H_VANISHED && hn[u] > H_VANISHED;
                const float f_up = coupled ? __fdividef(dtf * (float)kn[u], face_thick(H, Hp, c.use_harmonic)) : 0.0f;
                float ip, t, qq;
                pivot_row(H + f_dn * q_prev, f_up, ip, t, qq);
                const double fd = (double)f_dn, fu = (double)f_up, ipd = (double)ip;
                const double b = fd * (d_m - d_c) + fu * (dn[u] - d_c);
                w = b + mul_u(t_prev, w);
                const float vq = (float)(w * ipd);
                rows.put(k, t, vq);
                vsum += fabsf(vq);
                d_m = d_c;
                d_c = dn[u];
                t_prev = t;
                q_prev = qq;
                f_dn = f_up;
                h_c = hn[u];
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                hn[u] = hx[u];
                kn[u] = kx[u];
                dn[u] = dx[u];
            }
        }
    }
    rows.done_writing();

    // a group whose increment reaches MP_DELTA_MAX goes to the FP64 re-solve
    if (p.mp_redo && __any_sync(0xffffffffu, vsum > MP_DELTA_MAX)) {
        float dmax = 0.0f, delta = 0.0f;
        for (int kb = (w_hi - 1) >> 3; kb >= ((w_lo - 1) >> 3); --kb) {
            float t8[8], v8[8];
            rows.load8(kb, t8, v8);
#pragma unroll
            for (int q = 7; q >= 0; --q) {
                const int k = 8 * kb + q + 1;
                if (k > w_hi || k < w_lo) continue;
                delta = v8[q] + mul_u(t8[q], delta);
                dmax = fmaxf(dmax, fabsf(delta));
            }
        }
        if (__any_sync(0xffffffffu, dmax > MP_DELTA_MAX)) {
            if (lane == 0) {
                const unsigned base = atomicAdd(p.mp_redo, 1u);
                p.mp_redo[1 + base] = (g << 5) | (unsigned)tr;
            }
            return;
        }
    }

    const unsigned long long pol_once = l2_policy_evict_first();
    const int iT = c.idx_temperature, iS = c.idx_salinity, iPS = c.idx_pseudo_salt;
    const bool full_t = nonlocal && c.use_kpp && (tr == iT || tr == iS || tr == iPS);
    if (!full_t) {
        tracer_back_rows<false>(p, dt, trc, hp, rows, w_lo, w_hi, lo, hi, false, 0.0, 0.0, pol_once);
        return;
    }
    bool nl = live;
    double h_b = 0.0, q_kin = 0.0;
    if (nl) {
        double q_T_kin, q_S_kin;
        nl = nonlocal_column(p, c, col, hp, hi, h_b, q_T_kin, q_S_kin);
        q_kin = (tr == iT) ? q_T_kin : q_S_kin;
    }
    tracer_back_rows<true>(p, dt, trc, hp, rows, w_lo, w_hi, lo, hi, nl, h_b, q_kin, pol_once);
}

// One CTA per SM: warps [0, nt_warps) keep their rows in tensor memory
// (lane quarter warp % 4, columns (warp / 4) * 2 nzp), the others in
// shared memory.  Warp 0 allocates all 512 columns before the work and frees
// them after it.
template <int MAXW>
__global__ void __launch_bounds__(32 * MAXW, 1)
    k_tracers_mp_tm(const Params p, double dt, int nonlocal, int ngx, int nitems, int nt_warps, int nzp)
{
    extern __shared__ __align__(16) float smf[];
    __shared__ uint32_t tmem_slot;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) tmem_alloc_all(&tmem_slot);
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();
    const uint32_t tbase = tmem_slot;
    vphys_config cd = p.cfg;
    default_tracer_knobs(cd);
    // items are handed out one at a time in order (a warp that drew land
    // columns draws again at once), so neighbouring items -- the tracers of
    // one column group -- run at about the same time and share h and K in L2
    auto next = [&]() {
        unsigned it = 0;
        if (lane == 0) it = atomicAdd(p.work_ctr, 1u);
        return (int)__shfl_sync(0xffffffffu, it, 0);
    };
    if (warp < nt_warps) {
        TRows rows{tmem_warp_slot(tbase, warp, nzp)};
        for (int item = next(); item < nitems; item = next()) tracer_item_tm(p, cd, dt, nonlocal, ngx, item, rows, lane);
    } else {
        const size_t NB = (size_t)p.nz * MP_TR_COLS;
        float *tu = smf + (size_t)(warp - nt_warps) * 2 * NB + lane;
        SRows rows{tu, tu + NB, p.nz};
        for (int item = next(); item < nitems; item = next()) tracer_item_tm(p, cd, dt, nonlocal, ngx, item, rows, lane);
    }
    tmem_fence_before();
    __syncthreads();
    if (warp == 0) {
        tmem_fence_after();
        tmem_free_all(tbase);
    }
}

// The tensor-memory form applies to the default tracer knobs with ks = kt;
// false: the caller runs k_tracers_mp.
static bool launch_tracers_mp_tm(const Params &p, double dt, bool nonlocal, cudaStream_t stream)
{
    if (p.var_tr != VAR_TR_TMEM || !is_default_tracer_knobs(p.cfg) || !p.ks_equals_kt || p.ntr < 1 || !p.span ||
        !p.work_ctr)
        return false;
    const int nzp = (p.nz + 7) & ~7;          // levels rounded to a row block
    const int per_quarter = 512 / (2 * nzp);  // warps sharing one lane quarter
    int nt = 4 * (per_quarter < 3 ? per_quarter : 3);
    const size_t per_s = (size_t)p.nz * MP_TR_COLS * 2 * sizeof(float);
    // Rows in tensor memory only: shared-memory rows squeeze the L1 that the
    // tracers of a column group share for h and K (1440x1080x75, 4 tracers:
    // 12 tensor-memory warps 3.9-4.2 ms; 12 of them + 11 shared-memory warps
    // 6.05 ms; 11 shared-memory warps in the same kernel 4.65 ms).
    const int ns = 0;
    if (nt + ns < 1) return false;
    static bool attr_set = false;
    static int sms = 0;
    if (!attr_set) {
        cudaFuncSetAttribute(k_tracers_mp_tm<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
        attr_set = true;
    }
    const int ngx = (p.nx + MP_TR_COLS - 1) / MP_TR_COLS;
    const long long nitems = (long long)ngx * p.ny * p.ntr;
    if (nitems > 0x7fffffffLL) return false;
    const int nwarps = nt + ns;
    const int grid = (int)(nitems < (long long)sms * nwarps ? (nitems + nwarps - 1) / nwarps : sms);
    // nwarps <= 12: at most three warps per lane quarter, no shared-memory rows
    k_tracers_mp_tm<12><<<grid, 32 * nwarps, (size_t)ns * per_s, stream>>>(p, dt, nonlocal ? 1 : 0, ngx,
                                                                         (int)nitems, nt, nzp);
    if (p.mp_redo) launch_tracers_redo(p, dt, nonlocal, stream);
    return true;
}

// ---------------------------------------------------------------------------
// momentum: one thread per u or v face column
// ---------------------------------------------------------------------------
template <bool XF, bool DEF>
__device__ __forceinline__ void solve_face_mp(const Params &p, double dt, int i, int j, float *st, float *sv,
                                              float *sr, int bs)
{
    vphys_config cd = p.cfg;   // DEF: the default knobs folded in (is_default_face_knobs)
    if (DEF) default_face_knobs(cd);
    const vphys_config &c = cd;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const int nu = XF ? nx + 1 : nx;
    const size_t P = p.plane;
    const size_t PF = XF ? p.plane_u : p.plane_v;
    const size_t f = (size_t)i + (size_t)nu * j;
    double *__restrict__ uf = (XF ? p.u : p.v) + f;
    double *__restrict__ vrem = c.remnant ? ((XF ? p.visc_rem_u : p.visc_rem_v) + f) : nullptr;
    const unsigned long long pol_keep = l2_policy_evict_last();
    int il, ir, jb, ja;
    if (XF) {
        il = i - 1 > 0 ? i - 1 : 0;
        ir = i < nx - 1 ? i : nx - 1;
        jb = j;
        ja = j;
    } else {
        il = i;
        ir = i;
        jb = j - 1 > 0 ? j - 1 : 0;
        ja = j < ny - 1 ? j : ny - 1;
    }
    const size_t cl = (size_t)il + (size_t)nx * jb;
    const size_t cr = (size_t)ir + (size_t)nx * ja;
    if (!c.remnant && !c.implicit_stress && fmn(p.wet[cl], p.wet[cr]) == 0.0) {
        bool zero = true;
        for (int k = 1; k <= nz && zero; ++k) zero = (uf[PF * (size_t)(k - 1)] == 0.0);
        if (zero) return;
    }
    const double *__restrict__ hl = p.h + cl;
    const double *__restrict__ hr = p.h + cr;
    const double *__restrict__ kvl = p.kv + cl;
    const double *__restrict__ kvr = p.kv + cr;
    const int *ktp = XF ? p.k_top_u : p.k_top_v;
    const int *kbp = XF ? p.k_bot_u : p.k_bot_v;
    const int kb = kbp ? min(max(kbp[f], 1), nz) : 1;
    const int ktop = ktp ? min(max(ktp[f], 1), nz) : nz;
    const float bbl_thick = (float)c.hbbl_visc;
    const float kv_bbl = c.bbl_glue ? (float)(c.bbl_piston * c.hbbl_visc) : 0.0f;
    const float i_hbbl = __frcp_rn(bbl_thick + (float)EPS_HVEL);
    const float dtf = (float)dt;
    float zacc = 0.0f, zcol_l = 0.0f, zcol_r = 0.0f;
    if (c.hvel_mom6 && !c.hvel_harmonic) {   // column depths (k_column_depth)
        zcol_l = (float)p.zcol[cl];
        zcol_r = (float)p.zcol[cr];
    }
    const float d_min = fmn(-zcol_l, -zcol_r);
    int kb_live = kb;
    if (c.zlevel_faces) {
        for (int k = kb; k <= nz; ++k) {
            if (fmn(__ldg(hl + P * (size_t)(k - 1)), __ldg(hr + P * (size_t)(k - 1))) > H_VANISHED) {
                kb_live = k;
                break;
            }
        }
    }
    float hv_p, zi_p;
    double u_c = ld_hint(uf, pol_keep), u_m = 0.0;
    face_layer<float>(c, (float)__ldg(hl), (float)__ldg(hr), (float)u_c, 1, kb, d_min, i_hbbl, zacc, zcol_l, zcol_r,
                      hv_p, zi_p);
    float num_t = 0.0f, dz_t = 1.0f;
    bool cut_t = false;
    const float lam = (c.implicit_drag && !c.bbl_glue) ? (float)(XF ? p.lambda_bot_u : p.lambda_bot_v)[f] : 0.0f;
    double stress = 0.0;
    if (c.implicit_stress) {
        const double tau = (XF ? p.tau_x : p.tau_y)[f];
        stress = dt * tau * fmn(p.wet[cl], p.wet[cr]) * (1.0 / c.rho0);
    }
    // carried between rows: the coupling above the previous row, its q and t,
    // and the FP64 forward accumulations of the increment and of the remnant
    float f_prev = 0.0f, q_prev = 1.0f, t_prev = 0.0f;
    double w = 0.0, wr = 0.0;
    // level k + 1's data for row k; the loads of block k0 + MP_MOM_U are
    // issued before block k0 is computed (two register buffers)
    auto load_up = [&](int k0, double (&hl_)[MP_MOM_U], double (&hr_)[MP_MOM_U], double (&u_)[MP_MOM_U],
                       double (&kl_)[MP_MOM_U], double (&kr_)[MP_MOM_U]) {
#pragma unroll
        for (int q = 0; q < MP_MOM_U; ++q) {
            const int k = k0 + q;
            hl_[q] = hr_[q] = kl_[q] = kr_[q] = u_[q] = 0.0;
            if (k < nz) {
                const size_t o = P * (size_t)k;
                hl_[q] = __ldg(hl + o);
                hr_[q] = __ldg(hr + o);
                kl_[q] = __ldg(kvl + o);
                kr_[q] = __ldg(kvr + o);
                u_[q] = ld_hint(uf + PF * (size_t)k, pol_keep);
            }
        }
    };
    double hln[MP_MOM_U], hrn[MP_MOM_U], un[MP_MOM_U], kvln[MP_MOM_U], kvrn[MP_MOM_U];
    load_up(1, hln, hrn, un, kvln, kvrn);
    for (int k0 = 1; k0 <= nz; k0 += MP_MOM_U) {
        double hlx[MP_MOM_U], hrx[MP_MOM_U], ux[MP_MOM_U], kvlx[MP_MOM_U], kvrx[MP_MOM_U];
        load_up(k0 + MP_MOM_U, hlx, hrx, ux, kvlx, kvrx);
#pragma unroll
        for (int q = 0; q < MP_MOM_U; ++q) {
            const int k = k0 + q;
            if (k > nz) break;
            const float hv_0 = hv_p, zi_0 = zi_p;
            const float num_b = num_t, dz_b = dz_t;
            const bool cut_b = cut_t;
            double u_p = 0.0;
            if (k < nz) {
                u_p = un[q];
                face_layer<float>(c, (float)hln[q], (float)hrn[q], (float)u_p, k + 1, kb, d_min, i_hbbl, zacc,
                                  zcol_l, zcol_r, hv_p, zi_p);
                if (k >= kb_live && k <= ktop)
                    interface_coupling<float>(c, hv_0, hv_p, zi_0, dtf, kv_bbl, bbl_thick, (float)kvln[q],
                                              (float)kvrn[q], num_t, dz_t, cut_t);
            }
            // the row in conservative form (row k of the reference times hf_k)
            const float H = fmx(hv_0, (float)H_VANISHED);
            float f_up = 0.0f, f_dn = 0.0f, ex = 0.0f;
            if (k == kb_live && k <= ktop) {
                if (kb_live < nz && !cut_t) f_up = __fdividef(num_t, dz_t);
                if (c.bbl_glue) ex = __fdividef(dtf * kv_bbl, fmn(0.5f * hv_0, bbl_thick) + (float)EPS_HVEL);
                if (c.implicit_drag && !c.bbl_glue) ex = H * (dtf * lam);
            }
            if (k == ktop && k > kb_live && !cut_b) f_dn = __fdividef(num_b, dz_b);
            if (k > kb_live && k < ktop) {
                if (!cut_b) f_dn = __fdividef(num_b, dz_b);
                if (!cut_t) f_up = __fdividef(num_t, dz_t);
            }
            // FP64 residual of the old velocity (+ the wind stress of the top row)
            double b = (double)f_dn * (u_m - u_c) + (double)f_up * (u_p - u_c) - (double)ex * u_c;
            if (k == ktop && c.implicit_stress) b = b + (double)H * (stress / fmx((double)H, STRESS_H_MIN));
            // the row below couples into this one only through a shared interface
            const float t_in = (f_dn != 0.0f) ? t_prev : 0.0f;
            const float sx = H + ex + f_dn * q_prev;
            float ip, t, qq;
            pivot_row(sx, f_up, ip, t, qq);
            w = b + mul_u(t_in, w);
            const size_t s = (size_t)(k - 1) * bs;
            sv[s] = (float)(w * (double)ip);
            st[s] = t;
            if (vrem) {
                wr = (double)H + mul_u(t_in, wr);
                sr[s] = (float)(wr * (double)ip);
            }
            f_prev = f_up;
            q_prev = qq;
            t_prev = t;
            u_m = u_c;
            u_c = u_p;
        }
#pragma unroll
        for (int q = 0; q < MP_MOM_U; ++q) {
            hln[q] = hlx[q];
            hrn[q] = hrx[q];
            un[q] = ux[q];
            kvln[q] = kvlx[q];
            kvrn[q] = kvrx[q];
        }
    }
    (void)f_prev;
    // back-substitution: increment (+ the remnant, RHS 1, clipped at 1 as it goes)
    float delta = 0.0f, gam = 0.0f;
    auto load_down = [&](int k0, double (&u_)[MP_MOM_U]) {
#pragma unroll
        for (int q = 0; q < MP_MOM_U; ++q) {
            const int k = k0 - q;
            u_[q] = (k >= 1) ? ld_hint(uf + PF * (size_t)(k - 1), pol_keep) : 0.0;
        }
    };
    double uo[MP_MOM_U];
    load_down(nz, uo);
    for (int k0 = nz; k0 >= 1; k0 -= MP_MOM_U) {
        double uox[MP_MOM_U];
        load_down(k0 - MP_MOM_U, uox);
#pragma unroll
        for (int q = 0; q < MP_MOM_U; ++q) {
            const int k = k0 - q;
            if (k < 1) break;
            const size_t s = (size_t)(k - 1) * bs;
            const float tk = st[s];
            delta = sv[s] + mul_u(tk, delta);
            const size_t o = PF * (size_t)(k - 1);
            uf[o] = uo[q] + (double)delta;
            if (vrem) {
                gam = fminf(sr[s] + mul_u(tk, gam), 1.0f);
                vrem[o] = (double)gam;
            }
        }
#pragma unroll
        for (int q = 0; q < MP_MOM_U; ++q) uo[q] = uox[q];
    }
}

template <bool DEF>
__global__ void __launch_bounds__(MP_MOM_THREADS) k_momentum_mp(const Params p, double dt)
{
    extern __shared__ float smf[];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    const size_t NB = (size_t)p.nz * blockDim.x;
    float *st = smf + threadIdx.x, *sv = st + NB, *sr = sv + NB;
    if (blockIdx.z == 0) {
        if (i <= p.nx && j < p.ny) solve_face_mp<true, DEF>(p, dt, i, j, st, sv, sr, blockDim.x);
    } else {
        if (i < p.nx && j <= p.ny) solve_face_mp<false, DEF>(p, dt, i, j, st, sv, sr, blockDim.x);
    }
}

// One face of the mixed-precision solve at the default momentum knobs,
// driven by the TMA-staged ring (momentum_ring_cta): the arithmetic of
// solve_face_mp<., true> above, its t and v rows in the ring kernel's
// shared-memory row area, the old velocity read again from L2 by the
// back-substitution.
struct MixedFace {
    vphys_config c;
    double *uf;
    size_t PF;
    float *st, *sv;
    int tid, nz;
    bool valid;
    unsigned long long pol_keep;
    float dtf, bbl_thick, i_hbbl, zacc, zcol_l, zcol_r, d_min;
    float hv_p, zi_p, num_t, dz_t, q_prev, t_prev;
    double w, u_c, u_m;

    __device__ __forceinline__ void start(const Params &p, double dt, const FaceCells &fc, bool valid_, double *uf_,
                                          size_t PF_, unsigned char *rows, int tid_)
    {
        c = p.cfg;
        default_face_knobs(c);
        uf = uf_;
        PF = PF_;
        nz = p.nz;
        st = reinterpret_cast<float *>(rows);
        sv = st + (size_t)nz * MT_TW;
        tid = tid_;
        valid = valid_;
        pol_keep = l2_policy_evict_last();
        dtf = (float)dt;
        bbl_thick = (float)c.hbbl_visc;
        i_hbbl = __frcp_rn(bbl_thick + (float)EPS_HVEL);
        zacc = 0.0f;
        zcol_l = (float)p.zcol[fc.cl];
        zcol_r = (float)p.zcol[fc.cr];
        d_min = fmn(-zcol_l, -zcol_r);
        num_t = 0.0f;
        dz_t = 1.0f;
        q_prev = 1.0f;
        t_prev = 0.0f;
        w = 0.0;
        u_m = 0.0;
    }
    __device__ __forceinline__ void first(double hl, double hr, double uw)
    {
        u_c = uw;
        face_layer<float>(c, (float)hl, (float)hr, (float)u_c, 1, 1, d_min, i_hbbl, zacc, zcol_l, zcol_r, hv_p, zi_p);
    }
    template <bool NEXT>
    __device__ __forceinline__ void step(int k, double hl, double hr, double kvl, double kvr, double u_next)
    {
        const float hv_0 = hv_p, zi_0 = zi_p;
        const float num_b = num_t, dz_b = dz_t;
        double u_p = 0.0;
        if (NEXT) {
            u_p = u_next;
            face_layer<float>(c, (float)hl, (float)hr, (float)u_p, k + 1, 1, d_min, i_hbbl, zacc, zcol_l, zcol_r, hv_p,
                              zi_p);
            bool cut;
            interface_coupling<float>(c, hv_0, hv_p, zi_0, dtf, 0.0f, bbl_thick, (float)kvl, (float)kvr, num_t, dz_t,
                                      cut);
        }
        const float H = fmx(hv_0, (float)H_VANISHED);
        float f_up = 0.0f, f_dn = 0.0f;
        const float ex = 0.0f;
        if (k == 1 && 1 < nz) f_up = __fdividef(num_t, dz_t);
        if (k == nz && k > 1) f_dn = __fdividef(num_b, dz_b);
        if (k > 1 && k < nz) {
            f_dn = __fdividef(num_b, dz_b);
            f_up = __fdividef(num_t, dz_t);
        }
        const double b = (double)f_dn * (u_m - u_c) + (double)f_up * (u_p - u_c) - (double)ex * u_c;
        const float t_in = (f_dn != 0.0f) ? t_prev : 0.0f;
        const float sx = H + ex + f_dn * q_prev;
        float ip, t, qq;
        pivot_row(sx, f_up, ip, t, qq);
        w = b + mul_u(t_in, w);
        const size_t s = (size_t)(k - 1) * MT_TW + tid;
        sv[s] = (float)(w * (double)ip);
        st[s] = t;
        q_prev = qq;
        t_prev = t;
        u_m = u_c;
        u_c = u_p;
    }
    __device__ __forceinline__ void row(int m, double hl, double hr, double kvl, double kvr, double uw)
    {
        step<true>(m, hl, hr, kvl, kvr, uw);
    }
    __device__ __forceinline__ void last() { step<false>(nz, 0.0, 0.0, 0.0, 0.0, 0.0); }
    __device__ __forceinline__ void back()
    {
        float delta = 0.0f;
        for (int k0 = nz; k0 >= 1; k0 -= MP_MOM_UB) {
            double uo[MP_MOM_UB];
#pragma unroll
            for (int q = 0; q < MP_MOM_UB; ++q) {
                const int k = k0 - q;
                uo[q] = (k >= 1 && valid) ? ld_hint(uf + PF * (size_t)(k - 1), pol_keep) : 0.0;
            }
#pragma unroll
            for (int q = 0; q < MP_MOM_UB; ++q) {
                const int k = k0 - q;
                if (k < 1) break;
                const size_t s = (size_t)(k - 1) * MT_TW + tid;
                delta = sv[s] + mul_u(st[s], delta);
                if (valid) uf[PF * (size_t)(k - 1)] = uo[q] + (double)delta;
            }
        }
    }
};

__global__ void __launch_bounds__(MT_THREADS, 2)
    k_momentum_mp_tma(const __grid_constant__ MomMaps maps, const Params p, double dt, int ntiles)
{
    extern __shared__ __align__(128) unsigned char mt_smem[];
    momentum_ring_cta<MixedFace>(maps, p, dt, ntiles, mt_smem);
}

bool launch_momentum_mp_tma(const Params &p, double dt, cudaStream_t stream)
{
    MomMaps maps;
    int ntiles = 0;
    if (!momentum_ring_prepare(p, &maps, &ntiles, stream)) return false;
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_momentum_mp_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr_set = true;
    }
    const size_t smem = mt_smem_bytes(p.nz);
    const int grid = momentum_ring_grid((const void *)k_momentum_mp_tma, ntiles, smem);
    k_momentum_mp_tma<<<grid, MT_THREADS, smem, stream>>>(maps, p, dt, ntiles);
    return true;
}

template <bool TWO, int TPW>
static void launch_tracers_mp_t(const Params &p, double dt, bool nonlocal, cudaStream_t stream)
{
    const size_t smem = (size_t)p.nz * MP_TR_COLS * (1 + TPW) * sizeof(float);
    static bool attr_set = false;
    if (!attr_set) {
        const int mx = (int)((size_t)VPHYS_NZ_MAX * MP_TR_COLS * (1 + TPW) * sizeof(float));
        cudaFuncSetAttribute(k_tracers_mp<TWO, TPW, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        cudaFuncSetAttribute(k_tracers_mp<TWO, TPW, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        if (TPW == 1)
            cudaFuncSetAttribute(k_tracers_mp<TWO, 1, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        attr_set = true;
    }
    // one tracer per warp: every tracer its own group.  TPW per warp: the
    // tracers with the salt deposit (salinity, pseudo-salt: the same flux)
    // first, then the heat deposit, then the rest, TPW per group, so that a
    // group's deposits share their column scalars and profile
    const vphys_config &c = p.cfg;
    TracerGroups tg{};
    int n = 0;
    if (TPW == 1) {
        for (int t = 0; t < p.ntr; ++t) tg.perm[n++] = (signed char)t;
        tg.single = n;
        tg.ngroups = n;
    } else {
        const bool dep = nonlocal && c.use_kpp;
        for (int cls = 0; cls < 3; ++cls)
            for (int t = 0; t < p.ntr; ++t) {
                const int k = (dep && (t == c.idx_salinity || t == c.idx_pseudo_salt)) ? 0
                              : (dep && t == c.idx_temperature)                         ? 1
                                                                                        : 2;
                if (k == cls) tg.perm[n++] = (signed char)t;
            }
        tg.single = 0;
        tg.ngroups = (p.ntr + TPW - 1) / TPW;
    }
    const int ngx = (p.nx + MP_TR_COLS - 1) / MP_TR_COLS;
    const unsigned blocks = (unsigned)ngx * (unsigned)p.ny * (unsigned)tg.ngroups;
    if (is_default_tracer_knobs(p.cfg))
        k_tracers_mp<TWO, TPW, true><<<blocks, MP_TR_COLS, smem, stream>>>(p, dt, nonlocal ? 1 : 0, ngx, tg);
    else if (TPW == 1 && p.content_old)
        k_tracers_mp<TWO, 1, false, true><<<blocks, MP_TR_COLS, smem, stream>>>(p, dt, nonlocal ? 1 : 0, ngx, tg);
    else
        k_tracers_mp<TWO, TPW, false><<<blocks, MP_TR_COLS, smem, stream>>>(p, dt, nonlocal ? 1 : 0, ngx, tg);
    if (p.mp_redo) launch_tracers_redo(p, dt, nonlocal, stream);
}

void launch_tracers_mp(const Params &p, double dt, bool nonlocal, cudaStream_t stream)
{
    k_spans<<<dim3((p.nx + 127) / 128, p.ny), 128, 0, stream>>>(p);
    if (launch_tracers_mp_tm(p, dt, nonlocal, stream)) return;
    if (!p.ks_equals_kt) {
        launch_tracers_mp_t<true, 1>(p, dt, nonlocal, stream);
        return;
    }
    // tracers per warp (the variant vphys_autotune chose; a separate ks or
    // the column-content diagnostic keeps one per warp): sharing a warp saves
    // the repeated factorisation, at the price of a larger register and
    // shared-memory footprint per warp
    switch (p.content_old ? VAR_TR_SMEM1 : p.var_tr) {
    case VAR_TR_SMEM4: launch_tracers_mp_t<false, 4>(p, dt, nonlocal, stream); break;
    case VAR_TR_SMEM2: launch_tracers_mp_t<false, 2>(p, dt, nonlocal, stream); break;
    default: launch_tracers_mp_t<false, 1>(p, dt, nonlocal, stream); break;
    }
}

void launch_momentum_mp(const Params &p, double dt, cudaStream_t stream)
{
    if (p.var_mom == VAR_MOM_RING && launch_momentum_mp_tma(p, dt, stream)) return;
    const int bs = MP_MOM_THREADS;
    static bool attr_set = false;
    if (!attr_set) {
        const int mx = (int)((size_t)VPHYS_NZ_MAX * bs * sizeof(float) * 3);
        cudaFuncSetAttribute(k_momentum_mp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        cudaFuncSetAttribute(k_momentum_mp<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        attr_set = true;
    }
    const size_t smem = (size_t)p.nz * bs * sizeof(float) * (p.cfg.remnant ? 3 : 2);
    dim3 grid((p.nx + 1 + bs - 1) / bs, p.ny + 1, 2);
    if (is_default_face_knobs(p.cfg))
        k_momentum_mp<true><<<grid, bs, smem, stream>>>(p, dt);
    else
        k_momentum_mp<false><<<grid, bs, smem, stream>>>(p, dt);
}

}  // namespace vphys
