// vphys_kernels.cu -- the sm_100a kernels of the vertical-physics hot path.
//
// Data stay in the reference layout: level-major planes (i fastest), k = 1
// the bed.  One thread owns one cell column (or one u/v face column), so
// every per-level load and store of a warp touches 32 consecutive doubles of
// one plane (256 B, fully coalesced), and the serial k-recurrences (KPP walk,
// Thomas sweeps) run in registers with the per-column Thomas state in
// thread-private local memory (L1-resident, coalesced by construction).
//
// Kernels (one launch each, all asynchronous):
//   k_eos_wright   rho from (T, S)                     rdb_eos.F90:909-959
//   k_surface_flux surface heat/salt deposit           rdb_ocean_surface_flux.F90:959-1230
//   k_sw_penetration shortwave moved down the column   rdb_ocean_surface_flux.F90:1255-1530
//   k_stress_mag   |tau| at cell centres               rdb_ocean_surface_stress.F90:858-875
//   k_assemble     PP81 / seed, KPP passes 1 + 2, KV_ML_INVZ2, convection,
//                  split, guard, Bryan-Lewis or scalar gate: every interface
//                  of a column in one top-down register sweep
//                                                     rdb_ocean_vmix.F90:1007-1516, 1716-2434, 2677-2769
//   k_smooth_*     optional 1-2-1 horizontal smoothing  rdb_ocean_vmix.F90:2699-2748
//   k_momentum     u and v face columns: face thickness, coupling, fused
//                  Thomas sweep, optional remnant      rdb_ocean_vdiff.F90:1416-2115
//   (the tracer kernel lives in vphys_tracers.cu)
#include <cuda_runtime.h>

#include <cstdlib>

#include "vphys_device.cuh"
#include "vphys_faces.cuh"
#include "vphys_kernels.cuh"

namespace vphys {

// ---------------------------------------------------------------------------
// Wright EOS
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_eos_wright(const Params p)
{
    const size_t n = p.plane * (size_t)p.nz;
    const double *__restrict__ S = p.tr[p.cfg.idx_salinity];
    const double *__restrict__ T = p.tr[p.cfg.idx_temperature];
    const double p_ref = p.cfg.eos_p_ref, rho0 = p.cfg.rho0;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
        double hk = __ldg(p.h + idx);
        double r;
        if (hk > H_VANISHED) {
            double S_k = __ldg(S + idx), T_k = __ldg(T + idx);
            double T_sq = T_k * T_k;
            double T_cu = T_sq * T_k;
            double alpha_0 = WRIGHT_A0 + WRIGHT_A1 * T_k + WRIGHT_A2 * S_k;
            double p_0 = WRIGHT_B0 + WRIGHT_B1 * T_k + WRIGHT_B2 * T_sq + WRIGHT_B3 * T_cu + WRIGHT_B4 * S_k +
                         WRIGHT_B5 * S_k * T_k;
            double lambda = WRIGHT_C0 + WRIGHT_C1 * T_k + WRIGHT_C2 * T_sq + WRIGHT_C3 * T_cu + WRIGHT_C4 * S_k +
                            WRIGHT_C5 * S_k * T_k;
            double p_plus_p0 = p_ref + p_0;
            double denom = lambda + alpha_0 * p_plus_p0;
            r = p_plus_p0 / denom;
        } else {
            r = rho0;
        }
        p.rho[idx] = r;
    }
}

// ---------------------------------------------------------------------------
// Surface heat / salt deposit (ocean_surface_flux_apply_tracers,
// rdb_ocean_surface_flux.F90:959-1070 with apply_surface_src_2d_impl
// 1093-1142 and its nobudget twin for pseudo-salt 1175-1203): the content
// inv * Q(i,j) * wet(i,j) enters the first live layer from the top through
// rdb_conc_add_source; the budget books rdb_conc_accepted_source.  One thread
// per column; the walk reads one plane per vanished top layer.
// ---------------------------------------------------------------------------
__global__ void k_surface_flux(const Params p, double inv_heat, double inv_salt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= p.nx) return;
    const size_t col = (size_t)i + (size_t)p.nx * j;
    const size_t P = p.plane;
    int kt = p.nz;
    for (int k = p.nz; k >= 1; --k) {
        if (__ldg(p.h + col + P * (size_t)(k - 1)) > H_VANISHED) {
            kt = k;
            break;
        }
    }
    const size_t idx = col + P * (size_t)(kt - 1);
    const double hk = __ldg(p.h + idx);
    const double w = __ldg(p.wet + col);
    const int iT = p.cfg.idx_temperature, iS = p.cfg.idx_salinity, iPS = p.cfg.idx_pseudo_salt;
    const bool book = p.cfg.budgets && hk > H_VANISHED;
    const double *wd = p.wet_dyn;   // the dynamic mask composes after the static one
    if (iT >= 0) {
        double cell = inv_heat * __ldg(p.q_heat + col) * w;
        if (wd) cell = cell * __ldg(wd + col);
        p.tr[iT][idx] = conc_add_source(p.tr[iT][idx], hk, cell);
        if (p.cfg.budgets) p.heat_budget_surface[idx] += book ? cell : 0.0;
    }
    if (iS >= 0 || iPS >= 0) {
        double cell = inv_salt * __ldg(p.q_salt + col) * w;
        if (wd) cell = cell * __ldg(wd + col);
        if (iS >= 0) {
            p.tr[iS][idx] = conc_add_source(p.tr[iS][idx], hk, cell);
            if (p.cfg.budgets) p.salt_budget_surface[idx] += book ? cell : 0.0;
        }
        if (iPS >= 0) p.tr[iPS][idx] = conc_add_source(p.tr[iPS][idx], hk, cell);
    }
    // BOUND_SALINITY after the salt deposit (bound_salinity_top_impl,
    // rdb_ocean_surface_flux.F90:1072-1091): static wet mask, not booked
    if (p.cfg.bound_salinity && iS >= 0 && w > 0.5 && hk > H_DIV_EPS)
        p.tr[iS][idx] = fmx(p.tr[iS][idx], p.cfg.min_salinity);
}

// ---------------------------------------------------------------------------
// Shortwave penetration (ocean_surface_flux_apply_sw_penetration ->
// apply_sw_penetration_impl, rdb_ocean_surface_flux.F90:1255-1370,
// 1451-1530, with k_top = nz and k_bot = 1): the penetrating part
// I0 = sw_pen_frac Q_heat wet (SW_NET for Q_heat under sw_source = 1) of the surface lump leaves the first live layer
// and each live layer takes I0 (T(d_top) - T(d_bottom)), the deepest live
// layer the rest (opaque bed); vanished layers pass the light on.  One thread
// per column.
// ---------------------------------------------------------------------------
__global__ void k_sw_penetration(const Params p, double inv_scale)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= p.nx) return;
    const vphys_config &c = p.cfg;
    const int nz = p.nz;
    const size_t col = (size_t)i + (size_t)p.nx * j;
    const size_t P = p.plane;
    const double *__restrict__ hp = p.h + col;
    double *__restrict__ T = p.tr[c.idx_temperature] + col;
    int kt = nz;
    for (int k = nz; k >= 1; --k)
        if (__ldg(hp + P * (size_t)(k - 1)) > H_VANISHED) {
            kt = k;
            break;
        }
    int k_dep = 1;
    for (int k = 1; k <= nz; ++k)
        if (__ldg(hp + P * (size_t)(k - 1)) > H_VANISHED) {
            k_dep = k;
            break;
        }
    // the chlorophyll scheme absorbs all of the source (apply_sw_penetration_nb_impl, :1606-1668)
    const bool nbs = c.sw_chl != 0;
    const double *kap = p.sw_kappa;   // base pointer: null unless sw_chl
    double i0col = nbs ? __ldg(p.sw_src + col) * __ldg(p.wet + col)
                       : c.sw_pen_frac * __ldg(p.sw_src + col) * __ldg(p.wet + col);
    if (p.cover_frac) i0col = i0col * (1.0 - __ldg(p.cover_frac + col));   // no light under an ice shelf
    double d_top = 0.0;
    double trans_top = nbs ? sw_transmission_nb(d_top, kap, col, P, c.sw_nbands, c.sw_blue_frac) : sw_transmission(c, d_top);
    for (int k = nz; k >= k_dep; --k) {
        const size_t off = P * (size_t)(k - 1);
        const double hk = __ldg(hp + off);
        const double d_bot = d_top + hk;
        const double trans_bot = (k > k_dep) ? (nbs ? sw_transmission_nb(d_bot, kap, col, P, c.sw_nbands, c.sw_blue_frac)
                                                    : sw_transmission(c, d_bot))
                                             : 0.0;
        if (hk > H_VANISHED) {
            const double absorbed = i0col * (trans_top - trans_bot);
            double add = inv_scale * absorbed;
            if (k == kt) add = add - inv_scale * i0col;
            T[off] = conc_add_source(T[off], hk, add);
            if (c.budgets) p.heat_budget_surface[col + off] += add;
            trans_top = trans_bot;
        }
        d_top = d_bot;
    }
}

// The chlorophyll scheme's band opacities (sw_kappa_band_impl,
// rdb_ocean_sw_chl.F90:176-190, with sw_opacity_manizza,
// rdb_ocean_surface_flux.F90:784-793): a + b max(chl, 1e-4)^p on wet
// columns through the safe pow, the land value elsewhere.  One thread per
// column, every band.
__global__ void k_sw_chl_kappa(const Params p, const double *__restrict__ chl, double *__restrict__ kappa)
{
    const size_t col = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (col >= p.plane) return;
    const vphys_config &c = p.cfg;
    const bool wet = __ldg(p.wet + col) > 0.5;
    const double x = fmx(__ldg(chl + col), 1.0e-4);
    for (int n = 0; n < c.sw_nbands; ++n)
        kappa[col + (size_t)n * p.plane] =
            wet ? c.sw_opacity_coef[2 * n] + c.sw_opacity_coef[2 * n + 1] * sm_pow(x, c.sw_chl_power[n])
                : c.sw_opacity_land;
}

void launch_sw_chl_kappa(const Params &p, const double *chl, cudaStream_t stream)
{
    const unsigned blocks = (unsigned)((p.plane + 255) / 256);
    k_sw_chl_kappa<<<blocks, 256, 0, stream>>>(p, chl, (double *)p.sw_kappa);
}

__global__ void k_stress_mag(const Params p, double *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= p.nx) return;
    const int nx = p.nx;
    double tx = 0.5 * (p.tau_x[i + (size_t)(nx + 1) * j] + p.tau_x[i + 1 + (size_t)(nx + 1) * j]);
    double ty = 0.5 * (p.tau_y[i + (size_t)nx * j] + p.tau_y[i + (size_t)nx * (j + 1)]);
    out[i + (size_t)nx * j] = sqrt(tx * tx + ty * ty);
}

// ---------------------------------------------------------------------------
// Coefficient assembly: one thread per cell column.
// ---------------------------------------------------------------------------
constexpr int ASM_THREADS = 128;
// Layers per load block of the FP32 interface sweep (1440x1080x75: 1.97 ms
// loading each layer when its interface needs it, 1.60 ms with 2, 1.50 ms
// with 3 once the default-knob instantiation freed registers).  The FP64 sweep
// keeps the on-demand loads: its exact divisions already cover the load
// latency, and blocks measured slower there (default-knob instantiation:
// 2.14 ms on demand, 2.46 with 2, 2.43 with 3; VPHYS_ASM_U_D sets it).
#ifndef VPHYS_ASM_U_F
#define VPHYS_ASM_U_F 3
#endif

// The assembly knobs of the default (benchmark) configuration: PP81, KPP
// with constant buoyancy coefficients and no shortwave, Bryan-Lewis, no
// KV_ML_INVZ2, convection or guard.
// 1: the benchmark's knobs (PP81 + KPP + Bryan-Lewis, no other contributor,
// guard or shortwave); 2: the same without KPP (the reference time of the
// KPP stage); 0: anything else
__host__ __device__ __forceinline__ int default_assembly_kind(const vphys_config &c)
{
    const bool rest = c.interior_closure == VPHYS_INTERIOR_PP81 && c.bkgnd_profile && !(c.kv_ml_invz2 > 0.0) &&
                      !c.conv_enable && !c.vmix_guard && !c.buoyancy_coeffs && c.sw_pen_frac == 0.0 &&
                      !c.kappa_shear && !c.epbl;
    return rest ? (c.use_kpp ? 1 : 2) : 0;
}
__host__ __device__ __forceinline__ bool is_default_assembly_knobs(const vphys_config &c)
{
    return default_assembly_kind(c) == 1;
}
__device__ __forceinline__ void default_assembly_knobs(vphys_config &c, int kind)
{
    c.kappa_shear = 0;
    c.epbl = 0;
    c.interior_closure = VPHYS_INTERIOR_PP81;
    c.use_kpp = (kind == 1) ? 1 : 0;
    c.bkgnd_profile = 1;
    c.kv_ml_invz2 = 0.0;
    c.conv_enable = 0;
    c.vmix_guard = 0;
    c.buoyancy_coeffs = 0;
    c.sw_pen_frac = 0.0;
}

template <typename R, int DEF>
__global__ void __launch_bounds__(ASM_THREADS) k_assemble(const Params p)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= p.nx) return;
    // DEF: the default assembly knobs (is_default_assembly_knobs) as
    // compile-time constants, so the other options' branches fold out
    vphys_config cd = p.cfg;
    if (DEF) default_assembly_knobs(cd, DEF);
    const vphys_config &c = cd;
    const int nx = p.nx, nz = p.nz;
    const size_t P = p.plane, PU = p.plane_u, PV = p.plane_v;
    const size_t col = (size_t)i + (size_t)nx * j;
    const double *__restrict__ hp = p.h + col;
    const double *__restrict__ rp = p.rho + col;
    const double *__restrict__ up = p.u + (size_t)i + (size_t)(nx + 1) * j;
    const double *__restrict__ vp = p.v + (size_t)i + (size_t)nx * j;
    double *__restrict__ kvp = p.kv + col;
    double *__restrict__ ktp = p.kt + col;
    double *__restrict__ ksp = p.ks + col;
#define HH(k) __ldg(hp + P * (size_t)((k) - 1))
#define RR(k) __ldg(rp + P * (size_t)((k) - 1))
#define UC(k) (0.5 * (__ldg(up + PU * (size_t)((k) - 1)) + __ldg(up + PU * (size_t)((k) - 1) + 1)))
#define VC(k) (0.5 * (__ldg(vp + PV * (size_t)((k) - 1)) + __ldg(vp + PV * (size_t)((k) - 1) + nx)))

    const double rho0 = c.rho0;

    // first live layer from the top (rdb_vl_first_live); a column whose every
    // layer is exactly 0 m thick (land) is noted: its pass-1 walk finds no
    // crossing whatever rho holds (every delta_d is 0), so h_b = sum(h) = 0
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

    // lagged KPP BL depth (state); under EPBL its MLD, the depth convection
    // masks with (rdb_ocean_dyn.F90:1606-1610)
    double h_b = c.epbl ? p.mld_epbl[col] : p.bl_depth[col];
    double q_T_kin = 0.0, q_S_kin = 0.0, w_s = 0.0;
    bool destabilizing = false, kpp_active = false;
    if (c.use_kpp && !c.epbl) {   // EPBL replaces KPP (rdb_ocean_dyn.F90:1539)
        // ---- KPP pass 1 (rdb_ocean_vmix.F90:1288-1426) ----
        const double tau_mag = p.stress_mag[col];
        const double u_star = sqrt(xdiv(tau_mag, rho0));
        // pass 1 charges the shortwave that passes the lagged boundary layer
        q_T_kin = kpp_q_t_kin(c, p.q_heat[col], p.sw_src + col, p.sw_kappa, col, p.plane, h_b, HH(k_sfc));
        q_S_kin = xdiv(p.q_salt[col], rho0);
        double T_sfc = 0.0, S_sfc = 0.0;
        if (c.buoyancy_coeffs) {   // "eos": the surface layer's (T, S) (rdb_ocean_vmix.F90:1357-1376)
            T_sfc = p.tr[c.idx_temperature][col + P * (size_t)(k_sfc - 1)];
            S_sfc = p.tr[c.idx_salinity][col + P * (size_t)(k_sfc - 1)];
        }
        double B_0 = kpp_surface_b0(c, q_T_kin, q_S_kin, HH(k_sfc), T_sfc, S_sfc);
        {
            const double wstar3_lagged = fmx(0.0, -B_0) * h_b;
            const double cb = sm_cbrt(wstar3_lagged);
            const double w_s_col = sqrt(u_star * u_star + cb * cb);
            double hb_new = 0.0;   // all-zero column: no crossing, sum of zeros
            // learned KPP: the surrogate's h_b replaces the walk unless the
            // column is gated, sampled for the check, or in a fallback step
            const float pred = p.kpp_pred ? p.kpp_pred[col] : -1.0f;
            if (pred >= 0.0f) {
                hb_new = (double)pred;
            } else if (!all_zero) {
                const double u_ref = UC(k_sfc);
                const double v_ref = VC(k_sfc);
                const double b_ref = -(GRAVITY * RR(k_sfc) / rho0);
                const double h_sfc = HH(k_sfc);
                const double d_centre_ref = 0.5 * h_sfc;
                const double vt2_coef = c.c_vt2 / c.ri_crit;
                double ri_prev = 0.0, d_prev = d_centre_ref, d_centre_k = d_centre_ref;
                double h_above = h_sfc;
                bool crossing_found = false;
                for (int k = k_sfc - 1; k >= 1; --k) {
                    const double h_k = HH(k);
                    d_centre_k = d_centre_k + 0.5 * (h_above + h_k);
                    const double u_k = UC(k);
                    const double v_k = VC(k);
                    const double b_k = -(GRAVITY * RR(k) / rho0);
                    const double delta_d = d_centre_k - d_centre_ref;
                    const double delta_b = b_ref - b_k;
                    const double n_brunt = sqrt(fmx(0.0, xdiv(delta_b, delta_d)));
                    const double vt2 = vt2_coef * d_centre_k * n_brunt * w_s_col;
                    const double shear2 =
                        fmx((u_k - u_ref) * (u_k - u_ref) + (v_k - v_ref) * (v_k - v_ref) + vt2, c.shear2_floor);
                    const double ri_bulk = xdiv(delta_b * delta_d, shear2);
                    if (ri_bulk >= c.ri_crit) {
                        const double denom = ri_bulk - ri_prev;
                        double frac;
                        if (fabs(denom) > 1.0e-12)
                            frac = xdiv(c.ri_crit - ri_prev, denom);
                        else
                            frac = 0.5;
                        hb_new = d_prev + frac * (d_centre_k - d_prev);
                        crossing_found = true;
                        break;
                    }
                    ri_prev = ri_bulk;
                    d_prev = d_centre_k;
                    h_above = h_k;
                }
                if (!crossing_found) {
                    hb_new = 0.0;
                    for (int k = 1; k <= k_sfc; ++k) hb_new = hb_new + HH(k);
                }
                if (p.kpp_check) {
                    const float ck = p.kpp_check[col];
                    if (ck >= 0.0f) {   // sampled column: the network's h_b against pass 1
                        const double rel = fabs((double)ck - hb_new) / fmx(hb_new, 1.0);
                        atomicAdd(p.kpp_stats + 0, 1ull);
                        if (rel > (double)p.kpp_tol) atomicAdd(p.kpp_stats + 1, 1ull);
                        atomicAdd(p.kpp_stats + 8, (unsigned long long)(fmn(rel * rel, 1.0e6) * 1.0e6));
                    }
                }
            }
            h_b = hb_new;
            p.bl_depth[col] = h_b;
        }
        // ---- KPP pass 2 scalars (rdb_ocean_vmix.F90:1429-1491) ----
        if (c.sw_pen_frac != 0.0) {   // pass 2 charges what passes the new boundary layer
            q_T_kin = kpp_q_t_kin(c, p.q_heat[col], p.sw_src + col, p.sw_kappa, col, p.plane, h_b, HH(k_sfc));
            B_0 = kpp_surface_b0(c, q_T_kin, q_S_kin, HH(k_sfc), T_sfc, S_sfc);
        }
        p.b0[col] = B_0;
        destabilizing = B_0 < 0.0;
        const double wstar3 = fmx(0.0, -B_0) * h_b;
        const double w_star = sm_cbrt(wstar3);
        w_s = sqrt(u_star * u_star + w_star * w_star);
        kpp_active = (h_b > 0.0 && w_s > 0.0);
    }

    // ---- the interface sweep, in R (double: the exact path; float: the
    //      mixed-precision path, whose KPP pass 1 above stays FP64) ----
    const R r0 = (R)rho0, G = (R)GRAVITY;
    const R nu_bg = (R)c.pp81_nu_bg, kap_bg = (R)c.pp81_kappa_bg, nu0 = (R)c.pp81_nu0, alpha81 = (R)c.pp81_alpha;
    const R shear2_floor = (R)c.shear2_floor;
    const R kd_sfc = (R)c.bkgnd_kd_sfc, kd_deep = (R)c.bkgnd_kd_deep, z0 = (R)c.bkgnd_z0, bdelta = (R)c.bkgnd_delta;
    const R kv_max = (R)c.kv_max, kd_max = (R)c.kd_max, kt_bg = (R)c.kt_bg, ks_bg = (R)c.ks_bg;
    const R cs = (R)c.cs_nonlocal, qT = (R)q_T_kin, qS = (R)q_S_kin, hbR = (R)h_b, wsR = (R)w_s;
    const R invz2 = (R)c.kv_ml_invz2, conv_kd = (R)c.conv_kd, conv_pr = (R)c.conv_prandtl, conv_n2 = (R)c.conv_n2_thresh;
    const R ks_pr = (R)c.ks_prandtl_turb, epbl_pr = (R)c.epbl_prandtl;
    // gate constants (vmix_assemble, rdb_ocean_vmix.F90:2279-2348)
    const R pr_bl = (R)((c.bkgnd_prandtl > 0.0) ? c.bkgnd_prandtl : 1.0);
    const R kv_floor_scalar = (R)((c.bkgnd_prandtl > 0.0) ? c.bkgnd_prandtl * c.kt_bg + c.kv_bg : c.kv_bg);
    const R inv_pi = (R)(1.0 / PI_D);
    const bool pp81 = (c.interior_closure == VPHYS_INTERIOR_PP81);
    bool invz2_on = (c.kv_ml_invz2 > 0.0 && c.hmix_fixed > 0.0);
    const R hmix = (R)c.hmix_fixed;
    const R hmix_sq = hmix * hmix;
    const R dz_min_safe = rdiv(R(0.5) * hmix, (R)(nz > 1 ? nz : 1));
    const R HV = (R)H_VANISHED;

    // surface interface (k = nz+1): closed, every contributor leaves it at 0
    kvp[P * (size_t)nz] = 0.0;
    ktp[P * (size_t)nz] = 0.0;
    ksp[P * (size_t)nz] = 0.0;
    if (p.write_gamma) {
        p.gamma_t[col + P * (size_t)nz] = 0.0;
        p.gamma_s[col + P * (size_t)nz] = 0.0;
    }

    R depth = 0;   // sum of h over layers nz..q (interface q's depth)
    R d_run = 0;   // sum of h over layers k_sfc..q (KPP pass 2)
    // Layer values (rho, cell-centred u and v) are loaded only for interfaces
    // that use them: an interface between two 0-thickness layers (land,
    // below-bathymetry fillers) takes PP81's background branch and never
    // reads them.  The Bryan-Lewis value depends on the interface depth
    // alone, so it is re-evaluated only when the depth changes (it stays
    // constant through the fillers under the bathymetry).
    // rho and the cell-centred velocities stay FP64 in either precision: their
    // differences across an interface are formed in FP64 (a density step of
    // 1e-3 on 1027 would keep only 3 digits in FP32) and only then rounded to R
    R h_c = (R)HH(nz);
    double r_c = 0, uc_c = 0, vc_c = 0;
    bool have_c = false;
    R kdb_depth = 0, kdb_cached = 0;
    bool kdb_valid = false;
    unsigned bad = 0;
    // FP32 (PREF): the sweep's loads come ASM_U layers at a time, issued
    // before the block's arithmetic, so a column waits on memory once per
    // block instead of once per layer.  Layer values are read only from
    // k_lo - 1 up (k_lo: the lowest layer with h > 0): an interface q reads
    // layers q and q-1 only when h_{q-1} + h_q > 0, so no needed layer lies
    // lower, and the 0-thickness fillers under the bathymetry and land columns
    // load nothing.  The loaded values are the same either way.
#ifndef VPHYS_ASM_U_D
#define VPHYS_ASM_U_D 1   // FP64 sweep: on-demand loads (1) or blocks of this many layers
#endif
    constexpr bool PREF = sizeof(R) == sizeof(float) || VPHYS_ASM_U_D > 1;
    constexpr int ASM_U = (sizeof(R) == sizeof(float)) ? VPHYS_ASM_U_F : (PREF ? VPHYS_ASM_U_D : 1);
    int k_lo = nz + 2;
    if (PREF && !all_zero) {
        for (int k0 = 1; k0 <= nz && k_lo > nz; k0 += 8) {
            double hv[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) hv[u] = (k0 + u <= nz) ? HH(k0 + u) : 0.0;
#pragma unroll
            for (int u = 7; u >= 0; --u)
                if (hv[u] > 0.0) k_lo = k0 + u;
        }
    }
    const int k_need = k_lo - 1;
    for (int q0 = nz; q0 >= 1; q0 -= ASM_U) {
        double hb[ASM_U], rb[ASM_U], ub0[ASM_U], ub1[ASM_U], vb0[ASM_U], vb1[ASM_U];   // layer q0-1-u
#pragma unroll
        for (int u = 0; u < ASM_U; ++u) {
            const int L = q0 - 1 - u;
            hb[u] = rb[u] = ub0[u] = ub1[u] = vb0[u] = vb1[u] = 0.0;
            if (PREF && L >= 1) {
                hb[u] = HH(L);
                if (L >= k_need) {
                    rb[u] = RR(L);
                    ub0[u] = __ldg(up + PU * (size_t)(L - 1));
                    ub1[u] = __ldg(up + PU * (size_t)(L - 1) + 1);
                    vb0[u] = __ldg(vp + PV * (size_t)(L - 1));
                    vb1[u] = __ldg(vp + PV * (size_t)(L - 1) + nx);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < ASM_U; ++u) {
            const int q = q0 - u;
            if (q < 1) break;
            depth = depth + h_c;
            if (q <= k_sfc) d_run = d_run + h_c;
            R kvq = 0, ktq = 0, kdb = 0;
            R h_m = 0;
            double r_m = 0, uc_m = 0, vc_m = 0;
            bool have_m = false;
            if (q >= 2) {
                h_m = PREF ? (R)hb[u] : (R)HH(q - 1);
                if (c.bkgnd_profile) {
                    if (!(kdb_valid && depth == kdb_depth)) {
                        kdb_cached = kd_sfc + (kd_deep - kd_sfc) * (R(0.5) + ratan(rdiv(depth - z0, bdelta)) * inv_pi);
                        kdb_depth = depth;
                        kdb_valid = true;
                    }
                    kdb = kdb_cached;
                }
                const R dz_face = R(0.5) * (h_m + h_c);
                const bool need_layers = (pp81 && !(dz_face <= R(0))) || (c.conv_enable && !(dz_face <= HV));
                if (need_layers) {
                    if (!have_c) {
                        r_c = RR(q);
                        uc_c = UC(q);
                        vc_c = VC(q);
                        have_c = true;
                    }
                    r_m = PREF ? rb[u] : RR(q - 1);
                    uc_m = PREF ? 0.5 * (ub0[u] + ub1[u]) : UC(q - 1);
                    vc_m = PREF ? 0.5 * (vb0[u] + vb1[u]) : VC(q - 1);
                    have_m = true;
                }
                if (pp81) {
                    // ---- PP81 (rdb_ocean_vmix.F90:1046-1073) ----
                    if (dz_face <= R(0)) {
                        kvq = nu_bg;
                        ktq = kap_bg;
                    } else {
                        const auto rdz = rcp_of(dz_face);
                        const R du_dz = qdiv((R)(uc_c - uc_m), rdz);
                        const R dv_dz = qdiv((R)(vc_c - vc_m), rdz);
                        const R shear2 = fmx(du_dz * du_dz + dv_dz * dv_dz, shear2_floor);
                        const R n2 = -rdiv(G * (R)(r_c - r_m), r0 * dz_face);
                        const R ri = rdiv(n2, shear2);
                        const R denom = R(1) + alpha81 * fmx(ri, R(0));
                        const R ri_factor = rdiv(R(1), denom * denom);
                        kvq = nu_bg + nu0 * ri_factor;
                        ktq = kap_bg + rdiv(nu0 * ri_factor, denom);
                    }
                } else if (c.bkgnd_profile) {
                    // ---- interior "none" seed (rdb_ocean_vmix.F90:779-797) ----
                    kvq = pr_bl * kdb;
                    ktq = kdb;
                } else {
                    kvq = kv_floor_scalar;
                    ktq = kt_bg;
                }
            }
            // ---- KPP overlay (rdb_ocean_vmix.F90:1496-1514) ----
            R gt = 0, gs = 0;
            if (kpp_active && q > 1 && q <= k_sfc && d_run < hbR) {
                const R sigma = rdiv(d_run, hbR);
                const R g_shape = sigma * (R(1) - sigma) * (R(1) - sigma);
                const R kv_kpp = hbR * wsR * g_shape;
                kvq = fmx(kvq, kv_kpp);
                ktq = fmx(ktq, kv_kpp);
                if (destabilizing) {
                    const R gamma_factor = cs * g_shape;
                    gt = gamma_factor * qT;
                    gs = gamma_factor * qS;
                }
            }
            if (q >= 2) {
                // ---- kappa-shear merge after KPP, interior interfaces only
                //      (kappa_shear_merge_into_kv_kt, rdb_ocean_kappa_shear.F90:381-421) ----
                // ---- EPBL merge (epbl_merge_into_kv_kt / epbl_merge_max_shear,
                //      rdb_ocean_epbl.F90:1661-1718); with combine = max_shear and
                //      kappa-shear on, kappa-shear is merged first (rdb_ocean_dyn.F90:1553-1559)
                const bool shear_first = c.kappa_shear && c.epbl && c.epbl_combine == 3;
                if (c.epbl) {
                    const R kde = (R)p.kd_epbl[col + P * (size_t)(q - 1)];
                    if (shear_first) {
                        const R kds = (R)p.kd_shear[col + P * (size_t)(q - 1)];
                        ktq = ktq + kds;
                        kvq = kvq + ks_pr * kds;
                        ktq = ktq + fmx(kde - kds, R(0));
                        kvq = kvq + fmx(epbl_pr * kde - ks_pr * kds, R(0));
                    } else if (c.epbl_combine == 2) {
                        ktq = fmx(ktq, kde);
                        kvq = fmx(kvq, epbl_pr * kde);
                    } else {
                        ktq = ktq + kde;
                        kvq = kvq + epbl_pr * kde;
                    }
                }
                if (c.kappa_shear && !shear_first) {
                    const R kd = (R)p.kd_shear[col + P * (size_t)(q - 1)];
                    ktq = ktq + kd;
                    kvq = kvq + ks_pr * kd;
                }
                // ---- KV_ML_INVZ2 (rdb_ocean_vmix.F90:1757-1765) ----
                if (invz2_on) {
                    if (depth >= hmix) {
                        invz2_on = false;
                    } else {
                        const R zz = fmx(depth, dz_min_safe);
                        kvq = kvq + rdiv(invz2 * hmix_sq, zz * zz);
                    }
                }
                // ---- convection (rdb_ocean_vmix.F90:1835-1848) ----
                if (c.conv_enable) {
                    const R dz_face = R(0.5) * (h_m + h_c);
                    if (!(dz_face <= HV) && !(depth < hbR)) {
                        const R n2 = -rdiv(G * (R)(r_c - r_m), r0 * dz_face);
                        if (n2 < conv_n2) {
                            ktq = fmx(ktq, conv_kd);
                            kvq = fmx(kvq, conv_pr * conv_kd);
                        }
                    }
                }
            }
            // ---- split ks := kt, then the gate on interior interfaces ----
            R ksq = ktq;
            if (q >= 2 && q <= nz) {
                if (c.vmix_guard) {
                    bad += (kvq < R(0) || kvq != kvq);
                    bad += (ktq < R(0) || ktq != ktq);
                    bad += (ksq < R(0) || ksq != ksq);
                }
                if (c.bkgnd_profile) {
                    kvq = fmn(fmx(kvq, pr_bl * kdb), kv_max);
                    ktq = fmn(fmx(ktq, kdb), kd_max);
                    ksq = fmn(fmx(ksq, kdb), kd_max);
                } else {
                    kvq = fmn(fmx(kvq, kv_floor_scalar), kv_max);
                    ktq = fmn(fmx(ktq, kt_bg), kd_max);
                    ksq = fmn(fmx(ksq, ks_bg), kd_max);
                }
            }
            const size_t off = P * (size_t)(q - 1);
            kvp[off] = (double)kvq;
            ktp[off] = (double)ktq;
            ksp[off] = (double)ksq;
            if (p.write_gamma) {
                p.gamma_t[col + off] = (double)gt;
                p.gamma_s[col + off] = (double)gs;
            }
            h_c = h_m;
            r_c = r_m;
            uc_c = uc_m;
            vc_c = vc_m;
            have_c = have_m;
        }
    }
    if (bad) atomicAdd(p.guard_count, (unsigned long long)bad);
#undef HH
#undef RR
#undef UC
#undef VC
}

// ---------------------------------------------------------------------------
// 1-2-1 smoothing (rdb_ocean_vmix.F90:2699-2748): copy, then the stencil.
// ---------------------------------------------------------------------------
__global__ void k_copy(const double *__restrict__ src, double *__restrict__ dst, size_t n)
{
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x)
        dst[idx] = src[idx];
}

__global__ void k_smooth(const Params p, double *__restrict__ fld, const double *__restrict__ scratch)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;   // 0-based
    const int j = blockIdx.y;
    const int k = blockIdx.z + 2;                          // interfaces 2..nz (1-based)
    const int nx = p.nx, ny = p.ny;
    if (i < 1 || i > nx - 2 || j < 1 || j > ny - 2) return;
    const double *w = p.wet;
    auto W = [&](int ii, int jj) { return w[ii + (size_t)nx * jj]; };
    const size_t off = p.plane * (size_t)(k - 1);
    auto S = [&](int ii, int jj) { return scratch[off + ii + (size_t)nx * jj]; };
    double w_c = 4.0 * W(i, j);
    double w_e = 2.0 * W(i + 1, j);
    double w_w = 2.0 * W(i - 1, j);
    double w_n = 2.0 * W(i, j + 1);
    double w_s = 2.0 * W(i, j - 1);
    double w_ne = W(i + 1, j + 1);
    double w_nw = W(i - 1, j + 1);
    double w_se = W(i + 1, j - 1);
    double w_sw = W(i - 1, j - 1);
    double wsum = w_c + w_e + w_w + w_n + w_s + w_ne + w_nw + w_se + w_sw;
    double r;
    if (wsum <= 0.0 || W(i, j) == 0.0) {
        r = S(i, j);
    } else {
        r = (w_c * S(i, j) + w_e * S(i + 1, j) + w_w * S(i - 1, j) + w_n * S(i, j + 1) + w_s * S(i, j - 1) +
             w_ne * S(i + 1, j + 1) + w_nw * S(i - 1, j + 1) + w_se * S(i + 1, j - 1) + w_sw * S(i - 1, j - 1)) /
            wsum;
    }
    fld[off + i + (size_t)nx * j] = r;
}

// ---------------------------------------------------------------------------
// Momentum: one thread per (u face, v face) pair.
// ---------------------------------------------------------------------------
#ifndef VPHYS_MOM_THREADS
#define VPHYS_MOM_THREADS 128
#endif
constexpr int MOM_THREADS = VPHYS_MOM_THREADS;   // face columns per block (c' of each in shared memory)

#ifndef VPHYS_MOM_U
#define VPHYS_MOM_U 4
#endif
constexpr int MOM_U = VPHYS_MOM_U;   // levels per load block

// diffuse_velocity_columns_impl for one face column (rdb_ocean_vdiff.F90:1611-1925).
// The Thomas c' of every level sits in shared memory (cpp[(k-1)*bs]); the
// forward-swept d' is written in place over u with an L2 evict_last hint and
// read back by the back-substitution.
template <bool XF, bool DEF>
__device__ __forceinline__ void solve_face(const Params &p, double dt, int i, int j, double *cpp, int bs)
{
    // DEF: the default momentum knobs (hvel_mom6 z_clear, no remnant, BBL
    // glue, implicit stress or drag, z-level faces) as compile-time
    // constants, so their branches fold out of the per-level code
    vphys_config cd = p.cfg;
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
    const double *__restrict__ hl = p.h + cl;
    const double *__restrict__ hr = p.h + cr;
    const double *__restrict__ kvl = p.kv + cl;
    const double *__restrict__ kvr = p.kv + cr;
    const int *ktp = XF ? p.k_top_u : p.k_top_v;
    const int *kbp = XF ? p.k_bot_u : p.k_bot_v;
    // caller-supplied static indices, clamped into the column so that a bad
    // value can never index outside it (valid input: a no-op)
    const int kb = kbp ? min(max(kbp[f], 1), nz) : 1;
    const int ktop = ktp ? min(max(ktp[f], 1), nz) : nz;
    // A face touching land whose velocity is zero in every layer keeps it:
    // with a zero right-hand side every Thomas quantity is a zero, so the
    // solve is skipped (unless the remnant or the stress fold is wanted).
    if (!c.remnant && !c.implicit_stress && fmn(p.wet[cl], p.wet[cr]) == 0.0) {
        bool zero = true;
        for (int k = 1; k <= nz && zero; ++k) zero = (uf[PF * (size_t)(k - 1)] == 0.0);
        if (zero) return;
    }
    double kv_bbl = 0.0, bbl_thick = c.hbbl_visc;
    if (c.bbl_glue) {
        kv_bbl = c.bbl_piston * c.hbbl_visc;
        bbl_thick = c.hbbl_visc;
    }
    const double i_hbbl = 1.0 / (bbl_thick + EPS_HVEL);
    // column depths (k_column_depth: the same k = 1..nz accumulation)
    double zacc = 0.0, zcol_l = 0.0, zcol_r = 0.0;
    if (c.hvel_mom6 && !c.hvel_harmonic) {
        zcol_l = p.zcol[cl];
        zcol_r = p.zcol[cr];
    }
    const double d_min = fmn(-zcol_l, -zcol_r);
    int kb_live = kb;
    if (c.zlevel_faces) {
        for (int k = kb; k <= nz; ++k) {
            if (fmn(__ldg(hl + P * (size_t)(k - 1)), __ldg(hr + P * (size_t)(k - 1))) > H_VANISHED) {
                kb_live = k;
                break;
            }
        }
    }
    double hv_p, zi_p;
    double u_k = uf[0];
    face_layer<double>(c, __ldg(hl), __ldg(hr), u_k, 1, kb, d_min, i_hbbl, zacc, zcol_l, zcol_r, hv_p, zi_p);
    double num_t = 0.0, dz_t = 1.0;
    bool cut_t = false;
    double cp_prev = 0.0, dp_prev = 0.0, gp_prev = 0.0;
    const double lam = (c.implicit_drag && !c.bbl_glue) ? (XF ? p.lambda_bot_u : p.lambda_bot_v)[f] : 0.0;
    const double inv_rho0 = 1.0 / c.rho0;
    // level k + 1's data for row k; the loads of block k0 + MOM_U are issued
    // before block k0 is computed (two register buffers; a block's d' stores
    // go to its own levels, below the next block's loads)
    auto load_up = [&](int k0, double (&hl_)[MOM_U], double (&hr_)[MOM_U], double (&u_)[MOM_U],
                       double (&kl_)[MOM_U], double (&kr_)[MOM_U]) {
#pragma unroll
        for (int q = 0; q < MOM_U; ++q) {
            const int k = k0 + q;
            if (k < nz) {
                const size_t o = P * (size_t)k;
                hl_[q] = __ldg(hl + o);
                hr_[q] = __ldg(hr + o);
                kl_[q] = __ldg(kvl + o);
                kr_[q] = __ldg(kvr + o);
                u_[q] = uf[PF * (size_t)k];
            } else {
                hl_[q] = hr_[q] = kl_[q] = kr_[q] = u_[q] = 0.0;
            }
        }
    };
    double hln[MOM_U], hrn[MOM_U], un[MOM_U], kvln[MOM_U], kvrn[MOM_U];
    load_up(1, hln, hrn, un, kvln, kvrn);
    for (int k0 = 1; k0 <= nz; k0 += MOM_U) {
        double hlx[MOM_U], hrx[MOM_U], ux[MOM_U], kvlx[MOM_U], kvrx[MOM_U];
        load_up(k0 + MOM_U, hlx, hrx, ux, kvlx, kvrx);
#pragma unroll
        for (int q = 0; q < MOM_U; ++q) {
            const int k = k0 + q;
            if (k <= nz) {
                const double hv_0 = hv_p, zi_0 = zi_p;
                const double num_b = num_t, dz_b = dz_t;
                const bool cut_b = cut_t;
                double u_kp1 = 0.0;
                if (k < nz) {
                    u_kp1 = un[q];
                    face_layer<double>(c, hln[q], hrn[q], u_kp1, k + 1, kb, d_min, i_hbbl, zacc, zcol_l, zcol_r, hv_p, zi_p);
                    if (k >= kb_live && k <= ktop)
                        interface_coupling<double>(c, hv_0, hv_p, zi_0, dt, kv_bbl, bbl_thick, kvln[q], kvrn[q], num_t, dz_t,
                                           cut_t);
                }
                double a_k = 0.0, b_k = 1.0, c_k = 0.0;
                const double hf_k = fmx(hv_0, H_VANISHED);
                if (k == kb_live && k <= ktop) {
                    double alpha = 0.0;
                    if (kb_live < nz) {
                        alpha = xdiv(num_t, hf_k * dz_t);
                        if (cut_t) alpha = 0.0;
                    }
                    c_k = -alpha;
                    b_k = 1.0 + alpha;
                    if (c.bbl_glue) b_k = b_k + dt * kv_bbl / (hf_k * (fmn(0.5 * hv_0, bbl_thick) + EPS_HVEL));
                    if (c.implicit_drag && !c.bbl_glue) b_k = b_k + dt * lam;
                }
                if (k == ktop && k > kb_live) {
                    double beta = xdiv(num_b, hf_k * dz_b);
                    if (cut_b) beta = 0.0;
                    a_k = -beta;
                    b_k = 1.0 + beta;
                }
                if (k > kb_live && k < ktop) {
                    double beta = xdiv(num_b, hf_k * dz_b);
                    double alpha = xdiv(num_t, hf_k * dz_t);
                    if (cut_b) beta = 0.0;
                    if (cut_t) alpha = 0.0;
                    a_k = -beta;
                    c_k = -alpha;
                    b_k = 1.0 + alpha + beta;
                }
                double r_k = u_k;
                if (k == ktop && c.implicit_stress) {
                    const double tau = (XF ? p.tau_x : p.tau_y)[f];
                    const double wmin = fmn(p.wet[cl], p.wet[cr]);
                    r_k = r_k + xdiv(dt * tau * 1.0 * wmin * inv_rho0, fmx(hf_k, STRESS_H_MIN));
                }
                const Rcp denom = rcp_of((k == 1) ? b_k : b_k - a_k * cp_prev);
                const double cp = qdiv(c_k, denom);
                const double dp = qdiv((k == 1) ? r_k : r_k - a_k * dp_prev, denom);
                double gp = 0.0;
                if (vrem) gp = qdiv((k == 1) ? 1.0 : 1.0 - a_k * gp_prev, denom);
                cpp[(size_t)(k - 1) * bs] = cp;
                if (k < nz) {
                    st_hint(uf + PF * (size_t)(k - 1), dp, pol_keep);
                    if (vrem) st_hint(vrem + PF * (size_t)(k - 1), gp, pol_keep);
                }
                cp_prev = cp;
                dp_prev = dp;
                gp_prev = gp;
                u_k = u_kp1;
            }
        }
#pragma unroll
        for (int q = 0; q < MOM_U; ++q) {
            hln[q] = hlx[q];
            hrn[q] = hrx[q];
            un[q] = ux[q];
            kvln[q] = kvlx[q];
            kvrn[q] = kvrx[q];
        }
    }
    // back-substitution (momentum into u, remnant into visc_rem); the d' of
    // block k0 - MOM_U are loaded while block k0 is computed
    double u_next = dp_prev;
    double g_next = fmn(gp_prev, 1.0);
    uf[PF * (size_t)(nz - 1)] = u_next;
    if (vrem) vrem[PF * (size_t)(nz - 1)] = g_next;
    auto load_down = [&](int k0, double (&d_)[MOM_U], double (&g_)[MOM_U]) {
#pragma unroll
        for (int q = 0; q < MOM_U; ++q) {
            const int k = k0 - q;
            d_[q] = g_[q] = 0.0;
            if (k >= 1) {
                d_[q] = ld_hint(uf + PF * (size_t)(k - 1), pol_keep);
                if (vrem) g_[q] = ld_hint(vrem + PF * (size_t)(k - 1), pol_keep);
            }
        }
    };
    double dps[MOM_U], gps[MOM_U];
    load_down(nz - 1, dps, gps);
    for (int k0 = nz - 1; k0 >= 1; k0 -= MOM_U) {
        double dpx[MOM_U], gpx[MOM_U];
        load_down(k0 - MOM_U, dpx, gpx);
#pragma unroll
        for (int q = 0; q < MOM_U; ++q) {
            const int k = k0 - q;
            if (k >= 1) {
                const double cpk = cpp[(size_t)(k - 1) * bs];
                u_next = dps[q] - cpk * u_next;
                uf[PF * (size_t)(k - 1)] = u_next;
                if (vrem) {
                    g_next = fmn(gps[q] - cpk * g_next, 1.0);
                    vrem[PF * (size_t)(k - 1)] = g_next;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < MOM_U; ++q) {
            dps[q] = dpx[q];
            gps[q] = gpx[q];
        }
    }
}

// blockIdx.z = 0: u faces (i <= nx, j < ny); 1: v faces (i < nx, j <= ny)
template <bool DEF>
__global__ void __launch_bounds__(MOM_THREADS) k_momentum(const Params p, double dt)
{
    extern __shared__ double smem[];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    double *cpp = smem + threadIdx.x;
    if (blockIdx.z == 0) {
        if (i <= p.nx && j < p.ny) solve_face<true, DEF>(p, dt, i, j, cpp, blockDim.x);
    } else {
        if (i < p.nx && j <= p.ny) solve_face<false, DEF>(p, dt, i, j, cpp, blockDim.x);
    }
}

// ---------------------------------------------------------------------------
// Self-test of xdiv / qdiv against the IEEE quotient on seeded operands:
// random mantissas (plus all-ones and power-of-two ones), exponents in
// [emin, emin + erange), random signs, zeros one time in 16.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long st_mix(unsigned long long z)
{
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double st_make(unsigned long long r, int emin, int erange)
{
    unsigned long long mant = r & 0xFFFFFFFFFFFFFull;
    const int sel = (int)((r >> 52) & 15);
    if (sel == 0) mant = 0xFFFFFFFFFFFFFull;
    if (sel == 1) mant = 0;
    const int e = emin + (int)((r >> 56) % (unsigned long long)erange);
    const unsigned long long bits = ((r >> 63) << 63) | ((unsigned long long)(e + 1023) << 52) | mant;
    if (sel == 2) return ((r >> 63) ? -0.0 : 0.0);
    return __longlong_as_double((long long)bits);
}
__global__ void k_selftest_division(unsigned long long seed, long long per_thread, int emin, int erange,
                                    unsigned long long *bad)
{
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    unsigned long long nb = 0;
    for (long long n = 0; n < per_thread; ++n) {
        const unsigned long long r1 = st_mix(seed ^ ((unsigned long long)tid * 0x100000001b3ull + (unsigned long long)n * 0x9e37ull));
        const unsigned long long r2 = st_mix(r1 + 0x632be59bd9b4e019ull);
        const unsigned long long r3 = st_mix(r2 + 0x2545f4914f6cdd1dull);
        const double a = st_make(r1, emin, erange), b = st_make(r2, emin, erange), a2 = st_make(r3, emin, erange);
        if (b == 0.0) continue;
        const double ref = a / b, ref2 = a2 / b;
        const Rcp rb = rcp_of(b);
        const double q = qdiv(a, rb), q2 = qdiv(a2, rb), x = xdiv(a, b);
        nb += (__double_as_longlong(q) != __double_as_longlong(ref)) + (__double_as_longlong(q2) != __double_as_longlong(ref2)) +
              (__double_as_longlong(x) != __double_as_longlong(ref));
    }
    if (nb) atomicAdd(bad, nb);
}

void launch_selftest_division(unsigned long long seed, long long per_thread, int emin, int erange,
                              unsigned long long *bad, cudaStream_t stream)
{
    k_selftest_division<<<148 * 4, 256, 0, stream>>>(seed, per_thread, emin, erange, bad);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int grid_1d(size_t n, int threads)
{
    size_t b = (n + threads - 1) / threads;
    const size_t cap = 148ull * 16ull;
    return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

void launch_eos_wright(const Params &p, cudaStream_t stream)
{
    k_eos_wright<<<grid_1d(p.plane * (size_t)p.nz, 256), 256, 0, stream>>>(p);
}

void launch_surface_flux(const Params &p, double inv_heat, double inv_salt, cudaStream_t stream)
{
    dim3 grid((p.nx + 127) / 128, p.ny);
    k_surface_flux<<<grid, 128, 0, stream>>>(p, inv_heat, inv_salt);
}

void launch_sw_penetration(const Params &p, double inv_scale, cudaStream_t stream)
{
    dim3 grid((p.nx + 127) / 128, p.ny);
    k_sw_penetration<<<grid, 128, 0, stream>>>(p, inv_scale);
}

void launch_stress_mag(const Params &p, cudaStream_t stream)
{
    dim3 grid((p.nx + 127) / 128, p.ny);
    k_stress_mag<<<grid, 128, 0, stream>>>(p, const_cast<double *>(p.stress_mag));
}

void launch_assemble(const Params &p, cudaStream_t stream)
{
    dim3 grid((p.nx + ASM_THREADS - 1) / ASM_THREADS, p.ny);
    const int kind = default_assembly_kind(p.cfg);
    if (p.cfg.mixed_precision >= 2) {
        if (kind == 1)
            k_assemble<float, 1><<<grid, ASM_THREADS, 0, stream>>>(p);
        else if (kind == 2)
            k_assemble<float, 2><<<grid, ASM_THREADS, 0, stream>>>(p);
        else
            k_assemble<float, 0><<<grid, ASM_THREADS, 0, stream>>>(p);
    } else {
        if (kind == 1)
            k_assemble<double, 1><<<grid, ASM_THREADS, 0, stream>>>(p);
        else if (kind == 2)
            k_assemble<double, 2><<<grid, ASM_THREADS, 0, stream>>>(p);
        else
            k_assemble<double, 0><<<grid, ASM_THREADS, 0, stream>>>(p);
    }
}

void launch_smooth(const Params &p, double *fld, double *scratch, cudaStream_t stream)
{
    const size_t n = p.plane * (size_t)(p.nz + 1);
    k_copy<<<grid_1d(n, 256), 256, 0, stream>>>(fld, scratch, n);
    if (p.nz >= 2) {
        dim3 grid((p.nx + 127) / 128, p.ny, p.nz - 1);
        k_smooth<<<grid, 128, 0, stream>>>(p, fld, scratch);
    }
}

// -sum_{k=1..nz} h of every column, accumulated in the order of
// diffuse_velocity_columns_impl's z_clear pre-pass (rdb_ocean_vdiff.F90:1621-1700),
// so the momentum kernels read two numbers per face instead of 2*nz.
__global__ void k_column_depth(const Params p)
{
    constexpr int U = 8;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= p.nx) return;
    const size_t col = (size_t)i + (size_t)p.nx * j;
    const double *__restrict__ hp = p.h + col;
    const size_t P = p.plane;
    double z = 0.0;
    for (int k0 = 0; k0 < p.nz; k0 += U) {
        double hv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) hv[u] = (k0 + u < p.nz) ? __ldg(hp + P * (size_t)(k0 + u)) : 0.0;
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (k0 + u < p.nz) z = z - hv[u];
    }
    p.zcol[col] = z;
}

void launch_column_depth(const Params &p, cudaStream_t stream)
{
    k_column_depth<<<dim3((p.nx + 127) / 128, p.ny), 128, 0, stream>>>(p);
}

void launch_momentum(const Params &p, double dt, cudaStream_t stream)
{
    if (p.cfg.hvel_mom6 && !p.cfg.hvel_harmonic) launch_column_depth(p, stream);
    if (p.cfg.mixed_precision) {
        launch_momentum_mp(p, dt, stream);
        return;
    }
    static bool attr_set = false;
    if (!attr_set) {
        const int mx = (int)((size_t)VPHYS_NZ_MAX * MOM_THREADS * sizeof(double));
        cudaFuncSetAttribute(k_momentum<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        cudaFuncSetAttribute(k_momentum<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        attr_set = true;
    }
    dim3 grid((p.nx + 1 + MOM_THREADS - 1) / MOM_THREADS, p.ny + 1, 2);
    const size_t smem = (size_t)p.nz * MOM_THREADS * sizeof(double);
    if (is_default_face_knobs(p.cfg))
        k_momentum<true><<<grid, MOM_THREADS, smem, stream>>>(p, dt);
    else
        k_momentum<false><<<grid, MOM_THREADS, smem, stream>>>(p, dt);
}

}  // namespace vphys
