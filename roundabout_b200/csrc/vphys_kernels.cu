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
//   k_stress_mag   |tau| at cell centres               rdb_ocean_surface_stress.F90:858-875
//   k_assemble     PP81 / seed, KPP passes 1 + 2, KV_ML_INVZ2, convection,
//                  split, guard, Bryan-Lewis or scalar gate: every interface
//                  of a column in one top-down register sweep
//                                                     rdb_ocean_vmix.F90:1007-1516, 1716-2434, 2677-2769
//   k_smooth_*     optional 1-2-1 horizontal smoothing  rdb_ocean_vmix.F90:2699-2748
//   k_momentum     u and v face columns: face thickness, coupling, fused
//                  Thomas sweep, optional remnant      rdb_ocean_vdiff.F90:1416-2115
//   k_tracers<N>   tracer build + factorisation once per diffusivity, forward
//                  sweep of all N tracers, back-substitution, budgets, and
//                  the KPP non-local tendency fused into the store
//                                                     rdb_ocean_vdiff.F90:1107-1414,
//                                                     rdb_ocean_vmix.F90:1605-1714
#include <cuda_runtime.h>

#include "vphys_device.cuh"
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
            double alpha_0 = 7.057924e-4 + 3.480336e-7 * T_k + -1.112733e-7 * S_k;
            double p_0 = 5.790749e8 + 3.516535e6 * T_k + -4.002714e4 * T_sq + 2.084372e2 * T_cu + 5.944068e5 * S_k +
                         -9.643486e3 * S_k * T_k;
            double lambda = 1.704853e5 + 7.904722e2 * T_k + -7.984422e0 * T_sq + 5.140652e-2 * T_cu +
                            -2.302158e2 * S_k + -3.079464e0 * S_k * T_k;
            double p_plus_p0 = p_ref + p_0;
            double denom = lambda + alpha_0 * p_plus_p0;
            r = p_plus_p0 / denom;
        } else {
            r = rho0;
        }
        p.rho[idx] = r;
    }
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

__global__ void __launch_bounds__(ASM_THREADS) k_assemble(const Params p)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= p.nx) return;
    const vphys_config &c = p.cfg;
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

    // first live layer from the top (rdb_vl_first_live)
    int k_sfc = nz;
    for (int k = nz; k >= 1; --k) {
        if (HH(k) > H_VANISHED) {
            k_sfc = k;
            break;
        }
    }

    double h_b = p.bl_depth[col];   // lagged BL depth (state)
    double q_T_kin = 0.0, q_S_kin = 0.0, w_s = 0.0;
    bool destabilizing = false, kpp_active = false;
    if (c.use_kpp) {
        // ---- KPP pass 1 (rdb_ocean_vmix.F90:1288-1426) ----
        const double tau_mag = p.stress_mag[col];
        const double u_star = sqrt(tau_mag / rho0);
        q_T_kin = p.q_heat[col] / (rho0 * c.cp);
        q_S_kin = p.q_salt[col] / rho0;
        const double B_0 = (GRAVITY / rho0) * (c.alpha_T * q_T_kin - c.beta_S * q_S_kin);
        {
            const double wstar3_lagged = fmx(0.0, -B_0) * h_b;
            const double cb = sm_cbrt(wstar3_lagged);
            const double w_s_col = sqrt(u_star * u_star + cb * cb);
            const double u_ref = UC(k_sfc);
            const double v_ref = VC(k_sfc);
            const double b_ref = -(GRAVITY * RR(k_sfc) / rho0);
            const double h_sfc = HH(k_sfc);
            const double d_centre_ref = 0.5 * h_sfc;
            const double vt2_coef = c.c_vt2 / c.ri_crit;
            double ri_prev = 0.0, d_prev = d_centre_ref, d_centre_k = d_centre_ref;
            double h_above = h_sfc;
            bool crossing_found = false;
            double hb_new = 0.0;
            for (int k = k_sfc - 1; k >= 1; --k) {
                const double h_k = HH(k);
                d_centre_k = d_centre_k + 0.5 * (h_above + h_k);
                const double u_k = UC(k);
                const double v_k = VC(k);
                const double b_k = -(GRAVITY * RR(k) / rho0);
                const double delta_d = d_centre_k - d_centre_ref;
                const double delta_b = b_ref - b_k;
                const double n_brunt = sqrt(fmx(0.0, delta_b / delta_d));
                const double vt2 = vt2_coef * d_centre_k * n_brunt * w_s_col;
                const double shear2 =
                    fmx((u_k - u_ref) * (u_k - u_ref) + (v_k - v_ref) * (v_k - v_ref) + vt2, c.shear2_floor);
                const double ri_bulk = delta_b * delta_d / shear2;
                if (ri_bulk >= c.ri_crit) {
                    const double denom = ri_bulk - ri_prev;
                    double frac;
                    if (fabs(denom) > 1.0e-12)
                        frac = (c.ri_crit - ri_prev) / denom;
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
            h_b = hb_new;
            p.bl_depth[col] = h_b;
        }
        // ---- KPP pass 2 scalars (rdb_ocean_vmix.F90:1429-1491) ----
        p.b0[col] = B_0;
        destabilizing = B_0 < 0.0;
        const double wstar3 = fmx(0.0, -B_0) * h_b;
        const double w_star = sm_cbrt(wstar3);
        w_s = sqrt(u_star * u_star + w_star * w_star);
        kpp_active = (h_b > 0.0 && w_s > 0.0);
    }

    // gate constants (vmix_assemble, rdb_ocean_vmix.F90:2279-2348)
    const double pr_bl = (c.bkgnd_prandtl > 0.0) ? c.bkgnd_prandtl : 1.0;
    const double kv_floor_scalar = (c.bkgnd_prandtl > 0.0) ? c.bkgnd_prandtl * c.kt_bg + c.kv_bg : c.kv_bg;
    const double inv_pi = 1.0 / PI_D;
    const bool pp81 = (c.interior_closure == VPHYS_INTERIOR_PP81);
    bool invz2_on = (c.kv_ml_invz2 > 0.0 && c.hmix_fixed > 0.0);
    const double hmix = c.hmix_fixed;
    const double hmix_sq = hmix * hmix;
    const double dz_min_safe = 0.5 * hmix / (double)(nz > 1 ? nz : 1);

    // surface interface (k = nz+1): closed, every contributor leaves it at 0
    kvp[P * (size_t)nz] = 0.0;
    ktp[P * (size_t)nz] = 0.0;
    ksp[P * (size_t)nz] = 0.0;
    if (p.write_gamma) {
        p.gamma_t[col + P * (size_t)nz] = 0.0;
        p.gamma_s[col + P * (size_t)nz] = 0.0;
    }

    double depth = 0.0;   // sum of h over layers nz..q (interface q's depth)
    double d_run = 0.0;   // sum of h over layers k_sfc..q (KPP pass 2)
    double h_c = HH(nz), r_c = RR(nz), uc_c = UC(nz), vc_c = VC(nz);
    unsigned bad = 0;
    for (int q = nz; q >= 1; --q) {
        depth = depth + h_c;
        if (q <= k_sfc) d_run = d_run + h_c;
        double kvq = 0.0, ktq = 0.0, kdb = 0.0;
        double h_m = 0.0, r_m = 0.0, uc_m = 0.0, vc_m = 0.0;
        if (q >= 2) {
            h_m = HH(q - 1);
            r_m = RR(q - 1);
            if (c.bkgnd_profile)
                kdb = c.bkgnd_kd_sfc +
                      (c.bkgnd_kd_deep - c.bkgnd_kd_sfc) * (0.5 + sm_atan((depth - c.bkgnd_z0) / c.bkgnd_delta) * inv_pi);
            if (pp81) {
                // ---- PP81 (rdb_ocean_vmix.F90:1046-1073) ----
                uc_m = UC(q - 1);
                vc_m = VC(q - 1);
                const double dz_face = 0.5 * (h_m + h_c);
                if (dz_face <= 0.0) {
                    kvq = c.pp81_nu_bg;
                    ktq = c.pp81_kappa_bg;
                } else {
                    const double du_dz = (uc_c - uc_m) / dz_face;
                    const double dv_dz = (vc_c - vc_m) / dz_face;
                    const double shear2 = fmx(du_dz * du_dz + dv_dz * dv_dz, c.shear2_floor);
                    const double n2 = -(GRAVITY * (r_c - r_m) / (rho0 * dz_face));
                    const double ri = n2 / shear2;
                    const double denom = 1.0 + c.pp81_alpha * fmx(ri, 0.0);
                    const double ri_factor = 1.0 / (denom * denom);
                    kvq = c.pp81_nu_bg + c.pp81_nu0 * ri_factor;
                    ktq = c.pp81_kappa_bg + c.pp81_nu0 * ri_factor / denom;
                }
            } else if (c.bkgnd_profile) {
                // ---- interior "none" seed (rdb_ocean_vmix.F90:779-797) ----
                kvq = pr_bl * kdb;
                ktq = kdb;
            } else {
                kvq = kv_floor_scalar;
                ktq = c.kt_bg;
            }
        }
        // ---- KPP overlay (rdb_ocean_vmix.F90:1496-1514) ----
        double gt = 0.0, gs = 0.0;
        if (kpp_active && q > 1 && q <= k_sfc && d_run < h_b) {
            const double sigma = d_run / h_b;
            const double g_shape = sigma * (1.0 - sigma) * (1.0 - sigma);
            const double kv_kpp = h_b * w_s * g_shape;
            kvq = fmx(kvq, kv_kpp);
            ktq = fmx(ktq, kv_kpp);
            if (destabilizing) {
                const double gamma_factor = c.cs_nonlocal * g_shape;
                gt = gamma_factor * q_T_kin;
                gs = gamma_factor * q_S_kin;
            }
        }
        if (q >= 2) {
            // ---- KV_ML_INVZ2 (rdb_ocean_vmix.F90:1757-1765) ----
            if (invz2_on) {
                if (depth >= hmix) {
                    invz2_on = false;
                } else {
                    const double zz = fmx(depth, dz_min_safe);
                    kvq = kvq + c.kv_ml_invz2 * hmix_sq / (zz * zz);
                }
            }
            // ---- convection (rdb_ocean_vmix.F90:1835-1848) ----
            if (c.conv_enable) {
                const double dz_face = 0.5 * (h_m + h_c);
                if (!(dz_face <= H_VANISHED) && !(depth < h_b)) {
                    const double n2 = -(GRAVITY * (r_c - r_m) / (rho0 * dz_face));
                    if (n2 < c.conv_n2_thresh) {
                        ktq = fmx(ktq, c.conv_kd);
                        kvq = fmx(kvq, c.conv_prandtl * c.conv_kd);
                    }
                }
            }
        }
        // ---- split ks := kt, then the gate on interior interfaces ----
        double ksq = ktq;
        if (q >= 2 && q <= nz) {
            if (c.vmix_guard) {
                bad += (kvq < 0.0 || kvq != kvq);
                bad += (ktq < 0.0 || ktq != ktq);
                bad += (ksq < 0.0 || ksq != ksq);
            }
            if (c.bkgnd_profile) {
                kvq = fmn(fmx(kvq, pr_bl * kdb), c.kv_max);
                ktq = fmn(fmx(ktq, kdb), c.kd_max);
                ksq = fmn(fmx(ksq, kdb), c.kd_max);
            } else {
                kvq = fmn(fmx(kvq, kv_floor_scalar), c.kv_max);
                ktq = fmn(fmx(ktq, c.kt_bg), c.kd_max);
                ksq = fmn(fmx(ksq, c.ks_bg), c.kd_max);
            }
        }
        const size_t off = P * (size_t)(q - 1);
        kvp[off] = kvq;
        ktp[off] = ktq;
        ksp[off] = ksq;
        if (p.write_gamma) {
            p.gamma_t[col + off] = gt;
            p.gamma_s[col + off] = gs;
        }
        h_c = h_m;
        r_c = r_m;
        uc_c = uc_m;
        vc_c = vc_m;
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
constexpr int MOM_THREADS = 128;

__device__ __forceinline__ void face_layer(const vphys_config &c, double hl_c, double hr_c, double u_k, int k, int kb,
                                           double d_min, double i_hbbl, double &zacc, double &zcol_l,
                                           double &zcol_r, double &hvel, double &zint)
{
    // vdiff_face_layer (rdb_ocean_vdiff.F90:1964-2056)
    zint = 0.0;
    if (c.hvel_mom6 && !c.hvel_harmonic) {
        const double h_harm = 2.0 * hl_c * hr_c / (hl_c + hr_c + EPS_HVEL);
        const double h_arith = 0.5 * (hl_c + hr_c);
        const double h_delta = hr_c - hl_c;
        zcol_l = zcol_l + hl_c;
        zcol_r = zcol_r + hr_c;
        if (k >= kb) zacc = zacc + h_harm;
        const double z_clear = fmx(zcol_l, zcol_r) + d_min;
        zint = fmx(zacc, z_clear) * i_hbbl;
        hvel = h_arith;
        if (u_k * h_delta > 0.0) {
            const double z2 = zint;
            const double botfn = 1.0 / (1.0 + 0.09 * z2 * z2 * z2 * z2 * z2 * z2);
            hvel = (1.0 - botfn) * h_arith + botfn * h_harm;
        }
    } else if (c.hvel_mom6) {
        const double h_harm = 2.0 * hl_c * hr_c / (hl_c + hr_c + EPS_HVEL);
        const double h_arith = 0.5 * (hl_c + hr_c);
        const double h_delta = hr_c - hl_c;
        hvel = h_harm;
        if (c.hvel_upwind && u_k * h_delta < 0.0) {
            const double z2 = zacc;
            const double botfn = 1.0 / (1.0 + 0.09 * z2 * z2 * z2 * z2 * z2 * z2);
            hvel = (1.0 - botfn) * h_harm + botfn * h_arith;
        }
        if (k >= kb) zacc = zacc + h_harm * i_hbbl;
        zint = zacc;
    } else {
        hvel = 0.5 * (hl_c + hr_c);
    }
    if (c.zlevel_faces) hvel = fmn(hl_c, hr_c);
}

__device__ __forceinline__ void interface_coupling(const vphys_config &c, double hv_lo, double hv_hi, double zint_lo,
                                                   double dt, double kv_bbl, double bbl_thick, double kv_l,
                                                   double kv_r, double &num, double &dz, bool &cut)
{
    // vdiff_interface_coupling (rdb_ocean_vdiff.F90:2058-2115)
    const double hf_lo = fmx(hv_lo, H_VANISHED);
    const double hf_hi = fmx(hv_hi, H_VANISHED);
    if (c.hvel_mom6)
        dz = 0.5 * (hf_lo + hf_hi);
    else
        dz = face_thick(hf_lo, hf_hi, c.use_harmonic);
    double nu_f = 0.5 * (kv_l + kv_r);
    if (c.bbl_glue) {
        const double z = zint_lo;
        const double botfn_int = 1.0 / (1.0 + 0.09 * z * z * z * z * z * z);
        nu_f = fmx(0.0, nu_f + (kv_bbl - c.kv_bbl_bg) * botfn_int);
        if (dz > bbl_thick) dz = (1.0 - botfn_int) * dz + botfn_int * bbl_thick;
    }
    num = dt * nu_f;
    cut = c.zlevel_faces && (hv_lo <= H_VANISHED || hv_hi <= H_VANISHED);
}

template <bool XF>
__device__ __forceinline__ void solve_face(const Params &p, double dt, int i, int j, double *cdiag, double *rhs)
{
    // diffuse_velocity_columns_impl, one face column (rdb_ocean_vdiff.F90:1611-1925)
    const vphys_config &c = p.cfg;
    const int nx = p.nx, ny = p.ny, nz = p.nz;
    const int nu = XF ? nx + 1 : nx;
    const size_t P = p.plane;
    const size_t PF = XF ? p.plane_u : p.plane_v;
    const size_t f = (size_t)i + (size_t)nu * j;
    double *__restrict__ uf = (XF ? p.u : p.v) + f;
    double *__restrict__ vrem = c.remnant ? ((XF ? p.visc_rem_u : p.visc_rem_v) + f) : nullptr;
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
    double kv_bbl = 0.0, bbl_thick = c.hbbl_visc;
    if (c.bbl_glue) {
        kv_bbl = c.bbl_piston * c.hbbl_visc;
        bbl_thick = c.hbbl_visc;
    }
    const double i_hbbl = 1.0 / (bbl_thick + EPS_HVEL);
    double zacc = 0.0, zcol_l = 0.0, zcol_r = 0.0;
    if (c.hvel_mom6 && !c.hvel_harmonic) {
        for (int k = 1; k <= nz; ++k) {
            zcol_l = zcol_l - __ldg(hl + P * (size_t)(k - 1));
            zcol_r = zcol_r - __ldg(hr + P * (size_t)(k - 1));
        }
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
    double hv_0, hv_p, zi_0, zi_p;
    double u_next_in = uf[0];
    face_layer(c, __ldg(hl), __ldg(hr), u_next_in, 1, kb, d_min, i_hbbl, zacc, zcol_l, zcol_r, hv_p, zi_p);
    double num_t = 0.0, dz_t = 1.0;
    bool cut_t = false;
    double cp_prev = 0.0, dp_prev = 0.0, gp_prev = 0.0;
    const double lam = (c.implicit_drag && !c.bbl_glue) ? (XF ? p.lambda_bot_u : p.lambda_bot_v)[f] : 0.0;
    double stress_rhs = 0.0;
    const double inv_rho0 = 1.0 / c.rho0;
    double u_k = u_next_in;
    for (int k = 1; k <= nz; ++k) {
        hv_0 = hv_p;
        zi_0 = zi_p;
        const double num_b = num_t, dz_b = dz_t;
        const bool cut_b = cut_t;
        double u_kp1 = 0.0;
        if (k < nz) {
            u_kp1 = uf[PF * (size_t)k];
            face_layer(c, __ldg(hl + P * (size_t)k), __ldg(hr + P * (size_t)k), u_kp1, k + 1, kb, d_min, i_hbbl,
                       zacc, zcol_l, zcol_r, hv_p, zi_p);
            if (k >= kb_live && k <= ktop) {
                interface_coupling(c, hv_0, hv_p, zi_0, dt, kv_bbl, bbl_thick, __ldg(kvl + P * (size_t)k),
                                   __ldg(kvr + P * (size_t)k), num_t, dz_t, cut_t);
            }
        }
        double a_k = 0.0, b_k = 1.0, c_k = 0.0;
        const double hf_k = fmx(hv_0, H_VANISHED);
        if (k == kb_live && k <= ktop) {
            double alpha = 0.0;
            if (kb_live < nz) {
                alpha = num_t / (hf_k * dz_t);
                if (cut_t) alpha = 0.0;
            }
            c_k = -alpha;
            b_k = 1.0 + alpha;
            if (c.bbl_glue) b_k = b_k + dt * kv_bbl / (hf_k * (fmn(0.5 * hv_0, bbl_thick) + EPS_HVEL));
            if (c.implicit_drag && !c.bbl_glue) b_k = b_k + dt * lam;
        }
        if (k == ktop && k > kb_live) {
            double beta = num_b / (hf_k * dz_b);
            if (cut_b) beta = 0.0;
            a_k = -beta;
            b_k = 1.0 + beta;
        }
        if (k > kb_live && k < ktop) {
            double beta = num_b / (hf_k * dz_b);
            double alpha = num_t / (hf_k * dz_t);
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
            stress_rhs = dt * tau * 1.0 * wmin * inv_rho0 / fmx(hf_k, STRESS_H_MIN);
            r_k = r_k + stress_rhs;
        }
        double cp, dp, gp;
        if (k == 1) {
            cp = c_k / b_k;
            dp = r_k / b_k;
            gp = 1.0 / b_k;
        } else {
            const double denom = b_k - a_k * cp_prev;
            cp = c_k / denom;
            dp = (r_k - a_k * dp_prev) / denom;
            gp = (1.0 - a_k * gp_prev) / denom;
        }
        cdiag[k - 1] = cp;
        rhs[k - 1] = dp;
        if (vrem) vrem[PF * (size_t)(k - 1)] = gp;
        cp_prev = cp;
        dp_prev = dp;
        gp_prev = gp;
        u_k = u_kp1;
    }
    double u_next = dp_prev;
    double g_next = fmn(gp_prev, 1.0);
    uf[PF * (size_t)(nz - 1)] = u_next;
    if (vrem) vrem[PF * (size_t)(nz - 1)] = g_next;
    for (int k = nz - 1; k >= 1; --k) {
        const double cpk = cdiag[k - 1];
        u_next = rhs[k - 1] - cpk * u_next;
        uf[PF * (size_t)(k - 1)] = u_next;
        if (vrem) {
            g_next = fmn(vrem[PF * (size_t)(k - 1)] - cpk * g_next, 1.0);
            vrem[PF * (size_t)(k - 1)] = g_next;
        }
    }
}

__global__ void __launch_bounds__(MOM_THREADS) k_momentum(const Params p, double dt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i > p.nx) return;
    double cdiag[NZ_MAX], rhs[NZ_MAX];
    if (j < p.ny) solve_face<true>(p, dt, i, j, cdiag, rhs);
    if (i < p.nx) solve_face<false>(p, dt, i, j, cdiag, rhs);
}

// ---------------------------------------------------------------------------
// Tracers: build + factorise once per diffusivity, forward-sweep every
// tracer, back-substitute, then store with the budget and the KPP non-local
// tendency (applied after the diffusion, as vmix_apply_in_stage orders them).
// ---------------------------------------------------------------------------
constexpr int TR_THREADS = 128;

// Row k (1-based) of the tracer matrix (build_factorize_tracer_matrix,
// rdb_ocean_vdiff.F90:1285-1341); hm/hc/hp are the raw thicknesses of layers
// k-1, k, k+1, kb/kt the diffusivity at interfaces k and k+1.
__device__ __forceinline__ void tracer_row(int k, int nz, bool use_harmonic, double dt, double hm_raw, double hc_raw,
                                           double hp_raw, double K_k, double K_kp1, double &a, double &b, double &cc)
{
    if (k == 1) {
        const double hc = fmx(hc_raw, H_VANISHED);
        double alpha = 0.0;
        if (nz > 1) {
            const double hp = fmx(hp_raw, H_VANISHED);
            const double dz_face = face_thick(hc, hp, use_harmonic);
            alpha = dt * K_kp1 / (hc * dz_face);
            if (hc_raw <= H_VANISHED || hp_raw <= H_VANISHED) alpha = 0.0;
        }
        a = 0.0;
        cc = -alpha;
        b = 1.0 + alpha;
    } else if (k < nz) {
        const double hm = fmx(hm_raw, H_VANISHED);
        const double hc = fmx(hc_raw, H_VANISHED);
        const double hp = fmx(hp_raw, H_VANISHED);
        double beta = dt * K_k / (hc * face_thick(hm, hc, use_harmonic));
        double alpha = dt * K_kp1 / (hc * face_thick(hc, hp, use_harmonic));
        if (hc_raw <= H_VANISHED || hm_raw <= H_VANISHED) beta = 0.0;
        if (hc_raw <= H_VANISHED || hp_raw <= H_VANISHED) alpha = 0.0;
        a = -beta;
        cc = -alpha;
        b = 1.0 + alpha + beta;
    } else {
        const double hm = fmx(hm_raw, H_VANISHED);
        const double hc = fmx(hc_raw, H_VANISHED);
        const double dz_face = face_thick(hm, hc, use_harmonic);
        double beta = dt * K_k / (hc * dz_face);
        if (hc_raw <= H_VANISHED || hm_raw <= H_VANISHED) beta = 0.0;
        a = -beta;
        cc = 0.0;
        b = 1.0 + beta;
    }
}

template <int NTR, bool TWO>
__global__ void __launch_bounds__(TR_THREADS) k_tracers(const Params p, double dt, int diffuse, int nonlocal)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= p.nx) return;
    const vphys_config &c = p.cfg;
    const int nx = p.nx, nz = p.nz, ntr = p.ntr;
    const size_t P = p.plane;
    const size_t col = (size_t)i + (size_t)nx * j;
    const double *__restrict__ hp = p.h + col;
    const int iT = c.idx_temperature, iS = c.idx_salinity, iPS = c.idx_pseudo_salt;
#define HH(k) __ldg(hp + P * (size_t)((k) - 1))
    double *trc[NTR];
#pragma unroll
    for (int t = 0; t < NTR; ++t) trc[t] = (t < ntr) ? p.tr[t] + col : nullptr;

    double r[NTR][NZ_MAX];
    double cpA[NZ_MAX];
    double cpB[TWO ? NZ_MAX : 1];

    if (diffuse) {
        // ---- upward pass: rows, factorisation, forward sweep of every tracer ----
        const double *__restrict__ KA = p.kt + col;
        const double *__restrict__ KB = p.ks + col;
        double h_m = 0.0, h_c = HH(1), h_p = (nz > 1) ? HH(2) : 0.0;
        double KA_k = __ldg(KA), KA_kp1 = __ldg(KA + P);
        double KB_k = TWO ? __ldg(KB) : 0.0, KB_kp1 = TWO ? __ldg(KB + P) : 0.0;
        double cpA_prev = 0.0, cpB_prev = 0.0;
        for (int k = 1; k <= nz; ++k) {
            double aA, bA, cA;
            tracer_row(k, nz, c.use_harmonic, dt, h_m, h_c, h_p, KA_k, KA_kp1, aA, bA, cA);
            const double denA = (k == 1) ? bA : bA - aA * cpA_prev;
            cpA_prev = cA / denA;
            cpA[k - 1] = cpA_prev;
            double aB = 0.0, denB = 1.0;
            if (TWO) {
                double bB, cB;
                tracer_row(k, nz, c.use_harmonic, dt, h_m, h_c, h_p, KB_k, KB_kp1, aB, bB, cB);
                denB = (k == 1) ? bB : bB - aB * cpB_prev;
                cpB_prev = cB / denB;
                cpB[k - 1] = cpB_prev;
            }
#pragma unroll
            for (int t = 0; t < NTR; ++t) {
                if (t < ntr) {
                    const bool useA = !TWO || (t == iT);
                    const double a = useA ? aA : aB;
                    const double den = useA ? denA : denB;
                    const double x = trc[t][P * (size_t)(k - 1)];
                    r[t][k - 1] = (k == 1) ? x / den : (x - a * r[t][k - 2]) / den;
                }
            }
            h_m = h_c;
            h_c = h_p;
            h_p = (k + 2 <= nz) ? HH(k + 2) : 0.0;
            KA_k = KA_kp1;
            KA_kp1 = (k + 2 <= nz + 1) ? __ldg(KA + P * (size_t)(k + 1)) : 0.0;
            if (TWO) {
                KB_k = KB_kp1;
                KB_kp1 = (k + 2 <= nz + 1) ? __ldg(KB + P * (size_t)(k + 1)) : 0.0;
            }
        }
    }

    // ---- non-local column scalars, recomputed exactly as KPP pass 2 ----
    bool nl = nonlocal && c.use_kpp;
    int k_sfc = nz;
    double h_b = 0.0, q_T_kin = 0.0, q_S_kin = 0.0, cs = c.cs_nonlocal;
    if (nl) {
        for (int k = nz; k >= 1; --k) {
            if (HH(k) > H_VANISHED) {
                k_sfc = k;
                break;
            }
        }
        const double rho0 = c.rho0;
        h_b = p.bl_depth[col];
        const double u_star = sqrt(p.stress_mag[col] / rho0);
        q_T_kin = p.q_heat[col] / (rho0 * c.cp);
        q_S_kin = p.q_salt[col] / rho0;
        const double B_0 = (GRAVITY / rho0) * (c.alpha_T * q_T_kin - c.beta_S * q_S_kin);
        const double wstar3 = fmx(0.0, -B_0) * h_b;
        const double w_star = sm_cbrt(wstar3);
        const double w_s = sqrt(u_star * u_star + w_star * w_star);
        nl = (h_b > 0.0 && w_s > 0.0 && B_0 < 0.0);
    }
    const bool do_nl = nonlocal && c.use_kpp;
    double *heat = (c.budgets && diffuse && iT >= 0) ? p.heat_budget + col : nullptr;
    double *salt = (c.budgets && diffuse && iS >= 0) ? p.salt_budget + col : nullptr;

    // ---- downward pass: back-substitution, budgets, non-local, store ----
    double x_above[NTR];
#pragma unroll
    for (int t = 0; t < NTR; ++t) x_above[t] = 0.0;
    double gT_above = 0.0, gS_above = 0.0;   // gamma at the top interface of layer k
    double d_run = 0.0;
    double h_c = HH(nz), h_a = 0.0;
    for (int k = nz; k >= 1; --k) {
        const double h_b_layer = (k > 1) ? HH(k - 1) : 0.0;   // layer below
        double gT = 0.0, gS = 0.0;
        if (nl) {
            if (k <= k_sfc) d_run = d_run + h_c;
            if (k > 1 && k <= k_sfc && d_run < h_b) {
                const double sigma = d_run / h_b;
                const double g_shape = sigma * (1.0 - sigma) * (1.0 - sigma);
                const double gamma_factor = cs * g_shape;
                gT = gamma_factor * q_T_kin;
                gS = gamma_factor * q_S_kin;
            }
        }
        double fT = 0.0, fS = 0.0;
        if (do_nl) {
            double fT_up = 0.0, fT_dn = 0.0, fS_up = 0.0, fS_dn = 0.0;
            if (k < nz) {
                fT_up = nonlocal_face_flux(gT_above, h_c, h_a);
                fS_up = nonlocal_face_flux(gS_above, h_c, h_a);
            }
            if (k > 1) {
                fT_dn = nonlocal_face_flux(gT, h_b_layer, h_c);
                fS_dn = nonlocal_face_flux(gS, h_b_layer, h_c);
            }
            fT = dt * (fT_up - fT_dn);
            fS = dt * (fS_up - fS_dn);
        }
        const size_t off = P * (size_t)(k - 1);
#pragma unroll
        for (int t = 0; t < NTR; ++t) {
            if (t < ntr && (diffuse || t == iT || t == iS || t == iPS)) {
                double x;
                double x_old = trc[t][off];
                if (diffuse) {
                    const bool useA = !TWO || (t == iT);
                    const double cpk = useA ? cpA[k - 1] : cpB[TWO ? k - 1 : 0];
                    x = (k == nz) ? r[t][k - 1] : r[t][k - 1] - cpk * x_above[t];
                    x_above[t] = x;
                    if (t == iT && heat) {
                        const double p_new = h_c * x, p_old = h_c * x_old;
                        heat[off] = heat[off] + (p_new - p_old);
                    } else if (t == iS && salt) {
                        const double p_new = h_c * x, p_old = h_c * x_old;
                        salt[off] = salt[off] + (p_new - p_old);
                    }
                } else {
                    x = x_old;
                }
                if (do_nl) {
                    if (t == iT) x = conc_add_source(x, h_c, fT);
                    else if (t == iS || t == iPS) x = conc_add_source(x, h_c, fS);
                }
                trc[t][off] = x;
            }
        }
        gT_above = gT;
        gS_above = gS;
        h_a = h_c;
        h_c = h_b_layer;
    }
#undef HH
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

void launch_stress_mag(const Params &p, cudaStream_t stream)
{
    dim3 grid((p.nx + 127) / 128, p.ny);
    k_stress_mag<<<grid, 128, 0, stream>>>(p, const_cast<double *>(p.stress_mag));
}

void launch_assemble(const Params &p, cudaStream_t stream)
{
    dim3 grid((p.nx + ASM_THREADS - 1) / ASM_THREADS, p.ny);
    k_assemble<<<grid, ASM_THREADS, 0, stream>>>(p);
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

void launch_momentum(const Params &p, double dt, cudaStream_t stream)
{
    dim3 grid((p.nx + 1 + MOM_THREADS - 1) / MOM_THREADS, p.ny + 1);
    k_momentum<<<grid, MOM_THREADS, 0, stream>>>(p, dt);
}

template <int NTR>
static void launch_tracers_n(const Params &p, double dt, bool diffuse, bool nonlocal, cudaStream_t stream)
{
    dim3 grid((p.nx + TR_THREADS - 1) / TR_THREADS, p.ny);
    if (p.ks_equals_kt)
        k_tracers<NTR, false><<<grid, TR_THREADS, 0, stream>>>(p, dt, diffuse ? 1 : 0, nonlocal ? 1 : 0);
    else
        k_tracers<NTR, true><<<grid, TR_THREADS, 0, stream>>>(p, dt, diffuse ? 1 : 0, nonlocal ? 1 : 0);
}

void launch_tracers(const Params &p, double dt, bool diffuse, bool nonlocal, cudaStream_t stream)
{
    if (p.ntr <= 2)
        launch_tracers_n<2>(p, dt, diffuse, nonlocal, stream);
    else if (p.ntr <= 4)
        launch_tracers_n<4>(p, dt, diffuse, nonlocal, stream);
    else if (p.ntr <= 8)
        launch_tracers_n<8>(p, dt, diffuse, nonlocal, stream);
    else
        launch_tracers_n<16>(p, dt, diffuse, nonlocal, stream);
}

}  // namespace vphys
