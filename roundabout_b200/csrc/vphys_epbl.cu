// vphys_epbl.cu -- EPBL, the energetic planetary boundary layer (Reichl &
// Hallberg 2018), column form: epbl_compute -> epbl_column_kernel
// (src/parameterizations/vertical/rdb_ocean_epbl.F90:864-1659) with
// epbl_find_mstar (:630-688) and epbl_mixlen_shape (:690-714).
//
// One thread solves one column: the prep sweep (T0, S0 and the
// pressure-weighted potential-energy and column-height weights of each layer
// from the EOS derivatives), the surface energetics (B0, the convective
// release of the skin fluxes, u*, |f|), then up to epbl_mld_max_its
// mixed-layer-depth iterations, each a downward sweep that spends the
// wind and convective TKE on the largest diffusivity each interface can
// afford (closed-form energy solve with an embedded forward elimination) and
// moves the MLD guess (false position with a bisection fallback).  With
// shortwave penetration on (sw_pen_frac != 0) the prep also costs each
// layer's absorbed two-band heat (the TKE ledger of :1095-1185, opaque bed
// row k_bot = 1) and the sweep pays it (:1373-1425).  The column's nine
// per-layer arrays (h, the prep weights and the shortwave cost, 1-based,
// bottom-up as the reference stores them) live in the thread's local memory,
// sized by a compile-time bucket of nz.  Every value is formed by the same
// operations in the same order as the reference; built with -fmad=false it
// is bit-identical to the CPU restatement.
#include <cuda_runtime.h>

#include "vphys_device.cuh"
#include "vphys_kernels.cuh"

namespace vphys {
namespace {

constexpr double H_NEGLECT = H_DIV_EPS;   // rdb_ocean_epbl.F90:172-178

// eos_specvol_derivs (rdb_eos.F90:1551-1622)
__device__ __forceinline__ void specvol_derivs(const vphys_config &c, double T, double S, double pres, double &dsv_dt,
                                               double &dsv_ds)
{
    if (c.eos_variant == 1) {
        dsv_dt = xdiv(c.eos_alpha_t, c.rho0 * c.rho0);
        dsv_ds = xdiv(-c.eos_beta_s, c.rho0 * c.rho0);
        return;
    }
    const double T_sq = T * T;
    const double p_0 = WRIGHT_B0 + WRIGHT_B1 * T + WRIGHT_B2 * T_sq + WRIGHT_B3 * T_sq * T + WRIGHT_B4 * S +
                       WRIGHT_B5 * S * T;
    const double lambda = WRIGHT_C0 + WRIGHT_C1 * T + WRIGHT_C2 * T_sq + WRIGHT_C3 * T_sq * T + WRIGHT_C4 * S +
                          WRIGHT_C5 * S * T;
    const double dp0_dt = WRIGHT_B1 + 2.0 * WRIGHT_B2 * T + 3.0 * WRIGHT_B3 * T_sq + WRIGHT_B5 * S;
    const double dlam_dt = WRIGHT_C1 + 2.0 * WRIGHT_C2 * T + 3.0 * WRIGHT_C3 * T_sq + WRIGHT_C5 * S;
    const double dp0_ds = WRIGHT_B4 + WRIGHT_B5 * T;
    const double dlam_ds = WRIGHT_C4 + WRIGHT_C5 * T;
    const double big_p = pres + p_0;
    const double inv_p = 1.0 / big_p;
    const double inv_p2 = inv_p * inv_p;
    dsv_dt = WRIGHT_A1 + dlam_dt * inv_p - lambda * dp0_dt * inv_p2;
    dsv_ds = WRIGHT_A2 + dlam_ds * inv_p - lambda * dp0_ds * inv_p2;
}

// the RH18 fit (rdb_ocean_epbl.F90:664-670)
__device__ __noinline__ double rh18_mstar(const vphys_config &c, double b0, double ustar, double bld, double absf,
                                          double absf_floor)
{
    const double msn_term = c.epbl_rh18_cn2 * sm_exp(xdiv(c.epbl_rh18_cn3 * bld * absf, ustar));
    const double mstar_n = xdiv(c.epbl_rh18_cn1 * msn_term, 1.0 + msn_term);
    const double b0p = fmx(0.0, b0);
    const double u5 = (ustar * ustar) * (ustar * ustar) * ustar;
    const double mstar_s = c.epbl_rh18_cs1 * sm_pow(xdiv(b0p * b0p * bld, u5 * absf_floor), c.epbl_rh18_cs2);
    double mstar = mstar_n + mstar_s;
    if (c.epbl_mstar_cap > 0.0) mstar = fmn(c.epbl_mstar_cap, mstar);
    return mstar;
}

// fr^n for the mixing-length shape when n != 2
__device__ __noinline__ double shape_pow(double fr, double n) { return sm_pow(fr, n); }

// epbl_find_mstar: constant (1), OM4 (2), RH18 (3)
__device__ __forceinline__ double find_mstar(const vphys_config &c, double b0, double ustar, double bld, double absf)
{
    double mstar;
    const double absf_floor = fmx(absf, 1.0e-20);
    if (c.epbl_mstar_scheme == 2) {
        const double mstar_s = c.epbl_mstar_coef1 * sqrt(xdiv(fmx(0.0, b0), ustar * ustar * absf_floor));
        double mstar_n = 0.0;
        if (ustar > absf_floor * bld) mstar_n = c.epbl_c_ek * sm_log(xdiv(ustar, absf_floor * fmx(bld, 1.0e-10)));
        mstar = fmx(mstar_s, fmn(1.25, mstar_n));
        if (c.epbl_mstar_cap > 0.0) mstar = fmn(c.epbl_mstar_cap, mstar);
    } else if (c.epbl_mstar_scheme == 3) {
        mstar = rh18_mstar(c, b0, ustar, bld, absf, absf_floor);
    } else {
        mstar = c.epbl_mstar_const;
    }
    if (c.epbl_mstar_conv_adj > 0.0) {
        const double t1 = -bld * fmn(0.0, b0);
        const double t2 = 2.0 * mstar * (ustar * ustar * ustar);
        if (t2 > 0.0)
            mstar = xdiv(mstar * ((1.0 - c.epbl_mstar_conv_adj) * t1 + t2), t1 + t2);
        else
            mstar = mstar * (1.0 - c.epbl_mstar_conv_adj);
    }
    return mstar;
}

// ---- Langmuir enhancement, LF17 wind-only path (rdb_ocean_epbl.F90:716-862);
// the empirical constants of the cited formulas (Li & Fox-Kemper 2017,
// COARE 3.5), as the reference lists them at :59-71
// epbl_lf17_wave_state: COARE fixed-point u* -> U10, Stokes drift, Phillips peak wavenumber
// The Langmuir, RH18 and general-exponent paths are off by default; they are
// kept out of line so that their registers do not weigh on the default sweep.
__device__ __noinline__ void lf17_wave_state(double ustar_w, double rho_ocn, double &ustokes, double &kphil)
{
    const double ustar_air = ustar_w * sqrt(xdiv(rho_ocn, 1.225));
    const double z0_smooth = xdiv(0.11 * 1.0e-6, ustar_air);
    double u = ustar_air * sqrt(1000.0);
    bool converged = false;
    for (int itt = 1; itt <= 20; ++itt) {
        const double alpha_ch = fmn(0.028, 0.0017 * u + -0.005);
        const double z0w = fmx(z0_smooth + xdiv(alpha_ch * (ustar_air * ustar_air), GRAVITY), 1.0e-10);
        const double u_new = xdiv(ustar_air * sm_log(xdiv(10.0, z0w)), 0.40);
        if (fabs(u_new - u) <= 1.0e-3 * u) {
            u = u_new;
            converged = true;
            break;
        }
        u = u_new;
    }
    if (!converged) u = 25.82 * ustar_air;
    ustokes = 0.0162 * u;
    const double hm0 = 0.0246 * u * u;
    const double f_mean = xdiv(1.296 * 0.877 * GRAVITY, 2.0 * PI_D * 1.075 * u);
    const double vstokes = 0.125 * PI_D * 0.667 * f_mean * hm0 * hm0;
    kphil = xdiv(0.176 * ustokes, fmx(vstokes, 1.0e-30));
}

// one_m_exp_x: (1 - exp(-x))/x, a series below 1e-4
__device__ __forceinline__ double one_m_exp_x(double x)
{
    if (x < 1.0e-4) return 1.0 - x * (0.5 - xdiv(x, 6.0));
    return xdiv(1.0 - sm_exp(-x), x);
}

// epbl_lf17_la: the Langmuir number of the Stokes drift averaged over zsl
__device__ __noinline__ double lf17_la(double ustar_w, double zsl, double ustokes, double kphil)
{
    const double xkz = kphil * zsl;
    const double root2kz = sqrt(2.0 * xkz);
    const double r1 = (0.302 - 1.68 * xkz) * one_m_exp_x(2.0 * xkz);
    const double r3 = (0.1264 + 0.64 * xkz) * one_m_exp_x(5.12 * xkz);
    const double sqrt_pi = sqrt(PI_D);
    double r5;
    if (root2kz > 1.0e-3) {
        const double ec1 = sm_erfc(root2kz);
        const double ec2 = sm_erfc(1.6 * root2kz);
        r5 = sqrt_pi * (root2kz * (-0.84 * ec1 + 0.2 * ec2) + xdiv(0.1182 * (ec2 - ec1), root2kz));
    } else {
        r5 = -0.64 * sqrt_pi * root2kz + (-0.14184 + 1.0839648 * root2kz * root2kz);
    }
    const double ustokes_sl = fmx(ustokes * (0.715 + r1 + r3 + r5), 1.0e-10);
    return sqrt(xdiv(ustar_w, ustokes_sl));
}

// epbl_lt_enhance: La modified by the Ekman and Obukhov depth ratios, then
// mstar rescaled (capped) or incremented
__device__ __noinline__ double lt_enhance(const vphys_config &c, double la, double b0, double ustar, double bld,
                                          double absf, double mstar)
{
    const double vonkar = c.epbl_von_karman;
    const double mld_ek = xdiv(bld * absf, ustar);
    const double ek_ob = xdiv(fabs(b0 * vonkar), fmx(absf, 1.0e-20) * ustar * ustar);
    const double mld_ob = xdiv(fabs(bld * b0 * vonkar), ustar * ustar * ustar);
    const double lac_ek = (b0 >= 0.0) ? c.epbl_lt_lac4 : c.epbl_lt_lac5;
    const double lac_ob = (b0 >= 0.0) ? c.epbl_lt_lac2 : c.epbl_lt_lac3;
    double la_mod = la * ((1.0 + fmx(-0.5, c.epbl_lt_lac1 * mld_ek)) + lac_ek * ek_ob + lac_ob * mld_ob);
    la_mod = fmx(la_mod, 1.0e-10);
    if (c.epbl_lt_scheme == 2) return mstar + c.epbl_lt_enhance_coef * sm_pow(la_mod, c.epbl_lt_enhance_exp);
    return mstar * fmn(c.epbl_lt_max_enhance, 1.0 + c.epbl_lt_enhance_coef * sm_pow(la_mod, c.epbl_lt_enhance_exp));
}

// sw_pe_cost_shape (rdb_ocean_surface_flux.F90:1417-1449): the share of the
// skin PE cost that homogenising an exponential in-layer heating of optical
// depth tau incurs; Taylor branch below tau = 1e-2
__device__ __forceinline__ double sw_pe_cost_shape(double tau)
{
    if (tau <= 1.0e-2) return (1.0 / 6.0) * tau * (1.0 - (1.0 / 60.0) * tau * tau);
    const double em1 = 1.0 - sm_exp(-tau);
    return xdiv(tau * (1.0 + sm_exp(-tau)) - 2.0 * em1, tau * em1);
}

// The chlorophyll N-band ledger of one live layer (rdb_ocean_epbl.F90:
// 1143-1164): per band the heat absorbed between the layer's top and bottom
// (the bed opaque), weighted by the PE-cost shape at the band's optical depth.
static __device__ __noinline__ double sw_phi_nb(double i0, const double *kap, size_t col, size_t plane, int nb, double blue,
                                                double inv_rho0_cp, double dt, double d_top, double d_bot, double hk,
                                                bool bed)
{
    double phi_sum = 0.0;
    for (int n = 1; n <= nb; ++n) {
        const double kn = kap[col + (size_t)(n - 1) * plane];
        const double ea = sm_exp(-(kn * d_top));
        const double eb = bed ? 0.0 : sm_exp(-(kn * d_bot));
        const double heat_nb = i0 * sw_band_frac(n, nb, blue) * inv_rho0_cp * dt * (ea - eb);
        phi_sum = phi_sum + heat_nb * sw_pe_cost_shape(hk * kn);
    }
    return phi_sum;
}

// the turbulent velocity scale (cube root of the TKE rate, or RH18)
__device__ __forceinline__ double vstar_of(const vphys_config &c, double tke_here, double conv_perel, double ustar,
                                           double htot, double mld_guess, double dt)
{
    if (c.epbl_vstar_scheme == 2) {
        const double surf_scale = fmx(0.05, 1.0 - xdiv(htot, mld_guess));
        return c.epbl_vstar_scale_fac * surf_scale *
               (c.epbl_vstar_surf_fac * ustar + sm_cbrt(xdiv(c.epbl_wstar_ustar_coef * conv_perel, dt * c.rho0)));
    }
    return c.epbl_vstar_scale_fac * sm_cbrt(xdiv(tke_here, dt * c.rho0));
}

// the Ekman-limited mixing length times v* kappa
__device__ __forceinline__ double mixlen_kd(const vphys_config &c, double vstar, double htot, double hbs, double absf)
{
    const double num = htot * hbs * vstar;
    const double den = c.epbl_ekman_scale_coef * absf * htot * hbs + vstar;
    if (c.epbl_mld_iteration) return vstar * c.epbl_von_karman * fmx(c.epbl_min_mix_len, xdiv(num, den));
    return xdiv(vstar * c.epbl_von_karman * num, den);
}

// N = bucket + 2 (indices 1..nz+1 with nz <= bucket); DIAG: the TKE budget
// is kept and written (epbl_tke_diags), else its sums are dead code
template <int N, bool DIAG>
__global__ void __launch_bounds__(128, 4) k_epbl(const Params p, double dt, double inv_rho0_cp, double inv_rho0)
{
    const size_t col = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (col >= p.plane) return;
    const vphys_config &c = p.cfg;
    const int nz = p.nz;
    const size_t P = p.plane;
    const double rho0 = c.rho0;
    const double g_rho0 = GRAVITY * rho0;
    double *kdg = p.kd_epbl + col;
    const double *T = p.tr[c.idx_temperature] + col;
    const double *S = p.tr[c.idx_salinity] + col;

    double h[N], t0[N], s0[N], dpe_t[N], dpe_s[N], dch_t[N], dch_s[N], kd[N], ctke_sw[N];
    const bool sw_on = c.epbl_sw_ctke && c.sw_pen_frac != 0.0;
    const double i0_col = sw_on ? c.sw_pen_frac * p.sw_src[col] * p.wet[col] : 0.0;
    double d_top_sw = 0.0, e1_top = 1.0, e2_top = 1.0;
    int k_sfc = nz;   // first live layer from the top (nz when none is live)
    for (int k = nz; k >= 1; --k) {
        h[k] = p.h[col + P * (size_t)(k - 1)];
    }
    for (int k = nz; k >= 1; --k)
        if (h[k] > H_VANISHED) {
            k_sfc = k;
            break;
        }
    // ---- column prep (downward)
    double pres = 0.0, h_sum = 0.0, dsv_dt_sfc = 0.0, dsv_ds_sfc = 0.0;
    for (int k = nz; k >= 1; --k) {
        const double hk = h[k];
        double t0k = 0.0, s0k = 0.0;
        if (hk > 0.0) {
            t0k = T[P * (size_t)(k - 1)];
            s0k = S[P * (size_t)(k - 1)];
        }
        const double dmass = rho0 * hk;
        const double dpres = GRAVITY * dmass;
        const double p_mid = pres + 0.5 * dpres;
        double dsv_dt_k, dsv_ds_k;
        specvol_derivs(c, t0k, s0k, p_mid, dsv_dt_k, dsv_ds_k);
        t0[k] = t0k;
        s0[k] = s0k;
        dpe_t[k] = dmass * p_mid * dsv_dt_k;
        dpe_s[k] = dmass * p_mid * dsv_ds_k;
        dch_t[k] = dmass * dsv_dt_k;
        dch_s[k] = dmass * dsv_ds_k;
        if (k > k_sfc || !sw_on) {
            ctke_sw[k] = 0.0;   // dead layers above the live surface take no light
        } else if (c.sw_chl) {
            const double d_bot_sw = d_top_sw + hk;
            ctke_sw[k] = -0.5 * GRAVITY * rho0 * dch_t[k] *
                         sw_phi_nb(i0_col, p.sw_kappa, col, P, c.sw_nbands, c.sw_blue_frac, inv_rho0_cp, dt,
                                   d_top_sw, d_bot_sw, hk, k == 1);
            d_top_sw = d_bot_sw;
        } else {
            const double d_bot_sw = d_top_sw + hk;
            double heat_sw1, heat_sw2;
            if (k > 1) {
                const double e1_bot = sm_exp(xdiv(-d_bot_sw, c.sw_zeta1));
                const double e2_bot = sm_exp(xdiv(-d_bot_sw, c.sw_zeta2));
                heat_sw1 = i0_col * c.sw_band_ratio * inv_rho0_cp * dt * (e1_top - e1_bot);
                heat_sw2 = i0_col * (1.0 - c.sw_band_ratio) * inv_rho0_cp * dt * (e2_top - e2_bot);
                e1_top = e1_bot;
                e2_top = e2_bot;
            } else {   // opaque bed: the rest of the light
                heat_sw1 = i0_col * c.sw_band_ratio * inv_rho0_cp * dt * e1_top;
                heat_sw2 = i0_col * (1.0 - c.sw_band_ratio) * inv_rho0_cp * dt * e2_top;
            }
            ctke_sw[k] = -0.5 * GRAVITY * rho0 * dch_t[k] *
                         (heat_sw1 * sw_pe_cost_shape(xdiv(hk, c.sw_zeta1)) +
                          heat_sw2 * sw_pe_cost_shape(xdiv(hk, c.sw_zeta2)));
            d_top_sw = d_bot_sw;
        }
        if (k == k_sfc) {
            dsv_dt_sfc = dsv_dt_k;
            dsv_ds_sfc = dsv_ds_k;
        }
        if (k <= k_sfc) {
            pres = pres + dpres;
            h_sum = h_sum + hk;
        }
    }
    h_sum = h_sum + H_NEGLECT;

    // ---- surface forcing energetics
    const double q_t_kin = inv_rho0_cp * p.q_heat[col];
    const double q_s_kin = inv_rho0 * p.q_salt[col];
    const double b0 = g_rho0 * (dsv_dt_sfc * q_t_kin + dsv_ds_sfc * q_s_kin);
    // the skin carries the non-penetrating heat when the shortwave is charged per layer
    const double q_skin_kin = sw_on ? inv_rho0_cp * (p.q_heat[col] - i0_col) : q_t_kin;
    double ctke_sfc =
        -0.5 * GRAVITY * (rho0 * rho0) * h[k_sfc] * (q_skin_kin * dt * dsv_dt_sfc + q_s_kin * dt * dsv_ds_sfc);
    if (sw_on) ctke_sfc = ctke_sfc + ctke_sw[k_sfc];
    const double ustar = fmx(sqrt(xdiv(p.stress_mag[col], rho0)), c.epbl_ustar_min);
    const double f = p.coriolis ? p.coriolis[col] : 0.0;
    const double absf = sqrt((1.0 - c.epbl_omega_frac) * (f * f) + c.epbl_omega_frac * 4.0 * (c.epbl_omega * c.epbl_omega));
    const double idecay = xdiv(c.epbl_tke_decay * absf, ustar);
    const double mech_in = dt * rho0 * (ustar * ustar * ustar);
    // the LF17 wave state depends on u* alone: once per column
    double la_val = 0.0, lt_ustokes = 0.0, lt_kphil = 0.0;
    if (c.epbl_use_lt) lf17_wave_state(ustar, rho0, lt_ustokes, lt_kphil);

    double mld_found = 0.0;
    // the TKE budget of the last MLD iteration (:1641-1654), kept when asked for
    double d_wind = 0.0, d_conv = 0.0, d_forcing = 0.0, d_mixing = 0.0, d_mdecay = 0.0, d_cdecay = 0.0;
    if (p.wet[col] <= 0.0 || h_sum <= 2.0 * H_NEGLECT) {
        for (int k = 1; k <= nz + 1; ++k) kd[k] = 0.0;
    } else {
        double min_mld = 0.0, max_mld = h_sum, dmld_min = 0.0, dmld_max = 0.0;
        bool have_min = false, have_max = false;
        double mld_guess = 0.5 * (min_mld + max_mld);
        if (c.epbl_mld_use_prev_guess && p.mld_epbl[col] > 0.0) mld_guess = fmn(p.mld_epbl[col], max_mld);
        const int n_its = c.epbl_mld_iteration ? c.epbl_mld_max_its : 1;
        double dt_h = 0.0;   // carried from interface to interface, as the reference's local
        for (int obl_it = 1; obl_it <= n_its; ++obl_it) {
            d_wind = d_conv = d_forcing = d_mixing = d_mdecay = d_cdecay = 0.0;
            double mstar_val = find_mstar(c, b0, ustar, mld_guess, absf);
            if (c.epbl_use_lt) {
                la_val = lf17_la(ustar, c.epbl_la_frac_hbl * mld_guess, lt_ustokes, lt_kphil);
                mstar_val = lt_enhance(c, la_val, b0, ustar, mld_guess, absf, mstar_val);
            }
            double mech_tke = mstar_val * mech_in;
            d_wind = mech_tke;
            double conv_perel;
            if (ctke_sfc <= 0.0) {
                const double forcing_clip = fmx(ctke_sfc, -mech_tke);
                mech_tke = mech_tke + forcing_clip;
                conv_perel = 0.0;
                d_forcing = forcing_clip;
            } else {
                conv_perel = ctke_sfc;
                d_conv = c.epbl_nstar * ctke_sfc;
            }
            double h_ka = h[k_sfc] + H_NEGLECT;
            double hp_a = h_ka;
            double dpe_t_a = dpe_t[k_sfc], dpe_s_a = dpe_s[k_sfc], dch_t_a = dch_t[k_sfc], dch_s_a = dch_s[k_sfc];
            double th_a = h_ka * t0[k_sfc], sh_a = h_ka * s0[k_sfc];
            double te_lag = 0.0, se_lag = 0.0, kddt_prev = 0.0;
            double htot = h[k_sfc], z_int = h[k_sfc], pres_int = g_rho0 * h[k_sfc], mld_output = h[k_sfc];
            bool sfc_connected = true;
            for (int ki = k_sfc + 1; ki <= nz + 1; ++ki) kd[ki] = 0.0;

            for (int ki = k_sfc; ki >= 2; --ki) {
                const int ka = ki, kb = ki - 1;
                h_ka = h[ka] + H_NEGLECT;
                const double h_kb = h[kb] + H_NEGLECT;
                bool sfc_disconnect = false;
                const double exp_kh = sm_exp(-h_ka * idecay);
                d_mdecay = d_mdecay + (1.0 - exp_kh) * mech_tke;
                mech_tke = mech_tke * exp_kh;
                // the layer below accrues its shortwave cost; a release joins the convective reservoir
                const double ctke_sw_kb = ctke_sw[kb];
                if (ctke_sw_kb > 0.0) {
                    conv_perel = conv_perel + ctke_sw_kb;
                    d_conv = d_conv + c.epbl_nstar * ctke_sw_kb;
                }
                double nstar_fc = c.epbl_nstar;
                if (conv_perel > 0.0 && absf > 0.0) {
                    const double ah = absf * htot;
                    nstar_fc = xdiv(c.epbl_nstar * conv_perel,
                                    conv_perel + 0.2 * sqrt(0.5 * dt * rho0 * (ah * ah * ah) * conv_perel));
                }
                double tot_tke = mech_tke + nstar_fc * conv_perel;
                // a shortwave sink is paid first, both reservoirs drained in proportion
                if (ctke_sw_kb < 0.0) {
                    if (ctke_sw_kb + tot_tke < 0.0) {
                        d_mixing = d_mixing + tot_tke;
                        d_cdecay = d_cdecay + (c.epbl_nstar - nstar_fc) * conv_perel;
                        tot_tke = 0.0;
                        mech_tke = 0.0;
                        conv_perel = 0.0;
                    } else {
                        const double r_sw = xdiv(tot_tke + ctke_sw_kb, tot_tke);
                        d_mixing = d_mixing - ctke_sw_kb;
                        d_cdecay = d_cdecay + (1.0 - r_sw) * (c.epbl_nstar - nstar_fc) * conv_perel;
                        tot_tke = r_sw * tot_tke;
                        mech_tke = r_sw * mech_tke;
                        conv_perel = r_sw * conv_perel;
                    }
                }
                double kd_val;
                if (tot_tke <= 0.0 &&
                    0.0 <= (dch_t[kb] + dch_t[ka]) * (t0[ka] - t0[kb]) + (dch_s[kb] + dch_s[ka]) * (s0[ka] - s0[kb])) {
                    kd_val = 0.0;
                    sfc_disconnect = true;
                } else {
                    dt_h = xdiv(dt, fmx(0.5 * (h_ka + h_kb), 1.0e-15 * h_sum));
                    double tke_here = mech_tke + c.epbl_wstar_ustar_coef * conv_perel;
                    const double hb_hs = xdiv(h_sum - z_int, h_sum);
                    double shape_fn = 1.0;
                    {
                        const double ts = c.epbl_translay_scale;
                        if (c.epbl_mld_iteration && !(ts >= 1.0) && !(ts < 0.0) && !(mld_guess <= 0.0)) {
                            const double fr = fmx(0.0, xdiv(mld_guess - z_int, mld_guess));
                            shape_fn = (c.epbl_mixlen_exponent == 2.0) ? ts + (1.0 - ts) * fr * fr
                                                                       : ts + (1.0 - ts) * shape_pow(fr, c.epbl_mixlen_exponent);
                        }
                    }
                    const double hbs = fmn(hb_hs, shape_fn);
                    double kd_g0 = 0.0;
                    if (tke_here > 0.0) kd_g0 = mixlen_kd(c, vstar_of(c, tke_here, conv_perel, ustar, htot, mld_guess, dt),
                                                          htot, hbs, absf);
                    const double hp_b = h_kb;
                    const double th_b = h_kb * t0[kb];
                    const double sh_b = h_kb * s0[kb];
                    const double hps = hp_a + hp_b;
                    const double bdt1 = hp_a * hp_b;
                    const double dt_c = hp_a * th_b - hp_b * th_a;
                    const double ds_c = hp_a * sh_b - hp_b * sh_a;
                    double pec_core =
                        hp_b * (dpe_t_a * dt_c + dpe_s_a * ds_c) - hp_a * (dpe_t[kb] * dt_c + dpe_s[kb] * ds_c);
                    const double colht_core =
                        hp_b * (dch_t_a * dt_c + dch_s_a * ds_c) - hp_a * (dch_t[kb] * dt_c + dch_s[kb] * ds_c);
                    if (colht_core < 0.0) pec_core = pec_core - pres_int * colht_core;
                    const double dkddt = kd_g0 * dt_h;
                    const double pe_max = xdiv(pec_core, bdt1 * hps);
                    if (pe_max < 0.0) {
                        // convectively unstable: the Kd of the mixing length, the release banked
                        tke_here = mech_tke + c.epbl_wstar_ustar_coef * (conv_perel - pe_max);
                        if (tke_here > 0.0)
                            kd_val = mixlen_kd(c, vstar_of(c, tke_here, conv_perel, ustar, htot, mld_guess, dt), htot,
                                               hbs, absf);
                        else
                            kd_val = 0.0;
                        const double pe_g0 = xdiv(pec_core * dkddt, bdt1 * (bdt1 + dkddt * hps));
                        double dpe_conv = xdiv(pec_core * (kd_val * dt_h), bdt1 * (bdt1 + (kd_val * dt_h) * hps));
                        if (dpe_conv > 0.0) {
                            kd_val = kd_g0;
                            dpe_conv = pe_g0;
                        }
                        conv_perel = conv_perel - dpe_conv;
                        d_conv = d_conv - c.epbl_nstar * dpe_conv;
                        if (sfc_connected) mld_output = mld_output + h[kb];
                    } else {
                        // stable: the energy-limited Kd; the reservoirs drained
                        double tke_used, frac_bl;
                        if ((pec_core * dkddt <= tot_tke * (bdt1 * (bdt1 + dkddt * hps))) || (pec_core <= 0.0)) {
                            kd_val = kd_g0;
                            tke_used = xdiv(pec_core * dkddt, bdt1 * (bdt1 + dkddt * hps));
                            frac_bl = 1.0;
                        } else {
                            kd_val = xdiv(bdt1 * bdt1 * tot_tke, dt_h * (pec_core - bdt1 * hps * tot_tke));
                            tke_used = tot_tke;
                            frac_bl = xdiv(tot_tke * (bdt1 * (bdt1 + dkddt * hps)), pec_core * dkddt);
                        }
                        if (sfc_connected) mld_output = mld_output + frac_bl * h[kb];
                        if (frac_bl < 1.0) sfc_disconnect = true;
                        double r_reduc = 0.0;
                        if (tot_tke > 0.0 && tot_tke > tke_used) r_reduc = xdiv(tot_tke - tke_used, tot_tke);
                        d_mixing = d_mixing + tke_used;
                        d_cdecay = d_cdecay + (1.0 - r_reduc) * (c.epbl_nstar - nstar_fc) * conv_perel;
                        mech_tke = r_reduc * mech_tke;
                        conv_perel = r_reduc * conv_perel;
                    }
                }
                kd[ki] = kd_val;
                const double kddt_cur = kd_val * dt_h;
                const double b1 = 1.0 / (hp_a + kddt_cur);
                const double c1 = kddt_cur * b1;
                if (ki == k_sfc) {
                    te_lag = b1 * (h_ka * t0[ka]);
                    se_lag = b1 * (h_ka * s0[ka]);
                } else {
                    const double te_new = b1 * (h_ka * t0[ka] + kddt_prev * te_lag);
                    const double se_new = b1 * (h_ka * s0[ka] + kddt_prev * se_lag);
                    te_lag = te_new;
                    se_lag = se_new;
                }
                hp_a = h_kb + (hp_a * b1) * kddt_cur;
                dpe_t_a = dpe_t[kb] + c1 * dpe_t_a;
                dpe_s_a = dpe_s[kb] + c1 * dpe_s_a;
                dch_t_a = dch_t[kb] + c1 * dch_t_a;
                dch_s_a = dch_s[kb] + c1 * dch_s_a;
                th_a = h_kb * t0[kb] + kddt_cur * te_lag;
                sh_a = h_kb * s0[kb] + kddt_cur * se_lag;
                kddt_prev = kddt_cur;
                if (sfc_disconnect) {
                    htot = h[kb];
                    sfc_connected = false;
                } else {
                    htot = htot + h[kb];
                }
                z_int = z_int + h[kb];
                pres_int = pres_int + g_rho0 * h[kb];
            }
            kd[1] = 0.0;
            d_mdecay = d_mdecay + mech_tke;   // the stocks left at the bed count as dissipated
            d_cdecay = d_cdecay + c.epbl_nstar * conv_perel;
            mld_found = mld_output;
            if (!c.epbl_mld_iteration) break;
            if (fabs(mld_found - mld_guess) < c.epbl_mld_tol) break;
            if (obl_it == n_its) break;
            if (mld_found > mld_guess) {
                min_mld = mld_guess;
                dmld_min = mld_found - mld_guess;
                have_min = true;
            } else {
                max_mld = mld_guess;
                dmld_max = mld_found - mld_guess;
                have_max = true;
            }
            if (c.epbl_mld_bisection)
                mld_guess = 0.5 * (min_mld + max_mld);
            else if (have_min && have_max && obl_it > 2 && (obl_it - 1) % 4 > 0)
                mld_guess = min_mld + xdiv(dmld_min * (max_mld - min_mld), dmld_min - dmld_max);
            else if (mld_found > min_mld && mld_found < max_mld)
                mld_guess = mld_found;
            else
                mld_guess = 0.5 * (min_mld + max_mld);
        }
    }
    for (int k = 1; k <= nz + 1; ++k) kdg[P * (size_t)(k - 1)] = kd[k];
    p.mld_epbl[col] = mld_found;
    if (p.la_epbl) p.la_epbl[col] = la_val;
    if (DIAG && p.epbl_tke[0]) {
        p.epbl_tke[0][col] = xdiv(d_wind, dt);
        p.epbl_tke[1][col] = xdiv(d_conv, dt);
        p.epbl_tke[2][col] = xdiv(d_forcing, dt);
        p.epbl_tke[3][col] = xdiv(d_mixing, dt);
        p.epbl_tke[4][col] = xdiv(d_mdecay, dt);
        p.epbl_tke[5][col] = xdiv(d_cdecay, dt);
    }
}

}  // namespace

void launch_epbl(const Params &p, double dt, cudaStream_t stream)
{
    // the column-invariant multipliers, divided on the host in IEEE double
    // (epbl_compute passes 1/(rho0 cp) and 1/rho0, rdb_ocean_epbl.F90:906-927)
    const double inv_rho0_cp = 1.0 / (p.cfg.rho0 * p.cfg.cp);
    const double inv_rho0 = 1.0 / p.cfg.rho0;
    const int threads = 128;
    const unsigned blocks = (unsigned)((p.plane + threads - 1) / threads);
    const bool diag = p.cfg.epbl_tke_diags != 0;
#define VPHYS_EPBL_LAUNCH(NB)                                                                        \
    if (diag)                                                                                        \
        k_epbl<NB, true><<<blocks, threads, 0, stream>>>(p, dt, inv_rho0_cp, inv_rho0);              \
    else                                                                                             \
        k_epbl<NB, false><<<blocks, threads, 0, stream>>>(p, dt, inv_rho0_cp, inv_rho0)
    if (p.nz <= 32) {
        VPHYS_EPBL_LAUNCH(34);
    } else if (p.nz <= 80) {
        VPHYS_EPBL_LAUNCH(82);
    } else {
        VPHYS_EPBL_LAUNCH(NZ_MAX + 2);
    }
#undef VPHYS_EPBL_LAUNCH
}

}  // namespace vphys
