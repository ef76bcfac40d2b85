/* vphys_oracle_epbl.c -- EPBL (energetic planetary boundary layer; Reichl &
 * Hallberg 2018, Ocean Modelling 132, 112-129), column form: CPU FP64
 * restatement of src/parameterizations/vertical/rdb_ocean_epbl.F90.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of vphys_epbl (see vphys_oracle.h).
 * Built scope: the mstar schemes "constant", "om4" and "rh18", the cube-root
 * and RH18 velocity scales, the MLD iteration (false position / bisection,
 * optionally seeded by the previous MLD), the mixing-length shape, the two-band penetrating-shortwave TKE ledger (on whenever
 * sw_pen_frac != 0, source Q_heat, bed row k_bot = 1), and the three merges
 * (add, max, max_shear), the LF17 Langmuir enhancement of mstar and the TKE
 * budget diagnostics.
 *
 * Parity pins: the analytic and structural tests of the reference's
 * tests/test_ocean_epbl.F90 re-expressed in tests/test_oracle_epbl.py, and
 * the safe-math exp / log / cbrt the column uses, pinned to the reference's
 * golden bits (tests/test_oracle_safe_math.py).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "vphys_oracle.h"

static const double GRAVITY = 9.80665;   /* rdb_constants.F90:37 */
static const double H_VANISHED = 1.5e-4;
static const double H_NEGLECT = 1.0e-20; /* H_DIV_EPS */

#define C3(a, i, j, k) (a)[((size_t)(i) - 1) + (size_t)nx * (((size_t)(j) - 1) + (size_t)ny * ((size_t)(k) - 1))]
#define C2(a, i, j) (a)[((size_t)(i) - 1) + (size_t)nx * ((size_t)(j) - 1)]

static inline double fmx(double a, double b) { return a > b ? a : b; }
static inline double fmn(double a, double b) { return a < b ? a : b; }

/* Wright (1997) constants (rdb_eos.F90:200-217) */
#define W_A1 3.480336e-7
#define W_A2 -1.112733e-7
#define W_B0 5.790749e8
#define W_B1 3.516535e6
#define W_B2 -4.002714e4
#define W_B3 2.084372e2
#define W_B4 5.944068e5
#define W_B5 -9.643486e3
#define W_C0 1.704853e5
#define W_C1 7.904722e2
#define W_C2 -7.984422e0
#define W_C3 5.140652e-2
#define W_C4 -2.302158e2
#define W_C5 -3.079464e0

/* eos_specvol_derivs (rdb_eos.F90:1551-1622) */
static void specvol_derivs(const vphys_config *c, double T, double S, double pres, double *dsv_dt, double *dsv_ds)
{
    if (c->eos_variant == 1) {
        *dsv_dt = c->eos_alpha_t / (c->rho0 * c->rho0);
        *dsv_ds = -c->eos_beta_s / (c->rho0 * c->rho0);
        return;
    }
    double T_sq = T * T;
    double p_0 = W_B0 + W_B1 * T + W_B2 * T_sq + W_B3 * T_sq * T + W_B4 * S + W_B5 * S * T;
    double lambda = W_C0 + W_C1 * T + W_C2 * T_sq + W_C3 * T_sq * T + W_C4 * S + W_C5 * S * T;
    double dp0_dt = W_B1 + 2.0 * W_B2 * T + 3.0 * W_B3 * T_sq + W_B5 * S;
    double dlam_dt = W_C1 + 2.0 * W_C2 * T + 3.0 * W_C3 * T_sq + W_C5 * S;
    double dp0_ds = W_B4 + W_B5 * T;
    double dlam_ds = W_C4 + W_C5 * T;
    double big_p = pres + p_0;
    double inv_p = 1.0 / big_p;
    double inv_p2 = inv_p * inv_p;
    *dsv_dt = W_A1 + dlam_dt * inv_p - lambda * dp0_dt * inv_p2;
    *dsv_ds = W_A2 + dlam_ds * inv_p - lambda * dp0_ds * inv_p2;
}

/* epbl_find_mstar (rdb_ocean_epbl.F90:630-688): constant, OM4, RH18 */
static double find_mstar(const vphys_config *c, double b0, double ustar, double bld, double absf)
{
    double mstar;
    const double absf_floor = fmx(absf, 1.0e-20);
    if (c->epbl_mstar_scheme == 2) {
        double mstar_s = c->epbl_mstar_coef1 * sqrt(fmx(0.0, b0) / (ustar * ustar * absf_floor));
        double mstar_n = 0.0;
        if (ustar > absf_floor * bld)
            mstar_n = c->epbl_c_ek * vpo_sm_log(ustar / (absf_floor * fmx(bld, 1.0e-10)));
        mstar = fmx(mstar_s, fmn(1.25, mstar_n));
        if (c->epbl_mstar_cap > 0.0) mstar = fmn(c->epbl_mstar_cap, mstar);
    } else if (c->epbl_mstar_scheme == 3) {
        const double msn_term = c->epbl_rh18_cn2 * vpo_sm_exp(c->epbl_rh18_cn3 * bld * absf / ustar);
        const double mstar_n = c->epbl_rh18_cn1 * msn_term / (1.0 + msn_term);
        const double b0p = fmx(0.0, b0);
        const double u5 = (ustar * ustar) * (ustar * ustar) * ustar;
        const double mstar_s = c->epbl_rh18_cs1 * vpo_sm_pow(b0p * b0p * bld / (u5 * absf_floor), c->epbl_rh18_cs2);
        mstar = mstar_n + mstar_s;
        if (c->epbl_mstar_cap > 0.0) mstar = fmn(c->epbl_mstar_cap, mstar);
    } else {
        mstar = c->epbl_mstar_const;
    }
    if (c->epbl_mstar_conv_adj > 0.0) {
        const double t1 = -bld * fmn(0.0, b0);
        const double t2 = 2.0 * mstar * (ustar * ustar * ustar);
        if (t2 > 0.0)
            mstar = mstar * ((1.0 - c->epbl_mstar_conv_adj) * t1 + t2) / (t1 + t2);
        else
            mstar = mstar * (1.0 - c->epbl_mstar_conv_adj);
    }
    return mstar;
}

/* ---- Langmuir enhancement, LF17 wind-only path (rdb_ocean_epbl.F90:716-862).
 * The empirical constants are those of the cited formulas (Li & Fox-Kemper
 * 2017, COARE 3.5 of Edson et al. 2013), as the reference lists them at
 * :59-71. */
#define LT_VONKAR_WAVES 0.40
#define LT_NU_AIR 1.0e-6
#define LT_RHO_AIR 1.225
#define LT_CHARNOCK_MIN 0.028
#define LT_CHARNOCK_SLOPE 0.0017
#define LT_CHARNOCK_ICPT -0.005
#define LT_US_TO_U10 0.0162
#define LT_SWH_FROM_U10SQ 0.0246
#define LT_U19P5_TO_U10 1.075
#define LT_FM_INTO_FP 1.296
#define LT_R_LOSS 0.667
static const double LT_PI = 3.141592653589793115997963468544185161590576171875;

/* epbl_lf17_wave_state (:716-765): COARE fixed-point u* -> U10, then the
 * surface Stokes drift and the Phillips peak wavenumber */
static void lf17_wave_state(double ustar_w, double rho_ocn, double *u10, double *ustokes, double *kphil)
{
    const double ustar_air = ustar_w * sqrt(rho_ocn / LT_RHO_AIR);
    const double z0_smooth = 0.11 * LT_NU_AIR / ustar_air;
    double u = ustar_air * sqrt(1000.0);
    int converged = 0;
    for (int itt = 1; itt <= 20; ++itt) {
        const double alpha_ch = fmn(LT_CHARNOCK_MIN, LT_CHARNOCK_SLOPE * u + LT_CHARNOCK_ICPT);
        const double z0w = fmx(z0_smooth + alpha_ch * (ustar_air * ustar_air) / GRAVITY, 1.0e-10);
        const double u_new = ustar_air * vpo_sm_log(10.0 / z0w) / LT_VONKAR_WAVES;
        if (fabs(u_new - u) <= 1.0e-3 * u) {
            u = u_new;
            converged = 1;
            break;
        }
        u = u_new;
    }
    if (!converged) u = 25.82 * ustar_air;
    *u10 = u;
    *ustokes = LT_US_TO_U10 * u;
    const double hm0 = LT_SWH_FROM_U10SQ * u * u;
    const double f_mean = LT_FM_INTO_FP * 0.877 * GRAVITY / (2.0 * LT_PI * LT_U19P5_TO_U10 * u);
    const double vstokes = 0.125 * LT_PI * LT_R_LOSS * f_mean * hm0 * hm0;
    *kphil = 0.176 * *ustokes / fmx(vstokes, 1.0e-30);
}

/* one_m_exp_x (:806-816): (1 - exp(-x))/x, a series below 1e-4 */
static double one_m_exp_x(double x)
{
    if (x < 1.0e-4) return 1.0 - x * (0.5 - x / 6.0);
    return (1.0 - vpo_sm_exp(-x)) / x;
}

/* epbl_lf17_la (:767-804): the Langmuir number of the Stokes drift averaged
 * over the surface layer zsl */
static double lf17_la(double ustar_w, double zsl, double ustokes, double kphil)
{
    const double xkz = kphil * zsl;
    const double root2kz = sqrt(2.0 * xkz);
    const double r1 = (0.302 - 1.68 * xkz) * one_m_exp_x(2.0 * xkz);
    const double r3 = (0.1264 + 0.64 * xkz) * one_m_exp_x(5.12 * xkz);
    double r5;
    if (root2kz > 1.0e-3) {
        const double ec1 = vpo_sm_erfc(root2kz);
        const double ec2 = vpo_sm_erfc(1.6 * root2kz);
        r5 = sqrt(LT_PI) * (root2kz * (-0.84 * ec1 + 0.2 * ec2) + 0.1182 * (ec2 - ec1) / root2kz);
    } else {
        r5 = -0.64 * sqrt(LT_PI) * root2kz + (-0.14184 + 1.0839648 * root2kz * root2kz);
    }
    const double ustokes_sl = fmx(ustokes * (0.715 + r1 + r3 + r5), 1.0e-10);
    return sqrt(ustar_w / ustokes_sl);
}

/* epbl_lt_enhance (:818-862): La modified by the Ekman and Obukhov depth
 * ratios, then mstar rescaled (capped) or incremented */
static double lt_enhance(const vphys_config *c, double la, double b0, double ustar, double bld, double absf,
                         double mstar)
{
    const double vonkar = c->epbl_von_karman;
    const double mld_ek = bld * absf / ustar;
    const double ek_ob = fabs(b0 * vonkar) / (fmx(absf, 1.0e-20) * ustar * ustar);
    const double mld_ob = fabs(bld * b0 * vonkar) / (ustar * ustar * ustar);
    double la_mod;
    if (b0 >= 0.0)
        la_mod = la * ((1.0 + fmx(-0.5, c->epbl_lt_lac1 * mld_ek)) + c->epbl_lt_lac4 * ek_ob + c->epbl_lt_lac2 * mld_ob);
    else
        la_mod = la * ((1.0 + fmx(-0.5, c->epbl_lt_lac1 * mld_ek)) + c->epbl_lt_lac5 * ek_ob + c->epbl_lt_lac3 * mld_ob);
    la_mod = fmx(la_mod, 1.0e-10);
    if (c->epbl_lt_scheme == 2) return mstar + c->epbl_lt_enhance_coef * vpo_sm_pow(la_mod, c->epbl_lt_enhance_exp);
    const double enh = fmn(c->epbl_lt_max_enhance, 1.0 + c->epbl_lt_enhance_coef * vpo_sm_pow(la_mod, c->epbl_lt_enhance_exp));
    return mstar * enh;
}

void vpo_epbl_lf17(double ustar, double rho0, double zsl, double *u10, double *la)
{
    double ustokes, kphil;
    lf17_wave_state(ustar, rho0, u10, &ustokes, &kphil);
    *la = lf17_la(ustar, zsl, ustokes, kphil);
}

double vpo_epbl_lt_enhance(const vphys_config *c, double la, double b0, double ustar, double bld, double absf,
                           double mstar)
{
    return lt_enhance(c, la, b0, ustar, bld, absf, mstar);
}

/* sw_pe_cost_shape (rdb_ocean_surface_flux.F90:1417-1449): the fraction of
 * the skin PE cost that homogenising an exponentially distributed in-layer
 * heating of optical depth tau incurs; Taylor branch below tau = 1e-2. */
static double sw_pe_cost_shape(double tau)
{
    if (tau <= 1.0e-2) return (1.0 / 6.0) * tau * (1.0 - (1.0 / 60.0) * tau * tau);
    const double em1 = 1.0 - vpo_sm_exp(-tau);
    return (tau * (1.0 + vpo_sm_exp(-tau)) - 2.0 * em1) / (tau * em1);
}

/* epbl_mixlen_shape (:690-714) */
static double mixlen_shape(const vphys_config *c, double z_depth, double mld_guess)
{
    const double ts = c->epbl_translay_scale;
    if (!c->epbl_mld_iteration || ts >= 1.0 || ts < 0.0 || mld_guess <= 0.0) return 1.0;
    const double fr = fmx(0.0, (mld_guess - z_depth) / mld_guess);
    if (c->epbl_mixlen_exponent == 2.0) return ts + (1.0 - ts) * fr * fr;
    return ts + (1.0 - ts) * vpo_sm_pow(fr, c->epbl_mixlen_exponent);
}

/* the turbulent velocity scale and the mixing-length diffusivity of sweep
 * steps (6) and (8a) (:1431-1453, 1492-1510) */
static double vstar_of(const vphys_config *c, double tke_here, double conv_perel, double ustar, double htot,
                       double mld_guess, double dt)
{
    if (c->epbl_vstar_scheme == 2) {
        const double surf_scale = fmx(0.05, 1.0 - htot / mld_guess);
        return c->epbl_vstar_scale_fac * surf_scale *
               (c->epbl_vstar_surf_fac * ustar +
                vpo_sm_cbrt(c->epbl_wstar_ustar_coef * conv_perel / (dt * c->rho0)));
    }
    return c->epbl_vstar_scale_fac * vpo_sm_cbrt(tke_here / (dt * c->rho0));
}

static double mixlen_kd(const vphys_config *c, double vstar, double htot, double hbs, double absf)
{
    if (c->epbl_mld_iteration) {
        const double mixlen = fmx(c->epbl_min_mix_len,
                                  (htot * hbs * vstar) / (c->epbl_ekman_scale_coef * absf * htot * hbs + vstar));
        return vstar * c->epbl_von_karman * mixlen;
    }
    return vstar * c->epbl_von_karman * (htot * hbs * vstar) / (c->epbl_ekman_scale_coef * absf * htot * hbs + vstar);
}

static int first_live(const double *h, int nx, int ny, int i, int j, int kstart)
{
    for (int k = kstart; k >= 1; --k)
        if (C3(h, i, j, k) > H_VANISHED) return k;
    return kstart;
}

/* epbl_compute -> epbl_column_kernel (:864-1659): the column prep, the
 * surface energetics, the MLD iteration around the downward sweep. */
void vpo_epbl(const vphys_config *c, vpo_state *s, double dt)
{
    if (c->idx_temperature < 0 || c->idx_salinity < 0) return;
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const double *T = s->tr[c->idx_temperature];
    const double *S = s->tr[c->idx_salinity];
    const double rho0 = c->rho0;
    const double inv_rho0_cp = 1.0 / (rho0 * c->cp);
    const double inv_rho0 = 1.0 / rho0;
#pragma omp parallel for collapse(2) schedule(dynamic, 16)
    for (int j = 1; j <= ny; ++j) {
        for (int i = 1; i <= nx; ++i) {
            const int n = nz + 2;
            double t0[n], s0[n], dpe_t[n], dpe_s[n], dch_t[n], dch_s[n], ctke_sw[n];
            const int k_sfc = first_live(s->h, nx, ny, i, j, nz);
            /* the penetrating-shortwave ledger (:1095-1185): irradiance I0 and the
             * running depth of the layer top below the live surface */
            const int sw_on = c->epbl_sw_ctke && c->sw_pen_frac != 0.0;   /* sw_ctke_active (:905) */
            const double i0_col = sw_on ? c->sw_pen_frac * C2(vpo_sw_source(c, s), i, j) * C2(s->wet, i, j) : 0.0;
            double d_top_sw = 0.0, e1_top = 1.0, e2_top = 1.0;
            /* ---- column prep: T0, S0 and the pressure-weighted weights (downward) */
            double pres = 0.0, h_sum = 0.0, dsv_dt_sfc = 0.0, dsv_ds_sfc = 0.0;
            for (int k = nz; k >= 1; --k) {
                const double hk = C3(s->h, i, j, k);
                double t0k = 0.0, s0k = 0.0;
                if (hk > 0.0) {
                    t0k = C3(T, i, j, k);
                    s0k = C3(S, i, j, k);
                }
                const double dmass = rho0 * hk;
                const double dpres = GRAVITY * dmass;
                const double p_mid = pres + 0.5 * dpres;
                double dsv_dt_k, dsv_ds_k;
                specvol_derivs(c, t0k, s0k, p_mid, &dsv_dt_k, &dsv_ds_k);
                t0[k] = t0k;
                s0[k] = s0k;
                dpe_t[k] = dmass * p_mid * dsv_dt_k;
                dpe_s[k] = dmass * p_mid * dsv_ds_k;
                dch_t[k] = dmass * dsv_dt_k;
                dch_s[k] = dmass * dsv_ds_k;
                if (k > k_sfc) {
                    ctke_sw[k] = 0.0;   /* dead layers above the live surface take no light */
                } else if (sw_on && c->sw_chl) {
                    /* the chlorophyll N-band ledger (1143-1164): per band, the
                     * difference form with the opaque bed at k = 1 */
                    const double d_bot_sw = d_top_sw + hk;
                    double phi_sum = 0.0;
                    for (int n = 1; n <= c->sw_nbands; ++n) {
                        const double kn = s->sw_kappa[(size_t)(i - 1) + (size_t)nx * (j - 1) + (size_t)nx * ny * (n - 1)];
                        const double ea = vpo_sm_exp(-(kn * d_top_sw));
                        const double eb = (k > 1) ? vpo_sm_exp(-(kn * d_bot_sw)) : 0.0;
                        const double heat_nb =
                            i0_col * vpo_sw_band_frac(n, c->sw_nbands, c->sw_blue_frac) * inv_rho0_cp * dt * (ea - eb);
                        phi_sum = phi_sum + heat_nb * sw_pe_cost_shape(hk * kn);
                    }
                    ctke_sw[k] = -0.5 * GRAVITY * rho0 * dch_t[k] * phi_sum;
                    d_top_sw = d_bot_sw;
                } else if (sw_on) {
                    /* absorbed heat per band, difference form, opaque bed at k = 1 */
                    const double d_bot_sw = d_top_sw + hk;
                    double heat_sw1, heat_sw2;
                    if (k > 1) {
                        const double e1_bot = vpo_sm_exp(-d_bot_sw / c->sw_zeta1);
                        const double e2_bot = vpo_sm_exp(-d_bot_sw / c->sw_zeta2);
                        heat_sw1 = i0_col * c->sw_band_ratio * inv_rho0_cp * dt * (e1_top - e1_bot);
                        heat_sw2 = i0_col * (1.0 - c->sw_band_ratio) * inv_rho0_cp * dt * (e2_top - e2_bot);
                        e1_top = e1_bot;
                        e2_top = e2_bot;
                    } else {
                        heat_sw1 = i0_col * c->sw_band_ratio * inv_rho0_cp * dt * e1_top;
                        heat_sw2 = i0_col * (1.0 - c->sw_band_ratio) * inv_rho0_cp * dt * e2_top;
                    }
                    ctke_sw[k] = -0.5 * GRAVITY * rho0 * dch_t[k] *
                                 (heat_sw1 * sw_pe_cost_shape(hk / c->sw_zeta1) +
                                  heat_sw2 * sw_pe_cost_shape(hk / c->sw_zeta2));
                    d_top_sw = d_bot_sw;
                } else {
                    ctke_sw[k] = 0.0;
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

            /* ---- surface forcing energetics */
            const double q_t_kin = inv_rho0_cp * C2(s->q_heat, i, j);
            const double q_s_kin = inv_rho0 * C2(s->q_salt, i, j);
            const double b0 = GRAVITY * rho0 * (dsv_dt_sfc * q_t_kin + dsv_ds_sfc * q_s_kin);
            const double h_top = C3(s->h, i, j, k_sfc);
            double ctke_sfc;
            if (sw_on) {
                /* the skin carries only the non-penetrating heat; the shortwave
                 * absorbed in the surface layer is its own ledger entry */
                const double q_nonpen_kin = inv_rho0_cp * (C2(s->q_heat, i, j) - i0_col);
                ctke_sfc = -0.5 * GRAVITY * (rho0 * rho0) * h_top *
                               (q_nonpen_kin * dt * dsv_dt_sfc + q_s_kin * dt * dsv_ds_sfc) +
                           ctke_sw[k_sfc];
            } else {
                ctke_sfc = -0.5 * GRAVITY * (rho0 * rho0) * h_top * (q_t_kin * dt * dsv_dt_sfc + q_s_kin * dt * dsv_ds_sfc);
            }
            const double ustar = fmx(sqrt(C2(s->stress_mag, i, j) / rho0), c->epbl_ustar_min);
            const double f = s->coriolis ? C2(s->coriolis, i, j) : 0.0;
            const double absf = sqrt((1.0 - c->epbl_omega_frac) * (f * f) +
                                     c->epbl_omega_frac * 4.0 * (c->epbl_omega * c->epbl_omega));
            const double idecay = c->epbl_tke_decay * absf / ustar;
            const double mech_in = dt * rho0 * (ustar * ustar * ustar);
            /* the LF17 wave state depends on u* alone: once per column */
            double la_val = 0.0, lt_u10 = 0.0, lt_ustokes = 0.0, lt_kphil = 0.0;
            if (c->epbl_use_lt) lf17_wave_state(ustar, rho0, &lt_u10, &lt_ustokes, &lt_kphil);

            double mld_found = 0.0;
            /* the TKE budget of the last MLD iteration (:1641-1654) */
            double d_wind = 0.0, d_conv = 0.0, d_forcing = 0.0, d_mixing = 0.0, d_mdecay = 0.0, d_cdecay = 0.0;
            if (C2(s->wet, i, j) <= 0.0 || h_sum <= 2.0 * H_NEGLECT) {
                for (int k = 1; k <= nz + 1; ++k) C3(s->kd_epbl, i, j, k) = 0.0;
            } else {
                /* ---- outer MLD iteration */
                double min_mld = 0.0, max_mld = h_sum, dmld_min = 0.0, dmld_max = 0.0;
                int have_min = 0, have_max = 0;
                double mld_guess = 0.5 * (min_mld + max_mld);
                if (c->epbl_mld_use_prev_guess && C2(s->mld_epbl, i, j) > 0.0)
                    mld_guess = fmn(C2(s->mld_epbl, i, j), max_mld);
                const int n_its = c->epbl_mld_iteration ? c->epbl_mld_max_its : 1;
                double dt_h = 0.0;   /* carried between interfaces (the Fortran local) */
                for (int obl_it = 1; obl_it <= n_its; ++obl_it) {
                    d_wind = d_conv = d_forcing = d_mixing = d_mdecay = d_cdecay = 0.0;
                    double mstar_val = find_mstar(c, b0, ustar, mld_guess, absf);
                    if (c->epbl_use_lt) {
                        la_val = lf17_la(ustar, c->epbl_la_frac_hbl * mld_guess, lt_ustokes, lt_kphil);
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
                        d_conv = c->epbl_nstar * ctke_sfc;
                    }
                    double h_ka = C3(s->h, i, j, k_sfc) + H_NEGLECT;
                    double hp_a = h_ka;
                    double dpe_t_a = dpe_t[k_sfc], dpe_s_a = dpe_s[k_sfc];
                    double dch_t_a = dch_t[k_sfc], dch_s_a = dch_s[k_sfc];
                    double th_a = h_ka * t0[k_sfc], sh_a = h_ka * s0[k_sfc];
                    double te_lag = 0.0, se_lag = 0.0, kddt_prev = 0.0;
                    double htot = C3(s->h, i, j, k_sfc);
                    double z_int = C3(s->h, i, j, k_sfc);
                    double pres_int = GRAVITY * rho0 * C3(s->h, i, j, k_sfc);
                    double mld_output = C3(s->h, i, j, k_sfc);
                    int sfc_connected = 1;
                    for (int ki = k_sfc + 1; ki <= nz + 1; ++ki) C3(s->kd_epbl, i, j, ki) = 0.0;

                    for (int ki = k_sfc; ki >= 2; --ki) {
                        const int ka = ki, kb = ki - 1;
                        h_ka = C3(s->h, i, j, ka) + H_NEGLECT;
                        const double h_kb = C3(s->h, i, j, kb) + H_NEGLECT;
                        int sfc_disconnect = 0;
                        /* (1) mechanical TKE decays across the layer above */
                        const double exp_kh = vpo_sm_exp(-h_ka * idecay);
                        d_mdecay = d_mdecay + (1.0 - exp_kh) * mech_tke;
                        mech_tke = mech_tke * exp_kh;
                        /* (2) the layer below accrues its shortwave cost: a release
                         * (> 0) joins the convective reservoir */
                        double ctke_sw_kb = 0.0;
                        if (sw_on) {
                            ctke_sw_kb = ctke_sw[kb];
                            if (ctke_sw_kb > 0.0) {
                                conv_perel = conv_perel + ctke_sw_kb;
                                d_conv = d_conv + c->epbl_nstar * ctke_sw_kb;
                            }
                        }
                        /* (3) rotation-reduced convective efficiency */
                        double nstar_fc = c->epbl_nstar;
                        if (conv_perel > 0.0 && absf > 0.0) {
                            const double ah = absf * htot;
                            nstar_fc = c->epbl_nstar * conv_perel /
                                       (conv_perel + 0.2 * sqrt(0.5 * dt * rho0 * (ah * ah * ah) * conv_perel));
                        }
                        double tot_tke = mech_tke + nstar_fc * conv_perel;
                        /* (3b) a shortwave sink (< 0) is paid first, both reservoirs
                         * drained in proportion */
                        if (sw_on && ctke_sw_kb < 0.0) {
                            if (ctke_sw_kb + tot_tke < 0.0) {
                                d_mixing = d_mixing + tot_tke;
                                d_cdecay = d_cdecay + (c->epbl_nstar - nstar_fc) * conv_perel;
                                tot_tke = 0.0;
                                mech_tke = 0.0;
                                conv_perel = 0.0;
                            } else {
                                const double r_sw = (tot_tke + ctke_sw_kb) / tot_tke;
                                d_mixing = d_mixing - ctke_sw_kb;
                                d_cdecay = d_cdecay + (1.0 - r_sw) * (c->epbl_nstar - nstar_fc) * conv_perel;
                                tot_tke = r_sw * tot_tke;
                                mech_tke = r_sw * mech_tke;
                                conv_perel = r_sw * conv_perel;
                            }
                        }
                        double kd_val;
                        /* (5) static-stability short-circuit */
                        if (tot_tke <= 0.0 && 0.0 <= (dch_t[kb] + dch_t[ka]) * (t0[ka] - t0[kb]) +
                                                          (dch_s[kb] + dch_s[ka]) * (s0[ka] - s0[kb])) {
                            kd_val = 0.0;
                            sfc_disconnect = 1;
                        } else {
                            /* (6) velocity scale, mixing length, first-guess Kd */
                            dt_h = dt / fmx(0.5 * (h_ka + h_kb), 1.0e-15 * h_sum);
                            double tke_here = mech_tke + c->epbl_wstar_ustar_coef * conv_perel;
                            const double hb_hs = (h_sum - z_int) / h_sum;
                            const double shape_fn = mixlen_shape(c, z_int, mld_guess);
                            const double hbs = fmn(hb_hs, shape_fn);
                            double kd_g0 = 0.0;
                            if (tke_here > 0.0) {
                                const double vstar = vstar_of(c, tke_here, conv_perel, ustar, htot, mld_guess, dt);
                                kd_g0 = mixlen_kd(c, vstar, htot, hbs, absf);
                            }
                            /* (7), (8) closed-form energy solve */
                            const double hp_b = h_kb;
                            const double th_b = h_kb * t0[kb];
                            const double sh_b = h_kb * s0[kb];
                            const double hps = hp_a + hp_b;
                            const double bdt1 = hp_a * hp_b;
                            const double dt_c = hp_a * th_b - hp_b * th_a;
                            const double ds_c = hp_a * sh_b - hp_b * sh_a;
                            double pec_core = hp_b * (dpe_t_a * dt_c + dpe_s_a * ds_c) -
                                              hp_a * (dpe_t[kb] * dt_c + dpe_s[kb] * ds_c);
                            const double colht_core = hp_b * (dch_t_a * dt_c + dch_s_a * ds_c) -
                                                      hp_a * (dch_t[kb] * dt_c + dch_s[kb] * ds_c);
                            if (colht_core < 0.0) pec_core = pec_core - pres_int * colht_core;
                            const double dkddt = kd_g0 * dt_h;
                            const double pe_max = pec_core / (bdt1 * hps);
                            if (pe_max < 0.0) {
                                /* (8a) convectively unstable */
                                tke_here = mech_tke + c->epbl_wstar_ustar_coef * (conv_perel - pe_max);
                                if (tke_here > 0.0) {
                                    const double vstar =
                                        vstar_of(c, tke_here, conv_perel, ustar, htot, mld_guess, dt);
                                    kd_val = mixlen_kd(c, vstar, htot, hbs, absf);
                                } else {
                                    kd_val = 0.0;
                                }
                                const double pe_g0 = pec_core * dkddt / (bdt1 * (bdt1 + dkddt * hps));
                                double dpe_conv =
                                    pec_core * (kd_val * dt_h) / (bdt1 * (bdt1 + (kd_val * dt_h) * hps));
                                if (dpe_conv > 0.0) {
                                    kd_val = kd_g0;
                                    dpe_conv = pe_g0;
                                }
                                conv_perel = conv_perel - dpe_conv;
                                d_conv = d_conv - c->epbl_nstar * dpe_conv;
                                if (sfc_connected) mld_output = mld_output + C3(s->h, i, j, kb);
                            } else {
                                /* (8b) stable: energy-limited Kd; drain the reservoirs */
                                double tke_used, frac_bl;
                                if ((pec_core * dkddt <= tot_tke * (bdt1 * (bdt1 + dkddt * hps))) || (pec_core <= 0.0)) {
                                    kd_val = kd_g0;
                                    tke_used = pec_core * dkddt / (bdt1 * (bdt1 + dkddt * hps));
                                    frac_bl = 1.0;
                                } else {
                                    kd_val = (bdt1 * bdt1 * tot_tke) / (dt_h * (pec_core - bdt1 * hps * tot_tke));
                                    tke_used = tot_tke;
                                    frac_bl = tot_tke * (bdt1 * (bdt1 + dkddt * hps)) / (pec_core * dkddt);
                                }
                                if (sfc_connected) mld_output = mld_output + frac_bl * C3(s->h, i, j, kb);
                                if (frac_bl < 1.0) sfc_disconnect = 1;
                                double r_reduc = 0.0;
                                if (tot_tke > 0.0 && tot_tke > tke_used) r_reduc = (tot_tke - tke_used) / tot_tke;
                                d_mixing = d_mixing + tke_used;
                                d_cdecay = d_cdecay + (1.0 - r_reduc) * (c->epbl_nstar - nstar_fc) * conv_perel;
                                mech_tke = r_reduc * mech_tke;
                                conv_perel = r_reduc * conv_perel;
                            }
                        }
                        C3(s->kd_epbl, i, j, ki) = kd_val;
                        const double kddt_cur = kd_val * dt_h;
                        /* (9) advance the embedded forward elimination */
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
                            htot = C3(s->h, i, j, kb);
                            sfc_connected = 0;
                        } else {
                            htot = htot + C3(s->h, i, j, kb);
                        }
                        z_int = z_int + C3(s->h, i, j, kb);
                        pres_int = pres_int + GRAVITY * rho0 * C3(s->h, i, j, kb);
                    }
                    C3(s->kd_epbl, i, j, 1) = 0.0;
                    /* the stocks left at the bed count as dissipated */
                    d_mdecay = d_mdecay + mech_tke;
                    d_cdecay = d_cdecay + c->epbl_nstar * conv_perel;
                    mld_found = mld_output;
                    if (!c->epbl_mld_iteration) break;
                    if (fabs(mld_found - mld_guess) < c->epbl_mld_tol) break;
                    if (obl_it == n_its) break;
                    if (mld_found > mld_guess) {
                        min_mld = mld_guess;
                        dmld_min = mld_found - mld_guess;
                        have_min = 1;
                    } else {
                        max_mld = mld_guess;
                        dmld_max = mld_found - mld_guess;
                        have_max = 1;
                    }
                    if (c->epbl_mld_bisection)
                        mld_guess = 0.5 * (min_mld + max_mld);
                    else if (have_min && have_max && obl_it > 2 && (obl_it - 1) % 4 > 0)
                        mld_guess = min_mld + dmld_min * (max_mld - min_mld) / (dmld_min - dmld_max);
                    else if (mld_found > min_mld && mld_found < max_mld)
                        mld_guess = mld_found;
                    else
                        mld_guess = 0.5 * (min_mld + max_mld);
                }
            }
            C2(s->mld_epbl, i, j) = mld_found;
            if (s->la_epbl) C2(s->la_epbl, i, j) = la_val;
            if (c->epbl_tke_diags) {
                const double d[6] = {d_wind, d_conv, d_forcing, d_mixing, d_mdecay, d_cdecay};
                for (int q = 0; q < 6; ++q)
                    if (s->epbl_tke[q]) C2(s->epbl_tke[q], i, j) = d[q] / dt;
            }
        }
    }
}

/* epbl_merge_into_kv_kt (:1661-1688) and epbl_merge_max_shear (:1690-1718);
 * interior interfaces only.  With combine = max_shear (and kappa-shear on)
 * the kappa-shear merge comes first, additively (rdb_ocean_dyn.F90:1553-1559). */
void vpo_epbl_merge(const vphys_config *c, vpo_state *s)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const double pr = c->epbl_prandtl;
    const int shear_first = c->kappa_shear && c->epbl_combine == 3;
    if (shear_first) vpo_kappa_shear_merge(c, s);
#pragma omp parallel for
    for (int k = 2; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                const double kd = C3(s->kd_epbl, i, j, k);
                if (shear_first) {
                    const double kds = C3(s->kd_shear, i, j, k);
                    C3(s->kt, i, j, k) = C3(s->kt, i, j, k) + fmx(kd - kds, 0.0);
                    C3(s->kv, i, j, k) = C3(s->kv, i, j, k) + fmx(pr * kd - c->ks_prandtl_turb * kds, 0.0);
                } else if (c->epbl_combine == 2) {
                    C3(s->kt, i, j, k) = fmx(C3(s->kt, i, j, k), kd);
                    C3(s->kv, i, j, k) = fmx(C3(s->kv, i, j, k), pr * kd);
                } else {
                    C3(s->kt, i, j, k) = C3(s->kt, i, j, k) + kd;
                    C3(s->kv, i, j, k) = C3(s->kv, i, j, k) + pr * kd;
                }
            }
}
