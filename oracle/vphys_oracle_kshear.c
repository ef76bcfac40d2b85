/* vphys_oracle_kshear.c -- kappa-shear (Jackson, Hallberg & Legg 2008,
 * J. Phys. Oceanogr. 38, 1033-1053), column form: CPU FP64 restatement of
 * src/parameterizations/vertical/rdb_ocean_kappa_shear.F90.
 *
 * TEST INFRASTRUCTURE ONLY: the checker of vphys_kappa_shear (see
 * vphys_oracle.h).  Arrays are 1-based like the Fortran (element 0 unused):
 * inside the column solver layer k = 1..nz and interface k = 1..nz+1 run
 * SURFACE-DOWN (local k = 1 is the surface); the gather and scatter flip to
 * the bottom-up global order (kappa_shear_column_kernel, :480-648).
 *
 * Parity pins: the reference's golden profile (tests/test_ocean_kappa_shear.F90
 * :286-393, values from its Python prototype, 1e-6 relative) and the
 * structural tests of the same file (no source, activation, self-limiting,
 * merge); tests/test_oracle_kappa_shear.py re-expresses them.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "vphys_oracle.h"

static const double GRAVITY = 9.80665;     /* rdb_constants.F90:37 */
static const double H_VANISHED = 1.5e-4;

#define C3(a, i, j, k) (a)[((size_t)(i) - 1) + (size_t)nx * (((size_t)(j) - 1) + (size_t)ny * ((size_t)(k) - 1))]
#define C2(a, i, j) (a)[((size_t)(i) - 1) + (size_t)nx * ((size_t)(j) - 1)]

static inline double fmx(double a, double b) { return a > b ? a : b; }
static inline double fmn(double a, double b) { return a < b ? a : b; }

/* the knobs of ocean_kappa_shear_t (rdb_ocean_kappa_shear.F90:96-150) */
typedef struct ks_par {
    double ri_crit, shearmix_rate, fri_curvature, c_n, c_s, lambda, lz_rescale;
    double kappa_0, kappa_seed, kappa_trunc, tke_bg, tol_err, src_max_chg, vel_underflow, rho0;
    double alpha_t, beta_s;
    int max_inner_it, max_substep_it, eos_linear;
} ks_par;

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

/* eos_specvol_derivs (rdb_eos.F90:1551-1622): dSV/dT, dSV/dS of the Wright
 * variant, or of the linear one at the reference density. */
static void specvol_derivs(const ks_par *p, double T, double S, double pres, double *dsv_dt, double *dsv_ds)
{
    if (p->eos_linear) {
        *dsv_dt = p->alpha_t / (p->rho0 * p->rho0);
        *dsv_ds = -p->beta_s / (p->rho0 * p->rho0);
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

/* ks_src_func (:953-969) */
static double ks_src_func(double ri_crit, double shearmix_rate, double fri_curvature, double n2, double s2)
{
    double ksrc = 0.0;
    if (n2 < ri_crit * s2) {
        double dnom = ri_crit * s2 + fri_curvature * n2;
        if (dnom != 0.0 && s2 > 0.0) ksrc = 2.0 * shearmix_rate * sqrt(s2) * (ri_crit * s2 - n2) / dnom;
    }
    return ksrc;
}

/* ks_precompute (:971-1032) */
static void ks_precompute(int nz, double lz_rescale, const double *h, double *idz, double *idz_int, double *hint,
                          double *il2)
{
    double dbot[nz + 2];
    double i_lz2 = 1.0 / (lz_rescale * lz_rescale);
    for (int k = 1; k <= nz; ++k) idz[k] = 1.0 / h[k];
    idz_int[1] = 2.0 / h[1];
    for (int k = 2; k <= nz; ++k) idz_int[k] = 2.0 / (h[k - 1] + h[k]);
    idz_int[nz + 1] = 2.0 / h[nz];

    hint[1] = 0.0;
    if (nz >= 2) {
        hint[2] = h[1];
        for (int k = 2; k <= nz - 1; ++k) {
            double hk = h[k], hkm1 = h[k - 1], hkp1 = h[k + 1];
            double norm_l = 1.0 / (hk * (hkm1 + hkp1) + 2.0 * hkm1 * hkp1);
            double wt_a = (hk + hkp1) * hkm1 * norm_l;
            double wt_b = (hkm1 + hk) * hkp1 * norm_l;
            hint[k] = hint[k] + hk * wt_a;
            hint[k + 1] = hk * wt_b;
        }
        hint[nz] = hint[nz] + h[nz];
    }
    hint[nz + 1] = 0.0;

    dbot[nz + 1] = 0.0;
    for (int k = nz; k >= 1; --k) dbot[k] = dbot[k + 1] + h[k];
    il2[1] = 0.0;
    il2[nz + 1] = 0.0;
    double dtop = 0.0;
    for (int k = 2; k <= nz; ++k) {
        dtop = dtop + h[k - 1];
        if (dtop > 0.0 && dbot[k] > 0.0) {
            double t = dtop + dbot[k];
            double b = dtop * dbot[k];
            il2[k] = i_lz2 * (t * t) / (b * b);
        } else {
            il2[k] = 0.0;
        }
    }
}

/* ks_projected_state (:1034-1171): (u0, v0, T0, S0) mixed implicitly with
 * kappa over dt_now inside the layer band [ks, ke]; N2, S2 recomputed. */
static void ks_projected_state(int nz, double dt_now, int ks, int ke, double vel_underflow, const double *dbuoy_t,
                               const double *dbuoy_s, const double *h, const double *idz_int, const double *u0,
                               const double *v0, const double *t0, const double *s0, const double *kappa,
                               double *u_o, double *v_o, double *t_o, double *s_o, double *c1_o, double *n2_o,
                               double *s2_o)
{
    for (int k = 1; k <= nz; ++k) {
        u_o[k] = u0[k];
        v_o[k] = v0[k];
        t_o[k] = t0[k];
        s_o[k] = s0[k];
    }
    for (int k = 1; k <= nz + 1; ++k) c1_o[k] = 0.0;

    if (ks <= ke && dt_now > 0.0) {
        double a_b = dt_now * kappa[ks + 1] * idz_int[ks + 1];
        double b1 = 1.0 / (h[ks] + a_b);
        c1_o[ks + 1] = a_b * b1;
        double d1 = h[ks] * b1;
        u_o[ks] = b1 * h[ks] * u0[ks];
        v_o[ks] = b1 * h[ks] * v0[ks];
        t_o[ks] = b1 * h[ks] * t0[ks];
        s_o[ks] = b1 * h[ks] * s0[ks];
        double a_a;
        for (int k = ks + 1; k <= ke - 1; ++k) {
            a_a = a_b;
            a_b = dt_now * kappa[k + 1] * idz_int[k + 1];
            double bd1 = h[k] + d1 * a_a;
            b1 = 1.0 / (bd1 + a_b);
            c1_o[k + 1] = a_b * b1;
            d1 = bd1 * b1;
            u_o[k] = b1 * (h[k] * u0[k] + a_a * u_o[k - 1]);
            v_o[k] = b1 * (h[k] * v0[k] + a_a * v_o[k - 1]);
            t_o[k] = b1 * (h[k] * t0[k] + a_a * t_o[k - 1]);
            s_o[k] = b1 * (h[k] * s0[k] + a_a * s_o[k - 1]);
        }
        a_a = a_b;
        double b1nz;
        if (ke > ks) {
            b1 = 1.0 / (h[ke] + d1 * a_a);
            t_o[ke] = b1 * (h[ke] * t0[ke] + a_a * t_o[ke - 1]);
            s_o[ke] = b1 * (h[ke] * s0[ke] + a_a * s_o[ke - 1]);
            if (ke == nz)
                b1nz = 1.0 / ((h[ke] + d1 * a_a) + dt_now * kappa[nz + 1] * idz_int[nz + 1]);
            else
                b1nz = b1;
            u_o[ke] = b1nz * (h[ke] * u0[ke] + a_a * u_o[ke - 1]);
            v_o[ke] = b1nz * (h[ke] * v0[ke] + a_a * v_o[ke - 1]);
        } else {
            b1 = 1.0 / (h[ke] + a_a);
            t_o[ke] = b1 * h[ke] * t0[ke];
            s_o[ke] = b1 * h[ke] * s0[ke];
            if (ke == nz)
                b1nz = 1.0 / (h[ke] + a_a + dt_now * kappa[nz + 1] * idz_int[nz + 1]);
            else
                b1nz = b1;
            u_o[ke] = b1nz * h[ke] * u0[ke];
            v_o[ke] = b1nz * h[ke] * v0[ke];
        }
        if (fabs(u_o[ke]) < vel_underflow) u_o[ke] = 0.0;
        if (fabs(v_o[ke]) < vel_underflow) v_o[ke] = 0.0;
        for (int k = ke - 1; k >= ks; --k) {
            u_o[k] = u_o[k] + c1_o[k + 1] * u_o[k + 1];
            v_o[k] = v_o[k] + c1_o[k + 1] * v_o[k + 1];
            t_o[k] = t_o[k] + c1_o[k + 1] * t_o[k + 1];
            s_o[k] = s_o[k] + c1_o[k + 1] * s_o[k + 1];
            if (fabs(u_o[k]) < vel_underflow) u_o[k] = 0.0;
            if (fabs(v_o[k]) < vel_underflow) v_o[k] = 0.0;
        }
    } else {
        for (int k = 1; k <= nz; ++k) {
            if (fabs(u_o[k]) < vel_underflow) u_o[k] = 0.0;
            if (fabs(v_o[k]) < vel_underflow) v_o[k] = 0.0;
        }
    }

    n2_o[1] = 0.0;
    n2_o[nz + 1] = 0.0;
    s2_o[1] = 0.0;
    s2_o[nz + 1] = 0.0;
    for (int kk = 2; kk <= nz; ++kk) {
        double ua, va, ta, sa, ub, vb, tb, sb;
        if (kk - 1 >= ks && kk - 1 <= ke) {
            ua = u_o[kk - 1]; va = v_o[kk - 1]; ta = t_o[kk - 1]; sa = s_o[kk - 1];
        } else {
            ua = u0[kk - 1]; va = v0[kk - 1]; ta = t0[kk - 1]; sa = s0[kk - 1];
        }
        if (kk >= ks && kk <= ke) {
            ub = u_o[kk]; vb = v_o[kk]; tb = t_o[kk]; sb = s_o[kk];
        } else {
            ub = u0[kk]; vb = v0[kk]; tb = t0[kk]; sb = s0[kk];
        }
        double n2v = idz_int[kk] * (dbuoy_t[kk] * (ta - tb) + dbuoy_s[kk] * (sa - sb));
        if (n2v < 0.0) n2v = 0.0;
        n2_o[kk] = n2v;
        double du = ua - ub, dv = va - vb;
        s2_o[kk] = (du * du + dv * dv) * (idz_int[kk] * idz_int[kk]);
    }
}

/* ks_find_kappa_tke (:1173-1413): the inner Picard solve. */
static void ks_find_kappa_tke(const ks_par *p, int nz, double tke_min, double f2_val, double c_n2, double c_s2,
                              double ilambda2, const double *n2_in, const double *s2_in, const double *kappa_seed,
                              double *k_q_io, const double *idz, const double *hint, const double *il2,
                              const double *e1, double *tke_o, double *kappa_o, double *ksrc_sc, double *tkedec_sc,
                              double *aq_sc, double *dq_sc, double *cq_sc, double *dk_sc, double *ck_sc,
                              double *ild2_sc)
{
    const double kappa_0 = p->kappa_0, kappa_trunc = p->kappa_trunc, tke_bg = p->tke_bg;
    int ks_src = nz + 2, ke_src = 0;
    ksrc_sc[1] = 0.0;
    ksrc_sc[nz + 1] = 0.0;
    for (int kk = 2; kk <= nz; ++kk) {
        ksrc_sc[kk] = ks_src_func(p->ri_crit, p->shearmix_rate, p->fri_curvature, n2_in[kk], s2_in[kk]);
        if (ksrc_sc[kk] > 0.0) {
            if (ks_src > kk) ks_src = kk;
            ke_src = kk;
        }
    }
    if (ks_src > ke_src) {
        for (int kk = 1; kk <= nz + 1; ++kk) {
            tke_o[kk] = tke_min;
            kappa_o[kk] = 0.0;
            k_q_io[kk] = 0.0;
        }
        return;
    }
    for (int kk = 2; kk <= nz; ++kk) tkedec_sc[kk] = sqrt(c_n2 * n2_in[kk] + c_s2 * s2_in[kk]);

    tke_o[1] = tke_bg;
    for (int kk = 2; kk <= nz; ++kk) {
        if (kappa_seed[kk] > 0.0 && k_q_io[kk] > 0.0)
            tke_o[kk] = kappa_seed[kk] / k_q_io[kk];
        else
            tke_o[kk] = tke_min;
    }
    tke_o[nz + 1] = tke_min;
    for (int kk = 1; kk <= nz + 1; ++kk) kappa_o[kk] = kappa_seed[kk];
    kappa_o[1] = 0.0;
    kappa_o[nz + 1] = 0.0;

    int ks_kap = 2, ke_kap = nz, ks_kp = 2, ke_kp = nz;
    for (int it = 1; it <= p->max_inner_it; ++it) {
        /* (a) TKE sweep; ke_tke is an interface index, nz+1 = the bed */
        int ke_tke = (ke_kap > ke_kp ? ke_kap : ke_kp) + 1;
        if (ke_tke > nz + 1) ke_tke = nz + 1;
        int kmax = ke_tke < nz ? ke_tke : nz;
        for (int k = 1; k <= kmax; ++k) aq_sc[k] = (0.5 * (kappa_o[k] + kappa_o[k + 1]) + kappa_0) * idz[k];

        dq_sc[1] = -tke_o[1];
        tke_o[1] = tke_bg;
        cq_sc[2] = 0.0;
        double cqc_l = 1.0;
        for (int kk = 2; kk <= ke_tke - 1; ++kk) {
            dq_sc[kk] = -tke_o[kk];
            double tsrc_l = (kappa_o[kk] + kappa_0) * s2_in[kk] + tke_bg * tkedec_sc[kk];
            double bqd1_l = hint[kk] * (tkedec_sc[kk] + n2_in[kk] * k_q_io[kk]) + cqc_l * aq_sc[kk - 1];
            double bq_l = 1.0 / (bqd1_l + aq_sc[kk]);
            tke_o[kk] = bq_l * (hint[kk] * tsrc_l + aq_sc[kk - 1] * tke_o[kk - 1]);
            cq_sc[kk + 1] = aq_sc[kk] * bq_l;
            cqc_l = bqd1_l * bq_l;
        }
        if (ke_tke == nz + 1) {
            tke_o[nz + 1] = tke_min;
            dq_sc[nz + 1] = 0.0;
        } else {
            int kk = ke_tke;
            double tsrc_l = kappa_0 * s2_in[kk] + tke_bg * tkedec_sc[kk];
            double bq_l = 1.0 / (hint[kk] * tkedec_sc[kk] + cqc_l * aq_sc[kk - 1] + aq_sc[kk]);
            cq_sc[kk + 1] = aq_sc[kk] * bq_l;
            dq_sc[kk] = -tke_o[kk];
            double raw_l = bq_l * (hint[kk] * tsrc_l + aq_sc[kk - 1] * tke_o[kk - 1]);
            double dnom_l = 1.0 - cq_sc[kk + 1] * e1[kk + 1];
            if (fabs(dnom_l) > 1.0e-30)
                tke_o[kk] = fmx((raw_l + cq_sc[kk + 1] * (tke_o[kk + 1] - e1[kk + 1] * tke_o[kk])) / dnom_l, tke_min);
            else
                tke_o[kk] = fmx(raw_l, tke_min);
            dq_sc[kk] = tke_o[kk] + dq_sc[kk];
            for (int k2 = ke_tke + 1; k2 <= nz + 1; ++k2) {
                dq_sc[k2] = e1[k2] * dq_sc[k2 - 1];
                tke_o[k2] = fmx(tke_o[k2] + dq_sc[k2], tke_min);
                if (fabs(dq_sc[k2]) < 1.0e-16 * tke_o[k2]) break;
            }
        }
        for (int kk = ke_tke - 1; kk >= 1; --kk) {
            tke_o[kk] = fmx(tke_o[kk] + cq_sc[kk + 1] * tke_o[kk + 1], tke_min);
            dq_sc[kk] = tke_o[kk] + dq_sc[kk];
        }

        /* (b) kappa sweep with the truncation ramp and range tracking */
        ks_kp = ks_kap;
        ke_kp = ke_kap;
        for (int kk = 2; kk <= nz; ++kk) {
            if (tke_o[kk] > 0.0)
                ild2_sc[kk] = (n2_in[kk] * ilambda2 + f2_val) / tke_o[kk] + il2[kk];
            else
                ild2_sc[kk] = 1.0e30;
        }
        dk_sc[1] = 0.0;
        ck_sc[2] = 0.0;
        double ckc_l = 1.0;
        int ke_new = 0;
        for (int kk = 2; kk <= nz; ++kk) {
            dk_sc[kk] = -kappa_o[kk];
            double bkd1_l = hint[kk] * ild2_sc[kk] + ckc_l * idz[kk - 1];
            double bk_l = 1.0 / (bkd1_l + idz[kk]);
            kappa_o[kk] = bk_l * (idz[kk - 1] * kappa_o[kk - 1] + hint[kk] * ksrc_sc[kk]);
            ck_sc[kk + 1] = idz[kk] * bk_l;
            ckc_l = bkd1_l * bk_l;
            double trv = ckc_l * kappa_trunc;
            double tr2v = 2.0 * trv;
            if (kappa_o[kk] < trv) {
                kappa_o[kk] = 0.0;
                if (kk > ke_src) {
                    ke_kap = kk - 1;
                    k_q_io[kk] = 0.0;
                    break;
                }
            } else if (kappa_o[kk] < tr2v) {
                kappa_o[kk] = 2.0 * (kappa_o[kk] - trv);
            }
            ke_new = kk;
        }
        if (ke_new > 0) ke_kap = ke_new;
        if (ke_kap >= 1 && tke_o[ke_kap] > 0.0) k_q_io[ke_kap] = kappa_o[ke_kap] / tke_o[ke_kap];
        dk_sc[ke_kap] = dk_sc[ke_kap] + kappa_o[ke_kap];
        for (int kk = ke_kap + 2; kk <= ke_kp + 1; ++kk) {
            if (kk > nz) break;
            dk_sc[kk] = -kappa_o[kk];
            kappa_o[kk] = 0.0;
            k_q_io[kk] = 0.0;
        }
        int ks_new = 2;
        for (int kk = ke_kap - 1; kk >= 2; --kk) {
            kappa_o[kk] = kappa_o[kk] + ck_sc[kk + 1] * kappa_o[kk + 1];
            if (kappa_o[kk] <= kappa_trunc) {
                kappa_o[kk] = 0.0;
                if (kk < ks_src) {
                    ks_kap = kk + 1;
                    k_q_io[kk] = 0.0;
                    break;
                }
            } else if (kappa_o[kk] < 2.0 * kappa_trunc) {
                kappa_o[kk] = 2.0 * (kappa_o[kk] - kappa_trunc);
            }
            dk_sc[kk] = dk_sc[kk] + kappa_o[kk];
            if (tke_o[kk] > 0.0)
                k_q_io[kk] = kappa_o[kk] / tke_o[kk];
            else
                k_q_io[kk] = 0.0;
            ks_new = kk;
        }
        ks_kap = ks_new > 2 ? ks_new : 2;
        for (int kk = ks_kp; kk <= ks_kap - 2; ++kk) {
            if (kk < 2) continue;
            kappa_o[kk] = 0.0;
            k_q_io[kk] = 0.0;
        }

        /* (c) Picard convergence */
        int k_lo = ks_kap < ks_kp ? ks_kap : ks_kp;
        int k_hi = ke_kap > ke_kp ? ke_kap : ke_kp;
        int conv = 1;
        for (int kk = k_lo; kk <= k_hi; ++kk) {
            double lhs_l = fabs(dk_sc[kk]);
            double rhs_l = p->tol_err * (kappa_0 + kappa_o[kk] - 0.5 * dk_sc[kk]);
            if (lhs_l > rhs_l) {
                conv = 0;
                break;
            }
        }
        if (conv) break;
    }
    kappa_o[1] = 0.0;
    kappa_o[nz + 1] = 0.0;
}

/* the source-change test of one trial step of ks_adaptive_dt */
static int ks_dt_valid(const ks_par *p, int k_lo, int k_hi, double dt_try, const double *n2_pr, const double *s2_pr,
                       const double *tol_max, const double *tol_min_a, const double *tol_chg_a,
                       const double *kappa_src)
{
    double idtt = 0.0;
    if (dt_try > 0.0) idtt = 1.0 / dt_try;
    for (int kk = k_lo; kk <= k_hi; ++kk) {
        if (n2_pr[kk] < p->ri_crit * s2_pr[kk]) {
            double ksrc_tst = ks_src_func(p->ri_crit, p->shearmix_rate, p->fri_curvature, n2_pr[kk], s2_pr[kk]);
            double upper_t = fmx(tol_max[kk], kappa_src[kk] + idtt * tol_chg_a[kk]);
            double lower_t = fmn(tol_min_a[kk], kappa_src[kk] - idtt * tol_chg_a[kk]);
            if (ksrc_tst > upper_t || ksrc_tst < lower_t) return 0;
        } else {
            double lower_t = fmn(tol_min_a[kk], kappa_src[kk] - idtt * tol_chg_a[kk]);
            if (0.0 < lower_t) return 0;
        }
    }
    return 1;
}

/* ks_adaptive_dt (:1415-1543): halving pass, then a 5-step refinement. */
static double ks_adaptive_dt(const ks_par *p, int nz, double dt_rem, int itt_outer, const double *dbuoy_t,
                             const double *dbuoy_s, const double *h, const double *u_cur, const double *v_cur,
                             const double *t_cur, const double *s_cur, const double *kappa_out,
                             const double *kappa_src, const double *local_src, const double *local_src_avg,
                             int ks_kap, int ke_kap, const double *idz_int)
{
    const int n = nz + 2;
    double tol_max[n], tol_min_a[n], tol_chg_a[n];
    double u_pr[n], v_pr[n], t_pr[n], s_pr[n], c1_pr[n], n2_pr[n], s2_pr[n];
    double tol_dksrc_low;
    if (p->src_max_chg == 10.0)
        tol_dksrc_low = 0.95;
    else
        tol_dksrc_low = (p->src_max_chg - 0.5) / p->src_max_chg;
    double tol2_l = 2.0 * p->tol_err;
    for (int kk = 1; kk <= nz + 1; ++kk) {
        tol_max[kk] = kappa_src[kk] + p->src_max_chg * local_src[kk];
        tol_min_a[kk] = kappa_src[kk] - tol_dksrc_low * local_src[kk];
        tol_chg_a[kk] = tol2_l * local_src_avg[kk];
    }
    int k_lo = ks_kap - 1 > 2 ? ks_kap - 1 : 2;
    int k_hi = ke_kap + 1 < nz ? ke_kap + 1 : nz;
    int ks_lyr = ks_kap - 1 > 1 ? ks_kap - 1 : 1;
    int ke_lyr = ke_kap < nz ? ke_kap : nz;

    double dt_tst = dt_rem;
    int valid_dt = 0;
    int max_halvings = (p->max_substep_it + 1 - itt_outer) / 2;
    int nh = max_halvings > 1 ? max_halvings : 1;
    for (int ih = 1; ih <= nh; ++ih) {
        ks_projected_state(nz, 0.5 * dt_tst, ks_lyr, ke_lyr, p->vel_underflow, dbuoy_t, dbuoy_s, h, idz_int, u_cur,
                           v_cur, t_cur, s_cur, kappa_out, u_pr, v_pr, t_pr, s_pr, c1_pr, n2_pr, s2_pr);
        valid_dt = ks_dt_valid(p, k_lo, k_hi, dt_tst, n2_pr, s2_pr, tol_max, tol_min_a, tol_chg_a, kappa_src);
        if (valid_dt) break;
        dt_tst = 0.5 * dt_tst;
    }
    double dt_inc = 0.0;
    if (dt_tst < dt_rem && valid_dt) {
        dt_inc = 0.5 * dt_tst;
        for (int ir = 1; ir <= 5; ++ir) {
            double dt_try = dt_tst + dt_inc;
            ks_projected_state(nz, 0.5 * dt_try, ks_lyr, ke_lyr, p->vel_underflow, dbuoy_t, dbuoy_s, h, idz_int,
                               u_cur, v_cur, t_cur, s_cur, kappa_out, u_pr, v_pr, t_pr, s_pr, c1_pr, n2_pr, s2_pr);
            if (ks_dt_valid(p, k_lo, k_hi, dt_try, n2_pr, s2_pr, tol_max, tol_min_a, tol_chg_a, kappa_src))
                dt_tst = dt_try;
            dt_inc = 0.5 * dt_inc;
        }
    }
    return fmn(dt_tst * (1.0 + p->tol_err) + dt_inc, dt_rem);
}

/* ks_solve_column (:1545-1909): the whole column solve, surface-down. */
static void ks_solve_column(const ks_par *p, int nz, double dt, double f2_val, const double *h, const double *u_sd,
                            const double *v_sd, const double *t_sd, const double *s_sd, const double *idz,
                            const double *idz_int, const double *hint, const double *il2, double *kappa_avg_sd,
                            double *tke_avg_sd)
{
    const int n = nz + 2;
    double u_c[n], v_c[n], t_c[n], s_c[n], dbuoy_t[n], dbuoy_s[n], e1[n];
    double kappa[n], k_q[n], kappa_avg[n], tke_avg[n], n2[n], s2[n], tke[n];
    double ksrc[n], tkedec[n], aq[n], dq[n], cq[n], dk[n], ck[n], ild2[n], cqsav[n];
    double u_ps[n], v_ps[n], t_ps[n], s_ps[n], c1_ps[n], n2p[n], s2p[n], n2c[n], s2c[n];
    double kappa_out[n], kq_tmp[n], tke_pred[n], kappa_pred[n], kappa_mid[n], tke_fin[n], kappa_pred2[n];
    double local_src_avg[n], kappa_src[n], local_src[n];

    const double kappa_0 = p->kappa_0;
    const double k0dt = dt * kappa_0;
    const double tke_min = fmx(p->tke_bg, 1.0e-20);
    const double c_n2 = p->c_n * p->c_n;
    const double c_s2 = p->c_s * p->c_s;
    const double ilambda2 = 1.0 / (p->lambda * p->lambda);

    /* background-diffusion pre-step with kappa_0 */
    if (nz == 1) {
        double b1_l = 1.0 / (h[1] + k0dt * idz_int[2]);
        u_c[1] = b1_l * h[1] * u_sd[1];
        v_c[1] = b1_l * h[1] * v_sd[1];
        t_c[1] = t_sd[1];
        s_c[1] = s_sd[1];
    } else {
        double a1n = k0dt * idz_int[2];
        double b1_l = 1.0 / (h[1] + a1n);
        cqsav[2] = a1n * b1_l;
        double d1_l = h[1] * b1_l;
        u_c[1] = b1_l * h[1] * u_sd[1];
        v_c[1] = b1_l * h[1] * v_sd[1];
        t_c[1] = b1_l * h[1] * t_sd[1];
        s_c[1] = b1_l * h[1] * s_sd[1];
        double a1c;
        for (int k = 2; k <= nz - 1; ++k) {
            a1c = a1n;
            a1n = k0dt * idz_int[k + 1];
            double bd1_l = h[k] + d1_l * a1c;
            b1_l = 1.0 / (bd1_l + a1n);
            u_c[k] = b1_l * (h[k] * u_sd[k] + a1c * u_c[k - 1]);
            v_c[k] = b1_l * (h[k] * v_sd[k] + a1c * v_c[k - 1]);
            t_c[k] = b1_l * (h[k] * t_sd[k] + a1c * t_c[k - 1]);
            s_c[k] = b1_l * (h[k] * s_sd[k] + a1c * s_c[k - 1]);
            cqsav[k + 1] = a1n * b1_l;
            d1_l = bd1_l * b1_l;
        }
        a1c = a1n;
        double base_l = h[nz] + d1_l * a1c;
        double b1ns = 1.0 / (base_l + k0dt * idz_int[nz + 1]);
        double b1in = 1.0 / base_l;
        u_c[nz] = b1ns * (h[nz] * u_sd[nz] + a1c * u_c[nz - 1]);
        v_c[nz] = b1ns * (h[nz] * v_sd[nz] + a1c * v_c[nz - 1]);
        t_c[nz] = b1in * (h[nz] * t_sd[nz] + a1c * t_c[nz - 1]);
        s_c[nz] = b1in * (h[nz] * s_sd[nz] + a1c * s_c[nz - 1]);
        cqsav[nz + 1] = 0.0;
        for (int k = nz - 1; k >= 1; --k) {
            u_c[k] = u_c[k] + cqsav[k + 1] * u_c[k + 1];
            v_c[k] = v_c[k] + cqsav[k + 1] * v_c[k + 1];
            t_c[k] = t_c[k] + cqsav[k + 1] * t_c[k + 1];
            s_c[k] = s_c[k] + cqsav[k + 1] * s_c[k + 1];
        }
    }

    /* frozen interface buoyancy derivatives at the hydrostatic pressure */
    dbuoy_t[1] = 0.0;
    dbuoy_s[1] = 0.0;
    dbuoy_t[nz + 1] = 0.0;
    dbuoy_s[nz + 1] = 0.0;
    double p_int = 0.0;
    for (int kk = 2; kk <= nz; ++kk) {
        double dpres = GRAVITY * p->rho0 * h[kk - 1];
        p_int = p_int + dpres;
        double t_int = 0.5 * (t_c[kk - 1] + t_c[kk]);
        double s_int = 0.5 * (s_c[kk - 1] + s_c[kk]);
        double dsv_dt_k, dsv_ds_k;
        specvol_derivs(p, t_int, s_int, p_int, &dsv_dt_k, &dsv_ds_k);
        dbuoy_t[kk] = GRAVITY * p->rho0 * dsv_dt_k;
        dbuoy_s[kk] = GRAVITY * p->rho0 * dsv_ds_k;
    }

    /* initial N2, S2 */
    n2[1] = 0.0;
    n2[nz + 1] = 0.0;
    s2[1] = 0.0;
    s2[nz + 1] = 0.0;
    for (int kk = 2; kk <= nz; ++kk) {
        double n2v = idz_int[kk] * (dbuoy_t[kk] * (t_c[kk - 1] - t_c[kk]) + dbuoy_s[kk] * (s_c[kk - 1] - s_c[kk]));
        if (n2v < 0.0) n2v = 0.0;
        n2[kk] = n2v;
        double du = u_c[kk - 1] - u_c[kk], dv = v_c[kk - 1] - v_c[kk];
        s2[kk] = (du * du + dv * dv) * (idz_int[kk] * idz_int[kk]);
    }

    /* e1 tail recursion */
    e1[nz + 1] = 0.0;
    double ome_l = 1.0;
    double eden2_l = kappa_0 * idz[nz];
    for (int kk = nz; kk >= 2; --kk) {
        double eden1_l = hint[kk] * sqrt(c_n2 * n2[kk] + c_s2 * s2[kk]) + ome_l * eden2_l;
        eden2_l = kappa_0 * idz[kk - 1];
        double i_eden_l = 1.0 / (eden2_l + eden1_l);
        e1[kk] = eden2_l * i_eden_l;
        ome_l = eden1_l * i_eden_l;
    }
    e1[1] = 0.0;

    for (int kk = 1; kk <= nz + 1; ++kk) {
        k_q[kk] = 0.0;
        kappa_avg[kk] = 0.0;
        tke_avg[kk] = 0.0;
        kappa[kk] = p->kappa_seed;
    }
    kappa[1] = 0.0;
    kappa[nz + 1] = 0.0;
    double dt_rem = dt;
    local_src_avg[1] = 0.0;
    local_src_avg[nz + 1] = 0.0;
    for (int kk = 2; kk <= nz; ++kk) {
        if (hint[kk] > 0.0)
            local_src_avg[kk] = 0.1 * k0dt * idz_int[kk] / hint[kk];
        else
            local_src_avg[kk] = 0.0;
    }

    for (int io = 1; io <= p->max_substep_it; ++io) {
        /* step 1: K_src and the TKE seed */
        int ks_src = nz + 2, ke_src = 0;
        ksrc[1] = 0.0;
        ksrc[nz + 1] = 0.0;
        for (int kk = 2; kk <= nz; ++kk) {
            ksrc[kk] = ks_src_func(p->ri_crit, p->shearmix_rate, p->fri_curvature, n2[kk], s2[kk]);
            if (ksrc[kk] > 0.0) {
                if (ks_src > kk) ks_src = kk;
                ke_src = kk;
            }
        }
        for (int kk = 1; kk <= nz + 1; ++kk) kappa_src[kk] = ksrc[kk];
        for (int kk = 2; kk <= nz; ++kk) tkedec[kk] = sqrt(c_n2 * n2[kk] + c_s2 * s2[kk]);
        tke[1] = p->tke_bg;
        for (int kk = 2; kk <= nz; ++kk) {
            if (kappa[kk] > 0.0 && k_q[kk] > 0.0)
                tke[kk] = kappa[kk] / k_q[kk];
            else
                tke[kk] = tke_min;
        }
        tke[nz + 1] = tke_min;
        for (int kk = 1; kk <= nz + 1; ++kk) kappa_out[kk] = kappa[kk];

        if (ks_src > ke_src) {
            for (int kk = 1; kk <= nz + 1; ++kk) kappa_out[kk] = 0.0;
            for (int kk = 2; kk <= nz; ++kk) ild2[kk] = 0.0;
        } else {
            for (int kk = 1; kk <= nz + 1; ++kk) kq_tmp[kk] = k_q[kk];
            ks_find_kappa_tke(p, nz, tke_min, f2_val, c_n2, c_s2, ilambda2, n2, s2, kappa, kq_tmp, idz, hint, il2,
                              e1, tke, kappa_out, ksrc, tkedec, aq, dq, cq, dk, ck, ild2);
            for (int kk = 1; kk <= nz + 1; ++kk) k_q[kk] = kq_tmp[kk];
        }

        /* local_src of the adaptive-dt bands */
        local_src[1] = 0.0;
        local_src[nz + 1] = 0.0;
        for (int kk = 2; kk <= nz; ++kk) {
            if (hint[kk] > 0.0) {
                local_src[kk] = ksrc[kk] + kappa_0 * ((idz[kk - 1] + idz[kk]) / fmx(hint[kk], 1.0e-30) + ild2[kk]);
                double n2v = idz[kk - 1] * (kappa_out[kk - 1] - kappa_out[kk]) +
                             idz[kk] * (kappa_out[kk + 1] - kappa_out[kk]);
                if (n2v > 0.0) local_src[kk] = local_src[kk] + n2v / fmx(hint[kk], 1.0e-30);
            } else {
                local_src[kk] = ksrc[kk];
            }
        }

        /* step 2: active range of kappa_out */
        int ks_kap = nz + 2, ke_kap = 0;
        for (int kk = 2; kk <= nz; ++kk) {
            if (kappa_out[kk] > 0.0) {
                if (ks_kap > kk) ks_kap = kk;
                ke_kap = kk;
            }
        }
        if (ke_kap == nz) kappa_out[nz + 1] = 0.0;
        int no_mixing = ke_kap < ks_kap;

        /* step 3: dt_now */
        double dt_now;
        if (no_mixing || io == p->max_substep_it)
            dt_now = dt_rem;
        else
            dt_now = ks_adaptive_dt(p, nz, dt_rem, io, dbuoy_t, dbuoy_s, h, u_c, v_c, t_c, s_c, kappa_out, kappa_src,
                                    local_src, local_src_avg, ks_kap, ke_kap, idz_int);
        for (int kk = 2; kk <= nz; ++kk) local_src_avg[kk] = local_src_avg[kk] + dt_now * local_src[kk];
        double dt_wt = dt_now / dt;

        if (no_mixing) {
            for (int kk = 1; kk <= nz + 1; ++kk) tke_avg[kk] = tke_avg[kk] + dt_wt * tke[kk];
            dt_rem = 0.0;
        } else {
            /* predictor */
            int ks_ps = ks_kap - 1 > 1 ? ks_kap - 1 : 1;
            int ke_ps = ke_kap < nz ? ke_kap : nz;
            ks_projected_state(nz, dt_now, ks_ps, ke_ps, p->vel_underflow, dbuoy_t, dbuoy_s, h, idz_int, u_c, v_c,
                               t_c, s_c, kappa_out, u_ps, v_ps, t_ps, s_ps, c1_ps, n2p, s2p);
            for (int kk = 1; kk <= nz + 1; ++kk) kq_tmp[kk] = k_q[kk];
            ks_find_kappa_tke(p, nz, tke_min, f2_val, c_n2, c_s2, ilambda2, n2p, s2p, kappa_out, kq_tmp, idz, hint,
                              il2, e1, tke_pred, kappa_pred, ksrc, tkedec, aq, dq, cq, dk, ck, ild2);
            for (int kk = 1; kk <= nz + 1; ++kk) kappa_mid[kk] = 0.5 * (kappa_out[kk] + kappa_pred[kk]);
            int ks_mid = nz + 2, ke_mid = 0;
            for (int kk = 1; kk <= nz + 1; ++kk) {
                if (kappa_mid[kk] > 0.0) {
                    if (ks_mid > kk) ks_mid = kk;
                    ke_mid = kk;
                }
            }
            ks_ps = ks_mid - 1 > 1 ? ks_mid - 1 : 1;
            ke_ps = ke_mid < nz ? ke_mid : nz;

            /* corrector */
            ks_projected_state(nz, dt_now, ks_ps, ke_ps, p->vel_underflow, dbuoy_t, dbuoy_s, h, idz_int, u_c, v_c,
                               t_c, s_c, kappa_mid, u_ps, v_ps, t_ps, s_ps, c1_ps, n2c, s2c);
            ks_find_kappa_tke(p, nz, tke_min, f2_val, c_n2, c_s2, ilambda2, n2c, s2c, kappa_out, k_q, idz, hint, il2,
                              e1, tke_fin, kappa_pred2, ksrc, tkedec, aq, dq, cq, dk, ck, ild2);
            dt_rem = dt_rem - dt_now;
            for (int kk = 1; kk <= nz + 1; ++kk) {
                kappa_avg[kk] = kappa_avg[kk] + dt_wt * 0.5 * (kappa_out[kk] + kappa_pred2[kk]);
                tke_avg[kk] = tke_avg[kk] + dt_wt * 0.5 * (tke_pred[kk] + tke_fin[kk]);
                kappa[kk] = kappa_pred2[kk];
            }
            kappa[1] = 0.0;
            kappa[nz + 1] = 0.0;

            /* step 5: advance the real state for the next substep */
            if (dt_rem > 0.0) {
                for (int kk = 1; kk <= nz + 1; ++kk) kappa_mid[kk] = 0.5 * (kappa_out[kk] + kappa_pred2[kk]);
                ks_projected_state(nz, dt_now, 1, nz, p->vel_underflow, dbuoy_t, dbuoy_s, h, idz_int, u_c, v_c, t_c,
                                   s_c, kappa_mid, u_ps, v_ps, t_ps, s_ps, c1_ps, n2, s2);
                for (int k = 1; k <= nz; ++k) {
                    u_c[k] = u_ps[k];
                    v_c[k] = v_ps[k];
                    t_c[k] = t_ps[k];
                    s_c[k] = s_ps[k];
                }
            }
        }
        if (dt_rem <= 0.0) break;
    }

    for (int kk = 1; kk <= nz + 1; ++kk) {
        kappa_avg_sd[kk] = kappa_avg[kk];
        tke_avg_sd[kk] = tke_avg[kk];
    }
    kappa_avg_sd[1] = 0.0;
    kappa_avg_sd[nz + 1] = 0.0;
}

/* ---- the massless merge (rdb_massless.F90:51-180), surface-down.  Walking
 * down, a merged layer opens only when the current one already has mass and
 * the incoming layer is massive: a vanished layer folds into the massive
 * layer above it, a leading surface run into the first massive layer below,
 * a trailing bed run into the last massive layer above. */
static const double H_DIV_EPS = 1.0e-20;

/* massless_build_maps (:51-108): merged thicknesses hc[1..nzc]; kc[k] the
 * merged layer of layer k (kc[nz+1] = nzc+1); kf[K] the fractional position
 * of interface K inside merged layer kc[K] (0: on a merged interface). */
void vpo_massless_build_maps(const double *h, int nz, double h_min, int *nzc_out, double *hc, int *kc, double *kf)
{
    int nzc = 1;
    hc[1] = 0.0;
    for (int k = 1; k <= nz; ++k) {
        if (hc[nzc] > 0.0 && h[k] > h_min) {
            nzc = nzc + 1;
            hc[nzc] = 0.0;
        }
        kc[k] = nzc;
        hc[nzc] = hc[nzc] + h[k];
    }
    kc[nz + 1] = nzc + 1;
    kf[1] = 0.0;
    double dz_in = h[1];
    for (int k = 2; k <= nz; ++k) {
        if (kc[k] > kc[k - 1]) {
            kf[k] = 0.0;
            dz_in = h[k];
        } else {
            kf[k] = dz_in / fmx(hc[kc[k]], H_DIV_EPS);
            dz_in = dz_in + h[k];
        }
    }
    kf[nz + 1] = 0.0;
    *nzc_out = nzc;
}

/* massless_merge_fields (:110-154): thickness-weighted means on the merged grid */
void vpo_massless_merge_fields(const double *h, const int *kc, int nz, int nzc, const double *u, const double *v,
                               const double *t, const double *s, double *uc, double *vc, double *tc, double *sc)
{
    double hc_acc[nzc + 2];
    for (int kk = 1; kk <= nzc; ++kk) {
        hc_acc[kk] = 0.0;
        uc[kk] = 0.0;
        vc[kk] = 0.0;
        tc[kk] = 0.0;
        sc[kk] = 0.0;
    }
    for (int k = 1; k <= nz; ++k) {
        const int kk = kc[k];
        hc_acc[kk] = hc_acc[kk] + h[k];
        uc[kk] = uc[kk] + u[k] * h[k];
        vc[kk] = vc[kk] + v[k] * h[k];
        tc[kk] = tc[kk] + t[k] * h[k];
        sc[kk] = sc[kk] + s[k] * h[k];
    }
    for (int kk = 1; kk <= nzc; ++kk) {
        const double denom = fmx(hc_acc[kk], H_DIV_EPS);
        uc[kk] = uc[kk] / denom;
        vc[kk] = vc[kk] / denom;
        tc[kk] = tc[kk] / denom;
        sc[kk] = sc[kk] / denom;
    }
}

/* massless_interp_back (:156-180): an interface quantity of the merged grid
 * back on the original interfaces (lookup, or the linear blend inside a
 * merged layer) */
void vpo_massless_interp_back(const double *qc, const int *kc, const double *kf, int nz, double *q)
{
    for (int kk = 1; kk <= nz + 1; ++kk) {
        if (kf[kk] == 0.0)
            q[kk] = qc[kc[kk]];
        else
            q[kk] = (1.0 - kf[kk]) * qc[kc[kk]] + kf[kk] * qc[kc[kk] + 1];
    }
}

static void ks_params(const vphys_config *c, ks_par *p)
{
    p->ri_crit = c->ks_ri_crit;
    p->shearmix_rate = c->ks_shearmix_rate;
    p->fri_curvature = c->ks_fri_curvature;
    p->c_n = c->ks_c_n;
    p->c_s = c->ks_c_s;
    p->lambda = c->ks_lambda;
    p->lz_rescale = c->ks_lz_rescale;
    p->kappa_0 = c->ks_kappa_0;
    p->kappa_seed = c->ks_kappa_seed;
    p->kappa_trunc = c->ks_kappa_trunc;
    p->tke_bg = c->ks_tke_bg;
    p->tol_err = c->ks_tol_err;
    p->src_max_chg = c->ks_src_max_chg;
    p->vel_underflow = c->ks_vel_underflow;
    p->rho0 = c->rho0;
    p->alpha_t = c->eos_alpha_t;
    p->beta_s = c->eos_beta_s;
    p->max_inner_it = c->ks_max_inner_it;
    p->max_substep_it = c->ks_max_substep_it;
    p->eos_linear = c->eos_variant == 1;
}

/* kappa_shear_compute -> kappa_shear_column_kernel (:427-648), massless
 * merge off: gather with the surface-down flip and the H_VANISHED floor,
 * solve, scatter kd_shear / tke_shear with 0 at the bed and the surface. */
void vpo_kappa_shear(const vphys_config *c, vpo_state *s, double dt)
{
    if (c->idx_temperature < 0 || c->idx_salinity < 0) return;
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    ks_par p;
    ks_params(c, &p);
    const double *T = s->tr[c->idx_temperature];
    const double *S = s->tr[c->idx_salinity];
#pragma omp parallel for collapse(2) schedule(dynamic, 16)
    for (int j = 1; j <= ny; ++j) {
        for (int i = 1; i <= nx; ++i) {
            const int n = nz + 2;
            double h_sd[n], u_sd[n], v_sd[n], t_sd[n], s_sd[n];
            double idz[n], idz_int[n], hint[n], il2[n], kappa_avg_sd[n], tke_avg_sd[n];
            for (int k = 1; k <= nz + 1; ++k) {
                kappa_avg_sd[k] = 0.0;
                tke_avg_sd[k] = 0.0;
            }
            if (C2(s->wet, i, j) > 0.0) {
                for (int k = 1; k <= nz; ++k) {
                    int kg = nz + 1 - k;
                    h_sd[k] = C3(s->h, i, j, kg);
                    u_sd[k] = 0.5 * (s->u[(size_t)(i - 1) + (size_t)(nx + 1) * ((size_t)(j - 1) + (size_t)ny * (kg - 1))] +
                                     s->u[(size_t)i + (size_t)(nx + 1) * ((size_t)(j - 1) + (size_t)ny * (kg - 1))]);
                    v_sd[k] = 0.5 * (s->v[(size_t)(i - 1) + (size_t)nx * ((size_t)(j - 1) + (size_t)(ny + 1) * (kg - 1))] +
                                     s->v[(size_t)(i - 1) + (size_t)nx * ((size_t)j + (size_t)(ny + 1) * (kg - 1))]);
                }
                double f = s->coriolis ? C2(s->coriolis, i, j) : 0.0;
                double f2_val = f * f;
                /* merge only when asked and the column holds a vanished layer */
                int do_merge = 0;
                if (c->ks_massless_merge)
                    for (int k = 1; k <= nz; ++k)
                        if (h_sd[k] < H_VANISHED) {
                            do_merge = 1;
                            break;
                        }
                for (int k = 1; k <= nz; ++k) {
                    int kg = nz + 1 - k;
                    if (!do_merge) h_sd[k] = fmx(h_sd[k], H_VANISHED);
                    t_sd[k] = C3(T, i, j, kg);
                    s_sd[k] = C3(S, i, j, kg);
                }
                if (do_merge) {
                    int nzc, kc[n];
                    double kf[n], hc[n], uc[n], vc[n], tc[n], sc[n], kappa_c[n], tke_c[n];
                    vpo_massless_build_maps(h_sd, nz, H_VANISHED, &nzc, hc, kc, kf);
                    vpo_massless_merge_fields(h_sd, kc, nz, nzc, u_sd, v_sd, t_sd, s_sd, uc, vc, tc, sc);
                    ks_precompute(nzc, p.lz_rescale, hc, idz, idz_int, hint, il2);
                    ks_solve_column(&p, nzc, dt, f2_val, hc, uc, vc, tc, sc, idz, idz_int, hint, il2, kappa_c,
                                    tke_c);
                    vpo_massless_interp_back(kappa_c, kc, kf, nz, kappa_avg_sd);
                    vpo_massless_interp_back(tke_c, kc, kf, nz, tke_avg_sd);
                } else {
                    ks_precompute(nz, p.lz_rescale, h_sd, idz, idz_int, hint, il2);
                    ks_solve_column(&p, nz, dt, f2_val, h_sd, u_sd, v_sd, t_sd, s_sd, idz, idz_int, hint, il2,
                                    kappa_avg_sd, tke_avg_sd);
                }
            }
            for (int k = 1; k <= nz + 1; ++k) {
                int kg = nz + 2 - k;
                C3(s->kd_shear, i, j, kg) = kappa_avg_sd[k];
                C3(s->tke_shear, i, j, kg) = tke_avg_sd[k];
            }
            C3(s->kd_shear, i, j, 1) = 0.0;
            C3(s->kd_shear, i, j, nz + 1) = 0.0;
            C3(s->tke_shear, i, j, 1) = 0.0;
            C3(s->tke_shear, i, j, nz + 1) = 0.0;
        }
    }
}

/* kappa_shear_merge_into_kv_kt (:381-421), column form: interior
 * interfaces only. */
void vpo_kappa_shear_merge(const vphys_config *c, vpo_state *s)
{
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const double kv_fac = c->ks_prandtl_turb;
#pragma omp parallel for
    for (int k = 2; k <= nz; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                C3(s->kt, i, j, k) = C3(s->kt, i, j, k) + C3(s->kd_shear, i, j, k);
                C3(s->kv, i, j, k) = C3(s->kv, i, j, k) + kv_fac * C3(s->kd_shear, i, j, k);
            }
}
