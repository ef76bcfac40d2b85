// vphys_kshear.cu -- kappa-shear (Jackson, Hallberg & Legg 2008), column
// form: kappa_shear_compute -> kappa_shear_column_kernel
// (src/parameterizations/vertical/rdb_ocean_kappa_shear.F90:427-648) with the
// column solver ks_solve_column and its helpers (:953-1909).
//
// One thread solves one column.  The solve is a serial chain per column --
// Thomas sweeps inside Picard iterations inside adaptive substeps, with
// data-dependent trip counts -- so columns map to threads and the column's
// working arrays live in the thread's local memory (interleaved across the
// warp by the hardware, so a warp's accesses to one level coalesce; the
// L1/L2 hold the hot part).  Arrays are 1-based like the Fortran, surface-down
// (index 1 = the surface layer / interface), sized by a compile-time bucket of
// nz.  Where the reference keeps separate arrays whose lifetimes do not
// overlap (the projected state of the adaptive-dt trials and of the
// predictor/corrector; the step-1 source and the inner solve's source; the
// tolerance bands, recomputed per level from the same operands), one array
// serves: 43 arrays per column instead of ~60, with every value computed by
// the same operations in the same order as the reference, so the result is
// bit-identical to the CPU restatement (built without FMA contraction, as
// this file is with -fmad=false).
#include <cuda_runtime.h>

#include "vphys_device.cuh"
#include "vphys_kernels.cuh"

namespace vphys {
namespace {

struct KsPar {
    double ri_crit, shearmix_rate, fri_curvature, kappa_0, kappa_seed, kappa_trunc, tke_bg, tol_err;
    double src_max_chg, vel_underflow, rho0, alpha_t, beta_s, lz_rescale;
    double tke_min, c_n2, c_s2, ilambda2, tol_dksrc_low;
    int max_inner_it, max_substep_it, eos_linear;
};

template <int N>   // N = bucket + 2: indices 1..nz+1 with nz <= bucket
struct KsCol {
    // column constants
    double h[N], idz[N], idz_int[N], hint[N], il2[N], dbuoy_t[N], dbuoy_s[N], e1[N];
    // the column state advanced substep by substep
    double u_c[N], v_c[N], t_c[N], s_c[N];
    double kappa[N], k_q[N], kappa_avg[N], tke_avg[N], n2[N], s2[N], local_src_avg[N];
    // per substep
    double ksrc[N], tkedec[N], tke[N], kappa_out[N], kq_tmp[N], local_src[N], ild2[N];
    // inner (Picard) solve
    double aq[N], dq[N], cq[N], dk[N], ck[N];
    // projected state
    double u_ps[N], v_ps[N], t_ps[N], s_ps[N], c1[N], n2p[N], s2p[N];
    // predictor / corrector
    double tke_pred[N], kappa_pred[N], kappa_mid[N], tke_fin[N], kappa_pred2[N];
    int nwork;   // 4 per Picard iteration + 1 per projected-state sweep: the column's cost, for scheduling
};

// the massless merge's maps: the merged layer of each layer (kc[nz+1] =
// nzc+1) and each interface's fractional position inside its merged layer.
// Kept apart from KsCol so the solve's frame is the same with the merge off.
template <int N>
struct KsMap {
    int kc[N];
    double kf[N];
};

// ---- the massless merge (rdb_massless.F90:51-180), surface-down: walking
// down, a merged layer opens only when the current one has mass and the
// incoming layer is massive.  The raw column arrives in w.h, u_c, v_c, t_c,
// s_c and is moved to scratch (w.n2p for h, u_ps, v_ps, t_ps, s_ps); the
// merged column goes back to w.h, u_c, v_c, t_c, s_c (the thickness sums in
// w.s2p) with the maps in m.kc / m.kf.  Returns nzc.
template <int N>
__device__ __noinline__ int massless_merge(KsCol<N> &w, KsMap<N> &m, int nz)
{
    for (int k = 1; k <= nz; ++k) {
        w.n2p[k] = w.h[k];
        w.u_ps[k] = w.u_c[k];
        w.v_ps[k] = w.v_c[k];
        w.t_ps[k] = w.t_c[k];
        w.s_ps[k] = w.s_c[k];
    }
    const double *hr = w.n2p;
    double *hc = w.h;
    int nzc = 1;
    hc[1] = 0.0;
    for (int k = 1; k <= nz; ++k) {
        if (hc[nzc] > 0.0 && hr[k] > H_VANISHED) {
            nzc = nzc + 1;
            hc[nzc] = 0.0;
        }
        m.kc[k] = nzc;
        hc[nzc] = hc[nzc] + hr[k];
    }
    m.kc[nz + 1] = nzc + 1;
    m.kf[1] = 0.0;
    double dz_in = hr[1];
    for (int k = 2; k <= nz; ++k) {
        if (m.kc[k] > m.kc[k - 1]) {
            m.kf[k] = 0.0;
            dz_in = hr[k];
        } else {
            m.kf[k] = xdiv(dz_in, fmx(hc[m.kc[k]], H_DIV_EPS));
            dz_in = dz_in + hr[k];
        }
    }
    m.kf[nz + 1] = 0.0;
    double *acc = w.s2p;
    for (int kk = 1; kk <= nzc; ++kk) {
        acc[kk] = 0.0;
        w.u_c[kk] = 0.0;
        w.v_c[kk] = 0.0;
        w.t_c[kk] = 0.0;
        w.s_c[kk] = 0.0;
    }
    for (int k = 1; k <= nz; ++k) {
        const int kk = m.kc[k];
        acc[kk] = acc[kk] + hr[k];
        w.u_c[kk] = w.u_c[kk] + w.u_ps[k] * hr[k];
        w.v_c[kk] = w.v_c[kk] + w.v_ps[k] * hr[k];
        w.t_c[kk] = w.t_c[kk] + w.t_ps[k] * hr[k];
        w.s_c[kk] = w.s_c[kk] + w.s_ps[k] * hr[k];
    }
    for (int kk = 1; kk <= nzc; ++kk) {
        const double denom = fmx(acc[kk], H_DIV_EPS);
        w.u_c[kk] = xdiv(w.u_c[kk], denom);
        w.v_c[kk] = xdiv(w.v_c[kk], denom);
        w.t_c[kk] = xdiv(w.t_c[kk], denom);
        w.s_c[kk] = xdiv(w.s_c[kk], denom);
    }
    return nzc;
}

// massless_interp_back at one original interface K
template <int N>
__device__ __forceinline__ double interp_back(const KsMap<N> &m, const double *qc, int K)
{
    const int kc = m.kc[K];
    const double kf = m.kf[K];
    if (kf == 0.0) return qc[kc];
    return (1.0 - kf) * qc[kc] + kf * qc[kc + 1];
}

// the scatter of a merged column: kappa and TKE interpolated back onto the
// original interfaces, with the surface-down flip (local interface k ->
// global 0-based nz+1-k) and 0 on the surface and the bed
template <int N>
__device__ __noinline__ void scatter_merged(const KsCol<N> &w, const KsMap<N> &m, int nz, double *kd, double *tke, size_t col,
                                            size_t plane)
{
    kd[col + (size_t)nz * plane] = 0.0;
    tke[col + (size_t)nz * plane] = 0.0;
    for (int k = 2; k <= nz; ++k) {
        const size_t kg = (size_t)(nz + 1 - k);
        kd[col + kg * plane] = interp_back(m, w.kappa_avg, k);
        tke[col + kg * plane] = interp_back(m, w.tke_avg, k);
    }
    kd[col] = 0.0;
    tke[col] = 0.0;
}

// eos_specvol_derivs (rdb_eos.F90:1551-1622)
__device__ __forceinline__ void specvol_derivs(const KsPar &p, double T, double S, double pres, double &dsv_dt,
                                               double &dsv_ds)
{
    if (p.eos_linear) {
        dsv_dt = p.alpha_t / (p.rho0 * p.rho0);
        dsv_ds = -p.beta_s / (p.rho0 * p.rho0);
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

// ks_src_func (:953-969)
__device__ __forceinline__ double src_func(const KsPar &p, double n2, double s2)
{
    double ksrc = 0.0;
    if (n2 < p.ri_crit * s2) {
        const double dnom = p.ri_crit * s2 + p.fri_curvature * n2;
        if (dnom != 0.0 && s2 > 0.0) ksrc = xdiv(2.0 * p.shearmix_rate * sqrt(s2) * (p.ri_crit * s2 - n2), dnom);
    }
    return ksrc;
}

// ks_projected_state (:1034-1171): mix (u_c, v_c, t_c, s_c) with kap over
// dt_now inside layers [ks, ke] into the _ps arrays; N2, S2 into n2o, s2o.
//
// The reference first copies the whole input column into the outputs and
// zeroes c1; on the band path neither is observable (levels outside the band
// read the inputs, and every c1 the back-substitution reads is written by the
// forward sweep), so only the no-band path copies.
template <int N>
__device__ __noinline__ void projected_state(KsCol<N> &w, int nz, double dt_now, int ks, int ke, double vel_underflow,
                                             const double *__restrict__ kap, double *__restrict__ n2o,
                                             double *__restrict__ s2o)
{
    w.nwork += 1;
    const double *__restrict__ h = w.h;
    const double *__restrict__ idz_int = w.idz_int;
    const double *__restrict__ u0 = w.u_c, *__restrict__ v0 = w.v_c, *__restrict__ t0 = w.t_c, *__restrict__ s0 = w.s_c;
    double *__restrict__ u_o = w.u_ps, *__restrict__ v_o = w.v_ps, *__restrict__ t_o = w.t_ps, *__restrict__ s_o = w.s_ps;
    double *__restrict__ c1 = w.c1;

    if (ks <= ke && dt_now > 0.0) {
        double a_b = dt_now * kap[ks + 1] * idz_int[ks + 1];
        double b1 = 1.0 / (h[ks] + a_b);
        c1[ks + 1] = a_b * b1;
        double d1 = h[ks] * b1;
        u_o[ks] = b1 * h[ks] * u0[ks];
        v_o[ks] = b1 * h[ks] * v0[ks];
        t_o[ks] = b1 * h[ks] * t0[ks];
        s_o[ks] = b1 * h[ks] * s0[ks];
        double a_a;
        for (int k = ks + 1; k <= ke - 1; ++k) {
            a_a = a_b;
            a_b = dt_now * kap[k + 1] * idz_int[k + 1];
            const double bd1 = h[k] + d1 * a_a;
            b1 = 1.0 / (bd1 + a_b);
            c1[k + 1] = a_b * b1;
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
            b1nz = (ke == nz) ? 1.0 / ((h[ke] + d1 * a_a) + dt_now * kap[nz + 1] * idz_int[nz + 1]) : b1;
            u_o[ke] = b1nz * (h[ke] * u0[ke] + a_a * u_o[ke - 1]);
            v_o[ke] = b1nz * (h[ke] * v0[ke] + a_a * v_o[ke - 1]);
        } else {
            b1 = 1.0 / (h[ke] + a_a);
            t_o[ke] = b1 * h[ke] * t0[ke];
            s_o[ke] = b1 * h[ke] * s0[ke];
            b1nz = (ke == nz) ? 1.0 / (h[ke] + a_a + dt_now * kap[nz + 1] * idz_int[nz + 1]) : b1;
            u_o[ke] = b1nz * h[ke] * u0[ke];
            v_o[ke] = b1nz * h[ke] * v0[ke];
        }
        if (fabs(u_o[ke]) < vel_underflow) u_o[ke] = 0.0;
        if (fabs(v_o[ke]) < vel_underflow) v_o[ke] = 0.0;
        for (int k = ke - 1; k >= ks; --k) {
            u_o[k] = u_o[k] + c1[k + 1] * u_o[k + 1];
            v_o[k] = v_o[k] + c1[k + 1] * v_o[k + 1];
            t_o[k] = t_o[k] + c1[k + 1] * t_o[k + 1];
            s_o[k] = s_o[k] + c1[k + 1] * s_o[k + 1];
            if (fabs(u_o[k]) < vel_underflow) u_o[k] = 0.0;
            if (fabs(v_o[k]) < vel_underflow) v_o[k] = 0.0;
        }
    } else {
        for (int k = 1; k <= nz; ++k) {
            u_o[k] = (fabs(u0[k]) < vel_underflow) ? 0.0 : u0[k];
            v_o[k] = (fabs(v0[k]) < vel_underflow) ? 0.0 : v0[k];
            t_o[k] = t0[k];
            s_o[k] = s0[k];
        }
    }

    n2o[1] = 0.0;
    n2o[nz + 1] = 0.0;
    s2o[1] = 0.0;
    s2o[nz + 1] = 0.0;
    for (int kk = 2; kk <= nz; ++kk) {
        const bool in_a = kk - 1 >= ks && kk - 1 <= ke;
        const bool in_b = kk >= ks && kk <= ke;
        const double ua = in_a ? u_o[kk - 1] : u0[kk - 1], va = in_a ? v_o[kk - 1] : v0[kk - 1];
        const double ta = in_a ? t_o[kk - 1] : t0[kk - 1], sa = in_a ? s_o[kk - 1] : s0[kk - 1];
        const double ub = in_b ? u_o[kk] : u0[kk], vb = in_b ? v_o[kk] : v0[kk];
        const double tb = in_b ? t_o[kk] : t0[kk], sb = in_b ? s_o[kk] : s0[kk];
        double n2v = idz_int[kk] * (w.dbuoy_t[kk] * (ta - tb) + w.dbuoy_s[kk] * (sa - sb));
        if (n2v < 0.0) n2v = 0.0;
        n2o[kk] = n2v;
        const double du = ua - ub, dv = va - vb;
        s2o[kk] = (du * du + dv * dv) * (idz_int[kk] * idz_int[kk]);
    }
}

// ks_find_kappa_tke (:1173-1413): the Picard solve of the steady (kappa, TKE)
// pair for the buoyancy/shear profile (n2_in, s2_in), seeded from kseed and
// k_q; writes tke_o, kappa_o, updates k_q in place.  Uses w.ksrc, w.tkedec,
// w.ild2 and the aq..ck scratch.
// Every array argument is a different member of w from the ones the solve
// uses directly (the callers pass n2/s2 or n2p/s2p, kappa or kappa_out,
// k_q or kq_tmp, and the tke/kappa outputs of that call), hence __restrict__.
template <int N>
__device__ __noinline__ void find_kappa_tke(KsCol<N> &w, const KsPar &p, int nz, double f2_val,
                                            const double *__restrict__ n2_in, const double *__restrict__ s2_in,
                                            const double *__restrict__ kseed, double *__restrict__ k_q,
                                            double *__restrict__ tke_o, double *__restrict__ kappa_o)
{
    const double kappa_0 = p.kappa_0, kappa_trunc = p.kappa_trunc, tke_bg = p.tke_bg, tke_min = p.tke_min;
    const double *__restrict__ idz = w.idz, *__restrict__ hint = w.hint, *__restrict__ e1 = w.e1;
    double *__restrict__ ksrc = w.ksrc, *__restrict__ tkedec = w.tkedec, *__restrict__ ild2 = w.ild2;
    double *__restrict__ aq = w.aq, *__restrict__ dq = w.dq, *__restrict__ cq = w.cq, *__restrict__ dk = w.dk;
    double *__restrict__ ck = w.ck;
    const double *__restrict__ il2 = w.il2;
    int ks_src = nz + 2, ke_src = 0;
    ksrc[1] = 0.0;
    ksrc[nz + 1] = 0.0;
    for (int kk = 2; kk <= nz; ++kk) {
        ksrc[kk] = src_func(p, n2_in[kk], s2_in[kk]);
        if (ksrc[kk] > 0.0) {
            if (ks_src > kk) ks_src = kk;
            ke_src = kk;
        }
    }
    if (ks_src > ke_src) {
        for (int kk = 1; kk <= nz + 1; ++kk) {
            tke_o[kk] = tke_min;
            kappa_o[kk] = 0.0;
            k_q[kk] = 0.0;
        }
        return;
    }
    for (int kk = 2; kk <= nz; ++kk) tkedec[kk] = sqrt(p.c_n2 * n2_in[kk] + p.c_s2 * s2_in[kk]);
    tke_o[1] = tke_bg;
    for (int kk = 2; kk <= nz; ++kk)
        tke_o[kk] = (kseed[kk] > 0.0 && k_q[kk] > 0.0) ? xdiv(kseed[kk], k_q[kk]) : tke_min;
    tke_o[nz + 1] = tke_min;
    for (int kk = 1; kk <= nz + 1; ++kk) kappa_o[kk] = kseed[kk];
    kappa_o[1] = 0.0;
    kappa_o[nz + 1] = 0.0;

    int ks_kap = 2, ke_kap = nz, ks_kp = 2, ke_kp = nz;
    for (int it = 1; it <= p.max_inner_it; ++it) {
        w.nwork += 4;
        // (a) TKE sweep (ke_tke: an interface index, nz+1 = the bed)
        int ke_tke = (ke_kap > ke_kp ? ke_kap : ke_kp) + 1;
        if (ke_tke > nz + 1) ke_tke = nz + 1;
        const int kmax = ke_tke < nz ? ke_tke : nz;
#pragma unroll 4
        for (int k = 1; k <= kmax; ++k) aq[k] = (0.5 * (kappa_o[k] + kappa_o[k + 1]) + kappa_0) * idz[k];
        dq[1] = -tke_o[1];
        tke_o[1] = tke_bg;
        cq[2] = 0.0;
        double cqc_l = 1.0;
        for (int kk = 2; kk <= ke_tke - 1; ++kk) {
            dq[kk] = -tke_o[kk];
            const double tsrc_l = (kappa_o[kk] + kappa_0) * s2_in[kk] + tke_bg * tkedec[kk];
            const double bqd1_l = hint[kk] * (tkedec[kk] + n2_in[kk] * k_q[kk]) + cqc_l * aq[kk - 1];
            const double bq_l = 1.0 / (bqd1_l + aq[kk]);
            tke_o[kk] = bq_l * (hint[kk] * tsrc_l + aq[kk - 1] * tke_o[kk - 1]);
            cq[kk + 1] = aq[kk] * bq_l;
            cqc_l = bqd1_l * bq_l;
        }
        if (ke_tke == nz + 1) {
            tke_o[nz + 1] = tke_min;
            dq[nz + 1] = 0.0;
        } else {
            const int kk = ke_tke;
            const double tsrc_l = kappa_0 * s2_in[kk] + tke_bg * tkedec[kk];
            const double bq_l = 1.0 / (hint[kk] * tkedec[kk] + cqc_l * aq[kk - 1] + aq[kk]);
            cq[kk + 1] = aq[kk] * bq_l;
            dq[kk] = -tke_o[kk];
            const double raw_l = bq_l * (hint[kk] * tsrc_l + aq[kk - 1] * tke_o[kk - 1]);
            const double dnom_l = 1.0 - cq[kk + 1] * e1[kk + 1];
            if (fabs(dnom_l) > 1.0e-30)
                tke_o[kk] = fmx(xdiv(raw_l + cq[kk + 1] * (tke_o[kk + 1] - e1[kk + 1] * tke_o[kk]), dnom_l), tke_min);
            else
                tke_o[kk] = fmx(raw_l, tke_min);
            dq[kk] = tke_o[kk] + dq[kk];
            for (int k2 = ke_tke + 1; k2 <= nz + 1; ++k2) {
                dq[k2] = e1[k2] * dq[k2 - 1];
                tke_o[k2] = fmx(tke_o[k2] + dq[k2], tke_min);
                if (fabs(dq[k2]) < 1.0e-16 * tke_o[k2]) break;
            }
        }
        for (int kk = ke_tke - 1; kk >= 1; --kk) {
            tke_o[kk] = fmx(tke_o[kk] + cq[kk + 1] * tke_o[kk + 1], tke_min);
            dq[kk] = tke_o[kk] + dq[kk];
        }

        // (b) kappa sweep with the truncation ramp and range tracking
        ks_kp = ks_kap;
        ke_kp = ke_kap;
#pragma unroll 4
        for (int kk = 2; kk <= nz; ++kk)
            ild2[kk] = (tke_o[kk] > 0.0) ? xdiv(n2_in[kk] * p.ilambda2 + f2_val, tke_o[kk]) + il2[kk] : 1.0e30;
        dk[1] = 0.0;
        ck[2] = 0.0;
        double ckc_l = 1.0;
        int ke_new = 0;
        for (int kk = 2; kk <= nz; ++kk) {
            dk[kk] = -kappa_o[kk];
            const double bkd1_l = hint[kk] * ild2[kk] + ckc_l * idz[kk - 1];
            const double bk_l = 1.0 / (bkd1_l + idz[kk]);
            kappa_o[kk] = bk_l * (idz[kk - 1] * kappa_o[kk - 1] + hint[kk] * ksrc[kk]);
            ck[kk + 1] = idz[kk] * bk_l;
            ckc_l = bkd1_l * bk_l;
            const double trv = ckc_l * kappa_trunc;
            const double tr2v = 2.0 * trv;
            if (kappa_o[kk] < trv) {
                kappa_o[kk] = 0.0;
                if (kk > ke_src) {
                    ke_kap = kk - 1;
                    k_q[kk] = 0.0;
                    break;
                }
            } else if (kappa_o[kk] < tr2v) {
                kappa_o[kk] = 2.0 * (kappa_o[kk] - trv);
            }
            ke_new = kk;
        }
        if (ke_new > 0) ke_kap = ke_new;
        if (ke_kap >= 1 && tke_o[ke_kap] > 0.0) k_q[ke_kap] = xdiv(kappa_o[ke_kap], tke_o[ke_kap]);
        dk[ke_kap] = dk[ke_kap] + kappa_o[ke_kap];
        for (int kk = ke_kap + 2; kk <= ke_kp + 1; ++kk) {
            if (kk > nz) break;
            dk[kk] = -kappa_o[kk];
            kappa_o[kk] = 0.0;
            k_q[kk] = 0.0;
        }
        int ks_new = 2;
        for (int kk = ke_kap - 1; kk >= 2; --kk) {
            kappa_o[kk] = kappa_o[kk] + ck[kk + 1] * kappa_o[kk + 1];
            if (kappa_o[kk] <= kappa_trunc) {
                kappa_o[kk] = 0.0;
                if (kk < ks_src) {
                    ks_kap = kk + 1;
                    k_q[kk] = 0.0;
                    break;
                }
            } else if (kappa_o[kk] < 2.0 * kappa_trunc) {
                kappa_o[kk] = 2.0 * (kappa_o[kk] - kappa_trunc);
            }
            dk[kk] = dk[kk] + kappa_o[kk];
            k_q[kk] = (tke_o[kk] > 0.0) ? xdiv(kappa_o[kk], tke_o[kk]) : 0.0;
            ks_new = kk;
        }
        ks_kap = ks_new > 2 ? ks_new : 2;
        for (int kk = ks_kp; kk <= ks_kap - 2; ++kk) {
            if (kk < 2) continue;
            kappa_o[kk] = 0.0;
            k_q[kk] = 0.0;
        }

        // (c) Picard convergence
        const int k_lo = ks_kap < ks_kp ? ks_kap : ks_kp;
        const int k_hi = ke_kap > ke_kp ? ke_kap : ke_kp;
        bool conv = true;
        for (int kk = k_lo; kk <= k_hi; ++kk) {
            const double lhs_l = fabs(dk[kk]);
            const double rhs_l = p.tol_err * (kappa_0 + kappa_o[kk] - 0.5 * dk[kk]);
            if (lhs_l > rhs_l) {
                conv = false;
                break;
            }
        }
        if (conv) break;
    }
    kappa_o[1] = 0.0;
    kappa_o[nz + 1] = 0.0;
}

// the source-change test of one trial step of ks_adaptive_dt; the bands
// tol_max / tol_min_a / tol_chg_a (:1455-1459) formed per level from w.ksrc
// (the substep's K_src), w.local_src and w.local_src_avg
template <int N>
__device__ __forceinline__ bool dt_valid(const KsCol<N> &w, const KsPar &p, int k_lo, int k_hi, double dt_try)
{
    const double idtt = (dt_try > 0.0) ? 1.0 / dt_try : 0.0;
    const double tol2_l = 2.0 * p.tol_err;
    for (int kk = k_lo; kk <= k_hi; ++kk) {
        const double ksrc_acc = w.ksrc[kk];
        const double tol_min_a = ksrc_acc - p.tol_dksrc_low * w.local_src[kk];
        const double tol_chg_a = tol2_l * w.local_src_avg[kk];
        if (w.n2p[kk] < p.ri_crit * w.s2p[kk]) {
            const double ksrc_tst = src_func(p, w.n2p[kk], w.s2p[kk]);
            const double tol_max = ksrc_acc + p.src_max_chg * w.local_src[kk];
            const double upper_t = fmx(tol_max, ksrc_acc + idtt * tol_chg_a);
            const double lower_t = fmn(tol_min_a, ksrc_acc - idtt * tol_chg_a);
            if (ksrc_tst > upper_t || ksrc_tst < lower_t) return false;
        } else {
            const double lower_t = fmn(tol_min_a, ksrc_acc - idtt * tol_chg_a);
            if (0.0 < lower_t) return false;
        }
    }
    return true;
}

// ks_adaptive_dt (:1415-1543): a halving pass, then a 5-step refinement
template <int N>
__device__ __noinline__ double adaptive_dt(KsCol<N> &w, const KsPar &p, int nz, double dt_rem, int itt_outer,
                                           int ks_kap, int ke_kap)
{
    const int k_lo = ks_kap - 1 > 2 ? ks_kap - 1 : 2;
    const int k_hi = ke_kap + 1 < nz ? ke_kap + 1 : nz;
    const int ks_lyr = ks_kap - 1 > 1 ? ks_kap - 1 : 1;
    const int ke_lyr = ke_kap < nz ? ke_kap : nz;
    double dt_tst = dt_rem;
    bool valid = false;
    const int max_halvings = (p.max_substep_it + 1 - itt_outer) / 2;
    const int nh = max_halvings > 1 ? max_halvings : 1;
    for (int ih = 1; ih <= nh; ++ih) {
        projected_state(w, nz, 0.5 * dt_tst, ks_lyr, ke_lyr, p.vel_underflow, w.kappa_out, w.n2p, w.s2p);
        valid = dt_valid(w, p, k_lo, k_hi, dt_tst);
        if (valid) break;
        dt_tst = 0.5 * dt_tst;
    }
    double dt_inc = 0.0;
    if (dt_tst < dt_rem && valid) {
        dt_inc = 0.5 * dt_tst;
        for (int ir = 1; ir <= 5; ++ir) {
            const double dt_try = dt_tst + dt_inc;
            projected_state(w, nz, 0.5 * dt_try, ks_lyr, ke_lyr, p.vel_underflow, w.kappa_out, w.n2p, w.s2p);
            if (dt_valid(w, p, k_lo, k_hi, dt_try)) dt_tst = dt_try;
            dt_inc = 0.5 * dt_inc;
        }
    }
    return fmn(dt_tst * (1.0 + p.tol_err) + dt_inc, dt_rem);
}

// ks_precompute + ks_solve_column (:971-1032, 1545-1909) for one column whose
// gathered thickness (floored), centred velocities and T, S sit in w.h,
// w.u_c, w.v_c, w.t_c, w.s_c (the pre-step works in place: each level's
// inputs are read before its output is written).
template <int N>
__device__ __noinline__ void solve_column(KsCol<N> &w, const KsPar &p, int nz, double dt, double f2_val)
{
    double *h = w.h, *idz = w.idz, *idz_int = w.idz_int, *hint = w.hint, *il2 = w.il2;
    // ---- ks_precompute
    {
        const double i_lz2 = 1.0 / (p.lz_rescale * p.lz_rescale);
        for (int k = 1; k <= nz; ++k) idz[k] = 1.0 / h[k];
        idz_int[1] = 2.0 / h[1];
        for (int k = 2; k <= nz; ++k) idz_int[k] = 2.0 / (h[k - 1] + h[k]);
        idz_int[nz + 1] = 2.0 / h[nz];
        hint[1] = 0.0;
        if (nz >= 2) {
            hint[2] = h[1];
            for (int k = 2; k <= nz - 1; ++k) {
                const double hk = h[k], hkm1 = h[k - 1], hkp1 = h[k + 1];
                const double norm_l = 1.0 / (hk * (hkm1 + hkp1) + 2.0 * hkm1 * hkp1);
                const double wt_a = (hk + hkp1) * hkm1 * norm_l;
                const double wt_b = (hkm1 + hk) * hkp1 * norm_l;
                hint[k] = hint[k] + hk * wt_a;
                hint[k + 1] = hk * wt_b;
            }
            hint[nz] = hint[nz] + h[nz];
        }
        hint[nz + 1] = 0.0;
        // the depth below each interface, dbot (k = nz..1), kept in e1 until e1 is formed
        double *dbot = w.e1;
        dbot[nz + 1] = 0.0;
        for (int k = nz; k >= 1; --k) dbot[k] = dbot[k + 1] + h[k];
        il2[1] = 0.0;
        il2[nz + 1] = 0.0;
        double dtop = 0.0;
        for (int k = 2; k <= nz; ++k) {
            dtop = dtop + h[k - 1];
            if (dtop > 0.0 && dbot[k] > 0.0) {
                const double t = dtop + dbot[k];
                const double b = dtop * dbot[k];
                il2[k] = xdiv(i_lz2 * (t * t), b * b);
            } else {
                il2[k] = 0.0;
            }
        }
    }

    const double kappa_0 = p.kappa_0;
    const double k0dt = dt * kappa_0;
    double *u_c = w.u_c, *v_c = w.v_c, *t_c = w.t_c, *s_c = w.s_c;
    // ---- background pre-step with kappa_0 (no-slip bed for u, v; insulating T, S)
    if (nz == 1) {
        const double b1_l = 1.0 / (h[1] + k0dt * idz_int[2]);
        u_c[1] = b1_l * h[1] * u_c[1];
        v_c[1] = b1_l * h[1] * v_c[1];
    } else {
        double *cqsav = w.cq;
        double a1n = k0dt * idz_int[2];
        double b1_l = 1.0 / (h[1] + a1n);
        cqsav[2] = a1n * b1_l;
        double d1_l = h[1] * b1_l;
        u_c[1] = b1_l * h[1] * u_c[1];
        v_c[1] = b1_l * h[1] * v_c[1];
        t_c[1] = b1_l * h[1] * t_c[1];
        s_c[1] = b1_l * h[1] * s_c[1];
        double a1c;
        for (int k = 2; k <= nz - 1; ++k) {
            a1c = a1n;
            a1n = k0dt * idz_int[k + 1];
            const double bd1_l = h[k] + d1_l * a1c;
            b1_l = 1.0 / (bd1_l + a1n);
            u_c[k] = b1_l * (h[k] * u_c[k] + a1c * u_c[k - 1]);
            v_c[k] = b1_l * (h[k] * v_c[k] + a1c * v_c[k - 1]);
            t_c[k] = b1_l * (h[k] * t_c[k] + a1c * t_c[k - 1]);
            s_c[k] = b1_l * (h[k] * s_c[k] + a1c * s_c[k - 1]);
            cqsav[k + 1] = a1n * b1_l;
            d1_l = bd1_l * b1_l;
        }
        a1c = a1n;
        const double base_l = h[nz] + d1_l * a1c;
        const double b1ns = 1.0 / (base_l + k0dt * idz_int[nz + 1]);
        const double b1in = 1.0 / base_l;
        u_c[nz] = b1ns * (h[nz] * u_c[nz] + a1c * u_c[nz - 1]);
        v_c[nz] = b1ns * (h[nz] * v_c[nz] + a1c * v_c[nz - 1]);
        t_c[nz] = b1in * (h[nz] * t_c[nz] + a1c * t_c[nz - 1]);
        s_c[nz] = b1in * (h[nz] * s_c[nz] + a1c * s_c[nz - 1]);
        cqsav[nz + 1] = 0.0;
        for (int k = nz - 1; k >= 1; --k) {
            u_c[k] = u_c[k] + cqsav[k + 1] * u_c[k + 1];
            v_c[k] = v_c[k] + cqsav[k + 1] * v_c[k + 1];
            t_c[k] = t_c[k] + cqsav[k + 1] * t_c[k + 1];
            s_c[k] = s_c[k] + cqsav[k + 1] * s_c[k + 1];
        }
    }

    // ---- frozen interface buoyancy derivatives at the hydrostatic pressure
    double *n2 = w.n2, *s2 = w.s2;
    w.dbuoy_t[1] = 0.0;
    w.dbuoy_s[1] = 0.0;
    w.dbuoy_t[nz + 1] = 0.0;
    w.dbuoy_s[nz + 1] = 0.0;
    {
        const double g_rho0 = GRAVITY * p.rho0;
        double p_int = 0.0;
        for (int kk = 2; kk <= nz; ++kk) {
            const double dpres = g_rho0 * h[kk - 1];
            p_int = p_int + dpres;
            const double t_int = 0.5 * (t_c[kk - 1] + t_c[kk]);
            const double s_int = 0.5 * (s_c[kk - 1] + s_c[kk]);
            double dsv_dt_k, dsv_ds_k;
            specvol_derivs(p, t_int, s_int, p_int, dsv_dt_k, dsv_ds_k);
            w.dbuoy_t[kk] = g_rho0 * dsv_dt_k;
            w.dbuoy_s[kk] = g_rho0 * dsv_ds_k;
        }
    }
    // ---- initial N2, S2
    n2[1] = 0.0;
    n2[nz + 1] = 0.0;
    s2[1] = 0.0;
    s2[nz + 1] = 0.0;
    for (int kk = 2; kk <= nz; ++kk) {
        double n2v = idz_int[kk] * (w.dbuoy_t[kk] * (t_c[kk - 1] - t_c[kk]) + w.dbuoy_s[kk] * (s_c[kk - 1] - s_c[kk]));
        if (n2v < 0.0) n2v = 0.0;
        n2[kk] = n2v;
        const double du = u_c[kk - 1] - u_c[kk], dv = v_c[kk - 1] - v_c[kk];
        s2[kk] = (du * du + dv * dv) * (idz_int[kk] * idz_int[kk]);
    }
    // ---- e1 tail recursion
    {
        double *e1 = w.e1;
        e1[nz + 1] = 0.0;
        double ome_l = 1.0;
        double eden2_l = kappa_0 * idz[nz];
        for (int kk = nz; kk >= 2; --kk) {
            const double eden1_l = hint[kk] * sqrt(p.c_n2 * n2[kk] + p.c_s2 * s2[kk]) + ome_l * eden2_l;
            eden2_l = kappa_0 * idz[kk - 1];
            const double i_eden_l = 1.0 / (eden2_l + eden1_l);
            e1[kk] = eden2_l * i_eden_l;
            ome_l = eden1_l * i_eden_l;
        }
        e1[1] = 0.0;
    }

    double *kappa = w.kappa, *k_q = w.k_q, *kappa_avg = w.kappa_avg, *tke_avg = w.tke_avg;
    double *kappa_out = w.kappa_out, *local_src = w.local_src, *local_src_avg = w.local_src_avg;
    for (int kk = 1; kk <= nz + 1; ++kk) {
        k_q[kk] = 0.0;
        kappa_avg[kk] = 0.0;
        tke_avg[kk] = 0.0;
        kappa[kk] = p.kappa_seed;
    }
    kappa[1] = 0.0;
    kappa[nz + 1] = 0.0;
    double dt_rem = dt;
    local_src_avg[1] = 0.0;
    local_src_avg[nz + 1] = 0.0;
    for (int kk = 2; kk <= nz; ++kk) local_src_avg[kk] = (hint[kk] > 0.0) ? xdiv(0.1 * k0dt * idz_int[kk], hint[kk]) : 0.0;

    // ---- adaptive outer substepping
    for (int io = 1; io <= p.max_substep_it; ++io) {
        int ks_src = nz + 2, ke_src = 0;
        w.ksrc[1] = 0.0;
        w.ksrc[nz + 1] = 0.0;
        for (int kk = 2; kk <= nz; ++kk) {
            w.ksrc[kk] = src_func(p, n2[kk], s2[kk]);
            if (w.ksrc[kk] > 0.0) {
                if (ks_src > kk) ks_src = kk;
                ke_src = kk;
            }
        }
        if (ks_src > ke_src) {
            // no source: the TKE seed is what the step averages
            double *tke = w.tke;
            tke[1] = p.tke_bg;
            for (int kk = 2; kk <= nz; ++kk) tke[kk] = (kappa[kk] > 0.0 && k_q[kk] > 0.0) ? xdiv(kappa[kk], k_q[kk]) : p.tke_min;
            tke[nz + 1] = p.tke_min;
            for (int kk = 1; kk <= nz + 1; ++kk) kappa_out[kk] = 0.0;
            for (int kk = 2; kk <= nz; ++kk) w.ild2[kk] = 0.0;
        } else {
            // find_kappa_tke re-forms the same source, decay and TKE seed,
            // seeds kappa_out from kappa, and leaves in k_q what the
            // reference copies back from its k_q copy
            find_kappa_tke(w, p, nz, f2_val, n2, s2, kappa, k_q, w.tke, kappa_out);
        }

        // local_src of the adaptive-dt bands
        local_src[1] = 0.0;
        local_src[nz + 1] = 0.0;
        for (int kk = 2; kk <= nz; ++kk) {
            if (hint[kk] > 0.0) {
                const double hmax = fmx(hint[kk], 1.0e-30);
                double ls = w.ksrc[kk] + kappa_0 * (xdiv(idz[kk - 1] + idz[kk], hmax) + w.ild2[kk]);
                const double n2v = idz[kk - 1] * (kappa_out[kk - 1] - kappa_out[kk]) +
                                   idz[kk] * (kappa_out[kk + 1] - kappa_out[kk]);
                if (n2v > 0.0) ls = ls + xdiv(n2v, hmax);
                local_src[kk] = ls;
            } else {
                local_src[kk] = w.ksrc[kk];
            }
        }

        int ks_kap = nz + 2, ke_kap = 0;
        for (int kk = 2; kk <= nz; ++kk) {
            if (kappa_out[kk] > 0.0) {
                if (ks_kap > kk) ks_kap = kk;
                ke_kap = kk;
            }
        }
        if (ke_kap == nz) kappa_out[nz + 1] = 0.0;
        const bool no_mixing = ke_kap < ks_kap;

        const double dt_now = (no_mixing || io == p.max_substep_it) ? dt_rem
                                                                    : adaptive_dt(w, p, nz, dt_rem, io, ks_kap, ke_kap);
        for (int kk = 2; kk <= nz; ++kk) local_src_avg[kk] = local_src_avg[kk] + dt_now * local_src[kk];
        const double dt_wt = xdiv(dt_now, dt);

        if (no_mixing) {
            for (int kk = 1; kk <= nz + 1; ++kk) tke_avg[kk] = tke_avg[kk] + dt_wt * w.tke[kk];
            dt_rem = 0.0;
        } else {
            // predictor
            int ks_ps = ks_kap - 1 > 1 ? ks_kap - 1 : 1;
            int ke_ps = ke_kap < nz ? ke_kap : nz;
            projected_state(w, nz, dt_now, ks_ps, ke_ps, p.vel_underflow, kappa_out, w.n2p, w.s2p);
            for (int kk = 1; kk <= nz + 1; ++kk) w.kq_tmp[kk] = k_q[kk];
            find_kappa_tke(w, p, nz, f2_val, w.n2p, w.s2p, kappa_out, w.kq_tmp, w.tke_pred, w.kappa_pred);
            int ks_mid = nz + 2, ke_mid = 0;
            for (int kk = 1; kk <= nz + 1; ++kk) {
                const double km = 0.5 * (kappa_out[kk] + w.kappa_pred[kk]);
                w.kappa_mid[kk] = km;
                if (km > 0.0) {
                    if (ks_mid > kk) ks_mid = kk;
                    ke_mid = kk;
                }
            }
            ks_ps = ks_mid - 1 > 1 ? ks_mid - 1 : 1;
            ke_ps = ke_mid < nz ? ke_mid : nz;
            // corrector (the real K_Q now)
            projected_state(w, nz, dt_now, ks_ps, ke_ps, p.vel_underflow, w.kappa_mid, w.n2p, w.s2p);
            find_kappa_tke(w, p, nz, f2_val, w.n2p, w.s2p, kappa_out, k_q, w.tke_fin, w.kappa_pred2);
            dt_rem = dt_rem - dt_now;
            const double half_wt = dt_wt * 0.5;
            for (int kk = 1; kk <= nz + 1; ++kk) {
                kappa_avg[kk] = kappa_avg[kk] + half_wt * (kappa_out[kk] + w.kappa_pred2[kk]);
                tke_avg[kk] = tke_avg[kk] + half_wt * (w.tke_pred[kk] + w.tke_fin[kk]);
                kappa[kk] = w.kappa_pred2[kk];
            }
            kappa[1] = 0.0;
            kappa[nz + 1] = 0.0;
            // advance the real state for the next substep
            if (dt_rem > 0.0) {
                for (int kk = 1; kk <= nz + 1; ++kk) w.kappa_mid[kk] = 0.5 * (kappa_out[kk] + w.kappa_pred2[kk]);
                projected_state(w, nz, dt_now, 1, nz, p.vel_underflow, w.kappa_mid, n2, s2);
                for (int k = 1; k <= nz; ++k) {
                    u_c[k] = w.u_ps[k];
                    v_c[k] = w.v_ps[k];
                    t_c[k] = w.t_ps[k];
                    s_c[k] = w.s_ps[k];
                }
            }
        }
        if (dt_rem <= 0.0) break;
    }
}

// Minimum resident 64-thread blocks per SM: 16 caps the solve at 64
// registers (a few bytes of spill) for 32 warps per SM.  The solve waits on
// its local-memory columns (the working sets of the resident threads far
// exceed L1 and L2), so warps in flight buy more than registers:
// 1440x1080x75, ordered columns: 824 ms at 128 registers (16 warps/SM),
// 666 ms at 80, 588 ms at 64.
#ifndef VPHYS_KS_MINB
#define VPHYS_KS_MINB 16
#endif

// Thread t solves column order[t] (t itself without an order) and records
// the column's cost in work[col] (0 for land) for the next call's ordering.
// MERGE instantiates the massless merge; without it the kernel carries none
// of the merge's code (its call graph alone costs the solve registers).
template <int N, bool MERGE>
__global__ void __launch_bounds__(64, VPHYS_KS_MINB) k_kappa_shear(Params p, KsPar kp, double dt,
                                                                    const int *__restrict__ order, int *work)
{
    const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (t >= p.plane) return;
    const size_t col = order ? (size_t)order[t] : t;
    const int nx = p.nx, nz = p.nz;
    const int i = (int)(col % (size_t)nx), j = (int)(col / (size_t)nx);
    double *kd = p.kd_shear, *tke = p.tke_shear;
    const size_t plane = p.plane;
    if (!(p.wet[col] > 0.0)) {
        for (int k = 0; k <= nz; ++k) {
            kd[col + (size_t)k * plane] = 0.0;
            tke[col + (size_t)k * plane] = 0.0;
        }
        if (work) work[col] = 0;
        return;
    }
    KsCol<N> w;
    w.nwork = 0;
    const double *T = p.tr[p.cfg.idx_temperature], *S = p.tr[p.cfg.idx_salinity];
    const size_t ucol = (size_t)j * (nx + 1) + i, vcol = col;
    // the massless merge engages only when asked and the column holds a vanished layer
    bool do_merge = false;
    if (MERGE)
        for (int k = 1; k <= nz; ++k)
            if (p.h[col + (size_t)(nz - k) * plane] < H_VANISHED) {
                do_merge = true;
                break;
            }
    // gather with the flip (local k = 1 the surface) into the solve's arrays;
    // a merged column keeps its raw thicknesses, the others the H_VANISHED floor
    for (int k = 1; k <= nz; ++k) {
        const size_t kg = (size_t)(nz - k);   // 0-based global layer of local layer k
        const double hk = p.h[col + kg * plane];
        w.h[k] = do_merge ? hk : fmx(hk, H_VANISHED);
        w.u_c[k] = 0.5 * (p.u[ucol + kg * p.plane_u] + p.u[ucol + 1 + kg * p.plane_u]);
        w.v_c[k] = 0.5 * (p.v[vcol + kg * p.plane_v] + p.v[vcol + nx + kg * p.plane_v]);
        w.t_c[k] = T[col + kg * plane];
        w.s_c[k] = S[col + kg * plane];
    }
    const double f = p.coriolis ? p.coriolis[col] : 0.0;
    KsMap<MERGE ? N : 1> m;
    int nzs = nz;
    if constexpr (MERGE)
        if (do_merge) nzs = massless_merge(w, m, nz);
    solve_column(w, kp, nzs, dt, f * f);
    if constexpr (MERGE) {
        if (do_merge) {
            w.kappa_avg[1] = 0.0;   // ks_solve_column's closed top and bottom (:1905-1908), read by the interpolation
            w.kappa_avg[nzs + 1] = 0.0;
            scatter_merged(w, m, nz, kd, tke, col, plane);
        }
    }
    if (!do_merge) {
        // scatter with the flip: local interface k -> global interface nz+2-k
        // (1-based), 0 on the bed and the surface
        for (int k = 1; k <= nz + 1; ++k) {
            const size_t kg = (size_t)(nz + 1 - k);
            const bool edge = (k == 1 || k == nz + 1);
            kd[col + kg * plane] = edge ? 0.0 : w.kappa_avg[k];
            tke[col + kg * plane] = edge ? 0.0 : w.tke_avg[k];
        }
    }
    if (work) work[col] = w.nwork;
}

// ---- the solve order: columns bucketed by their last cost, heaviest first.
// A warp then carries columns of like cost (a warp runs as long as its
// slowest lane) and the long columns start first.  Which thread solves which
// column changes nothing in any column's result.
constexpr int KS_NB = 1024;

__device__ __forceinline__ int ks_bucket(int work)
{
    const int key = work >> 3;
    return KS_NB - 1 - (key < KS_NB - 1 ? key : KS_NB - 1);
}

__global__ void k_ks_hist(const int *__restrict__ work, size_t n, unsigned *hist)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int b = ks_bucket(work[i]);
        // one atomic per distinct bucket of the warp (land comes in runs)
        const unsigned peers = __match_any_sync(__activemask(), b);
        if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&hist[b], (unsigned)__popc(peers));
    }
}

// exclusive scan of the KS_NB bucket counts, in place (one block of KS_NB threads)
__global__ void __launch_bounds__(KS_NB) k_ks_scan(unsigned *hist)
{
    __shared__ unsigned sh[KS_NB];
    const int t = threadIdx.x;
    const unsigned v = hist[t];
    sh[t] = v;
    __syncthreads();
    for (int off = 1; off < KS_NB; off <<= 1) {
        const unsigned a = (t >= off) ? sh[t - off] : 0u;
        __syncthreads();
        sh[t] += a;
        __syncthreads();
    }
    hist[t] = sh[t] - v;
}

__global__ void k_ks_scatter(const int *__restrict__ work, size_t n, unsigned *offs, int *order)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int b = ks_bucket(work[i]);
        const unsigned peers = __match_any_sync(__activemask(), b);
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(peers) - 1;
        unsigned base = 0;
        if (lane == leader) base = atomicAdd(&offs[b], (unsigned)__popc(peers));
        base = __shfl_sync(peers, base, leader);
        order[base + __popc(peers & ((1u << lane) - 1u))] = (int)i;
    }
}

KsPar ks_par_of(const vphys_config &c)
{
    KsPar k{};
    k.ri_crit = c.ks_ri_crit;
    k.shearmix_rate = c.ks_shearmix_rate;
    k.fri_curvature = c.ks_fri_curvature;
    k.kappa_0 = c.ks_kappa_0;
    k.kappa_seed = c.ks_kappa_seed;
    k.kappa_trunc = c.ks_kappa_trunc;
    k.tke_bg = c.ks_tke_bg;
    k.tol_err = c.ks_tol_err;
    k.src_max_chg = c.ks_src_max_chg;
    k.vel_underflow = c.ks_vel_underflow;
    k.rho0 = c.rho0;
    k.alpha_t = c.eos_alpha_t;
    k.beta_s = c.eos_beta_s;
    k.lz_rescale = c.ks_lz_rescale;
    k.max_inner_it = c.ks_max_inner_it;
    k.max_substep_it = c.ks_max_substep_it;
    k.eos_linear = c.eos_variant == 1;
    // column-invariant scalars, formed on the host in IEEE double exactly as
    // ks_solve_column (:1604-1608) and ks_adaptive_dt (:1446-1451) form them
    k.tke_min = c.ks_tke_bg > 1.0e-20 ? c.ks_tke_bg : 1.0e-20;
    k.c_n2 = c.ks_c_n * c.ks_c_n;
    k.c_s2 = c.ks_c_s * c.ks_c_s;
    k.ilambda2 = 1.0 / (c.ks_lambda * c.ks_lambda);
    k.tol_dksrc_low = (c.ks_src_max_chg == 10.0) ? 0.95 : (c.ks_src_max_chg - 0.5) / c.ks_src_max_chg;
    return k;
}

}  // namespace

void launch_kappa_shear(const Params &p, double dt, int *work, int *order, unsigned *hist, bool ordered,
                        cudaStream_t stream)
{
    const KsPar kp = ks_par_of(p.cfg);
    const size_t n = p.plane;
    const int *ord = nullptr;
    if (ordered && work && order && hist) {
        const int fill = (int)((n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184);
        cudaMemsetAsync(hist, 0, KS_NB * sizeof(unsigned), stream);
        k_ks_hist<<<fill, 256, 0, stream>>>(work, n, hist);
        k_ks_scan<<<1, KS_NB, 0, stream>>>(hist);
        k_ks_scatter<<<fill, 256, 0, stream>>>(work, n, hist, order);
        ord = order;
    }
    const int threads = 64;
    const unsigned blocks = (unsigned)((n + threads - 1) / threads);
#define VPHYS_KS_LAUNCH(M)                                                                 \
    if (p.nz <= 32)                                                                        \
        k_kappa_shear<34, M><<<blocks, threads, 0, stream>>>(p, kp, dt, ord, work);        \
    else if (p.nz <= 80)                                                                   \
        k_kappa_shear<82, M><<<blocks, threads, 0, stream>>>(p, kp, dt, ord, work);        \
    else                                                                                   \
        k_kappa_shear<NZ_MAX + 2, M><<<blocks, threads, 0, stream>>>(p, kp, dt, ord, work);
    if (p.cfg.ks_massless_merge) {
        VPHYS_KS_LAUNCH(true)
    } else {
        VPHYS_KS_LAUNCH(false)
    }
#undef VPHYS_KS_LAUNCH
}

}  // namespace vphys
