// vphys_tracers.cu -- implicit vertical diffusion of every tracer with the KPP
// non-local tendency fused into the store (rdb_ocean_vdiff.F90:1107-1414,
// rdb_ocean_vmix.F90:1605-1714).
//
// One thread per cell column; the block's 128 columns are consecutive in i,
// so every per-level access of a warp is one coalesced 256-B segment.
//
// * Only the column's live span [k_lo, k_hi] (first live layer from the bed,
//   first live layer from the surface) is solved: every row outside it is an
//   identity row of the reference's matrix (both couplings gated to zero by
//   H_VANISHED), whose solution is its input, its budget increment zero and
//   its non-local deposit refused -- the values are unchanged (up to the sign
//   of a zero), so those cells are neither read nor written.  Land columns
//   cost one scan of h.
// * The matrix is factorised once per diffusivity (kt, and ks when it differs)
//   in the same upward pass that forward-sweeps every tracer.  The pivots'
//   c' live in shared memory; the forward-swept right-hand sides are written
//   in place into the tracer arrays with an L2 evict_last hint and read back
//   by the downward pass, so the round trip stays in L2 and HBM sees each
//   tracer value read once and written once.
// * Loads are issued a block of U levels ahead of the arithmetic, so each
//   thread keeps several independent loads in flight under the serial
//   Thomas recurrence.
#include <cuda_runtime.h>

#include "vphys_device.cuh"
#include "vphys_kernels.cuh"

#ifndef VPHYS_TR_THREADS
#define VPHYS_TR_THREADS 128
#endif

namespace vphys {


// Row k (1-based) of the tracer matrix (build_factorize_tracer_matrix,
// rdb_ocean_vdiff.F90:1285-1341); hm/hc/hp are the raw thicknesses of layers
// k-1, k, k+1, K_k / K_kp1 the diffusivity at interfaces k and k+1.
__device__ __forceinline__ void tracer_row(int k, int nz, bool use_harmonic, double dt, double hm_raw, double hc_raw,
                                           double hp_raw, double K_k, double K_kp1, double &a, double &b, double &cc)
{
    if (k == 1) {
        const double hc = fmx(hc_raw, H_VANISHED);
        double alpha = 0.0;
        if (nz > 1) {
            const double hp = fmx(hp_raw, H_VANISHED);
            const double dz_face = face_thick(hc, hp, use_harmonic);
            alpha = xdiv(dt * K_kp1, hc * dz_face);
            if (hc_raw <= H_VANISHED || hp_raw <= H_VANISHED) alpha = 0.0;
        }
        a = 0.0;
        cc = -alpha;
        b = 1.0 + alpha;
    } else if (k < nz) {
        const double hm = fmx(hm_raw, H_VANISHED);
        const double hc = fmx(hc_raw, H_VANISHED);
        const double hp = fmx(hp_raw, H_VANISHED);
        double beta = xdiv(dt * K_k, hc * face_thick(hm, hc, use_harmonic));
        double alpha = xdiv(dt * K_kp1, hc * face_thick(hc, hp, use_harmonic));
        if (hc_raw <= H_VANISHED || hm_raw <= H_VANISHED) beta = 0.0;
        if (hc_raw <= H_VANISHED || hp_raw <= H_VANISHED) alpha = 0.0;
        a = -beta;
        cc = -alpha;
        b = 1.0 + alpha + beta;
    } else {
        const double hm = fmx(hm_raw, H_VANISHED);
        const double hc = fmx(hc_raw, H_VANISHED);
        const double dz_face = face_thick(hm, hc, use_harmonic);
        double beta = xdiv(dt * K_k, hc * dz_face);
        if (hc_raw <= H_VANISHED || hm_raw <= H_VANISHED) beta = 0.0;
        a = -beta;
        cc = 0.0;
        b = 1.0 + beta;
    }
}

// The columns of one warp: column (i, j) on this lane, `tid` its slot in the
// block's shared memory of `bs` columns.  CI: with the diffusion, the
// compensated column content before it (terms bottom-up, in the upward pass)
// and after it (top-down, in the downward pass) into p.content_old / _new.
template <int NTR, bool TWO, bool DEF, bool CI = false>
__device__ __forceinline__ void tracer_columns(const Params &p, double dt, int diffuse, int nonlocal, int i, int j,
                                               double *smem, int tid, int bs)
{
    // levels per load block: 2 up to 8 tracers, else 1 (1440x1080x75, 4
    // tracers: 5.25 ms with 4, 4.18 with 2, 4.37 with 1 -- the larger
    // unrolled body costs more in instruction-cache misses and registers than
    // the deeper prefetch gains)
#ifdef VPHYS_TR_U
    constexpr int TR_U = VPHYS_TR_U;
#else
    constexpr int TR_U = NTR <= 8 ? 2 : 1;
#endif
    // PIPE: the loads of the next level block are issued before the current
    // block is computed (two register buffers).  Up to VPHYS_TR_PIPE_MAX
    // tracers per thread; above it the doubled load code of the unrolled
    // tracer loop costs more than the overlap gains, and each block loads
    // just before its arithmetic.
#ifndef VPHYS_TR_PIPE_MAX
#define VPHYS_TR_PIPE_MAX 4
#endif
    constexpr bool PIPE = NTR <= VPHYS_TR_PIPE_MAX;
    vphys_config cd = p.cfg;   // DEF: the default knobs folded in (is_default_tracer_knobs)
    if (DEF) default_tracer_knobs(cd);
    const vphys_config &c = cd;
    const int nx = p.nx, nz = p.nz, ntr = p.ntr;
    const size_t P = p.plane;
    const bool in_grid = i < nx;
    const size_t col = (size_t)(in_grid ? i : 0) + (size_t)nx * j;
    const double *__restrict__ hp = p.h + col;
    const int iT = c.idx_temperature, iS = c.idx_salinity, iPS = c.idx_pseudo_salt;
    double *cpA = smem + tid;                       // cpA[(k-1)*bs]
    double *cpB = smem + (size_t)nz * bs + tid;     // only when TWO
    const unsigned long long pol_keep = l2_policy_evict_last();
    const unsigned long long pol_once = l2_policy_evict_first();
#define HH(k) __ldg(hp + P * (size_t)((k) - 1))

    // ---- this column's live span; rows outside it are identity rows ----
    int k_lo = 0, k_hi = 0;
    double h_below = 0.0, h_lo = 0.0, h_hi = 0.0;
    if (in_grid) {
        for (int k = 1; k <= nz; ++k) {
            const double hk = HH(k);
            if (hk > H_VANISHED) {
                k_lo = k;
                h_lo = hk;
                break;
            }
            h_below = hk;
        }
        if (k_lo > 0) {
            k_hi = k_lo;
            h_hi = h_lo;
            for (int k = nz; k > k_lo; --k) {
                const double hk = HH(k);
                if (hk > H_VANISHED) {
                    k_hi = k;
                    h_hi = hk;
                    break;
                }
            }
        }
    }
    const bool live = k_lo > 0;
    // the warp sweeps the union of its lanes' spans with a uniform k, so its
    // loads stay coalesced and the row-type branches stay uniform; a lane
    // outside its own span is predicated off (no load, no store)
    const unsigned full = 0xffffffffu;
    const int w_lo = __reduce_min_sync(full, live ? k_lo : 0x7fffffff);
    const int w_hi = __reduce_max_sync(full, live ? k_hi : 0);
    if (w_hi == 0) {   // no live layer anywhere in this warp
        if (CI && diffuse && in_grid)
            for (int t = 0; t < ntr; ++t) p.content_old[col + P * (size_t)t] = p.content_new[col + P * (size_t)t] = 0.0;
        return;
    }
    double c_old[NTR], e_old[NTR], c_new[NTR], e_new[NTR];   // CI: Neumaier sums and their compensations
#pragma unroll
    for (int t = 0; t < NTR; ++t) c_old[t] = e_old[t] = c_new[t] = e_new[t] = 0.0;

    double *trc[NTR];
#pragma unroll
    for (int t = 0; t < NTR; ++t) trc[t] = (t < ntr) ? p.tr[t] + col : nullptr;
    // With heat/salt budgets the reference needs h*c_new - h*c_old, so the
    // forward-swept values of T and S go to a scratch plane instead of over
    // the input (rbuf); every other tracer is swept in place.
    double *heat = (c.budgets && diffuse && iT >= 0) ? p.heat_budget + col : nullptr;
    double *salt = (c.budgets && diffuse && iS >= 0) ? p.salt_budget + col : nullptr;
    double *rbuf[NTR];
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
        rbuf[t] = trc[t];
        if (t < ntr && heat && t == iT) rbuf[t] = p.budget_scratch + col;
        if (t < ntr && salt && t == iS) rbuf[t] = p.budget_scratch + P * (size_t)nz + col;
    }

    if (diffuse) {
        // ---- upward pass: rows, factorisation, forward sweep of every tracer ----
        const double *__restrict__ KA = p.kt + col;
        const double *__restrict__ KB = p.ks + col;
        double h_m = h_below, h_c = h_lo;
        double KA_k = 0.0, KB_k = 0.0;   // interface k_lo: gated off when k_lo > 1
        double cpA_prev = 0.0, cpB_prev = 0.0;
        double r_prev[NTR];
#pragma unroll
        for (int t = 0; t < NTR; ++t) r_prev[t] = 0.0;
        // the loads of block k0 + TR_U are issued before block k0 is computed
        // (two register buffers; the block's stores go to its own levels)
        auto load_up = [&](int k0, double (&xs_)[TR_U][NTR], double (&hps_)[TR_U], double (&kap_)[TR_U],
                           double (&kbp_)[TR_U]) {
#pragma unroll
            for (int u = 0; u < TR_U; ++u) {
                const int k = k0 + u;
                const bool act = live && k >= k_lo && k <= k_hi;
                const size_t off = P * (size_t)(k - 1);
                hps_[u] = (act && k < nz) ? __ldg(hp + off + P) : 0.0;
                kap_[u] = (act && k < nz) ? ld_hint(KA + off + P, pol_once) : 0.0;
                kbp_[u] = (TWO && act && k < nz) ? ld_hint(KB + off + P, pol_once) : 0.0;
#pragma unroll
                for (int t = 0; t < NTR; ++t) xs_[u][t] = (act && t < ntr) ? trc[t][off] : 0.0;
            }
        };
        double xs[TR_U][NTR], hps[TR_U], kap[TR_U], kbp[TR_U];
        if constexpr (PIPE) load_up(w_lo, xs, hps, kap, kbp);
        for (int k0 = w_lo; k0 <= w_hi; k0 += TR_U) {
            double xs_n[TR_U][NTR], hps_n[TR_U], kap_n[TR_U], kbp_n[TR_U];
            if constexpr (PIPE)
                load_up(k0 + TR_U, xs_n, hps_n, kap_n, kbp_n);
            else
                load_up(k0, xs, hps, kap, kbp);
#pragma unroll
            for (int u = 0; u < TR_U; ++u) {
                const int k = k0 + u;
                if (k > w_hi) break;
                const bool act = live && k >= k_lo && k <= k_hi;
                if (act) {
                    const size_t off = P * (size_t)(k - 1);
                    const double h_p = hps[u];
                    double aA, bA, cA;
                    tracer_row(k, nz, c.use_harmonic, dt, h_m, h_c, h_p, KA_k, kap[u], aA, bA, cA);
                    const Rcp denA = rcp_of((k == 1) ? bA : bA - aA * cpA_prev);
                    cpA_prev = qdiv(cA, denA);
                    cpA[(size_t)(k - 1) * bs] = cpA_prev;
                    double aB = 0.0;
                    Rcp denB = denA;
                    if (TWO) {
                        double bB, cB;
                        tracer_row(k, nz, c.use_harmonic, dt, h_m, h_c, h_p, KB_k, kbp[u], aB, bB, cB);
                        denB = rcp_of((k == 1) ? bB : bB - aB * cpB_prev);
                        cpB_prev = qdiv(cB, denB);
                        cpB[(size_t)(k - 1) * bs] = cpB_prev;
                        KB_k = kbp[u];
                    }
#pragma unroll
                    for (int t = 0; t < NTR; ++t) {
                        if (t < ntr) {
                            const bool useA = !TWO || (t == iT);
                            const double a = useA ? aA : aB;
                            const double num = (k == 1) ? xs[u][t] : xs[u][t] - a * r_prev[t];
                            const double r = qdiv(num, useA ? denA : denB);
                            r_prev[t] = r;
                            st_hint(rbuf[t] + off, r, pol_keep);
                        }
                    }
                    if (CI) {
#pragma unroll
                        for (int t = 0; t < NTR; ++t)
                            if (t < ntr) neumaier_add(c_old[t], e_old[t], h_c * xs[u][t]);
                    }
                    KA_k = kap[u];
                    h_m = h_c;
                    h_c = h_p;
                }
            }
            if constexpr (PIPE) {
#pragma unroll
                for (int u = 0; u < TR_U; ++u) {
                    hps[u] = hps_n[u];
                    kap[u] = kap_n[u];
                    kbp[u] = kbp_n[u];
#pragma unroll
                    for (int t = 0; t < NTR; ++t) xs[u][t] = xs_n[u][t];
                }
            }
        }
    }

    // ---- non-local column scalars, recomputed exactly as KPP pass 2 ----
    const bool do_nl = nonlocal && c.use_kpp;
    bool nl = do_nl && live;
    double h_b = 0.0, q_T_kin = 0.0, q_S_kin = 0.0;
    if (nl) {
        const double rho0 = c.rho0;
        h_b = p.bl_depth[col];
        const double u_star = sqrt(xdiv(p.stress_mag[col], rho0));
        // the heat flux pass 2 charged (shortwave: what passes h_b, or the
        // surface layer k_hi)
        q_T_kin = kpp_q_t_kin(c, p.q_heat[col], p.sw_src + col, p.sw_kappa, col, p.plane, h_b, h_hi);
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
        nl = (h_b > 0.0 && w_s > 0.0 && B_0 < 0.0);
    }

    // ---- downward pass: back-substitution, budgets, non-local deposit and
    //      the store (the reference's k_sfc is this column's k_hi) ----
    double x_above[NTR];
#pragma unroll
    for (int t = 0; t < NTR; ++t) x_above[t] = 0.0;
    double gT_above = 0.0, gS_above = 0.0;
    double d_run = 0.0;
    double h_c = h_hi, h_a = 0.0;   // layer above k_hi is vanished: its flux is closed
    // sigma = d_run / h_b with one reciprocal per column (qdiv: the quotient bit for bit)
    const Rcp r_hb = rcp_of(nl ? h_b : 1.0);
    // the loads of block k0 - TR_U are issued before block k0 is computed
    auto load_down = [&](int k0, double (&rs_)[TR_U][NTR], double (&hbs_)[TR_U]) {
#pragma unroll
        for (int u = 0; u < TR_U; ++u) {
            const int k = k0 - u;
            const bool act = live && k >= k_lo && k <= k_hi;
            const size_t off = P * (size_t)(k - 1);
            hbs_[u] = (act && k > 1) ? __ldg(hp + off - P) : 0.0;
#pragma unroll
            for (int t = 0; t < NTR; ++t)
                rs_[u][t] = (act && t < ntr && (diffuse || t == iT || t == iS || t == iPS))
                                ? ld_hint((diffuse ? rbuf[t] : trc[t]) + off, pol_keep)
                                : 0.0;
        }
    };
    double rs[TR_U][NTR], hbs[TR_U];
    if constexpr (PIPE) load_down(w_hi, rs, hbs);
    for (int k0 = w_hi; k0 >= w_lo; k0 -= TR_U) {
        double rs_n[TR_U][NTR], hbs_n[TR_U];
        if constexpr (PIPE)
            load_down(k0 - TR_U, rs_n, hbs_n);
        else
            load_down(k0, rs, hbs);
#pragma unroll
        for (int u = 0; u < TR_U; ++u) {
            const int k = k0 - u;
            if (k < w_lo) break;
            const bool act = live && k >= k_lo && k <= k_hi;
            if (act) {
                const size_t off = P * (size_t)(k - 1);
                const double h_bl = hbs[u];
                double gT = 0.0, gS = 0.0;
                if (nl) {
                    d_run = d_run + h_c;
                    if (k > 1 && d_run < h_b) {
                        const double sigma = qdiv(d_run, r_hb);
                        const double g_shape = sigma * (1.0 - sigma) * (1.0 - sigma);
                        const double gamma_factor = c.cs_nonlocal * g_shape;
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
                        fT_dn = nonlocal_face_flux(gT, h_bl, h_c);
                        fS_dn = nonlocal_face_flux(gS, h_bl, h_c);
                    }
                    fT = dt * (fT_up - fT_dn);
                    fS = dt * (fS_up - fS_dn);
                }
                // conc_add_source's quotients src / (h + H_DIV_EPS), one reciprocal for
                // the layer (salinity and pseudo-salt share fS); a zero source adds
                // itself, as xdiv(+-0, b > 0) = +-0
                double incT = fT, incS = fS;
                if (do_nl && (fT != 0.0 || fS != 0.0)) {
                    const Rcp r_h = rcp_of(h_c + H_DIV_EPS);
                    if (fT != 0.0) incT = qdiv(fT, r_h);
                    if (fS != 0.0) incS = qdiv(fS, r_h);
                }
#pragma unroll
                for (int t = 0; t < NTR; ++t) {
                    if (t < ntr && (diffuse || t == iT || t == iS || t == iPS)) {
                        double x = rs[u][t];
                        if (diffuse) {
                            const bool useA = !TWO || (t == iT);
                            const double cpk = useA ? cpA[(size_t)(k - 1) * bs] : cpB[(size_t)(k - 1) * bs];
                            x = x - cpk * x_above[t];   // x_above = 0 at k_hi: the top row
                            x_above[t] = x;
                            if ((t == iT && heat) || (t == iS && salt)) {
                                double *bud = (t == iT) ? heat : salt;
                                const double x_old = trc[t][off];
                                const double p_new = h_c * x, p_old = h_c * x_old;
                                bud[off] = bud[off] + (p_new - p_old);
                            }
                        }
                        if (do_nl && h_c > H_VANISHED) {
                            if (t == iT) x = x + incT;
                            else if (t == iS || t == iPS) x = x + incS;
                        }
                        if (CI && diffuse) neumaier_add(c_new[t], e_new[t], h_c * x);
                        trc[t][off] = x;
                    }
                }
                gT_above = gT;
                gS_above = gS;
                h_a = h_c;
                h_c = h_bl;
            }
        }
        if constexpr (PIPE) {
#pragma unroll
            for (int u = 0; u < TR_U; ++u) {
                hbs[u] = hbs_n[u];
#pragma unroll
                for (int t = 0; t < NTR; ++t) rs[u][t] = rs_n[u][t];
            }
        }
    }
    if (CI && diffuse && in_grid) {
#pragma unroll
        for (int t = 0; t < NTR; ++t)
            if (t < ntr) {
                p.content_old[col + P * (size_t)t] = c_old[t] + e_old[t];
                p.content_new[col + P * (size_t)t] = c_new[t] + e_new[t];
            }
    }
#undef HH
}

template <int NTR, bool TWO, bool DEF, bool CI>
__global__ void __launch_bounds__(128) k_tracers(const Params p, double dt, int diffuse, int nonlocal)
{
    extern __shared__ double smem[];
    tracer_columns<NTR, TWO, DEF, CI>(p, dt, diffuse, nonlocal, blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y,
                                      smem, threadIdx.x, blockDim.x);
}

// The FP64 re-solve of the (32-column group, tracer) pairs that the
// mixed-precision kernel listed (mp_redo[0] entries after the count, each
// group << 5 | tracer) and left untouched: each runs the exact path above as
// a one-tracer problem -- the tracer's roles (T, S, pseudo-salt) and its
// diffusivity carried over -- so those columns come out bitwise as on the
// FP64 path.  One warp per entry, the grid strides over the list.
__global__ void __launch_bounds__(32) k_tracers_redo(const Params p, double dt, int nonlocal, int ngx)
{
    extern __shared__ double smem[];
    const unsigned n = *(volatile const unsigned *)p.mp_redo;
    for (unsigned e = blockIdx.x; e < n; e += gridDim.x) {
        const unsigned ent = p.mp_redo[1 + e];
        const int tix = (int)(ent & 31u);
        const unsigned g = ent >> 5;
        const int gi = (int)(g % (unsigned)ngx), j = (int)(g / (unsigned)ngx);
        const int li = gi * 32 + (int)threadIdx.x;
        Params q = p;
        const vphys_config &c = p.cfg;
        q.ntr = 1;
        q.tr[0] = p.tr[tix];
        q.cfg.idx_temperature = (tix == c.idx_temperature) ? 0 : -1;
        q.cfg.idx_salinity = (tix == c.idx_salinity) ? 0 : -1;
        q.cfg.idx_pseudo_salt = (tix == c.idx_pseudo_salt) ? 0 : -1;
        if (!p.ks_equals_kt && tix != c.idx_temperature) q.kt = p.ks;   // the second factorisation's tracers
        if (p.content_old) {
            q.content_old = p.content_old + p.plane * (size_t)tix;   // the tracer's plane of the content fields
            q.content_new = p.content_new + p.plane * (size_t)tix;
            tracer_columns<1, false, false, true>(q, dt, 1, nonlocal, li, j, smem, threadIdx.x, 32);
        } else {
            tracer_columns<1, false, false>(q, dt, 1, nonlocal, li, j, smem, threadIdx.x, 32);
        }
        __syncwarp();
    }
}

static void redo_attr()
{
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_tracers_redo, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)((size_t)VPHYS_NZ_MAX * 32 * sizeof(double)));
        attr_set = true;
    }
}

void launch_tracers_redo(const Params &p, double dt, bool nonlocal, cudaStream_t stream)
{
    redo_attr();
    const int ngx = (p.nx + 31) / 32;
    const size_t smem = (size_t)p.nz * 32 * sizeof(double);
    k_tracers_redo<<<148 * 8, 32, smem, stream>>>(p, dt, nonlocal ? 1 : 0, ngx);
}


template <int NTR, bool TWO>
static void launch_tracers_n(const Params &p, double dt, bool diffuse, bool nonlocal, cudaStream_t stream)
{
    // two factorisations keep two c' arrays: halve the block to stay within
    // the 227 KB of shared memory per block at nz = VPHYS_NZ_MAX
    const int bs = TWO ? VPHYS_TR_THREADS / 2 : VPHYS_TR_THREADS;
    const size_t smem = (size_t)p.nz * bs * sizeof(double) * (TWO ? 2 : 1);
    static bool attr_set = false;
    if (!attr_set) {
        const int mx = (int)((size_t)VPHYS_NZ_MAX * bs * sizeof(double) * (TWO ? 2 : 1));
        cudaFuncSetAttribute(k_tracers<NTR, TWO, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        cudaFuncSetAttribute(k_tracers<NTR, TWO, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        cudaFuncSetAttribute(k_tracers<NTR, TWO, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
        attr_set = true;
    }
    dim3 grid((p.nx + bs - 1) / bs, p.ny);
    if (is_default_tracer_knobs(p.cfg))
        k_tracers<NTR, TWO, true, false><<<grid, bs, smem, stream>>>(p, dt, diffuse ? 1 : 0, nonlocal ? 1 : 0);
    else if (p.content_old && diffuse)
        k_tracers<NTR, TWO, false, true><<<grid, bs, smem, stream>>>(p, dt, 1, nonlocal ? 1 : 0);
    else
        k_tracers<NTR, TWO, false, false><<<grid, bs, smem, stream>>>(p, dt, diffuse ? 1 : 0, nonlocal ? 1 : 0);
}

void launch_tracers(const Params &p, double dt, bool diffuse, bool nonlocal, cudaStream_t stream)
{
    if (diffuse && p.cfg.mixed_precision) {
        launch_tracers_mp(p, dt, nonlocal, stream);
        return;
    }
    const bool two = !p.ks_equals_kt;
    if (p.ntr <= 2) {
        two ? launch_tracers_n<2, true>(p, dt, diffuse, nonlocal, stream) : launch_tracers_n<2, false>(p, dt, diffuse, nonlocal, stream);
    } else if (p.ntr <= 4) {
        two ? launch_tracers_n<4, true>(p, dt, diffuse, nonlocal, stream) : launch_tracers_n<4, false>(p, dt, diffuse, nonlocal, stream);
    } else if (p.ntr <= 8) {
        two ? launch_tracers_n<8, true>(p, dt, diffuse, nonlocal, stream) : launch_tracers_n<8, false>(p, dt, diffuse, nonlocal, stream);
    } else {
        two ? launch_tracers_n<16, true>(p, dt, diffuse, nonlocal, stream) : launch_tracers_n<16, false>(p, dt, diffuse, nonlocal, stream);
    }
}

}  // namespace vphys
