/* vphys_oracle.h -- CPU FP64 restatement of Roundabout's vertical-physics
 * hot path.  TEST INFRASTRUCTURE ONLY: the checker for the CUDA library
 * (tests/, __graft_entry__.smoke(), and bench.py's cpu_baseline / reference
 * arm).  Nothing in the product links or calls it.
 *
 * Parity pins: the safe-math port (cbrt, atan) is checked bit for bit
 * against the reference's own golden vectors (tests/test_safe_math_golden.inc,
 * transcribed by tests/golden/make_safe_math_golden.py); the physics is
 * checked against the reference's analytic known-answer tests
 * (tests/test_ocean_pp81.F90, test_ocean_kpp.F90, test_ocean_kpp_nonlocal.F90,
 * test_ocean_kpp_convective.F90, test_ocean_buoyancy_flux.F90,
 * test_ocean_vdiff.F90, test_ocean_vdiff_implicit_stress_drag.F90,
 * test_ocean_vdiff_bbl.F90, test_ocean_visc_rem.F90,
 * test_ocean_vmix_assembly.F90, test_ocean_bkgnd_mixing.F90,
 * test_ocean_vmix_no_pp81.F90, test_ocean_convection.F90,
 * test_ocean_kv_ml_invz2.F90, test_ocean_wright_eos.F90,
 * test_ocean_sw_chl.F90, test_ocean_epbl_max_shear.F90) re-expressed in
 * tests/test_oracle_*.py;
 * kappa-shear (vphys_oracle_kshear.c) against the reference's golden kd
 * profile (tests/test_ocean_kappa_shear.F90:286-393, 1e-6 relative); EPBL
 * (vphys_oracle_epbl.c) against the physical tests of test_ocean_epbl.F90.
 * The Fortran reference itself cannot be compiled here (no Fortran
 * compiler), so bitwise parity with its binary output is unpinned.
 *
 * Loop order and operation order follow the Fortran source line by line;
 * build with -ffp-contract=off (the reference's CPU builds' setting), no
 * -ffast-math.
 */
#ifndef VPHYS_ORACLE_H
#define VPHYS_ORACLE_H

#include "../include/vphys.h"

#ifdef __cplusplus
extern "C" {
#endif

/* All arrays of one column-physics state, Fortran layout (see vphys.h). */
typedef struct vpo_state {
    int nx, ny, nz, ntr;
    double *h, *rho, *u, *v;
    double *kv, *kt, *ks, *kd_bg;          /* kd_bg: (nx,ny,nz+1) scratch */
    double *bl_depth, *b0, *stress_mag, *q_heat, *q_salt, *wet;
    double *tau_x, *tau_y, *lambda_bot_u, *lambda_bot_v;
    double *visc_rem_u, *visc_rem_v;
    double *gamma_t, *gamma_s;
    double *heat_budget, *salt_budget;
    int *k_top_u, *k_top_v, *k_bot_u, *k_bot_v;   /* 1-based */
    double **tr;                            /* ntr pointers */
    double *heat_budget_surface, *salt_budget_surface;
    double *coriolis;                       /* (nx,ny) f; NULL reads as 0 */
    double *kd_shear, *tke_shear;           /* (nx,ny,nz+1) kappa-shear kd_int, tke_int */
    double *kd_epbl;                        /* (nx,ny,nz+1) EPBL kd_int */
    double *mld_epbl;                       /* (nx,ny) EPBL mixed-layer depth */
    double *la_epbl;                        /* (nx,ny) EPBL Langmuir number */
    double *epbl_tke[6];                    /* (nx,ny) EPBL TKE budget terms, written when epbl_tke_diags */
    double *sw_net;                         /* (nx,ny) the shortwave source under sw_source = 1 */
    double *wet_dyn;                        /* (nx,ny) dynamic wet mask, read under use_wet_dyn */
    double *sw_chl;                         /* (nx,ny) surface chlorophyll, mg m-3 */
    double *sw_kappa;                       /* (nx,ny,VPHYS_SW_NB_MAX) chlorophyll-scheme band opacities */
    double *cover_frac;                     /* (nx,ny) ice-shelf cover fraction, read under use_cover_frac */
} vpo_state;

void vpo_sw_chl_kappa(const vphys_config *c, vpo_state *s);
double vpo_sw_band_frac(int n, int nb, double blue);
double vpo_sw_transmission_nb(const vphys_config *c, const vpo_state *s, int i, int j, double d);

/* The shortwave source the configuration selects (ocean_surfflux_set_sw's
 * sw_from_qsw, rdb_ocean_surface_flux.F90:715-740): Q_heat, or the net
 * shortwave under sw_source = 1. */
static inline const double *vpo_sw_source(const vphys_config *c, const vpo_state *s)
{
    return c->sw_source ? s->sw_net : s->q_heat;
}

void vpo_set_threads(int n);
int vpo_get_threads(void);

double vpo_sm_cbrt(double x);
double vpo_sm_atan(double x);

void vpo_eos_wright(const vphys_config *c, vpo_state *s);
void vpo_stress_mag(vpo_state *s);

void vpo_pp81(const vphys_config *c, vpo_state *s);
void vpo_seed_interior_none(const vphys_config *c, vpo_state *s);
void vpo_kpp_overlay(const vphys_config *c, vpo_state *s);
void vpo_kv_ml_invz2(const vphys_config *c, vpo_state *s);
void vpo_convection(const vphys_config *c, vpo_state *s);
void vpo_split(const vphys_config *c, vpo_state *s);
int vpo_assemble_gate(const vphys_config *c, vpo_state *s);
int vpo_build_coefficients(const vphys_config *c, vpo_state *s);

void vpo_vdiff_momentum(const vphys_config *c, vpo_state *s, double dt);
void vpo_vdiff_tracers(const vphys_config *c, vpo_state *s, double dt);
void vpo_nonlocal(const vphys_config *c, vpo_state *s, double dt);
void vpo_surface_flux(const vphys_config *c, vpo_state *s, double dt);
void vpo_eos_buoyancy_coeffs(double T, double S, double p, double *alpha_T, double *beta_S);
double vpo_sm_exp(double x);
double vpo_sm_log(double x);
double vpo_sm_pow(double x, double y);
double vpo_sm_erfc(double x);
void vpo_sw_penetration(const vphys_config *c, vpo_state *s, double dt);

/* kappa-shear, column form (vphys_oracle_kshear.c) */
void vpo_kappa_shear(const vphys_config *c, vpo_state *s, double dt);
void vpo_kappa_shear_merge(const vphys_config *c, vpo_state *s);
/* the massless merge of kappa-shear, 1-based surface-down arrays */
void vpo_massless_build_maps(const double *h, int nz, double h_min, int *nzc, double *hc, int *kc, double *kf);
void vpo_massless_merge_fields(const double *h, const int *kc, int nz, int nzc, const double *u, const double *v,
                               const double *t, const double *s, double *uc, double *vc, double *tc, double *sc);
void vpo_massless_interp_back(const double *qc, const int *kc, const double *kf, int nz, double *q);

/* EPBL, column form (vphys_oracle_epbl.c) */
void vpo_epbl(const vphys_config *c, vpo_state *s, double dt);
void vpo_epbl_merge(const vphys_config *c, vpo_state *s);
/* the LF17 wave state and Langmuir number, and the mstar enhancement, alone */
void vpo_epbl_lf17(double ustar, double rho0, double zsl, double *u10, double *la);
double vpo_epbl_lt_enhance(const vphys_config *c, double la, double b0, double ustar, double bld, double absf,
                           double mstar);

int vpo_step(const vphys_config *c, vpo_state *s, double dt, int n_steps);

/* Compensated (Neumaier) FP64 content sum_k h_k c_k of every column and
 * tracer over the column's live span (first live layer from the bed to the
 * first from the surface; 0 without one), the terms added bottom-up
 * (descending = 0) or top-down (descending = 1); out[t * nx * ny + col]. */
void vpo_column_content(const vpo_state *s, int descending, double *out);

#ifdef __cplusplus
}
#endif
#endif
