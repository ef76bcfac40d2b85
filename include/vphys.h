/* vphys.h -- C ABI of the B200-native vertical-physics library (libvphys.so).
 *
 * The library replaces, behind plain C entry points, the vertical-physics
 * hot path of Roundabout (JorgeG94/roundabout):
 *
 *   vmix_compute_pp81 -> vmix_apply_kpp_overlay -> vmix_split_kd_heat_salt
 *   -> vmix_assemble -> vdiff_apply_momentum -> vdiff_apply_tracers
 *   -> vmix_apply_nonlocal_tendencies            (+ the Wright EOS precursor)
 *
 * i.e. the body of `vmix_build_coefficients` + `vmix_apply_in_stage`
 * (src/core/ocean/dynamics/split_rk2/rdb_ocean_dyn.F90:1473-1634, 1636-1900).
 * Every entry point cites the reference routine it replaces.
 *
 * Conventions (identical to the reference, include/rdb_ocean.h:1-60):
 *   - every array is FP64, Fortran order (i fastest, then j, then k);
 *   - layers are bottom-up: k = 1 (index 0 here) is the BED, k = nz the surface;
 *   - cell arrays are (nx, ny, nz); interface arrays (kv, kt, ks) are
 *     (nx, ny, nz+1) with interface k at the bottom of layer k;
 *   - u-face arrays are (nx+1, ny, nz), v-face arrays (nx, ny+1, nz);
 *   - 2-D column arrays are (nx, ny); 2-D u/v face arrays (nx+1, ny) / (nx, ny+1);
 *   - tracers are stored as CONCENTRATION; a layer with h <= 1.5e-4 m
 *     (H_VANISHED) is an inert filler that keeps its value.
 *
 * Memory: the handle owns one device buffer per field (allocated at create,
 * in HBM); vphys_bind() replaces any of them by a caller-owned device pointer
 * (zero copy: a Fortran caller passes `c_loc` of an OpenACC/CUDA device
 * array, a Python caller a torch tensor's data_ptr()).  vphys_set_field() /
 * vphys_get_field() copy between host memory and the current device buffer.
 *
 * Errors: every entry point returns an int status (VPHYS_OK = 0); the
 * specific reason is pushed onto an error ring read by vphys_last_error()
 * (same snprintf-style contract as rdb_ocean_last_error,
 * include/rdb_ocean.h:314).  Nothing traps or aborts.
 *
 * Threading: a handle is bound to one CUDA stream (vphys_set_stream); it is
 * not thread-safe per handle.  Entry points enqueue work on that stream and
 * return without synchronising, except where stated.
 */
#ifndef VPHYS_H
#define VPHYS_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (values of the reference where one exists:
 *      include/rdb_ocean.h:79-89) ------------------------------------ */
#define VPHYS_OK 0
#define VPHYS_ERR_CONFIG 2          /* RDB_OCEAN_ERR_CONFIG_VALIDATE */
#define VPHYS_ERR_BAD_HANDLE 10     /* RDB_OCEAN_ERR_BAD_HANDLE */
#define VPHYS_ERR_NOT_INITIALISED 12
#define VPHYS_ERR_NOT_FOUND 13      /* unknown field id */
#define VPHYS_ERR_BAD_SHAPE 14      /* RDB_OCEAN_ERR_BAD_SHAPE */
#define VPHYS_ERR_CUDA 30           /* a CUDA runtime call failed */
#define VPHYS_ERR_GUARD 31          /* vmix_guard tripped: negative/NaN K
                                       (vmix_assemble status=1,
                                       rdb_ocean_vmix.F90:2264-2277) */
#define VPHYS_ERR_TOO_DEEP 32       /* nz > VPHYS_NZ_MAX */
#define VPHYS_ERR_ALLOC 33          /* device allocation failed */
#define VPHYS_ERR_TOO_LARGE 34      /* request beyond a fixed capacity */

/* Largest nz the column kernels accept; the reference's own per-column
 * stack bound NZ_STACK_MAX (src/core/rdb_constants.F90:107-124) is 128 and
 * must cover nz + 1. */
#define VPHYS_NZ_MAX 127

/* interior_closure tags (rdb_ocean_vmix.F90:146-158) */
#define VPHYS_INTERIOR_PP81 1
#define VPHYS_INTERIOR_NONE 4

/* most bands of the chlorophyll shortwave scheme (MAX_SW_BANDS) */
#define VPHYS_SW_NB_MAX 6

/* ---- configuration ---------------------------------------------------
 * Every knob the path reads, with the reference default
 * (ocean_vmix_t rdb_ocean_vmix.F90:198-483; ocean_vdiff_t
 * rdb_ocean_vdiff.F90:78-260; namelist defaults src/core/rdb_config.F90:
 * 1872-1893, 1936-1945).  vphys_config_default() fills them. */
typedef struct vphys_config {
    /* closure selection */
    int use_closure;          /* 1: PP81/none + contributors + assembly */
    int interior_closure;     /* VPHYS_INTERIOR_PP81 (default) | _NONE */
    int use_kpp;              /* KPP overlay (default 0 in ocean_vmix_t) */
    int bkgnd_profile;        /* Bryan-Lewis background (default 0) */
    int vmix_guard;           /* negative/NaN guard before the clip (0) */
    int kd_smooth_iterations; /* 1-2-1 smoothing passes (0) */
    int conv_enable;          /* convective adjustment contributor (0) */
    int surface_flux;         /* 1: vphys_step deposits q_heat / q_salt into the top live layer of
                                 T, S and pseudo-salt after the EOS (ocean_surface_flux_apply_tracers) */
    /* PP81 (rdb_ocean_vmix.F90:233-265) */
    double pp81_nu0;          /* 1e-2 */
    double pp81_nu_bg;        /* 1e-4 */
    double pp81_kappa_bg;     /* 1e-5 */
    double pp81_alpha;        /* 5 */
    double rho0;              /* 1035 */
    double shear2_floor;      /* 1e-10 */
    /* KPP (rdb_ocean_vmix.F90:306-339) */
    double ri_crit;           /* 0.3 */
    double cs_nonlocal;       /* 6.3 */
    double c_vt2;             /* 1.8 */
    double alpha_T;           /* dimensional, kg m-3 K-1 (1.7e-4 default) */
    double beta_S;            /* dimensional, kg m-3 psu-1 (7.6e-4 default) */
    double cp;                /* 3992 (SEAWATER_CP_DEFAULT) */
    /* KV_ML_INVZ2 surface band (rdb_ocean_vmix.F90:309-322) */
    double kv_ml_invz2;       /* 0 = off */
    double hmix_fixed;        /* 20 */
    /* convection (rdb_ocean_vmix.F90:532-555) */
    double conv_kd;           /* 1 */
    double conv_prandtl;      /* 1 */
    double conv_n2_thresh;    /* 0 */
    /* assembly gate (rdb_ocean_vmix.F90:341-371) */
    double kv_bg;             /* = pp81_nu_bg */
    double kt_bg;             /* = pp81_kappa_bg */
    double ks_bg;             /* = pp81_kappa_bg */
    double kv_max;            /* huge */
    double kd_max;            /* huge */
    /* Bryan-Lewis (rdb_ocean_vmix.F90:383-410) */
    double bkgnd_kd_sfc;      /* 1e-5 */
    double bkgnd_kd_deep;     /* 1.3e-4 */
    double bkgnd_z0;          /* 2500 */
    double bkgnd_delta;       /* 222 */
    double bkgnd_prandtl;     /* -1 (off) */
    /* Wright EOS reference pressure (rdb_eos.F90:909-959) */
    double eos_p_ref;         /* 0 Pa */
    /* momentum vdiff (ocean_vdiff_t) */
    int hvel_mom6;            /* 1 (namelist default) */
    int hvel_harmonic;        /* 0 */
    int hvel_upwind;          /* 1 */
    int use_harmonic;         /* 0 */
    int implicit_stress;      /* 0: wind stress folded into the top row */
    int implicit_drag;        /* 0: bottom drag folded into the bed row */
    int zlevel_faces;         /* 0 */
    int bbl_glue;             /* 0 (latched off without a bottom drag) */
    double hbbl_visc;         /* 10 */
    double bbl_piston;        /* 3e-4 */
    double kv_bbl_bg;         /* 1e-4 */
    /* tracer registry roles (0-based tracer index, -1 = absent);
     * rdb_multilayer_state.F90:550-551 puts S first, T second */
    int idx_temperature;      /* 1 */
    int idx_salinity;         /* 0 */
    int idx_pseudo_salt;      /* -1 */
    /* step options */
    int eos_in_step;          /* 1: vphys_step runs the Wright EOS first */
    int remnant;              /* 1: momentum also writes visc_rem_u/v */
    int budgets;              /* 1: tracers accumulate heat/salt budgets */
    int mixed_precision;      /* 0: FP64 throughout (bitwise the reference's arithmetic);
                                 1: FP64 assembly, FP32 Thomas sweeps + FP64 residual correction;
                                 2: as 1 with the assembly's interface sweep in FP32 too */
    int learned_kpp;          /* 1: the KPP boundary-layer depth comes from the attached MLP surrogate
                                 (vphys_kpp_attach), with the range gate and the sampled plain-KPP
                                 check; 0: the reference's bulk-Richardson search */
    int buoyancy_coeffs;      /* KPP surface buoyancy flux coefficients (&ocean_vmix_nml buoyancy_coeffs):
                                 0 "constant": alpha_T / beta_S above; 1 "eos": -d(rho)/dT and d(rho)/dS of
                                 the Wright EOS at the first live layer's (T, S) and eos_p_ref
                                 (eos_buoyancy_coeffs, rdb_eos.F90:1624-1736; the constants on a vanished
                                 surface layer) */
    int kpp_sw_method;        /* which shortwave KPP's B0 charges (kpp_sw_method, rdb_ocean_vmix.F90:132-136,
                                 335): VPHYS_KPP_SW_ALL 1 (all of Q_heat), _MXL 2 (default: Q_heat minus the
                                 penetrating part that passes the boundary layer), _LV1 (minus what passes
                                 the surface layer); read only when sw_pen_frac != 0 */
    /* two-band shortwave penetration (ocean_surface_flux_t, rdb_ocean_surface_flux.F90:229-258):
     * the penetrating irradiance I0 = sw_pen_frac * Q_heat, transmission
     * T(d) = R exp(-d/zeta1) + (1-R) exp(-d/zeta2).  sw_pen_frac = 0 (default)
     * turns both the KPP correction and the deposit off. */
    double sw_pen_frac;       /* 0 */
    double sw_band_ratio;     /* R, 0.58 */
    double sw_zeta1;          /* m, 0.35 */
    double sw_zeta2;          /* m, 23 */
    /* kappa-shear interior closure, column form (ocean_kappa_shear_t,
     * rdb_ocean_kappa_shear.F90:86-224; Jackson, Hallberg & Legg 2008).
     * kappa_shear = 1: vphys_step refreshes kd_shear once a step
     * (vphys_kappa_shear, kappa_shear_compute) and every assembly adds
     * kd_shear to kt and ks_prandtl_turb * kd_shear to kv after KPP, before
     * the split and the floors (kappa_shear_merge_into_kv_kt,
     * rdb_ocean_dyn.F90:1564-1583).  The vertex form (at_vertex) and the
     * massless merge are not built. */
    int kappa_shear;          /* 0 */
    int ks_max_inner_it;      /* Picard iterations, 50 (MAX_RINO_IT) */
    int ks_max_substep_it;    /* adaptive substeps, 13 (MAX_KAPPA_SHEAR_IT) */
    int eos_variant;          /* the shared EOS whose specific-volume derivatives kappa-shear and EPBL
                                 read (eos_specvol_derivs, rdb_eos.F90:1551-1622): 0 Wright 1997, 1 linear
                                 (eos_alpha_t, eos_beta_s, rho0).  The density precursor stays Wright. */
    double ks_ri_crit;        /* 0.25 */
    double ks_shearmix_rate;  /* 0.089 */
    double ks_fri_curvature;  /* -0.97 */
    double ks_c_n;            /* 0.24 */
    double ks_c_s;            /* 0.14 */
    double ks_lambda;         /* 0.82 */
    double ks_lz_rescale;     /* 1 */
    double ks_kappa_0;        /* 1e-7 m2/s */
    double ks_kappa_seed;     /* 1 m2/s */
    double ks_kappa_trunc;    /* 1e-9 m2/s */
    double ks_tke_bg;         /* 0 m2/s2 */
    double ks_tol_err;        /* 0.1 */
    double ks_src_max_chg;    /* 10 */
    double ks_prandtl_turb;   /* 1 */
    double ks_vel_underflow;  /* 0 m/s */
    double eos_alpha_t;       /* linear EOS only: kg m-3 K-1 */
    double eos_beta_s;        /* linear EOS only: kg m-3 psu-1 */
    /* EPBL, the energetic planetary boundary layer, column form (ocean_epbl_t,
     * rdb_ocean_epbl.F90:116-318; Reichl & Hallberg 2018).  epbl = 1 takes the
     * boundary layer from KPP, which it switches off as the reference does
     * (rdb_ocean_dyn.F90:1539): vphys_step refreshes KD_EPBL and MLD_EPBL
     * once a step (vphys_epbl, epbl_compute) and every assembly merges
     * KD_EPBL into kt and epbl_prandtl * KD_EPBL into kv (epbl_combine);
     * convection then masks below MLD_EPBL.  With sw_pen_frac != 0 the
     * two-band shortwave absorbed in each layer is charged to the TKE budget
     * (the reference's epbl_sw_ctke ledger, source Q_HEAT); epbl_use_lt adds
     * the Langmuir enhancement of mstar. */
    int epbl;                 /* 0 */
    int epbl_mstar_scheme;    /* 1 constant, 2 OM4 (default), 3 RH18 */
    int epbl_vstar_scheme;    /* 1 cube root (default), 2 RH18 */
    int epbl_combine;         /* 1 add (default), 2 max, 3 max_shear (needs kappa_shear: shear merged first) */
    int epbl_mld_iteration;   /* 1 */
    int epbl_mld_max_its;     /* 20 */
    int epbl_mld_bisection;   /* 0: false position with a bisection fallback */
    int epbl_mld_use_prev_guess; /* 0 */
    double epbl_mstar_const;  /* 1.2 */
    double epbl_mstar_cap;    /* -1 (off) */
    double epbl_mstar_coef1;  /* 0.3 */
    double epbl_c_ek;         /* 0.085 */
    double epbl_mstar_conv_adj; /* 0 */
    double epbl_nstar;        /* 0.2 */
    double epbl_tke_decay;    /* 2.5 */
    double epbl_wstar_ustar_coef; /* 1 */
    double epbl_vstar_scale_fac; /* 1 */
    double epbl_vstar_surf_fac; /* 1.2 */
    double epbl_von_karman;   /* 0.41 */
    double epbl_ekman_scale_coef; /* 1 */
    double epbl_min_mix_len;  /* 0 m */
    double epbl_mixlen_exponent; /* 2 */
    double epbl_translay_scale; /* 0.1 */
    double epbl_mld_tol;      /* 1 m */
    double epbl_omega;        /* 7.2921e-5 1/s */
    double epbl_omega_frac;   /* 0 */
    double epbl_ustar_min;    /* 1e-8 m/s */
    double epbl_prandtl;      /* 1 */
    /* RH18 mstar fit (epbl_mstar_scheme 3): mstar = cn1 e/(1+e) with
     * e = cn2 exp(cn3 BLD |f|/u*), plus cs1 (B0+^2 BLD/(u*^5 |f|))^cs2 */
    double epbl_rh18_cn1;     /* 0.275 */
    double epbl_rh18_cn2;     /* 8 */
    double epbl_rh18_cn3;     /* -5 */
    double epbl_rh18_cs1;     /* 0.2 */
    double epbl_rh18_cs2;     /* 0.4 */
    /* Langmuir enhancement of mstar (Reichl & Li 2019) from the LF17
     * statistical wave state of u* alone (Li & Fox-Kemper 2017; COARE 3.5
     * u* -> U10): epbl_lf17_wave_state, epbl_lf17_la, epbl_lt_enhance
     * (rdb_ocean_epbl.F90:716-862) */
    int epbl_use_lt;          /* 0 */
    int epbl_lt_scheme;       /* 1 rescale (default), 2 additive */
    double epbl_lt_enhance_coef; /* 0.447 */
    double epbl_lt_enhance_exp; /* -1.33 */
    double epbl_lt_max_enhance; /* 5 */
    double epbl_la_frac_hbl;  /* 0.04: the surface layer the Stokes drift is averaged over, a fraction of the MLD */
    double epbl_lt_lac1;      /* -0.87 */
    double epbl_lt_lac2;      /* 0 */
    double epbl_lt_lac3;      /* 0 */
    double epbl_lt_lac4;      /* 0.95 */
    double epbl_lt_lac5;      /* 0.95 */
    /* 1: vphys_epbl also writes the TKE budget of the last MLD iteration per
     * column, W m-2, into the EPBL_TKE_* fields (tke_diags,
     * rdb_ocean_epbl.F90:1647-1654); wind + conv + forcing - mixing -
     * mech_decay - conv_decay = 0 to round-off */
    int epbl_tke_diags;       /* 0 */
    /* kappa-shear: a column holding layers thinner than H_VANISHED is solved
     * on its massive sub-grid -- vanished layers folded into a massive
     * neighbour by thickness-weighted means, the interface results
     * interpolated back (massless_merge, rdb_massless.F90:51-180) -- instead
     * of flooring them at H_VANISHED; healthy columns are unchanged, bit for
     * bit */
    int ks_massless_merge;    /* 0 */
    /* the shortwave source of the penetration deposit, KPP's B0 charge and
     * EPBL's shortwave TKE ledger (sw_source, rdb_ocean_surface_flux.F90:
     * 715-740, 1256-1399; rdb_ocean_vmix.F90:1076-1118; rdb_ocean_epbl.F90:
     * 895-920): 0 "net_heat", I0 = sw_pen_frac Q_heat; 1 "q_sw",
     * I0 = sw_pen_frac SW_NET (the net shortwave q_sw + sw_ice, >= 0).  The
     * surface deposit itself always books Q_heat. */
    int sw_source;            /* 0 */
    /* OM3 BOUND_SALINITY: after the surface deposit, S = max(S, min_salinity)
     * on the first live layer of every wet column whose thickness exceeds
     * H_DIV_EPS (bound_salinity_top_impl, rdb_ocean_surface_flux.F90:
     * 1072-1091); non-conserving, not booked in the budgets */
    int bound_salinity;       /* 0 */
    /* 1: the WET_DYN field (the dynamic wet/dry cell mask) multiplies the
     * surface deposit of T, S and pseudo-salt, so a dry column takes no flux
     * (apply_surface_src_2d_dyn_impl, rdb_ocean_surface_flux.F90:1144-1225) */
    int use_wet_dyn;          /* 0 */
    double min_salinity;      /* 0 */
    /* EPBL charges the penetrating shortwave per layer in its TKE ledger
     * (epbl_sw_ctke, rdb_ocean_epbl.F90:356-360, 905); 0 treats all of the
     * heat flux as a skin flux even with sw_pen_frac != 0 */
    int epbl_sw_ctke;         /* 1 */
    /* Manizza (2005) chlorophyll N-band shortwave (sw_scheme = "manizza05";
     * rdb_ocean_surface_flux.F90:742-812, 1606-1668, rdb_ocean_sw_chl.F90):
     * the whole shortwave (sw_pen_frac must be 1) is absorbed in sw_nbands
     * bands, T(d) = sum_n frac_n exp(-kappa_n d), with frac the visible 0.42
     * split blue / red by sw_blue_frac and the rest shared evenly by bands
     * 3..n, and kappa_n the per-column opacities of the SW_KAPPA field
     * (vphys_sw_chl_apply fills them from the CHL field).  Read by the
     * penetration, KPP's B0 charge and EPBL's shortwave ledger. */
    int sw_chl;               /* 0 */
    int sw_nbands;            /* 3, in [3, VPHYS_SW_NB_MAX] */
    double sw_blue_frac;      /* 0.5 */
    double sw_opacity_coef[2 * VPHYS_SW_NB_MAX]; /* (a_n, b_n) pairs, m-1: 0.0232 0.074, 0.225 0.037, 2.86 0 */
    double sw_chl_power[VPHYS_SW_NB_MAX];        /* p_n: 0.674, 0.629, 0 */
    double sw_opacity_land;   /* 10: kappa on land columns */
    /* 1: the penetrating shortwave of a column is scaled by 1 - COVER_FRAC,
     * the ice-shelf cover fraction, so no light reaches the water under a
     * shelf (apply_sw_penetration_cover_impl / _nb_cover_impl,
     * rdb_ocean_surface_flux.F90:1532-1604, 1670-1730) */
    int use_cover_frac;       /* 0 */
    /* 1: the tracer diffusion writes, per column and tracer, the content
     * sum_k h_k c_k over the column's live span before the solve (terms
     * added bottom-up) and after it (with the fused non-local deposit; terms
     * added top-down), each an FP64 Neumaier-compensated sum, into the
     * CONTENT_OLD / CONTENT_NEW fields.  No counterpart in the reference: a
     * conservation diagnostic (the exact solve keeps it to FP64 round-off) */
    int column_integrals;     /* 0 */
} vphys_config;

#define VPHYS_KPP_SW_ALL 1
#define VPHYS_KPP_SW_MXL 2
#define VPHYS_KPP_SW_LV1 3

/* ---- field ids (vphys_bind / vphys_set_field / vphys_get_field) ----- */
enum vphys_field {
    VPHYS_FIELD_H = 0,          /* in      (nx, ny, nz)     layer thickness */
    VPHYS_FIELD_RHO = 1,        /* in/out  (nx, ny, nz)     potential density */
    VPHYS_FIELD_U = 2,          /* in/out  (nx+1, ny, nz)   u_face_x_layer */
    VPHYS_FIELD_V = 3,          /* in/out  (nx, ny+1, nz)   v_face_y_layer */
    VPHYS_FIELD_KV = 4,         /* out     (nx, ny, nz+1) */
    VPHYS_FIELD_KT = 5,         /* out     (nx, ny, nz+1) */
    VPHYS_FIELD_KS = 6,         /* out     (nx, ny, nz+1) */
    VPHYS_FIELD_BL_DEPTH = 7,   /* in/out  (nx, ny)  lagged KPP h_b (state) */
    VPHYS_FIELD_B0 = 8,         /* out     (nx, ny)  surface buoyancy flux */
    VPHYS_FIELD_STRESS_MAG = 9, /* in      (nx, ny)  |tau| at cell centres */
    VPHYS_FIELD_Q_HEAT = 10,    /* in      (nx, ny)  W m-2 */
    VPHYS_FIELD_Q_SALT = 11,    /* in      (nx, ny) */
    VPHYS_FIELD_WET = 12,       /* in      (nx, ny)  1 wet, 0 land */
    VPHYS_FIELD_TAU_X = 13,     /* in      (nx+1, ny) */
    VPHYS_FIELD_TAU_Y = 14,     /* in      (nx, ny+1) */
    VPHYS_FIELD_LAMBDA_BOT_U = 15, /* in   (nx+1, ny)  1/s */
    VPHYS_FIELD_LAMBDA_BOT_V = 16, /* in   (nx, ny+1) */
    VPHYS_FIELD_VISC_REM_U = 17,   /* out  (nx+1, ny, nz) */
    VPHYS_FIELD_VISC_REM_V = 18,   /* out  (nx, ny+1, nz) */
    VPHYS_FIELD_GAMMA_T = 19,   /* out     (nx, ny, nz+1) KPP non-local T flux */
    VPHYS_FIELD_GAMMA_S = 20,   /* out     (nx, ny, nz+1) */
    VPHYS_FIELD_HEAT_BUDGET = 21, /* in/out (nx, ny, nz) */
    VPHYS_FIELD_SALT_BUDGET = 22, /* in/out (nx, ny, nz) */
    VPHYS_FIELD_K_TOP_U = 23,   /* in int32 (nx+1, ny), 1-based (default nz) */
    VPHYS_FIELD_K_TOP_V = 24,   /* in int32 (nx, ny+1) */
    VPHYS_FIELD_K_BOT_U = 25,   /* in int32 (nx+1, ny), 1-based (default 1) */
    VPHYS_FIELD_K_BOT_V = 26,   /* in int32 (nx, ny+1) */
    VPHYS_FIELD_CORIOLIS = 27,  /* in      (nx, ny)  f at cell centres, 1/s: read by the learned KPP's
                                   features and by kappa-shear (f^2) */
    VPHYS_FIELD_HEAT_BUDGET_SURFACE = 28, /* in/out (nx, ny, nz) the surface deposit's heat contributor */
    VPHYS_FIELD_SALT_BUDGET_SURFACE = 29, /* in/out (nx, ny, nz) */
    VPHYS_FIELD_KD_SHEAR = 30,  /* in/out  (nx, ny, nz+1) kappa-shear diffusivity kd_int, 0 at bed and surface */
    VPHYS_FIELD_TKE_SHEAR = 31, /* out     (nx, ny, nz+1) kappa-shear time-mean TKE tke_int */
    VPHYS_FIELD_KD_EPBL = 32,   /* in/out  (nx, ny, nz+1) EPBL diffusivity kd_int, 0 at bed and surface */
    VPHYS_FIELD_MLD_EPBL = 33,  /* in/out  (nx, ny) EPBL mixed-layer depth (the previous one seeds the
                                   iteration when epbl_mld_use_prev_guess) */
    VPHYS_FIELD_LA_EPBL = 34,   /* out     (nx, ny) EPBL Langmuir number of the last MLD iteration (0 when
                                   epbl_use_lt is 0) */
    VPHYS_FIELD_EPBL_TKE_WIND = 35,       /* out (nx, ny) W m-2: mstar u*^3 rho0 (epbl_tke_diags) */
    VPHYS_FIELD_EPBL_TKE_CONV = 36,       /* out (nx, ny) convective release, nstar-weighted */
    VPHYS_FIELD_EPBL_TKE_FORCING = 37,    /* out (nx, ny) <= 0: surface stabilisation paid from the wind */
    VPHYS_FIELD_EPBL_TKE_MIXING = 38,     /* out (nx, ny) spent raising potential energy */
    VPHYS_FIELD_EPBL_TKE_MECH_DECAY = 39, /* out (nx, ny) mechanical TKE decayed (and left at the bed) */
    VPHYS_FIELD_EPBL_TKE_CONV_DECAY = 40, /* out (nx, ny) convective TKE lost to rotation (and left at the bed) */
    VPHYS_FIELD_SW_NET = 41,    /* in      (nx, ny) W m-2 >= 0: the net shortwave q_sw + sw_ice, the source
                                   when sw_source = 1 (allocated then) */
    VPHYS_FIELD_WET_DYN = 42,   /* in      (nx, ny) dynamic wet/dry cell mask, 1 wet, 0 dry (use_wet_dyn = 1;
                                   allocated then, filled with 1) */
    VPHYS_FIELD_SW_CHL = 43,    /* in      (nx, ny) surface chlorophyll, mg m-3 (sw_chl = 1; filled with the
                                   1e-4 floor) */
    VPHYS_FIELD_SW_KAPPA = 44,  /* in/out  (nx, ny, VPHYS_SW_NB_MAX) band opacities, m-1, the first
                                   sw_nbands planes read (sw_chl = 1; filled with 1) */
    VPHYS_FIELD_COVER_FRAC = 45, /* in     (nx, ny) ice-shelf cover fraction in [0, 1] (use_cover_frac = 1;
                                   filled with 0) */
    VPHYS_FIELD_CONTENT_OLD = 46, /* out   (nx, ny, ntracer) compensated column content before the diffusion
                                   (column_integrals = 1) */
    VPHYS_FIELD_CONTENT_NEW = 47, /* out   (nx, ny, ntracer) the same after it */
    VPHYS_FIELD_TRACER0 = 64    /* in/out  (nx, ny, nz); tracer t is
                                   VPHYS_FIELD_TRACER0 + t */
};

typedef struct vphys_handle_s *vphys_handle;

/* ---- lifecycle ------------------------------------------------------- */

/* Fill *cfg with the reference defaults listed above (each field cites its
 * namelist key and type default). */
int vphys_config_default(vphys_config *cfg);

/* Allocate a handle for an (nx, ny, nz) grid with ntracer tracers and
 * allocate every field in HBM (zeroed; k_top = nz, k_bot = 1, wet = 1).
 * Replaces ocean_vmix_init + ocean_vdiff_init + vmix_seed_backgrounds
 * (rdb_ocean_vmix.F90:798-913, rdb_ocean_vdiff.F90:328-372): kv = kv_bg,
 * kt = ks = kt_bg on interior interfaces, 0 on the bed and surface ones.
 * nz must be in [1, VPHYS_NZ_MAX].  On failure *out is NULL. */
int vphys_create(int nx, int ny, int nz, int ntracer, const vphys_config *cfg,
                 vphys_handle *out);

/* Idempotent on NULL; frees every handle-owned buffer; *h = NULL.  Replaces
 * rdb_ocean_destroy (include/rdb_ocean.h:119). */
int vphys_destroy(vphys_handle *h);

/* Replace the configuration (validated; VPHYS_ERR_CONFIG on a bad one).  No
 * counterpart in the reference's C ABI, whose configuration is the namelist
 * text of rdb_ocean_create_from_string (include/rdb_ocean.h:108). */
int vphys_set_config(vphys_handle h, const vphys_config *cfg);
int vphys_get_config(vphys_handle h, vphys_config *cfg);

/* Run the handle's work on this CUDA stream (cudaStream_t as void*;
 * NULL = the legacy default stream).  No counterpart in the reference. */
int vphys_set_stream(vphys_handle h, void *stream);

/* Zero-copy: use the caller's device array for `field` from now on.
 * The pointer must stay valid while the handle uses it.  The handle's own
 * buffer for the field is freed (a bound state is never held twice); NULL
 * unbinds and gives the field a fresh handle-owned buffer with its default
 * contents.  Synchronises the device when a buffer is freed.  The other
 * direction of the reference's zero-copy getters rdb_ocean_get_*_ptr
 * (include/rdb_ocean.h:338-387), which vphys_get_ptr replaces. */
int vphys_bind(vphys_handle h, int field, void *device_ptr);

/* Synchronous host<->device copies of a whole field (n = element count,
 * checked against the field's shape: VPHYS_ERR_BAD_SHAPE).  Double fields
 * take double*, the K_TOP/K_BOT fields int32*.  Replace the setters
 * rdb_ocean_set_h / _u / _v / _wind / _heat_flux / _salt_flux / _tracer
 * (include/rdb_ocean.h:419-447) and, for reading, rdb_ocean_refresh_host
 * (:327) with the host arrays. */
int vphys_set_field(vphys_handle h, int field, const void *host, size_t n);
int vphys_get_field(vphys_handle h, int field, void *host, size_t n);

/* The same copies enqueued on the handle's stream without waiting (the
 * counterparts of the setters and getters above, include/rdb_ocean.h:419-447,
 * made asynchronous): they return once the copy is queued, in stream order
 * with vphys_step.  The host buffer must stay valid, and untouched by the
 * caller, until vphys_synchronize(h) returns; page-locked (pinned) host
 * memory lets the copy run while the host and other streams work, so a
 * caller with two handles on two streams can overlap one domain's upload
 * with another's download. */
int vphys_set_field_async(vphys_handle h, int field, const void *host, size_t n);
int vphys_get_field_async(vphys_handle h, int field, void *host, size_t n);

/* Current device pointer and shape of a field, like
 * rdb_ocean_get_kv_ptr(handle, ptr, nx, ny, nz, gen)
 * (include/rdb_ocean.h:378-385); *gen = number of completed vphys_step
 * steps.  The pointer is a DEVICE pointer. */
int vphys_get_ptr(vphys_handle h, int field, void **ptr, int *nx, int *ny,
                  int *nz, int *gen);

/* ---- the hot path, stage by stage ------------------------------------ */

/* Wright (1997) EOS at eos_p_ref: rho from (T, S, h); vanished layers take
 * rho0.  Replaces eos_wright_impl (src/equation_of_state/rdb_eos.F90:909-959). */
int vphys_eos_wright(vphys_handle h);

/* |tau| at cell centres from the face stresses TAU_X/TAU_Y into STRESS_MAG.
 * Replaces ocean_surfstress_derived_impl
 * (rdb_ocean_surface_stress.F90:858-875). */
int vphys_stress_mag(vphys_handle h);

/* The surface heat and salt fluxes deposited on the first live layer from
 * the top: T += dt*Q_HEAT*WET/(rho0*cp)/(h+eps), S and pseudo-salt +=
 * dt*Q_SALT*WET/rho0/(h+eps) (rdb_conc_add_source; a vanished layer takes
 * nothing).  With budgets on, HEAT_BUDGET_SURFACE / SALT_BUDGET_SURFACE book
 * the accepted content (pseudo-salt books none).  Replaces
 * ocean_surface_flux_apply_tracers (rdb_ocean_surface_flux.F90:959-1070,
 * apply_surface_src_2d_impl 1093-1142, the nobudget twin 1175-1203), called
 * after the EOS at rdb_ocean_dyn.F90:1363; vphys_step runs it there when
 * surface_flux is 1. */
int vphys_surface_flux(vphys_handle h, double dt);

/* The penetrating shortwave moved down the column after the surface
 * deposit: I0 = sw_pen_frac * Q_HEAT * WET leaves the first live layer and
 * each live layer takes I0 (T(d_top) - T(d_bottom)) * dt/(rho0 cp), the
 * deepest live layer the rest (an opaque bed); vanished layers pass the light
 * on.  Column heat is unchanged; HEAT_BUDGET_SURFACE books the moves when
 * budgets are on.  A no-op when sw_pen_frac is 0 or there is no temperature
 * tracer.  Replaces ocean_surface_flux_apply_sw_penetration with
 * apply_sw_penetration_impl (rdb_ocean_surface_flux.F90:1255-1530), called
 * at rdb_ocean_dyn.F90:1375 right after the surface deposit; vphys_step runs
 * it there when surface_flux is 1. */
int vphys_sw_penetration(vphys_handle h, double dt);

/* The band opacities of the chlorophyll shortwave scheme from the CHL field:
 * SW_KAPPA(:,:,n) = a_n + b_n max(chl, 1e-4)^p_n on wet columns (the safe
 * pow, rdb_sm_pow), sw_opacity_land on land, for n = 1..sw_nbands.
 * Replaces sw_chl_fill_kappa / sw_kappa_band_impl / sw_opacity_manizza
 * (rdb_ocean_sw_chl.F90:160-190, rdb_ocean_surface_flux.F90:784-793), run by
 * sw_chl_apply after each chlorophyll read.  VPHYS_ERR_CONFIG unless
 * sw_chl = 1. */
int vphys_sw_chl_apply(vphys_handle h);

/* Kappa-shear, column form: per wet column, the JHL08 steady (kappa, TKE)
 * pair solved surface-down on the interfaces with adaptive substepping over
 * dt (a kappa_0 background pre-step, frozen EOS buoyancy derivatives at the
 * hydrostatic pressure, predictor-corrector substeps, Picard inner solves),
 * from H, U and V averaged to cell centres, the temperature and salinity
 * tracers, and CORIOLIS (f^2).  Writes KD_SHEAR (the time-mean diffusivity,
 * 0 on the bed and surface interfaces and in land columns) and TKE_SHEAR.
 * Layers thinner than H_VANISHED enter at H_VANISHED.  A no-op without a
 * temperature or salinity tracer.  Replaces kappa_shear_compute ->
 * kappa_shear_column_kernel (rdb_ocean_kappa_shear.F90:427-648, the solver
 * 953-1909); vphys_step runs it before the assembly when kappa_shear is 1,
 * and the assembly adds KD_SHEAR (rdb_ocean_dyn.F90:1564-1583). */
int vphys_kappa_shear(vphys_handle h, double dt);

/* EPBL, column form: per wet column the energetics of the surface forcing
 * (mstar u*^3 of wind work, the convective release of the surface buoyancy
 * loss) spent down the column on the largest diffusivity each interface can
 * afford (a closed-form energy solve with an embedded forward elimination),
 * iterated on the mixed-layer depth (false position, up to
 * epbl_mld_max_its).  Reads H, T, S, STRESS_MAG, Q_HEAT, Q_SALT, WET,
 * CORIOLIS; writes KD_EPBL (0 on the bed and surface interfaces and in land
 * columns), MLD_EPBL and LA_EPBL.  A no-op without a temperature or salinity tracer.
 * Replaces epbl_compute -> epbl_column_kernel (rdb_ocean_epbl.F90:864-1659);
 * vphys_step runs it before the assembly when epbl is 1, and the assembly
 * merges KD_EPBL (epbl_merge_into_kv_kt / epbl_merge_max_shear, 1661-1718). */
int vphys_epbl(vphys_handle h, double dt);

/* Mixed-precision tracer solves (mixed_precision >= 1): the number of
 * (32-column group, tracer) pairs whose one-step increment reached 2 units
 * in the last solve and were re-solved on the FP64 path (bitwise the exact
 * results).  Synchronises the handle's stream; 0 when nothing is mixed.  No
 * counterpart in the reference. */
int vphys_mixed_redo_count(vphys_handle h, unsigned *groups);

/* The whole coefficient build: interior closure (PP81 or background seed),
 * KPP overlay (+ bl_depth, b0, gamma_t/gamma_s), the kappa-shear merge
 * (kt += KD_SHEAR, kv += ks_prandtl_turb * KD_SHEAR when kappa_shear is 1),
 * KV_ML_INVZ2, convection,
 * heat/salt split, assembly gate (guard, Bryan-Lewis or scalar floors,
 * ceilings, optional 1-2-1 smoothing).  Replaces vmix_build_coefficients
 * (rdb_ocean_dyn.F90:1473-1634) with vmix_compute_pp81
 * (rdb_ocean_vmix.F90:1007-1074), vmix_apply_kpp_overlay (1076-1516),
 * vmix_add_kv_ml_invz2 (1716-1766), vmix_apply_convection (1768-1849),
 * vmix_split_kd_heat_salt (1850-1934), vmix_assemble (2183-2366).
 * Returns VPHYS_ERR_GUARD (after finishing the clip, like the reference's
 * status=1 path) when vmix_guard is on and a negative/NaN K was seen; this
 * return synchronises the stream. */
int vphys_assemble(vphys_handle h);

/* Backward-Euler vertical viscosity on U and V with kv.  Replaces
 * vdiff_apply_momentum -> diffuse_velocity_columns_impl
 * (rdb_ocean_vdiff.F90:455-718, 1416-1926). */
int vphys_vdiff_momentum(vphys_handle h, double dt);

/* Backward-Euler vertical diffusion: kt on temperature, ks on salinity and
 * every other tracer.  Replaces vdiff_apply_tracers
 * (rdb_ocean_vdiff.F90:1107-1414).  One factorisation serves every tracer
 * only while ks is the assembly gate's bitwise copy of kt (written by
 * vphys_assemble or vphys_step under floors that agree, and neither field
 * written by the caller since, bound to a caller's buffer or handed out by
 * vphys_get_ptr); otherwise kt and ks are factorised separately. */
int vphys_vdiff_tracers(vphys_handle h, double dt);

/* KPP non-local tendencies on T (gamma_t), S and pseudo-salt (gamma_s),
 * using the gamma of the last vphys_assemble.  Replaces
 * vmix_apply_nonlocal_tendencies (rdb_ocean_vmix.F90:1605-1714).  The
 * kernel re-derives gamma per column from h, BL_DEPTH, B0, STRESS_MAG,
 * Q_HEAT, Q_SALT and the shortwave fields rather than storing it, so those
 * must hold what vphys_assemble read (as in the reference's stage order,
 * where nothing writes them in between); the same holds for
 * vphys_vdiff_tracers_nonlocal. */
int vphys_nonlocal(vphys_handle h, double dt);

/* The tracer diffusion followed by the KPP non-local tendencies, as one fused
 * launch: the launch vphys_step runs for this stage.  Replaces the pair of
 * calls vdiff_apply_tracers then vmix_apply_nonlocal_tendencies that
 * vmix_apply_in_stage makes back to back (rdb_ocean_dyn.F90:1856-1860;
 * rdb_ocean_vdiff.F90:1107-1414, rdb_ocean_vmix.F90:1605-1714); the result
 * equals vphys_vdiff_tracers then vphys_nonlocal.  Asynchronous. */
int vphys_vdiff_tracers_nonlocal(vphys_handle h, double dt);

/* The in-project autotuner of the mixed-precision solves (no counterpart in
 * the reference, whose solves have one form each).  Times every kernel
 * variant of the mixed face solve and of the mixed tracer solve that the
 * handle's configuration admits, on the handle's own state (after an EOS and
 * an assembly, reps timed runs each after a warm-up, the state restored
 * before every run), keeps the fastest of each for the handle's later steps,
 * and restores the whole state (every field reads back as before the call).
 * Variants: face solve 0 registers, 1 TMA-staged ring; tracer solve 0, 1, 2
 * rows in shared memory with 1, 2 or 4 tracers per warp, 3 rows in tensor
 * memory.  ms[0..1] receive the face-solve times and ms[2..5] the tracer
 * times in milliseconds (-1: not admitted; ms may be NULL), chosen[0..1] the
 * picks (may be NULL).  Needs device memory for a copy of the state while it
 * runs.  Without mixed_precision it only reports the current picks.
 * Synchronous. */
int vphys_autotune(vphys_handle h, double dt, int reps, double *ms, int n_ms, int *chosen);

/* Pins the kernel variants of the mixed solves (the numbering of
 * vphys_autotune); a variant the configuration does not admit falls back to
 * the register form (face solve) or one tracer per warp (tracer solve).  No
 * counterpart in the reference. */
int vphys_set_variants(vphys_handle h, int momentum, int tracers);

/* n_steps of the whole chain (the body of vmix_apply_in_stage on a thermo
 * step, rdb_ocean_dyn.F90:1636-1900): [EOS] -> assemble -> momentum ->
 * tracers -> non-local, with the tracer solve and the non-local tendency
 * fused.  Asynchronous; safe to capture in a CUDA graph once the handle's
 * buffers are allocated.  n_steps <= 0 is a successful no-op. */
int vphys_step(vphys_handle h, double dt, int n_steps);

/* vphys_step as one CUDA graph: the launches of n_steps steps are captured
 * once (on a private stream) and replayed with cudaGraphLaunch on the
 * handle's stream; a change of any bound pointer, of the configuration, of
 * dt, n_steps or of the attached surrogate recaptures.  Results are those of
 * vphys_step(h, dt, n_steps).  (The learned KPP's sampled-check columns are
 * fixed per capture.)  Asynchronous.  No counterpart in the reference: the
 * CUDA-graph form of vphys_step. */
int vphys_step_graph(vphys_handle h, double dt, int n_steps);

/* Block until the handle's stream is idle; VPHYS_ERR_CUDA on a CUDA error.
 * No counterpart in the reference (whose calls return synchronised). */
int vphys_synchronize(vphys_handle h);

/* ---- errors ------------------------------------------------------------
 * Ring of recent messages, index 0 = most recent.  Copies up to cap bytes
 * (NUL-terminated if room), returns the full message length; 0 when idx is
 * out of range or cap <= 0 (rdb_ocean_last_error, include/rdb_ocean.h:314). */
int vphys_last_error(int idx, char *buf, int cap);

/* Library version string (static storage).  No counterpart in the
 * reference's C ABI. */
const char *vphys_version(void);

/* Device self-test of the exact division used by the kernels (a zero-guarded
 * quotient and a shared-reciprocal quotient with Markstein's correction):
 * compares both with the IEEE quotient a/b on n_pairs seeded operand pairs,
 * exponents in [emin, emin+erange), and writes the number of differing bits
 * patterns to *mismatches (0 expected).  Synchronous.  No counterpart in the
 * reference. */
int vphys_selftest_division(long long n_pairs, unsigned long long seed, int emin, int erange,
                            unsigned long long *mismatches);

/* Allocation-free 1-2-1 smoothing.  No counterpart in the reference.  It is
 * the same wet-masked 1-2-1 horizontal smoothing that vphys_assemble applies
 * when kd_smooth_iterations > 0, offered to callers that cannot call
 * cudaMalloc -- a host that owns all device memory through its own pool
 * (an OpenACC/Fortran model, a framework caching allocator) or code running
 * where allocating is not allowed.  `fld` is a device (nx, ny, nz+1)
 * interface field (kv, kt or ks), smoothed in place on interfaces 2..nz for
 * `iterations` passes; `wet` the device (nx, ny) wet mask; `stream` a
 * cudaStream_t (NULL: legacy default stream).  The copy of a plane that the
 * stencil reads lives in a fixed device array of 2^23 doubles (64 MiB) that
 * every GPU loading the library holds until exit; nx*ny above 2^23 returns
 * VPHYS_ERR_TOO_LARGE.  Nothing is allocated or freed.  The first call on a
 * device looks up that array's device address (once per device); make it
 * before any stream capture.  All calls share the array, so calls whose work
 * overlaps on the GPU race.  Asynchronous. */
int vphys_smooth_121_static(double *fld, const double *wet, int nx, int ny, int nz, int iterations,
                            void *stream);

/* sizeof(vphys_config) as compiled into the library, so a binding in another
 * language can verify its mirror of the struct before passing one.  No
 * counterpart in the reference (its configuration is namelist text). */
size_t vphys_config_sizeof(void);

/* ---- learned KPP surrogate: building blocks ---------------------------------
 * No counterpart in the reference (whose KPP is the bulk-Richardson search of
 * vmix_kpp_overlay_impl, rdb_ocean_vmix.F90:1121-1516); these serve the MLP
 * that stands in for it when cfg.learned_kpp is set.  All pointers are device
 * pointers; all calls are asynchronous on `stream` (cudaStream_t, NULL: the
 * legacy default stream).
 *
 * vphys_gemm_tn_bf16: C[M,N] = alpha * A[M,K] . B[N,K]^T on the tcgen05 tensor
 * cores, BF16 operands (row-major, K contiguous, rows lda / ldb elements apart,
 * 16-byte aligned, K, lda, ldb multiples of 8),
 * FP32 accumulation, 16 <= N <= 256 with N % 16 == 0.  Epilogue, per element:
 * v = alpha*acc (+ bias[col]) (* GELU'(zin[row*ld_z+col]) when zin);
 * out_f32[row*ld_f32+col] = v; a = act ? GELU(v) : v (tanh form);
 * out_bf16[row*ld_bf16+col] = bf16(a); out_bf16_t[col*ld_t+row] = bf16(a).
 * Every output may be NULL.  A stalled pipeline writes a non-zero code to
 * *err (device int) instead of hanging. */
/* The surrogate's weights and settings (device pointers stay owned by the
 * caller and must outlive the attachment).  Shapes: w1 BF16 [256, 160]
 * (inputs beyond 154 zero), w2 [256, 256], w3 [80, 256] (outputs beyond 77
 * unused), each row-major [out, in]; b1, b2 [256], b3 [80] FP32; feat_mean /
 * feat_istd [160] FP32 (features are (x - mean) * istd); the OBL-depth output
 * y0 is de-standardised as h_b = 10 m * exp(y0 * target_std0 + target_mean0). */
typedef struct vphys_kpp_model {
    const void *w1, *w2, *w3;
    const float *b1, *b2, *b3;
    const float *feat_mean, *feat_istd;
    float target_mean0, target_std0;
    float gate_limit;       /* |standardised feature| beyond which a column takes the plain KPP (e.g. 6) */
    float check_fraction;   /* fraction of columns re-run by the plain KPP each step (e.g. 0.01) */
    float check_tolerance;  /* relative h_b error counted as a failed check (e.g. 0.25) */
    float fail_fraction;    /* failed share of the checked columns that sends the next step to the plain KPP */
} vphys_kpp_model;

/* Attach (m != NULL) or detach (m == NULL) the surrogate; allocates one
 * inference's scratch (about 1.7 kB per column).  With cfg.learned_kpp and
 * cfg.use_kpp, vphys_assemble and vphys_step then run features -> MLP ->
 * gate/check before the assembly, whose pass 1 runs only where needed. */
int vphys_kpp_attach(vphys_handle h, const vphys_kpp_model *m);
/* Counters (synchronises the handle's stream): [0] checked in the last step,
 * [1] failed, [2] fallback flag of the last step, [3] gated in the last step,
 * [4] checked in total, [5] failed in total, [6] fallback steps, [7] gated in
 * total, [8] sum of squared relative h_b errors of the checks * 1e6, [9]
 * steps, [10] tensor-core GEMM error code (0).  n: entries wanted (<= 16). */
int vphys_kpp_stats(vphys_handle h, unsigned long long *out, int n);
/* Features of the handle's current state: raw FP32 [ncols, 154] and/or
 * standardised BF16 X [ncols, 160] / XT [160, ld_t] (mean, istd NULL: raw
 * values), the per-column gate flag and column depth (-1: no live layer). */
int vphys_kpp_features(vphys_handle h, const float *mean, const float *istd, float gate_limit, float *raw, void *X,
                       void *XT, long long ld_t, unsigned char *gate, float *colH);
/* Training targets [ncols, 80] FP32 from the state left by a plain assembly. */
int vphys_kpp_targets(vphys_handle h, float *T);
/* Training helpers: dY = scale*w*(Y - T) (+ loss += sum w (Y-T)^2); column
 * sums; column sums and sums of squares (FP64); standardisation into BF16 /
 * transposed BF16 / FP32; one Adam step (step >= 1) refreshing BF16 copies. */
int vphys_mlp_loss(const float *Y, const float *T, const float *w, int rows, int cols, float scale, float *dY32,
                   void *dY, void *dYT, float *loss, void *stream);
int vphys_mlp_colsum(const float *G, int rows, int cols, int ld, float *out, void *stream);
int vphys_mlp_colstats(const float *X, long long rows, int cols, int ld, double *sum, double *sumsq, void *stream);
int vphys_mlp_standardize(const float *raw, long long rows, int cols_in, int ld_in, const float *mean,
                          const float *istd, int cols_out, void *X, void *XT, long long ld_t, float *out32,
                          void *stream);
int vphys_mlp_adam(float *w, float *m, float *v, const float *g, int rows, int cols, float lr, float b1, float b2,
                   float eps, int step, void *wb, void *wbt, void *stream);

int vphys_gemm_tn_bf16(const void *A, long long lda, const void *B, long long ldb, int M, int N, int K,
                       float alpha, const float *bias, const float *zin, int ld_z, int act, float *out_f32,
                       int ld_f32, void *out_bf16, int ld_bf16, void *out_bf16_t, int ld_t, int *err, void *stream);

/* The surrogate's forward pass in one launch (the three layers of
 * vphys_kpp's in-step inference): Y[M,80] = (GELU(GELU(X W1^T + b1) W2^T + b2))
 * W3^T + b3 with X [M,160] BF16, W1 [256,160], W2 [256,256], W3 [80,256] BF16
 * (K contiguous), b1/b2 [256], b3 [80] and Y FP32.  The hidden activations
 * stay in shared memory (BF16, as the three separate GEMMs round them), so Y
 * equals three vphys_gemm_tn_bf16 calls bit for bit.  Every pointer 16-byte
 * aligned; M <= 0 is a no-op.  *err as for vphys_gemm_tn_bf16. */
int vphys_mlp3_bf16(const void *X, int M, const void *W1, const float *b1, const void *W2, const float *b2,
                    const void *W3, const float *b3, float *Y, int *err, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* VPHYS_H */
