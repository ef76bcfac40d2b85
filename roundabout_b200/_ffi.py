"""ctypes bindings to libvphys.so (include/vphys.h).

Mirrors the conventions of the reference's python/rdb/_ffi.py: stdlib ctypes
only, every prototype declared so a mismatched call raises instead of
corrupting memory, status codes kept byte-for-byte in sync with the C header,
and a library search order of

  1. ``VPHYS_LIB`` environment variable (explicit path to the .so);
  2. the in-tree build ``roundabout_b200/csrc/_build/libvphys.so``.

There is no CPU fallback: if the library is missing, `get_lib()` raises
`LibraryNotFoundError`.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

# ---- status codes: keep in sync with include/vphys.h -------------------
OK = 0
ERR_CONFIG = 2
ERR_BAD_HANDLE = 10
ERR_NOT_INITIALISED = 12
ERR_NOT_FOUND = 13
ERR_BAD_SHAPE = 14
ERR_CUDA = 30
ERR_GUARD = 31
ERR_TOO_DEEP = 32
ERR_ALLOC = 33
ERR_TOO_LARGE = 34

NZ_MAX = 127
INTERIOR_PP81 = 1
INTERIOR_NONE = 4

# ---- field ids ---------------------------------------------------------
FIELD_H = 0
FIELD_RHO = 1
FIELD_U = 2
FIELD_V = 3
FIELD_KV = 4
FIELD_KT = 5
FIELD_KS = 6
FIELD_BL_DEPTH = 7
FIELD_B0 = 8
FIELD_STRESS_MAG = 9
FIELD_Q_HEAT = 10
FIELD_Q_SALT = 11
FIELD_WET = 12
FIELD_TAU_X = 13
FIELD_TAU_Y = 14
FIELD_LAMBDA_BOT_U = 15
FIELD_LAMBDA_BOT_V = 16
FIELD_VISC_REM_U = 17
FIELD_VISC_REM_V = 18
FIELD_GAMMA_T = 19
FIELD_GAMMA_S = 20
FIELD_HEAT_BUDGET = 21
FIELD_SALT_BUDGET = 22
FIELD_K_TOP_U = 23
FIELD_K_TOP_V = 24
FIELD_K_BOT_U = 25
FIELD_K_BOT_V = 26
FIELD_CORIOLIS = 27
FIELD_HEAT_BUDGET_SURFACE = 28
FIELD_SALT_BUDGET_SURFACE = 29
FIELD_KD_SHEAR = 30
FIELD_TKE_SHEAR = 31
FIELD_KD_EPBL = 32
FIELD_MLD_EPBL = 33
FIELD_LA_EPBL = 34
FIELD_EPBL_TKE = {"wind": 35, "conv": 36, "forcing": 37, "mixing": 38, "mech_decay": 39, "conv_decay": 40}
FIELD_SW_NET = 41
FIELD_WET_DYN = 42
FIELD_SW_CHL = 43
FIELD_SW_KAPPA = 44
FIELD_COVER_FRAC = 45
FIELD_CONTENT_OLD = 46
FIELD_CONTENT_NEW = 47
SW_NB_MAX = 6
FIELD_TRACER0 = 64

FIELD_NAMES = {
    "h": FIELD_H, "rho": FIELD_RHO, "u": FIELD_U, "v": FIELD_V, "kv": FIELD_KV, "kt": FIELD_KT,
    "ks": FIELD_KS, "bl_depth": FIELD_BL_DEPTH, "b0": FIELD_B0, "stress_mag": FIELD_STRESS_MAG,
    "q_heat": FIELD_Q_HEAT, "q_salt": FIELD_Q_SALT, "wet": FIELD_WET, "tau_x": FIELD_TAU_X,
    "tau_y": FIELD_TAU_Y, "lambda_bot_u": FIELD_LAMBDA_BOT_U, "lambda_bot_v": FIELD_LAMBDA_BOT_V,
    "visc_rem_u": FIELD_VISC_REM_U, "visc_rem_v": FIELD_VISC_REM_V, "gamma_t": FIELD_GAMMA_T,
    "gamma_s": FIELD_GAMMA_S, "heat_budget": FIELD_HEAT_BUDGET, "salt_budget": FIELD_SALT_BUDGET,
    "k_top_u": FIELD_K_TOP_U, "k_top_v": FIELD_K_TOP_V, "k_bot_u": FIELD_K_BOT_U,
    "k_bot_v": FIELD_K_BOT_V, "coriolis": FIELD_CORIOLIS,
    "heat_budget_surface": FIELD_HEAT_BUDGET_SURFACE, "salt_budget_surface": FIELD_SALT_BUDGET_SURFACE,
    "kd_shear": FIELD_KD_SHEAR, "tke_shear": FIELD_TKE_SHEAR, "kd_epbl": FIELD_KD_EPBL, "mld_epbl": FIELD_MLD_EPBL,
    "la_epbl": FIELD_LA_EPBL, "sw_net": FIELD_SW_NET, "wet_dyn": FIELD_WET_DYN, "sw_chl": FIELD_SW_CHL,
    "sw_kappa": FIELD_SW_KAPPA, "cover_frac": FIELD_COVER_FRAC,
    "content_old": FIELD_CONTENT_OLD, "content_new": FIELD_CONTENT_NEW,
    **{f"epbl_tke_{k}": v for k, v in FIELD_EPBL_TKE.items()},
}
INT_FIELDS = (FIELD_K_TOP_U, FIELD_K_TOP_V, FIELD_K_BOT_U, FIELD_K_BOT_V)


def field_shape(field: int, nx: int, ny: int, nz: int, ntr: int = 1):
    """Fortran-order shape of a field (matches the counts of vphys_create)."""
    if field in (FIELD_CONTENT_OLD, FIELD_CONTENT_NEW):
        return (nx, ny, max(1, ntr))
    if field >= FIELD_TRACER0 or field in (FIELD_H, FIELD_RHO, FIELD_HEAT_BUDGET, FIELD_SALT_BUDGET,
                                           FIELD_HEAT_BUDGET_SURFACE, FIELD_SALT_BUDGET_SURFACE):
        return (nx, ny, nz)
    if field in (FIELD_U, FIELD_VISC_REM_U):
        return (nx + 1, ny, nz)
    if field in (FIELD_V, FIELD_VISC_REM_V):
        return (nx, ny + 1, nz)
    if field in (FIELD_KV, FIELD_KT, FIELD_KS, FIELD_GAMMA_T, FIELD_GAMMA_S, FIELD_KD_SHEAR, FIELD_TKE_SHEAR,
                 FIELD_KD_EPBL):
        return (nx, ny, nz + 1)
    if field in (FIELD_BL_DEPTH, FIELD_B0, FIELD_STRESS_MAG, FIELD_Q_HEAT, FIELD_Q_SALT, FIELD_WET, FIELD_CORIOLIS,
                 FIELD_MLD_EPBL, FIELD_LA_EPBL, FIELD_SW_NET, FIELD_WET_DYN, FIELD_SW_CHL,
                 FIELD_COVER_FRAC) or field in FIELD_EPBL_TKE.values():
        return (nx, ny)
    if field in (FIELD_TAU_X, FIELD_LAMBDA_BOT_U, FIELD_K_TOP_U, FIELD_K_BOT_U):
        return (nx + 1, ny)
    if field in (FIELD_TAU_Y, FIELD_LAMBDA_BOT_V, FIELD_K_TOP_V, FIELD_K_BOT_V):
        return (nx, ny + 1)
    if field == FIELD_SW_KAPPA:
        return (nx, ny, SW_NB_MAX)
    raise KeyError(field)


class VphysConfig(ctypes.Structure):
    """Mirror of `struct vphys_config` (include/vphys.h), field for field."""
    _fields_ = [
        ("use_closure", ctypes.c_int), ("interior_closure", ctypes.c_int), ("use_kpp", ctypes.c_int),
        ("bkgnd_profile", ctypes.c_int), ("vmix_guard", ctypes.c_int), ("kd_smooth_iterations", ctypes.c_int),
        ("conv_enable", ctypes.c_int), ("surface_flux", ctypes.c_int),
        ("pp81_nu0", ctypes.c_double), ("pp81_nu_bg", ctypes.c_double), ("pp81_kappa_bg", ctypes.c_double),
        ("pp81_alpha", ctypes.c_double), ("rho0", ctypes.c_double), ("shear2_floor", ctypes.c_double),
        ("ri_crit", ctypes.c_double), ("cs_nonlocal", ctypes.c_double), ("c_vt2", ctypes.c_double),
        ("alpha_T", ctypes.c_double), ("beta_S", ctypes.c_double), ("cp", ctypes.c_double),
        ("kv_ml_invz2", ctypes.c_double), ("hmix_fixed", ctypes.c_double),
        ("conv_kd", ctypes.c_double), ("conv_prandtl", ctypes.c_double), ("conv_n2_thresh", ctypes.c_double),
        ("kv_bg", ctypes.c_double), ("kt_bg", ctypes.c_double), ("ks_bg", ctypes.c_double),
        ("kv_max", ctypes.c_double), ("kd_max", ctypes.c_double),
        ("bkgnd_kd_sfc", ctypes.c_double), ("bkgnd_kd_deep", ctypes.c_double), ("bkgnd_z0", ctypes.c_double),
        ("bkgnd_delta", ctypes.c_double), ("bkgnd_prandtl", ctypes.c_double),
        ("eos_p_ref", ctypes.c_double),
        ("hvel_mom6", ctypes.c_int), ("hvel_harmonic", ctypes.c_int), ("hvel_upwind", ctypes.c_int),
        ("use_harmonic", ctypes.c_int), ("implicit_stress", ctypes.c_int), ("implicit_drag", ctypes.c_int),
        ("zlevel_faces", ctypes.c_int), ("bbl_glue", ctypes.c_int),
        ("hbbl_visc", ctypes.c_double), ("bbl_piston", ctypes.c_double), ("kv_bbl_bg", ctypes.c_double),
        ("idx_temperature", ctypes.c_int), ("idx_salinity", ctypes.c_int), ("idx_pseudo_salt", ctypes.c_int),
        ("eos_in_step", ctypes.c_int), ("remnant", ctypes.c_int), ("budgets", ctypes.c_int),
        ("mixed_precision", ctypes.c_int), ("learned_kpp", ctypes.c_int),
        ("buoyancy_coeffs", ctypes.c_int), ("kpp_sw_method", ctypes.c_int),
        ("sw_pen_frac", ctypes.c_double), ("sw_band_ratio", ctypes.c_double), ("sw_zeta1", ctypes.c_double),
        ("sw_zeta2", ctypes.c_double),
        ("kappa_shear", ctypes.c_int), ("ks_max_inner_it", ctypes.c_int), ("ks_max_substep_it", ctypes.c_int),
        ("eos_variant", ctypes.c_int),
        ("ks_ri_crit", ctypes.c_double), ("ks_shearmix_rate", ctypes.c_double), ("ks_fri_curvature", ctypes.c_double),
        ("ks_c_n", ctypes.c_double), ("ks_c_s", ctypes.c_double), ("ks_lambda", ctypes.c_double),
        ("ks_lz_rescale", ctypes.c_double), ("ks_kappa_0", ctypes.c_double), ("ks_kappa_seed", ctypes.c_double),
        ("ks_kappa_trunc", ctypes.c_double), ("ks_tke_bg", ctypes.c_double), ("ks_tol_err", ctypes.c_double),
        ("ks_src_max_chg", ctypes.c_double), ("ks_prandtl_turb", ctypes.c_double),
        ("ks_vel_underflow", ctypes.c_double), ("eos_alpha_t", ctypes.c_double), ("eos_beta_s", ctypes.c_double),
        ("epbl", ctypes.c_int), ("epbl_mstar_scheme", ctypes.c_int), ("epbl_vstar_scheme", ctypes.c_int),
        ("epbl_combine", ctypes.c_int), ("epbl_mld_iteration", ctypes.c_int), ("epbl_mld_max_its", ctypes.c_int),
        ("epbl_mld_bisection", ctypes.c_int), ("epbl_mld_use_prev_guess", ctypes.c_int),
    ] + [(n, ctypes.c_double) for n in (
        "epbl_mstar_const", "epbl_mstar_cap", "epbl_mstar_coef1", "epbl_c_ek", "epbl_mstar_conv_adj", "epbl_nstar",
        "epbl_tke_decay", "epbl_wstar_ustar_coef", "epbl_vstar_scale_fac", "epbl_vstar_surf_fac", "epbl_von_karman",
        "epbl_ekman_scale_coef", "epbl_min_mix_len", "epbl_mixlen_exponent", "epbl_translay_scale", "epbl_mld_tol",
        "epbl_omega", "epbl_omega_frac", "epbl_ustar_min", "epbl_prandtl", "epbl_rh18_cn1", "epbl_rh18_cn2",
        "epbl_rh18_cn3", "epbl_rh18_cs1", "epbl_rh18_cs2")] + [
        ("epbl_use_lt", ctypes.c_int), ("epbl_lt_scheme", ctypes.c_int)] + [(n, ctypes.c_double) for n in (
            "epbl_lt_enhance_coef", "epbl_lt_enhance_exp", "epbl_lt_max_enhance", "epbl_la_frac_hbl",
            "epbl_lt_lac1", "epbl_lt_lac2", "epbl_lt_lac3", "epbl_lt_lac4", "epbl_lt_lac5")] + [
        ("epbl_tke_diags", ctypes.c_int), ("ks_massless_merge", ctypes.c_int),
        ("sw_source", ctypes.c_int), ("bound_salinity", ctypes.c_int), ("use_wet_dyn", ctypes.c_int),
        ("min_salinity", ctypes.c_double), ("epbl_sw_ctke", ctypes.c_int),
        ("sw_chl", ctypes.c_int), ("sw_nbands", ctypes.c_int), ("sw_blue_frac", ctypes.c_double),
        ("sw_opacity_coef", ctypes.c_double * (2 * SW_NB_MAX)), ("sw_chl_power", ctypes.c_double * SW_NB_MAX),
        ("sw_opacity_land", ctypes.c_double), ("use_cover_frac", ctypes.c_int),
        ("column_integrals", ctypes.c_int)]

    def as_dict(self):
        out = {}
        for n, _ in self._fields_:
            v = getattr(self, n)
            out[n] = list(v) if isinstance(v, ctypes.Array) else v   # the band-coefficient arrays by value
        return out


class LibraryNotFoundError(FileNotFoundError):
    """Raised when libvphys.so has not been built."""


PKG_DIR = Path(__file__).resolve().parent
BUILD_DIR = PKG_DIR / "csrc" / "_build"
LIB_NAME = "libvphys.so"


def find_library() -> Path:
    env = os.environ.get("VPHYS_LIB")
    if env:
        p = Path(env)
        if p.exists():
            return p
        raise LibraryNotFoundError(f"VPHYS_LIB={env} does not exist")
    p = BUILD_DIR / LIB_NAME
    if p.exists():
        return p
    raise LibraryNotFoundError(
        f"{p} not found: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
        "or `python -m roundabout_b200.build`")


class KppModel(ctypes.Structure):
    """Mirror of `struct vphys_kpp_model` (include/vphys.h)."""

    _fields_ = [("w1", ctypes.c_void_p), ("w2", ctypes.c_void_p), ("w3", ctypes.c_void_p),
                ("b1", ctypes.c_void_p), ("b2", ctypes.c_void_p), ("b3", ctypes.c_void_p),
                ("feat_mean", ctypes.c_void_p), ("feat_istd", ctypes.c_void_p),
                ("target_mean0", ctypes.c_float), ("target_std0", ctypes.c_float),
                ("gate_limit", ctypes.c_float), ("check_fraction", ctypes.c_float),
                ("check_tolerance", ctypes.c_float), ("fail_fraction", ctypes.c_float)]


_V = ctypes.c_void_p
_I = ctypes.c_int
_F = ctypes.c_float
_LL = ctypes.c_longlong

_PROTOTYPES = {
    "vphys_config_default": (ctypes.c_int, [ctypes.POINTER(VphysConfig)]),
    "vphys_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(VphysConfig), ctypes.POINTER(ctypes.c_void_p)]),
    "vphys_destroy": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p)]),
    "vphys_set_config": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(VphysConfig)]),
    "vphys_get_config": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(VphysConfig)]),
    "vphys_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "vphys_bind": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "vphys_set_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]),
    "vphys_set_field_async": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]),
    "vphys_get_field_async": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]),
    "vphys_get_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]),
    "vphys_get_ptr": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "vphys_eos_wright": (ctypes.c_int, [ctypes.c_void_p]),
    "vphys_stress_mag": (ctypes.c_int, [ctypes.c_void_p]),
    "vphys_surface_flux": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "vphys_sw_penetration": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "vphys_sw_chl_apply": (ctypes.c_int, [ctypes.c_void_p]),
    "vphys_kappa_shear": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "vphys_epbl": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "vphys_mixed_redo_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint)]),
    "vphys_assemble": (ctypes.c_int, [ctypes.c_void_p]),
    "vphys_vdiff_momentum": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "vphys_vdiff_tracers": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "vphys_nonlocal": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "vphys_vdiff_tracers_nonlocal": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "vphys_set_variants": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "vphys_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                      ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "vphys_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]),
    "vphys_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "vphys_last_error": (ctypes.c_int, [ctypes.c_int, ctypes.c_char_p, ctypes.c_int]),
    "vphys_version": (ctypes.c_char_p, []),
    "vphys_config_sizeof": (ctypes.c_size_t, []),
    "vphys_smooth_121_static": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "vphys_selftest_division": (ctypes.c_int, [ctypes.c_longlong, ctypes.c_ulonglong, ctypes.c_int, ctypes.c_int,
                                                ctypes.POINTER(ctypes.c_ulonglong)]),
    "vphys_step_graph": (_I, [_V, ctypes.c_double, _I]),
    "vphys_kpp_attach": (_I, [_V, ctypes.POINTER(KppModel)]),
    "vphys_kpp_stats": (_I, [_V, ctypes.POINTER(ctypes.c_ulonglong), _I]),
    "vphys_kpp_features": (_I, [_V, _V, _V, _F, _V, _V, _V, _LL, _V, _V]),
    "vphys_kpp_targets": (_I, [_V, _V]),
    "vphys_mlp_loss": (_I, [_V, _V, _V, _I, _I, _F, _V, _V, _V, _V, _V]),
    "vphys_mlp_colsum": (_I, [_V, _I, _I, _I, _V, _V]),
    "vphys_mlp_colstats": (_I, [_V, _LL, _I, _I, _V, _V, _V]),
    "vphys_mlp_standardize": (_I, [_V, _LL, _I, _I, _V, _V, _I, _V, _V, _LL, _V, _V]),
    "vphys_mlp_adam": (_I, [_V, _V, _V, _V, _I, _I, _F, _F, _F, _F, _I, _V, _V, _V]),
    "vphys_gemm_tn_bf16": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_longlong,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]),
    "vphys_mlp3_bf16": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
}

EXPORTED_SYMBOLS = tuple(_PROTOTYPES)

_lib = None


def get_lib():
    """Load libvphys.so once and declare every prototype."""
    global _lib
    if _lib is None:
        L = ctypes.CDLL(str(find_library()))
        for name, (res, args) in _PROTOTYPES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error(idx: int = 0) -> str:
    L = get_lib()
    buf = ctypes.create_string_buffer(1024)
    n = L.vphys_last_error(idx, buf, len(buf))
    return buf.value.decode(errors="replace") if n > 0 else ""


class VphysError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        super().__init__(f"{where} failed with status {status}: {last_error(0)}")


def check(status: int, where: str):
    if status != OK:
        raise VphysError(status, where)
    return status
