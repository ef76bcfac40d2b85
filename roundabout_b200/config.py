"""Configuration of the vertical-physics path.

`default_config()` returns a `VphysConfig` holding the reference defaults
(ocean_vmix_t, src/parameterizations/vertical/rdb_ocean_vmix.F90:198-483;
ocean_vdiff_t, rdb_ocean_vdiff.F90:78-260; namelist defaults
src/core/rdb_config.F90:1872-1893, 1936-1945) -- the same values
`vphys_config_default()` writes in C.

The closure classes mirror the vertical closures of python/rdb/closures.py
(PacanowskiPhilander, KPP, Langmuir, EPBL, KappaShear, ConvectiveAdjustment,
BryanLewisBackground, ConstantBackground, NearSurfaceViscosity,
HarmonicFaceThickness, ThermoSubcycling, ImplicitVerticalFriction,
DiffusivityLimits; TidalMixing, DoubleDiffusion and HenyeyBackground raise
when applied): the same names, keywords, defaults and knob targets, each
writing only its own knobs into the config through `apply(cfg)`.  Keywords
that exist only here are listed in each class and default to the reference's
behaviour.
"""
from __future__ import annotations

import sys

from ._ffi import INTERIOR_NONE, INTERIOR_PP81, VphysConfig

HUGE = sys.float_info.max


def default_config() -> VphysConfig:
    c = VphysConfig()
    c.use_closure = 1
    c.interior_closure = INTERIOR_PP81
    c.use_kpp = 0
    c.bkgnd_profile = 0
    c.vmix_guard = 0
    c.kd_smooth_iterations = 0
    c.conv_enable = 0
    c.surface_flux = 0
    c.buoyancy_coeffs = 0
    c.kpp_sw_method = 2
    c.sw_pen_frac = 0.0
    c.sw_band_ratio = 0.58
    c.sw_zeta1 = 0.35
    c.sw_zeta2 = 23.0
    c.pp81_nu0 = 1.0e-2
    c.pp81_nu_bg = 1.0e-4
    c.pp81_kappa_bg = 1.0e-5
    c.pp81_alpha = 5.0
    c.rho0 = 1035.0
    c.shear2_floor = 1.0e-10
    c.ri_crit = 0.3
    c.cs_nonlocal = 6.3
    c.c_vt2 = 1.8
    c.alpha_T = 1.7e-4
    c.beta_S = 7.6e-4
    c.cp = 3992.0
    c.kv_ml_invz2 = 0.0
    c.hmix_fixed = 20.0
    c.conv_kd = 1.0
    c.conv_prandtl = 1.0
    c.conv_n2_thresh = 0.0
    c.kv_bg = 1.0e-4
    c.kt_bg = 1.0e-5
    c.ks_bg = 1.0e-5
    c.kv_max = HUGE
    c.kd_max = HUGE
    c.bkgnd_kd_sfc = 1.0e-5
    c.bkgnd_kd_deep = 1.3e-4
    c.bkgnd_z0 = 2500.0
    c.bkgnd_delta = 222.0
    c.bkgnd_prandtl = -1.0
    c.eos_p_ref = 0.0
    c.hvel_mom6 = 1
    c.hvel_harmonic = 0
    c.hvel_upwind = 1
    c.use_harmonic = 0
    c.implicit_stress = 0
    c.implicit_drag = 0
    c.zlevel_faces = 0
    c.bbl_glue = 0
    c.hbbl_visc = 10.0
    c.bbl_piston = 3.0e-4
    c.kv_bbl_bg = 1.0e-4
    c.idx_temperature = 1
    c.idx_salinity = 0
    c.idx_pseudo_salt = -1
    c.eos_in_step = 0
    c.remnant = 0
    c.budgets = 0
    c.mixed_precision = 0
    c.learned_kpp = 0
    c.kappa_shear = 0
    c.ks_max_inner_it = 50
    c.ks_max_substep_it = 13
    c.eos_variant = 0
    c.ks_ri_crit = 0.25
    c.ks_shearmix_rate = 0.089
    c.ks_fri_curvature = -0.97
    c.ks_c_n = 0.24
    c.ks_c_s = 0.14
    c.ks_lambda = 0.82
    c.ks_lz_rescale = 1.0
    c.ks_kappa_0 = 1.0e-7
    c.ks_kappa_seed = 1.0
    c.ks_kappa_trunc = 1.0e-9
    c.ks_tke_bg = 0.0
    c.ks_tol_err = 0.1
    c.ks_src_max_chg = 10.0
    c.ks_prandtl_turb = 1.0
    c.ks_vel_underflow = 0.0
    c.eos_alpha_t = 0.0
    c.eos_beta_s = 0.0
    c.epbl = 0
    c.epbl_mstar_scheme = 2
    c.epbl_vstar_scheme = 1
    c.epbl_combine = 1
    c.epbl_mld_iteration = 1
    c.epbl_mld_max_its = 20
    c.epbl_mld_bisection = 0
    c.epbl_mld_use_prev_guess = 0
    c.epbl_mstar_const = 1.2
    c.epbl_mstar_cap = -1.0
    c.epbl_mstar_coef1 = 0.3
    c.epbl_c_ek = 0.085
    c.epbl_mstar_conv_adj = 0.0
    c.epbl_nstar = 0.2
    c.epbl_tke_decay = 2.5
    c.epbl_wstar_ustar_coef = 1.0
    c.epbl_vstar_scale_fac = 1.0
    c.epbl_vstar_surf_fac = 1.2
    c.epbl_von_karman = 0.41
    c.epbl_ekman_scale_coef = 1.0
    c.epbl_min_mix_len = 0.0
    c.epbl_mixlen_exponent = 2.0
    c.epbl_translay_scale = 0.1
    c.epbl_mld_tol = 1.0
    c.epbl_omega = 7.2921e-05
    c.epbl_omega_frac = 0.0
    c.epbl_ustar_min = 1e-08
    c.epbl_prandtl = 1.0
    c.epbl_rh18_cn1 = 0.275
    c.epbl_rh18_cn2 = 8.0
    c.epbl_rh18_cn3 = -5.0
    c.epbl_rh18_cs1 = 0.2
    c.epbl_rh18_cs2 = 0.4
    c.epbl_use_lt = 0
    c.epbl_lt_scheme = 1
    c.epbl_lt_enhance_coef = 0.447
    c.epbl_lt_enhance_exp = -1.33
    c.epbl_lt_max_enhance = 5.0
    c.epbl_la_frac_hbl = 0.04
    c.epbl_lt_lac1 = -0.87
    c.epbl_lt_lac2 = 0.0
    c.epbl_lt_lac3 = 0.0
    c.epbl_lt_lac4 = 0.95
    c.epbl_lt_lac5 = 0.95
    c.epbl_tke_diags = 0
    c.ks_massless_merge = 0
    c.sw_source = 0
    c.bound_salinity = 0
    c.use_wet_dyn = 0
    c.min_salinity = 0.0
    c.epbl_sw_ctke = 1
    c.sw_chl = 0
    c.sw_nbands = 3
    c.sw_blue_frac = 0.5
    for n, v in enumerate((0.0232, 0.074, 0.225, 0.037, 2.86, 0.0)):
        c.sw_opacity_coef[n] = v
    c.sw_chl_power[0] = 0.674
    c.sw_chl_power[1] = 0.629
    c.sw_opacity_land = 10.0
    c.use_cover_frac = 0
    c.column_integrals = 0
    return c


def hot_path_config(ntracers: int = 4, pseudo_salt_index: int | None = 3) -> VphysConfig:
    """The benchmark configuration: PP81 + KPP + Bryan-Lewis, Wright EOS in
    the step, dimensional alpha_T = 0.2 / beta_S = 0.77 (the kpp_basin example,
    validation_examples/ocean/epbl_mld/kpp_basin.nml), tracers S, T, then
    passives (ideal age, pseudo-salt)."""
    c = default_config()
    c.use_kpp = 1
    c.bkgnd_profile = 1
    c.alpha_T = 0.2
    c.beta_S = 0.77
    c.eos_in_step = 1
    c.idx_salinity = 0
    c.idx_temperature = 1
    c.idx_pseudo_salt = pseudo_salt_index if (pseudo_salt_index is not None and pseudo_salt_index < ntracers) else -1
    return c


def seed_backgrounds(cfg: VphysConfig):
    """vmix_seed_backgrounds (rdb_ocean_vmix.F90:843-913): kv_bg/kt_bg/ks_bg
    follow pp81_nu_bg / pp81_kappa_bg."""
    cfg.kv_bg = cfg.pp81_nu_bg
    cfg.kt_bg = cfg.pp81_kappa_bg
    cfg.ks_bg = cfg.pp81_kappa_bg
    return cfg


# ---------------------------------------------------------------------------
# Closure objects (python/rdb/closures.py:20-413)
# ---------------------------------------------------------------------------
class PacanowskiPhilander:
    """PP81 interior closure (python/rdb/closures.py:20-47):
    `PacanowskiPhilander(nu0=1e-2, nu_bg=1e-3, kappa_bg=1e-4, alpha=5.0,
    shear2_floor=1e-9, enabled=True)`.  `enabled=False` turns the whole
    closure off (`use_closure = .false.`), which selects the reference's
    scalar-K vdiff path; this library refuses that configuration with
    VPHYS_ERR_CONFIG when the handle is created or reconfigured."""

    def __init__(self, nu0=1e-2, nu_bg=1e-3, kappa_bg=1e-4, alpha=5.0, shear2_floor=1e-9, enabled=True):
        self.nu0, self.nu_bg, self.kappa_bg = nu0, nu_bg, kappa_bg
        self.alpha, self.shear2_floor = alpha, shear2_floor
        self.enabled = bool(enabled)

    def apply(self, cfg):
        cfg.use_closure = int(self.enabled)
        if not self.enabled:
            return cfg
        cfg.interior_closure = INTERIOR_PP81
        cfg.pp81_nu0 = float(self.nu0)
        cfg.pp81_nu_bg = float(self.nu_bg)
        cfg.pp81_kappa_bg = float(self.kappa_bg)
        cfg.pp81_alpha = float(self.alpha)
        cfg.shear2_floor = float(self.shear2_floor)
        return seed_backgrounds(cfg)


class KPP:
    """KPP boundary-layer overlay (python/rdb/closures.py:50-85):
    `KPP(ri_crit=0.3, cs_nonlocal=6.3, c_vt2=1.8, shortwave_method="mxl_sw",
    enabled=True)`; `shortwave_method` is the reference's kpp_sw_method
    string ("all_sw", "mxl_sw", "lv1_sw": parse_kpp_sw_method,
    rdb_ocean_vmix.F90:1561-1577).  Extra keywords of this library, left
    unset by default: `alpha_T`, `beta_S` (the constant buoyancy
    coefficients of KPP's B0)."""

    _SW = {"all_sw": 1, "mxl_sw": 2, "lv1_sw": 3}

    def __init__(self, ri_crit=0.3, cs_nonlocal=6.3, c_vt2=1.8, shortwave_method="mxl_sw", enabled=True,
                 alpha_T=None, beta_S=None):
        if shortwave_method not in self._SW:
            raise ValueError(f"KPP: shortwave_method must be one of {sorted(self._SW)}")
        self.ri_crit, self.cs_nonlocal, self.c_vt2 = ri_crit, cs_nonlocal, c_vt2
        self.shortwave_method = shortwave_method
        self.alpha_T, self.beta_S = alpha_T, beta_S
        self.enabled = bool(enabled)

    def apply(self, cfg):
        cfg.use_kpp = int(self.enabled)
        if not self.enabled:
            return cfg
        cfg.ri_crit = float(self.ri_crit)
        cfg.cs_nonlocal = float(self.cs_nonlocal)
        cfg.c_vt2 = float(self.c_vt2)
        cfg.kpp_sw_method = self._SW[self.shortwave_method]
        if self.alpha_T is not None:
            cfg.alpha_T = float(self.alpha_T)
        if self.beta_S is not None:
            cfg.beta_S = float(self.beta_S)
        return cfg


class BryanLewisBackground:
    """Depth-varying background Kd (python/rdb/closures.py:237-260):
    `BryanLewisBackground(kd_surface=1e-5, kd_deep=1.3e-4, z0=2500.0,
    delta=222.0, prandtl=1.0)`."""

    def __init__(self, kd_surface=1e-5, kd_deep=1.3e-4, z0=2500.0, delta=222.0, prandtl=1.0):
        self.kd_surface, self.kd_deep, self.z0, self.delta, self.prandtl = kd_surface, kd_deep, z0, delta, prandtl

    def apply(self, cfg):
        cfg.bkgnd_profile = 1
        cfg.bkgnd_kd_sfc = float(self.kd_surface)
        cfg.bkgnd_kd_deep = float(self.kd_deep)
        cfg.bkgnd_z0 = float(self.z0)
        cfg.bkgnd_delta = float(self.delta)
        cfg.bkgnd_prandtl = float(self.prandtl)
        return cfg


class ConstantBackground:
    """The scalar background floor (python/rdb/closures.py:284-295):
    `ConstantBackground(kv=1e-3, kt=1e-4)` writes pp81_nu_bg /
    pp81_kappa_bg, from which the vmix initialisation seeds the kv/kt/ks
    floors (vmix_seed_backgrounds, rdb_ocean_vmix.F90:843-913)."""

    def __init__(self, kv=1e-3, kt=1e-4):
        self.kv, self.kt = kv, kt

    def apply(self, cfg):
        cfg.pp81_nu_bg = float(self.kv)
        cfg.pp81_kappa_bg = float(self.kt)
        return seed_backgrounds(cfg)


class NearSurfaceViscosity:
    """KV_ML_INVZ2 surface band (python/rdb/closures.py:298-319):
    `NearSurfaceViscosity(kv=0.0, hmix=20.0)`."""

    def __init__(self, kv=0.0, hmix=20.0):
        self.kv, self.hmix = kv, hmix

    def apply(self, cfg):
        cfg.kv_ml_invz2 = float(self.kv)
        cfg.hmix_fixed = float(self.hmix)
        return cfg


class ConvectiveAdjustment:
    """(python/rdb/closures.py:200-213) `ConvectiveAdjustment(kd=1.0,
    prandtl=1.0, n2_threshold=0.0)`."""

    def __init__(self, kd=1.0, prandtl=1.0, n2_threshold=0.0):
        self.kd, self.prandtl, self.n2_threshold = kd, prandtl, n2_threshold

    def apply(self, cfg):
        cfg.conv_enable = 1
        cfg.conv_kd = float(self.kd)
        cfg.conv_prandtl = float(self.prandtl)
        cfg.conv_n2_thresh = float(self.n2_threshold)
        return cfg


class ShortwavePenetration:
    """Two-band shortwave penetration (python/rdb/forcing.py:93-115:
    `ShortwavePenetration(fraction=0.0, band_ratio=0.58, zeta1=0.35,
    zeta2=23.0, source="net_heat", epbl_tke_ledger=True)`).  `source="q_sw"`
    reads the SW_NET field (q_sw + sw_ice) as the irradiance of the
    penetration, KPP's B0 charge and EPBL's ledger; any other source is
    refused, as sw_source_is_implemented does
    (rdb_ocean_surface_flux.F90:814-822).  All inert at fraction=0."""

    _SOURCE = {"net_heat": 0, "q_sw": 1}

    def __init__(self, fraction=0.0, band_ratio=0.58, zeta1=0.35, zeta2=23.0, source="net_heat",
                 epbl_tke_ledger=True):
        if source not in self._SOURCE:
            raise ValueError(f"ShortwavePenetration: source must be one of {sorted(self._SOURCE)}")
        self.fraction, self.band_ratio, self.zeta1, self.zeta2 = fraction, band_ratio, zeta1, zeta2
        self.source, self.epbl_tke_ledger = source, epbl_tke_ledger

    def apply(self, cfg):
        cfg.sw_pen_frac = float(self.fraction)
        cfg.sw_band_ratio = float(self.band_ratio)
        cfg.sw_zeta1 = float(self.zeta1)
        cfg.sw_zeta2 = float(self.zeta2)
        cfg.sw_source = self._SOURCE[self.source]
        cfg.epbl_sw_ctke = 1 if self.epbl_tke_ledger else 0
        return cfg


class Langmuir:
    """Langmuir enhancement of EPBL's mstar (python/rdb/closures.py:88-105:
    `Langmuir(scheme="rescale", coef=0.447, exponent=-1.33, max_enhance=5.0,
    sl_fraction=0.04)`), passed as `EPBL(langmuir=...)`."""

    _SCHEME = {"rescale": 1, "additive": 2}

    def __init__(self, scheme="rescale", coef=0.447, exponent=-1.33, max_enhance=5.0, sl_fraction=0.04):
        if scheme not in self._SCHEME:
            raise ValueError(f"Langmuir: scheme must be one of {sorted(self._SCHEME)}")
        self.scheme, self.coef, self.exponent = scheme, coef, exponent
        self.max_enhance, self.sl_fraction = max_enhance, sl_fraction

    def _apply(self, cfg):
        cfg.epbl_use_lt = 1
        cfg.epbl_lt_scheme = self._SCHEME[self.scheme]
        cfg.epbl_lt_enhance_coef = float(self.coef)
        cfg.epbl_lt_enhance_exp = float(self.exponent)
        cfg.epbl_lt_max_enhance = float(self.max_enhance)
        cfg.epbl_la_frac_hbl = float(self.sl_fraction)
        return cfg


class EPBL:
    """Reichl-Hallberg energetics PBL, column form (python/rdb/closures.py:107-150:
    `EPBL(mstar_scheme="om4", mstar=1.2, nstar=0.2, prandtl=1.0, combine="add",
    mld_iteration=True, mld_use_prev_guess=False, langmuir=None)`).  Like the
    reference it switches KPP off; `langmuir` is a `Langmuir`."""

    _MSTAR = {"constant": 1, "om4": 2, "rh18": 3}
    _COMBINE = {"add": 1, "max": 2, "max_shear": 3}

    def __init__(self, mstar_scheme="om4", mstar=1.2, nstar=0.2, prandtl=1.0, combine="add", mld_iteration=True,
                 mld_use_prev_guess=False, langmuir=None):
        if mstar_scheme not in self._MSTAR:
            raise ValueError(f"EPBL: mstar_scheme must be one of {sorted(self._MSTAR)}")
        if combine not in self._COMBINE:
            raise ValueError(f"EPBL: combine must be one of {sorted(self._COMBINE)}")
        if langmuir is not None and not isinstance(langmuir, Langmuir):
            raise TypeError("EPBL: langmuir must be a Langmuir")
        self.langmuir = langmuir
        self.mstar_scheme, self.mstar, self.nstar = mstar_scheme, mstar, nstar
        self.prandtl, self.combine = prandtl, combine
        self.mld_iteration, self.mld_use_prev_guess = mld_iteration, mld_use_prev_guess

    def apply(self, cfg):
        cfg.epbl = 1
        cfg.use_kpp = 0
        cfg.epbl_mstar_scheme = self._MSTAR[self.mstar_scheme]
        cfg.epbl_mstar_const = float(self.mstar)
        cfg.epbl_nstar = float(self.nstar)
        cfg.epbl_prandtl = float(self.prandtl)
        cfg.epbl_combine = self._COMBINE[self.combine]
        cfg.epbl_mld_iteration = int(bool(self.mld_iteration))
        cfg.epbl_mld_use_prev_guess = int(bool(self.mld_use_prev_guess))
        if self.langmuir is not None:
            self.langmuir._apply(cfg)
        return cfg


class KappaShear:
    """JHL08 prognostic interior shear turbulence, column form
    (python/rdb/closures.py:152-180: `KappaShear(ri_crit=0.25, prandtl=1.0,
    at_vertex=False, ...)`).  The vertex (corner) form is not built here:
    `at_vertex=True` raises.  The iteration-control knobs are the `ks_*`
    fields of the config."""

    def __init__(self, ri_crit=0.25, prandtl=1.0, at_vertex=False, vertex_geometric_mean=False, vertex_kdmin=0.0):
        if at_vertex or vertex_geometric_mean:
            raise NotImplementedError("KappaShear: the vertex (corner) form is not built; use the column form")
        self.ri_crit, self.prandtl = ri_crit, prandtl

    def apply(self, cfg):
        cfg.kappa_shear = 1
        cfg.ks_ri_crit = float(self.ri_crit)
        cfg.ks_prandtl_turb = float(self.prandtl)
        return cfg


class HarmonicFaceThickness:
    """MOM6 HARMONIC_VISC (python/rdb/closures.py:322-336):
    `HarmonicFaceThickness()` sets the namelist's harmonic_visc, which the
    vdiff set-up copies into `use_harmonic`
    (rdb_ocean_setup_vmix.F90:378-379): harmonic-mean face thickness in the
    vertical-friction and diffusion matrices."""

    def apply(self, cfg):
        cfg.use_harmonic = 1
        return cfg


class ThermoSubcycling:
    """(python/rdb/closures.py:339-352) `ThermoSubcycling(ratio=1)`: the
    thermo step runs every `ratio` dynamics steps.  vphys_step IS the
    thermo step of this path, so the caller calls it every `ratio` steps;
    the object only checks the ratio."""

    def __init__(self, ratio=1):
        if int(ratio) < 1:
            raise ValueError("ThermoSubcycling: ratio must be >= 1")
        self.ratio = int(ratio)

    def apply(self, cfg):
        return cfg


class ImplicitVerticalFriction:
    """Implicit vertical friction (python/rdb/closures.py:355-392):
    `ImplicitVerticalFriction(stress=False, drag=False,
    harmonic_thickness=True, harmonic_visc=False, bbl_glue=True, hbbl=10.0,
    bbl_piston=3e-4)`.  `harmonic_thickness` -> hvel_mom6 (MOM6's momentum
    face thickness), `harmonic_visc` -> hvel_harmonic (which branch of it),
    `bbl_glue` -> the BBL glue.  As in the reference's vdiff set-up, the
    glue latches off unless a bottom drag is configured
    (rdb_ocean_setup_vmix.F90:385-393, "No drag configured => the latch
    leaves the glue OFF"); `bottom_drag=True` (an extra keyword of this
    library, for a caller whose bottom-drag configuration is set) keeps it.
    `upwind` (extra, default True as in the namelist) is hvel_upwind."""

    def __init__(self, stress=False, drag=False, harmonic_thickness=True, harmonic_visc=False, bbl_glue=True,
                 hbbl=10.0, bbl_piston=3e-4, bottom_drag=False, upwind=True):
        self.stress, self.drag = stress, drag
        self.harmonic_thickness, self.bbl_glue = harmonic_thickness, bbl_glue
        self.harmonic_visc = harmonic_visc
        self.hbbl, self.bbl_piston = hbbl, bbl_piston
        self.bottom_drag, self.upwind = bottom_drag, upwind

    def apply(self, cfg):
        cfg.implicit_stress = int(bool(self.stress))
        cfg.implicit_drag = int(bool(self.drag))
        cfg.hvel_mom6 = int(bool(self.harmonic_thickness))
        cfg.hvel_harmonic = int(bool(self.harmonic_visc))
        cfg.bbl_glue = int(bool(self.bbl_glue) and bool(self.bottom_drag))
        cfg.hbbl_visc = float(self.hbbl)
        cfg.bbl_piston = float(self.bbl_piston)
        cfg.hvel_upwind = int(bool(self.upwind))
        return cfg


class DiffusivityLimits:
    """The floors/ceilings/smoothing gate (python/rdb/closures.py:395-405):
    `DiffusivityLimits(kv_max=1e6, kd_max=1e6, smoothing=0)`; `guard` (an
    extra keyword of this library, default off) is vmix_guard."""

    def __init__(self, kv_max=1e6, kd_max=1e6, smoothing=0, guard=False):
        self.kv_max, self.kd_max, self.smoothing, self.guard = kv_max, kd_max, smoothing, guard

    def apply(self, cfg):
        cfg.kv_max = float(self.kv_max)
        cfg.kd_max = float(self.kd_max)
        cfg.kd_smooth_iterations = int(self.smoothing)
        cfg.vmix_guard = int(bool(self.guard))
        return cfg


class _NotOnThisPath:
    """A reference closure whose contribution this library does not build;
    applying it raises, so a reference script fails loudly instead of
    running without it."""

    what = ""

    def __init__(self, *args, **kwargs):
        self.args, self.kwargs = args, kwargs

    def apply(self, cfg):
        raise NotImplementedError(f"{type(self).__name__}: {self.what} is not built in this library")


class TidalMixing(_NotOnThisPath):
    """(python/rdb/closures.py:183-197) St-Laurent/Simmons tidal mixing."""

    what = "the tidal-mixing contributor"


class DoubleDiffusion(_NotOnThisPath):
    """(python/rdb/closures.py:216-234) salt fingering and diffusive convection."""

    what = "the double-diffusion split of kt/ks"


class HenyeyBackground(_NotOnThisPath):
    """(python/rdb/closures.py:263-281) the latitude-scaled background."""

    what = "the Henyey background"


def compose(*closures, base: VphysConfig | None = None) -> VphysConfig:
    cfg = base if base is not None else default_config()
    for c in closures:
        c.apply(cfg)
    return cfg
