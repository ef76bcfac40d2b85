"""The Python closure objects mirror python/rdb/closures.py of the reference.

tests/golden/closures_table.json (made by tests/golden/make_closures_table.py
from the reference's source, parsed and never executed) lists, for every
class, the keyword defaults and the knob each keyword writes.  For every
vertical closure of that table this checks roundabout_b200.config's class of
the same name: the same keywords with the same defaults, and each keyword
landing -- at its default and at another value -- in the knob of this
library's vphys_config that stands for the reference's knob.  The
reference's three contributors this library does not build raise when
applied.
"""
import inspect
import json
from pathlib import Path

import pytest

from roundabout_b200 import config as C

TABLE = json.loads((Path(__file__).resolve().parent / "golden" / "closures_table.json").read_text())

# reference knob -> (vphys_config field, transform of the keyword's value)
_SW = {"all_sw": 1, "mxl_sw": 2, "lv1_sw": 3}
_MSTAR = {"constant": 1, "om4": 2, "rh18": 3}
_COMBINE = {"add": 1, "max": 2, "max_shear": 3}
_LT = {"rescale": 1, "additive": 2}
KNOB = {
    "ocean_vmix.use_closure": ("use_closure", int), "ocean_vmix.pp81_nu0": ("pp81_nu0", float),
    "ocean_vmix.pp81_nu_bg": ("pp81_nu_bg", float), "ocean_vmix.pp81_kappa_bg": ("pp81_kappa_bg", float),
    "ocean_vmix.pp81_alpha": ("pp81_alpha", float), "ocean_vmix.shear2_floor": ("shear2_floor", float),
    "ocean_vmix.use_kpp": ("use_kpp", int), "ocean_vmix.kpp_ri_crit": ("ri_crit", float),
    "ocean_vmix.kpp_cs_nonlocal": ("cs_nonlocal", float), "ocean_vmix.kpp_c_vt2": ("c_vt2", float),
    "ocean_thermo.kpp_sw_method": ("kpp_sw_method", _SW.__getitem__),
    "ocean_epbl.enable": ("epbl", int), "ocean_epbl.mstar_scheme": ("epbl_mstar_scheme", _MSTAR.__getitem__),
    "ocean_epbl.mstar": ("epbl_mstar_const", float), "ocean_epbl.nstar": ("epbl_nstar", float),
    "ocean_epbl.prandtl": ("epbl_prandtl", float), "ocean_epbl.combine": ("epbl_combine", _COMBINE.__getitem__),
    "ocean_epbl.mld_iteration": ("epbl_mld_iteration", int),
    "ocean_epbl.mld_use_prev_guess": ("epbl_mld_use_prev_guess", int),
    "ocean_epbl.use_lt": ("epbl_use_lt", int), "ocean_epbl.lt_scheme": ("epbl_lt_scheme", _LT.__getitem__),
    "ocean_epbl.lt_enhance_coef": ("epbl_lt_enhance_coef", float),
    "ocean_epbl.lt_enhance_exp": ("epbl_lt_enhance_exp", float),
    "ocean_epbl.lt_max_enhance": ("epbl_lt_max_enhance", float),
    "ocean_epbl.la_frac_hbl": ("epbl_la_frac_hbl", float),
    "ocean_kappa_shear.enable": ("kappa_shear", int), "ocean_kappa_shear.ri_crit": ("ks_ri_crit", float),
    "ocean_kappa_shear.prandtl_turb": ("ks_prandtl_turb", float),
    "ocean_conv.enable": ("conv_enable", int), "ocean_conv.kd_conv": ("conv_kd", float),
    "ocean_conv.prandtl_conv": ("conv_prandtl", float), "ocean_conv.n2_thresh": ("conv_n2_thresh", float),
    "ocean_vmix.bkgnd_profile": ("bkgnd_profile", int), "ocean_vmix.bkgnd_kd_sfc": ("bkgnd_kd_sfc", float),
    "ocean_vmix.bkgnd_kd_deep": ("bkgnd_kd_deep", float), "ocean_vmix.bkgnd_z0": ("bkgnd_z0", float),
    "ocean_vmix.bkgnd_delta": ("bkgnd_delta", float), "ocean_vmix.bkgnd_prandtl": ("bkgnd_prandtl", float),
    "ocean_vmix.kv_ml_invz2": ("kv_ml_invz2", float), "ocean_vmix.hmix_fixed": ("hmix_fixed", float),
    "ocean_vmix.harmonic_visc": ("use_harmonic", int),
    "ocean_vdiff.implicit_stress": ("implicit_stress", int), "ocean_vdiff.implicit_drag": ("implicit_drag", int),
    "ocean_vdiff.hvel_mom6": ("hvel_mom6", int), "ocean_vdiff.hvel_harmonic": ("hvel_harmonic", int),
    "ocean_vdiff.bbl_glue": ("bbl_glue", int), "ocean_vdiff.hbbl_visc": ("hbbl_visc", float),
    "ocean_vdiff.bbl_piston": ("bbl_piston", float),
    "ocean_vmix.kv_max": ("kv_max", float), "ocean_vmix.kd_max": ("kd_max", float),
    "ocean_vmix.kd_smooth_iterations": ("kd_smooth_iterations", int),
}
MIRRORED = ["PacanowskiPhilander", "KPP", "Langmuir", "EPBL", "KappaShear", "ConvectiveAdjustment",
            "BryanLewisBackground", "ConstantBackground", "NearSurfaceViscosity", "HarmonicFaceThickness",
            "ThermoSubcycling", "ImplicitVerticalFriction", "DiffusivityLimits"]
NOT_BUILT = ["TidalMixing", "DoubleDiffusion", "HenyeyBackground"]
# keywords of the reference that select a form this library does not build (they raise)
UNBUILT_KW = {"KappaShear": {"at_vertex", "vertex_geometric_mean", "vertex_kdmin"}, "ThermoSubcycling": {"ratio"}}
# keywords that only take effect together with one of this library's extra keywords
EXTRA_FOR = {("ImplicitVerticalFriction", "bbl_glue"): {"bottom_drag": True}}
OTHER = {"mxl_sw": "lv1_sw", "om4": "rh18", "add": "max_shear", "rescale": "additive"}


def _other(v):
    if isinstance(v, bool):
        return not v
    if isinstance(v, str):
        return OTHER[v]
    if isinstance(v, int):
        return v + 2
    return v * 3.0 + 0.25


def _applied(cls_name, **kw):
    obj = getattr(C, cls_name)(**kw)
    cfg = C.default_config()
    if cls_name == "Langmuir":
        obj._apply(cfg)
    else:
        obj.apply(cfg)
    return cfg


@pytest.mark.parametrize("name", MIRRORED)
def test_same_keywords_and_defaults(name):
    ref = TABLE[name]["defaults"]
    sig = inspect.signature(getattr(C, name).__init__).parameters
    for kw, dflt in ref.items():
        assert kw in sig, f"{name}: keyword {kw} missing"
        assert sig[kw].default == dflt, f"{name}.{kw}: default {sig[kw].default!r}, reference {dflt!r}"


@pytest.mark.parametrize("name", MIRRORED)
def test_each_keyword_writes_the_same_knob(name):
    entry = TABLE[name]
    skip = UNBUILT_KW.get(name, set())
    for knob, src in entry["assigns"]:
        if "kw" in src and src["kw"] in skip:
            continue
        field, conv = KNOB[knob]
        if "const" in src:
            assert getattr(_applied(name), field) == conv(src["const"]), (name, knob)
            continue
        kw = src["kw"]
        extra = EXTRA_FOR.get((name, kw), {})
        base = entry["defaults"][kw]
        got = getattr(_applied(name, **extra), field)
        assert got == conv(base), f"{name}({kw}={base!r}) -> {field} = {got!r}"
        if kw == "enabled":
            continue   # enabled=False turns the object's other knobs off
        new = _other(base)
        got = getattr(_applied(name, **{kw: new}, **extra), field)
        assert got == conv(new), f"{name}({kw}={new!r}) -> {field} = {got!r}"


def test_switches_off():
    assert _applied("PacanowskiPhilander", enabled=False).use_closure == 0
    assert _applied("KPP", enabled=False).use_kpp == 0
    assert _applied("EPBL").use_kpp == 0


def test_glue_latches_off_without_a_bottom_drag():
    """The reference's vdiff set-up leaves the glue off when no bottom drag
    is configured (rdb_ocean_setup_vmix.F90:385-393)."""
    assert _applied("ImplicitVerticalFriction").bbl_glue == 0
    assert _applied("ImplicitVerticalFriction", bottom_drag=True).bbl_glue == 1


def test_backgrounds_seed_the_floors():
    cfg = _applied("ConstantBackground", kv=2e-3, kt=3e-4)
    assert (cfg.kv_bg, cfg.kt_bg, cfg.ks_bg) == (2e-3, 3e-4, 3e-4)


@pytest.mark.parametrize("name", NOT_BUILT)
def test_unbuilt_contributors_raise(name):
    assert name in TABLE
    with pytest.raises(NotImplementedError):
        getattr(C, name)().apply(C.default_config())


def test_vertex_shear_raises():
    with pytest.raises(NotImplementedError):
        C.KappaShear(at_vertex=True)
