"""The C ABI without a GPU: libvphys.so loads, exports every entry point that
include/vphys.h declares, agrees with the Python mirror of its config struct
and its defaults, and fails cleanly (status + error-ring message, no abort)
where a device would be needed."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def lib():
    from roundabout_b200 import build as b

    b.build()
    from roundabout_b200 import _ffi

    return _ffi.get_lib()


def declared_symbols():
    text = (ROOT / "include" / "vphys.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|size_t|const char \*)\s*(vphys_\w+)\s*\(", text, re.M)))


def test_every_declared_symbol_is_exported(lib):
    from roundabout_b200 import _ffi

    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), f"{s} declared in include/vphys.h but not exported"
        assert s in _ffi.EXPORTED_SYMBOLS, f"{s} has no ctypes prototype in _ffi.py"


def test_config_struct_layout_and_defaults(lib):
    from roundabout_b200 import _ffi
    from roundabout_b200.config import default_config

    assert lib.vphys_config_sizeof() == ctypes.sizeof(_ffi.VphysConfig)
    c = _ffi.VphysConfig()
    assert lib.vphys_config_default(ctypes.byref(c)) == _ffi.OK
    py = default_config()
    assert c.as_dict() == py.as_dict()


def test_errors_are_reported_not_raised(lib):
    from roundabout_b200 import _ffi

    h = ctypes.c_void_p()
    st = lib.vphys_create(4, 4, 200, 2, None, ctypes.byref(h))
    assert st == _ffi.ERR_TOO_DEEP and h.value is None
    assert "VPHYS_NZ_MAX" in _ffi.last_error(0)
    bad = _ffi.VphysConfig()
    lib.vphys_config_default(ctypes.byref(bad))
    bad.use_closure = 0
    assert lib.vphys_create(4, 4, 4, 2, ctypes.byref(bad), ctypes.byref(h)) == _ffi.ERR_CONFIG
    assert "scalar" in _ffi.last_error(0)
    assert lib.vphys_step(None, 1.0, 1) == _ffi.ERR_BAD_HANDLE
    nothing = ctypes.c_void_p()
    assert lib.vphys_destroy(ctypes.byref(nothing)) == _ffi.OK
    buf = ctypes.create_string_buffer(4)
    n = lib.vphys_last_error(0, buf, 4)
    assert n > 3 and len(buf.value) == 3          # snprintf-style truncation
    assert lib.vphys_last_error(10_000, buf, 4) == 0


def test_create_without_a_device_fails_cleanly(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from roundabout_b200 import _ffi

    h = ctypes.c_void_p()
    st = lib.vphys_create(8, 8, 4, 2, None, ctypes.byref(h))
    assert st in (_ffi.ERR_ALLOC, _ffi.ERR_CUDA) and h.value is None
    assert _ffi.last_error(0)


def test_python_driver_raises_without_a_device(lib):
    """The Python driver has no CPU fallback: without a device it raises a
    typed error carrying the library's message."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from roundabout_b200 import _ffi
    from roundabout_b200.column import VerticalPhysics

    with pytest.raises(_ffi.VphysError) as err:
        VerticalPhysics(8, 8, 4, 2)
    assert err.value.status in (_ffi.ERR_ALLOC, _ffi.ERR_CUDA)
    assert "vphys_create" in str(err.value)


def test_kappa_shear_knobs_are_validated(lib):
    """The kappa-shear knobs are checked at create, before any device work."""
    from roundabout_b200 import _ffi
    from roundabout_b200.config import KappaShear, default_config

    h = ctypes.c_void_p()
    for name, value in (("ks_max_inner_it", 0), ("ks_max_substep_it", -1), ("eos_variant", 2), ("ks_lambda", 0.0),
                        ("kappa_shear", 2), ("ks_massless_merge", 2), ("sw_source", 2), ("bound_salinity", -1),
                        ("use_wet_dyn", 3), ("epbl_sw_ctke", 2), ("sw_chl", 2),
                        ("use_cover_frac", 2)):
        bad = default_config()
        setattr(bad, name, value)
        assert lib.vphys_create(4, 4, 4, 2, ctypes.byref(bad), ctypes.byref(h)) == _ffi.ERR_CONFIG, name
        assert h.value is None
    cfg = KappaShear(ri_crit=0.3, prandtl=0.8).apply(default_config())
    assert cfg.kappa_shear == 1 and cfg.ks_ri_crit == 0.3 and cfg.ks_prandtl_turb == 0.8
    with pytest.raises(NotImplementedError):
        KappaShear(at_vertex=True)


def test_epbl_knobs_are_validated(lib):
    """EPBL's unbuilt options are refused at create (no device work)."""
    from roundabout_b200 import _ffi
    from roundabout_b200.config import EPBL, Langmuir, default_config

    h = ctypes.c_void_p()
    for over in (dict(epbl_mstar_scheme=4), dict(learned_kpp=1), dict(epbl_combine=4), dict(epbl_mld_max_its=0),
                 dict(epbl_ustar_min=0.0)):
        bad = default_config()
        bad.epbl = 1
        for k, v in over.items():
            setattr(bad, k, v)
        assert lib.vphys_create(4, 4, 4, 2, ctypes.byref(bad), ctypes.byref(h)) == _ffi.ERR_CONFIG, over
        assert h.value is None
    cfg = EPBL(mstar_scheme="om4", combine="max_shear", mld_use_prev_guess=True).apply(default_config())
    assert (cfg.epbl, cfg.use_kpp, cfg.epbl_mstar_scheme, cfg.epbl_combine, cfg.epbl_mld_use_prev_guess) == (1, 0, 2, 3, 1)
    assert EPBL(mstar_scheme="rh18").apply(default_config()).epbl_mstar_scheme == 3
    with pytest.raises(ValueError):
        EPBL(mstar_scheme="rh19")
    with pytest.raises(TypeError):
        EPBL(langmuir=object())
    lt = EPBL(langmuir=Langmuir(scheme="additive", coef=0.3)).apply(default_config())
    assert (lt.epbl_use_lt, lt.epbl_lt_scheme, lt.epbl_lt_enhance_coef) == (1, 2, 0.3)


def test_every_named_field_has_a_shape():
    """Each field the python mirror names maps to a Fortran-order shape."""
    from roundabout_b200 import _ffi

    for name, fid in _ffi.FIELD_NAMES.items():
        shp = _ffi.field_shape(fid, 5, 4, 3)
        assert len(shp) in (2, 3) and all(n > 0 for n in shp), name


def test_chlorophyll_knobs_are_validated(lib):
    """The chlorophyll scheme needs sw_pen_frac = 1 (or 0, which selects 1),
    3..6 bands and a positive clear-water opacity per band
    (rdb_config_validate.F90:291-310)."""
    from roundabout_b200 import _ffi
    from roundabout_b200.config import default_config

    h = ctypes.c_void_p()
    for over in (dict(sw_pen_frac=0.5), dict(sw_pen_frac=1.0, sw_nbands=2), dict(sw_pen_frac=1.0, sw_nbands=7),
                 dict(sw_pen_frac=1.0, sw_nbands=4)):
        bad = default_config()
        bad.sw_chl = 1
        for k, v in over.items():
            setattr(bad, k, v)
        assert lib.vphys_create(4, 4, 4, 2, ctypes.byref(bad), ctypes.byref(h)) == _ffi.ERR_CONFIG, over
        assert h.value is None


@pytest.mark.gpu
def test_chlorophyll_unset_fraction_selects_one(lib):
    """sw_chl = 1 with sw_pen_frac left at 0 ("unset") is accepted and stored
    as 1, as the reference's set_sw_chl does (rdb_ocean_sw_chl.F90:87-103)."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from roundabout_b200 import _ffi
    from roundabout_b200.config import default_config

    cfg = default_config()
    cfg.sw_chl = 1
    cfg.sw_pen_frac = 0.0
    h = ctypes.c_void_p()
    assert lib.vphys_create(4, 4, 4, 2, ctypes.byref(cfg), ctypes.byref(h)) == _ffi.OK
    got = _ffi.VphysConfig()
    assert lib.vphys_get_config(h, ctypes.byref(got)) == _ffi.OK
    assert got.sw_pen_frac == 1.0 and got.sw_chl == 1
    cfg.sw_pen_frac = 0.0
    assert lib.vphys_set_config(h, ctypes.byref(cfg)) == _ffi.OK
    assert lib.vphys_get_config(h, ctypes.byref(got)) == _ffi.OK
    assert got.sw_pen_frac == 1.0
    assert lib.vphys_destroy(ctypes.byref(h)) == _ffi.OK
