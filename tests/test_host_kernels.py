"""The CUDA source of the kappa-shear and EPBL column kernels, compiled as
host C++ and run thread by thread on the CPU, against the oracle -- bit for
bit.

The kernels' arithmetic is plain IEEE FP64 in a fixed order with no FMA
contraction (the GPU build uses -fmad=false; here g++ -ffp-contract=off), so
the same source gives the same bits on the host.  This checks the device
code itself -- its index arithmetic, the memory reuse that departs from the
reference's layout, the device ports of the safe-math functions -- on CPU in
every run of the suite; the GPU tests (tests/test_gpu_kappa_shear.py,
tests/test_gpu_epbl.py) check the same source on the B200.
tests/host_kernels/prelude.h stands in for the CUDA qualifiers and intrinsics.
"""
import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from tests._cases import columns, hot_cfg, oracle_state

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "roundabout_b200" / "csrc"
HERE = Path(__file__).resolve().parent / "host_kernels"
_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a):
    return a.ctypes.data_as(_dp)


def _build(tmp: Path, source: str, launcher: str, driver: str) -> ctypes.CDLL:
    text = (CSRC / source).read_text()
    body = "\n".join(l for l in text[: text.index(f"void {launcher}(")].splitlines() if not l.startswith("#include"))
    unit = tmp / (Path(source).stem + "_host.cpp")
    unit.write_text('#include "prelude.h"\n' + body + "\n}  // namespace vphys\n" + (HERE / driver).read_text())
    lib = tmp / (Path(source).stem + "_host.so")
    cmd = ["g++", "-O2", "-ffp-contract=off", "-fno-fast-math", "-std=c++17", "-fPIC", "-shared",
           f"-I{HERE}", f"-I{CSRC}", "-o", str(lib), str(unit)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return ctypes.CDLL(str(lib))


@pytest.fixture(scope="module")
def host_libs(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    tmp = tmp_path_factory.mktemp("host_kernels")
    return {"kshear": _build(tmp, "vphys_kshear.cu", "launch_kappa_shear", "kshear_driver.inc"),
            "epbl": _build(tmp, "vphys_epbl.cu", "launch_epbl", "epbl_driver.inc")}


def _beta_plane(st):
    st.coriolis[...] = (1.0e-4 + 2.0e-7 * np.arange(st.ny))[None, :]


@pytest.mark.parametrize("shape", [(20, 12, 12), (12, 9, 40), (10, 6, 75), (7, 5, 1), (9, 4, 3), (6, 5, 100)])
@pytest.mark.parametrize("knobs", [{}, dict(eos_variant=1, eos_alpha_t=0.2, eos_beta_s=0.77, ks_vel_underflow=1e-3,
                                            ks_tke_bg=1e-12, ks_src_max_chg=8.0, ks_lz_rescale=0.5),
                                   dict(ks_massless_merge=1)])
def test_kappa_shear_source_matches_oracle(oracle, host_libs, shape, knobs):
    nx, ny, nz = shape
    cols = columns(nx=nx, ny=ny, nz=nz, seed=nx * ny + nz, thin_frac=0.15)
    cols.h[: nx // 3, :, -1] = 1.0e-4
    cfg = hot_cfg(kappa_shear=1, **knobs)
    st = oracle_state(oracle, cols, cfg)
    _beta_plane(st)
    st.call("vpo_kappa_shear", cfg, 3600.0)
    kd, tke = np.zeros_like(st.kd_shear), np.zeros_like(st.tke_shear)
    host_libs["kshear"].host_kappa_shear(ctypes.byref(cfg), nx, ny, nz, _ptr(st.h), _ptr(st.u), _ptr(st.v),
                                         _ptr(st.tracers[cfg.idx_temperature]), _ptr(st.tracers[cfg.idx_salinity]),
                                         _ptr(st.wet), _ptr(st.coriolis), ctypes.c_double(3600.0), _ptr(kd),
                                         _ptr(tke))
    assert np.array_equal(kd, st.kd_shear)
    assert np.array_equal(tke, st.tke_shear)
    if nz >= 12:
        assert st.kd_shear.max() > 0.0


EPBL_KNOBS = {
    "om4": dict(),
    "constant_rh18vstar_linear": dict(epbl_mstar_scheme=1, eos_variant=1, eos_alpha_t=0.2, eos_beta_s=0.77,
                                      epbl_vstar_scheme=2, epbl_mstar_conv_adj=0.5, epbl_omega_frac=0.3),
    "no_iteration": dict(epbl_mld_iteration=0, epbl_mstar_cap=0.8, epbl_min_mix_len=0.5),
    "shortwave_diags": dict(sw_pen_frac=0.6, epbl_tke_diags=1),
    "rh18_exponent": dict(epbl_mstar_scheme=3, epbl_mixlen_exponent=3.0, epbl_mstar_cap=0.9),
    "langmuir": dict(epbl_use_lt=1, epbl_tke_diags=1),
    "langmuir_additive": dict(epbl_use_lt=1, epbl_lt_scheme=2, sw_pen_frac=0.5),
    "shortwave_qsw": dict(sw_pen_frac=0.7, sw_source=1, epbl_tke_diags=1),
    "shortwave_no_ledger": dict(sw_pen_frac=0.7, epbl_sw_ctke=0),
    "chlorophyll_4band": dict(sw_pen_frac=1.0, sw_chl=1, sw_nbands=4, epbl_tke_diags=1),
}


@pytest.mark.parametrize("shape", [(20, 12, 12), (12, 9, 40), (10, 6, 75), (7, 5, 1), (9, 4, 2), (6, 5, 100)])
@pytest.mark.parametrize("knobs", sorted(EPBL_KNOBS))
def test_epbl_source_matches_oracle(oracle, host_libs, shape, knobs):
    nx, ny, nz = shape
    cols = columns(nx=nx, ny=ny, nz=nz, seed=nx * ny + 3 * nz, thin_frac=0.15)
    cols.h[: nx // 3, :, -1] = 1.0e-4
    cfg = hot_cfg(epbl=1, **EPBL_KNOBS[knobs])
    st = oracle_state(oracle, cols, cfg)
    _beta_plane(st)
    st.q_heat[...] *= 3.0
    st.sw_net[...] = np.abs(st.q_heat) * 0.8 + 40.0
    if cfg.sw_chl:
        cfg.sw_opacity_coef[6], cfg.sw_opacity_coef[7], cfg.sw_chl_power[3] = 0.8, 0.05, 0.5
        st.sw_chl[...] = np.abs(np.sin(np.arange(nx * ny))).reshape((nx, ny), order="F") * 3.0
        st.call("vpo_sw_chl_kappa", cfg)
    st.call("vpo_epbl", cfg, 3600.0)
    kd, mld, la = np.zeros_like(st.kd_epbl), np.zeros_like(st.mld_epbl), np.zeros_like(st.la_epbl)
    tke6 = np.zeros(6 * nx * ny)
    host_libs["epbl"].host_epbl(ctypes.byref(cfg), nx, ny, nz, _ptr(st.h), _ptr(st.tracers[cfg.idx_temperature]),
                                _ptr(st.tracers[cfg.idx_salinity]), _ptr(st.wet), _ptr(st.coriolis),
                                _ptr(st.stress_mag), _ptr(st.q_heat), _ptr(st.q_salt), _ptr(st.sw_net), _ptr(st.sw_kappa),
                                ctypes.c_double(3600.0),
                                _ptr(kd), _ptr(mld), _ptr(la), _ptr(tke6))
    assert np.array_equal(kd, st.kd_epbl)
    assert np.array_equal(mld, st.mld_epbl)
    assert np.array_equal(la, st.la_epbl)
    if cfg.epbl_tke_diags:
        for q in range(6):
            plane = tke6[q * nx * ny:(q + 1) * nx * ny].reshape((nx, ny), order="F")
            assert np.array_equal(plane, st.epbl_tke[q]), q
