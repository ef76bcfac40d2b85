"""Parity of EPBL (vphys_epbl, and the merge inside the assembly and
vphys_step with epbl = 1) with the CPU oracle.

The column solve is epbl_compute -> epbl_column_kernel
(rdb_ocean_epbl.F90:864-1659): bitwise on kd_epbl and mld_epbl for the
OM4, RH18 and constant mstar, both velocity scales, mixing-length
exponents 2 and 3, the LF17 Langmuir enhancement (rescale and additive), the TKE budget
diagnostics, the MLD iteration with false
position, bisection, the previous-MLD seed or none, both EOS variants, the
penetrating-shortwave TKE ledger (two-band from Q_heat or the q_sw source, or the chlorophyll N-band), nz from 1 to 100, vanished top layers and
land; the merges (add, max,
max_shear with kappa-shear) bitwise through the assembly and whole steps,
with convection masked below EPBL's MLD; the mixed step within 1e-6.
"""
import numpy as np
import pytest

from tests._cases import assert_bitwise, columns, hot_cfg, oracle_state

pytestmark = pytest.mark.gpu

DT = 3600.0


@pytest.fixture(scope="module")
def VP():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from roundabout_b200.column import VerticalPhysics

    return VerticalPhysics


def beta_plane(ny, nx):
    f = (1.0e-4 + 2.0e-11 * 1.0e4 * np.arange(ny))[None, :]
    return np.asfortranarray(np.broadcast_to(f, (nx, ny)))


KNOBS = {
    "om4": dict(),
    "const_linear_rh18": dict(epbl_mstar_scheme=1, eos_variant=1, eos_alpha_t=0.2, eos_beta_s=0.77,
                              epbl_vstar_scheme=2, epbl_mstar_conv_adj=0.5, epbl_omega_frac=0.3),
    "no_iteration": dict(epbl_mld_iteration=0, epbl_mstar_cap=0.8, epbl_min_mix_len=0.5),
    "bisection_prev": dict(epbl_mld_bisection=1, epbl_mld_use_prev_guess=1, epbl_mld_max_its=7),
    "shortwave": dict(sw_pen_frac=0.6, epbl_tke_diags=1),
    "rh18_exponent": dict(epbl_mstar_scheme=3, epbl_mstar_cap=0.9, epbl_mixlen_exponent=3.0, epbl_vstar_scheme=2),
    "langmuir": dict(epbl_use_lt=1, epbl_tke_diags=1),
    "langmuir_additive_sw": dict(epbl_use_lt=1, epbl_lt_scheme=2, sw_pen_frac=0.5, epbl_lt_lac2=0.1),
    "shortwave_qsw": dict(sw_pen_frac=0.7, sw_source=1, epbl_tke_diags=1),
    "shortwave_no_ledger": dict(sw_pen_frac=0.7, epbl_sw_ctke=0),
    "chlorophyll": dict(sw_pen_frac=1.0, sw_chl=1, epbl_tke_diags=1),
    "shortwave_linear": dict(epbl_mstar_scheme=1, sw_pen_frac=1.0, eos_variant=1, eos_alpha_t=0.2, eos_beta_s=0.77,
                             sw_zeta1=1.5, sw_zeta2=9.0),
}


def setup(VP, oracle, cols, cfg, prev_mld=None):
    f = beta_plane(cols.ny, cols.nx)
    st = oracle_state(oracle, cols, cfg)
    st.coriolis[...] = f
    st.q_heat[...] *= 3.0
    vp = VP(cols.nx, cols.ny, cols.nz, len(cols.tracers), cfg)
    vp.load_columns(cols)
    vp.set("coriolis", f)
    vp.set("q_heat", st.q_heat)
    if cfg.sw_source:
        st.sw_net[...] = np.abs(st.q_heat) * 0.8 + 40.0
        vp.set("sw_net", st.sw_net)
    if cfg.sw_chl:
        st.sw_chl[...] = np.abs(np.sin(np.arange(cols.nx * cols.ny))).reshape((cols.nx, cols.ny), order="F") * 3.0
        st.call("vpo_sw_chl_kappa", cfg)
        vp.set("sw_chl", st.sw_chl)
        vp.sw_chl_apply()
    if prev_mld is not None:
        st.mld_epbl[...] = prev_mld
        vp.set("mld_epbl", prev_mld)
    return st, vp


@pytest.mark.parametrize("shape,thin", [((24, 20, 12), 0.0), ((30, 18, 40), 0.15), ((16, 12, 75), 0.1),
                                        ((9, 7, 1), 0.0), ((9, 7, 2), 0.0), ((11, 5, 3), 0.2), ((8, 6, 100), 0.1),
                                        ((150, 3, 33), 0.1)])
@pytest.mark.parametrize("knobs", sorted(KNOBS))
def test_epbl_standalone(VP, oracle, shape, thin, knobs):
    nx, ny, nz = shape
    cols = columns(nx=nx, ny=ny, nz=nz, seed=nx + 5 * nz, thin_frac=thin)
    cols.h[: nx // 4, :, -1] = 1.0e-4       # vanished top layers: the column starts at the first live one
    cfg = hot_cfg(epbl=1, **KNOBS[knobs])
    prev = None
    if knobs == "bisection_prev":
        prev = np.asfortranarray(np.abs(np.sin(np.arange(nx * ny))).reshape(nx, ny) * 80.0)
    st, vp = setup(VP, oracle, cols, cfg, prev)
    st.call("vpo_epbl", cfg, DT)
    vp.epbl(DT)
    assert_bitwise("kd_epbl", vp.get("kd_epbl"), st.kd_epbl)
    assert_bitwise("mld_epbl", vp.get("mld_epbl"), st.mld_epbl)
    assert_bitwise("la_epbl", vp.get("la_epbl"), st.la_epbl)
    if cfg.epbl_tke_diags:
        for q, name in enumerate(("wind", "conv", "forcing", "mixing", "mech_decay", "conv_decay")):
            assert_bitwise(f"epbl_tke_{name}", vp.get(f"epbl_tke_{name}"), st.epbl_tke[q])
    if nz >= 12:
        assert st.kd_epbl.max() > 0.0


@pytest.mark.parametrize("combine,shear", [(1, 0), (2, 0), (3, 0), (3, 1), (1, 1)])
def test_assemble_merges_epbl(VP, oracle, combine, shear):
    cols = columns(nx=40, ny=24, nz=30, seed=61, thin_frac=0.1)
    cfg = hot_cfg(epbl=1, epbl_combine=combine, epbl_prandtl=0.7, kappa_shear=shear, ks_prandtl_turb=0.8,
                  conv_enable=1)
    st, vp = setup(VP, oracle, cols, cfg)
    st.call("vpo_eos_wright", cfg)
    st.call("vpo_epbl", cfg, DT)
    if shear:
        st.call("vpo_kappa_shear", cfg, DT)
    assert st.call("vpo_build_coefficients", cfg) == 0
    vp.eos()
    vp.epbl(DT)
    if shear:
        vp.kappa_shear(DT)
    vp.assemble()
    for n in ("kv", "kt", "ks", "kd_epbl", "mld_epbl", "bl_depth"):
        assert_bitwise(n, vp.get(n), getattr(st, n))
    assert (st.bl_depth == 0.0).all()          # KPP did not run


@pytest.mark.parametrize("shear,sw", [(0, 0), (1, 0), (0, 1)])
def test_step_with_epbl(VP, oracle, shear, sw):
    cols = columns(nx=30, ny=18, nz=24, seed=62, thin_frac=0.1)
    cfg = hot_cfg(epbl=1, budgets=1, surface_flux=1, kappa_shear=shear, epbl_combine=3 if shear else 1,
                  epbl_mld_use_prev_guess=1, conv_enable=1, sw_pen_frac=0.5 if sw else 0.0)
    st, vp = setup(VP, oracle, cols, cfg)
    assert st.call("vpo_step", cfg, DT, 3) == 0
    vp.step(DT, 3)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    for n in ("kv", "kt", "ks", "u", "v", "kd_epbl", "mld_epbl", "heat_budget"):
        assert_bitwise(n, vp.get(n), getattr(st, n))


def test_step_graph_with_epbl(VP, oracle):
    cols = columns(nx=40, ny=24, nz=16, seed=63, thin_frac=0.1)
    cfg = hot_cfg(epbl=1)
    st, vp = setup(VP, oracle, cols, cfg)
    assert st.call("vpo_step", cfg, DT, 4) == 0
    vp.step_graph(DT, 2)
    vp.step_graph(DT, 2)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    assert_bitwise("mld_epbl", vp.get("mld_epbl"), st.mld_epbl)


@pytest.mark.parametrize("mixed", [1, 2])
def test_mixed_step_with_epbl(VP, oracle, mixed):
    ntr = 6
    cols = columns(nx=48, ny=32, nz=40, seed=64, ntr=ntr, thin_frac=0.15, passive_init="uniform")
    cfg = hot_cfg(ntr=ntr, epbl=1)
    st, _ = setup(VP, oracle, cols, cfg)
    _, vp = setup(VP, oracle, cols, hot_cfg(ntr=ntr, epbl=1, mixed_precision=mixed))
    assert st.call("vpo_step", cfg, DT, 1) == 0
    vp.step(DT, 1)
    err = max(float(np.abs(np.asarray(vp.get_tracer(t)) - st.tracers[t]).max()) for t in range(ntr))
    assert err <= 1.0e-6, err
    assert_bitwise("kd_epbl", vp.get("kd_epbl"), st.kd_epbl)
