"""Parity of the surface heat/salt deposit (vphys_surface_flux, and inside
vphys_step with surface_flux = 1) with the CPU oracle.

The deposit is ocean_surface_flux_apply_tracers (rdb_ocean_surface_flux.F90:
959-1070): bitwise on the FP64 path, standalone and in a whole step; the
mixed-precision step keeps its 1e-6 per-step bar with the deposit on.
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


def loaded(VP, cols, cfg):
    vp = VP(cols.nx, cols.ny, cols.nz, len(cols.tracers), cfg)
    vp.load_columns(cols)
    return vp


@pytest.mark.parametrize("shape", [(24, 20, 12), (7, 5, 1), (130, 9, 20)])
@pytest.mark.parametrize("budgets", [0, 1])
def test_surface_flux_standalone(VP, oracle, shape, budgets):
    nx, ny, nz = shape
    cols = columns(nx=nx, ny=ny, nz=nz, seed=nx + 3 * nz, thin_frac=0.2)
    cols.h[: nx // 3, :, -1] = 1.0e-4          # vanished top filler on part of the domain
    if nz > 2:
        cols.h[: nx // 5, :, -2] = 0.0          # and a second one on some of it
    cfg = hot_cfg(budgets=budgets, surface_flux=1)
    st = oracle_state(oracle, cols, cfg)
    vp = loaded(VP, cols, cfg)
    for _ in range(3):
        st.call("vpo_surface_flux", cfg, DT)
        vp.surface_flux(DT)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    if budgets:
        assert_bitwise("heat_budget_surface", vp.get("heat_budget_surface"), st.heat_budget_surface)
        assert_bitwise("salt_budget_surface", vp.get("salt_budget_surface"), st.salt_budget_surface)
        assert np.abs(st.heat_budget_surface).max() > 0.0


def test_surface_flux_content_equals_budget(VP, oracle):
    """The column heat content gained is the booked contribution (the
    contributors-match-analytic case, test_ocean_surface_flux.F90:220-300)."""
    cols = columns(nx=32, ny=16, nz=10, seed=41, land_frac=0.2)
    cfg = hot_cfg(budgets=1, surface_flux=1)
    vp = loaded(VP, cols, cfg)
    T0 = np.asarray(vp.get_tracer(1)).copy()
    for _ in range(4):
        vp.surface_flux(DT)
    gained = ((np.asarray(vp.get_tracer(1)) - T0) * cols.h).sum()
    booked = np.asarray(vp.get("heat_budget_surface")).sum()
    assert abs(gained - booked) <= 1e-9 * max(abs(booked), 1e-30)


@pytest.mark.parametrize("shape", [(24, 20, 12), (33, 17, 3)])
def test_step_with_surface_flux(VP, oracle, shape):
    nx, ny, nz = shape
    cols = columns(nx=nx, ny=ny, nz=nz, seed=nx + ny, thin_frac=0.1)
    cfg = hot_cfg(budgets=1, surface_flux=1)
    st = oracle_state(oracle, cols, cfg)
    vp = loaded(VP, cols, cfg)
    assert st.call("vpo_step", cfg, DT, 3) == 0
    vp.step(DT, 3)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    for n in ("kv", "kt", "ks", "u", "v", "bl_depth", "b0", "rho", "heat_budget", "heat_budget_surface",
              "salt_budget_surface"):
        assert_bitwise(n, vp.get(n), getattr(st, n))


def test_step_graph_with_surface_flux(VP, oracle):
    cols = columns(nx=40, ny=24, nz=16, seed=43, thin_frac=0.1)
    cfg = hot_cfg(surface_flux=1)
    st = oracle_state(oracle, cols, cfg)
    vp = loaded(VP, cols, cfg)
    assert st.call("vpo_step", cfg, DT, 4) == 0
    vp.step_graph(DT, 2)
    vp.step_graph(DT, 2)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])


def test_mixed_step_with_surface_flux(VP, oracle):
    """A 1 mm top layer under 100 W/m2 warms by ~87 K: its column group is
    re-solved in FP64, and the step keeps the 1e-6 bar."""
    ntr = 6
    cols = columns(nx=48, ny=32, nz=40, seed=44, ntr=ntr, thin_frac=0.15, passive_init="uniform")
    cfg = hot_cfg(ntr=ntr, surface_flux=1)
    st = oracle_state(oracle, cols, cfg)
    vp = loaded(VP, cols, hot_cfg(ntr=ntr, surface_flux=1, mixed_precision=1))
    assert st.call("vpo_step", cfg, DT, 1) == 0
    vp.step(DT, 1)
    assert vp.mixed_redo_count() > 0
    err = max(float(np.abs(np.asarray(vp.get_tracer(t)) - st.tracers[t]).max()) for t in range(ntr))
    assert err <= 1.0e-6, err


def test_surface_flux_rejects_bad_flag(VP):
    from roundabout_b200 import _ffi

    cols = columns(nx=8, ny=4, nz=3, seed=45)
    with pytest.raises(_ffi.VphysError):
        loaded(VP, cols, hot_cfg(surface_flux=2))


SW = dict(sw_pen_frac=0.5, sw_band_ratio=0.58, sw_zeta1=0.35, sw_zeta2=23.0)


@pytest.mark.parametrize("budgets", [0, 1])
def test_sw_penetration_standalone(VP, oracle, budgets):
    """ocean_surface_flux_apply_sw_penetration after the surface deposit,
    bitwise, with vanished top fillers and thin layers."""
    cols = columns(nx=40, ny=12, nz=20, seed=46, thin_frac=0.2)
    cols.h[:10, :, -1] = 1.0e-4
    cfg = hot_cfg(budgets=budgets, surface_flux=1, **SW)
    st = oracle_state(oracle, cols, cfg)
    vp = loaded(VP, cols, cfg)
    for _ in range(2):
        st.call("vpo_surface_flux", cfg, DT)
        st.call("vpo_sw_penetration", cfg, DT)
        vp.surface_flux(DT)
        vp.sw_penetration(DT)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    if budgets:
        assert_bitwise("heat_budget_surface", vp.get("heat_budget_surface"), st.heat_budget_surface)


@pytest.mark.parametrize("method", [1, 2, 3])
def test_assemble_with_shortwave(VP, oracle, method):
    """KPP's B0 charging only the absorbed shortwave (MXL: inside the
    boundary layer, LV1: inside the surface layer): the assembly bitwise."""
    cols = columns(seed=47)
    cfg = hot_cfg(kpp_sw_method=method, **SW)
    st = oracle_state(oracle, cols, cfg)
    st.q_heat[...] = np.abs(st.q_heat) + 50.0    # sunlit: a penetrating part to subtract
    st.call("vpo_eos_wright", cfg)
    st.bl_depth[...] = np.abs(np.sin(np.arange(st.bl_depth.size))).reshape(st.bl_depth.shape, order="F") * 60.0
    vp = loaded(VP, cols, cfg)
    vp.set("q_heat", st.q_heat)
    vp.eos()
    vp.set("bl_depth", st.bl_depth)
    vp.get("gamma_t")
    assert st.call("vpo_build_coefficients", cfg) == 0
    vp.assemble()
    for n in ("kv", "kt", "ks", "bl_depth", "b0", "gamma_t"):
        assert_bitwise(n, vp.get(n), getattr(st, n))


@pytest.mark.parametrize("eos_coeffs", [0, 1])
def test_step_with_shortwave(VP, oracle, eos_coeffs):
    """Whole steps with the surface deposit, the shortwave moved down the
    column and KPP's corrected B0 (and its non-local deposit): bitwise."""
    cols = columns(nx=30, ny=18, nz=16, seed=48, thin_frac=0.1)
    cfg = hot_cfg(budgets=1, surface_flux=1, buoyancy_coeffs=eos_coeffs, **SW)
    st = oracle_state(oracle, cols, cfg)
    vp = loaded(VP, cols, cfg)
    assert st.call("vpo_step", cfg, DT, 3) == 0
    vp.step(DT, 3)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    for n in ("kv", "kt", "u", "bl_depth", "b0", "heat_budget", "heat_budget_surface"):
        assert_bitwise(n, vp.get(n), getattr(st, n))
    c0 = hot_cfg(budgets=1, surface_flux=1, buoyancy_coeffs=eos_coeffs)
    s0 = oracle_state(oracle, cols, c0)
    s0.call("vpo_step", c0, DT, 3)
    assert np.abs(s0.tracers[1] - st.tracers[1]).max() > 1e-6   # the shortwave changed the answer


def test_mixed_step_with_shortwave(VP, oracle):
    ntr = 6
    cols = columns(nx=48, ny=32, nz=40, seed=49, ntr=ntr, thin_frac=0.15, passive_init="uniform")
    cfg = hot_cfg(ntr=ntr, surface_flux=1, **SW)
    st = oracle_state(oracle, cols, cfg)
    vp = loaded(VP, cols, hot_cfg(ntr=ntr, surface_flux=1, mixed_precision=1, **SW))
    assert st.call("vpo_step", cfg, DT, 1) == 0
    vp.step(DT, 1)
    err = max(float(np.abs(np.asarray(vp.get_tracer(t)) - st.tracers[t]).max()) for t in range(ntr))
    assert err <= 1.0e-6, err


def _sunlit_qsw(st):
    """A net shortwave unlike Q_heat's own share, zero on every third row."""
    st.q_heat[...] = np.abs(st.q_heat) + 60.0
    st.sw_net[...] = 0.5 * st.q_heat + 150.0 * (np.arange(st.nx)[:, None] % 3 == 0)
    st.sw_net[:, ::3] = 0.0


def test_qsw_penetration_standalone(VP, oracle):
    """sw_source = "q_sw": the penetration moves sw_pen_frac q_sw down the
    column (apply_sw_penetration_impl with sw_net), bitwise."""
    cols = columns(nx=40, ny=12, nz=20, seed=91, thin_frac=0.2)
    cols.h[:10, :, -1] = 1.0e-4
    cfg = hot_cfg(budgets=1, surface_flux=1, sw_source=1, **SW)
    st = oracle_state(oracle, cols, cfg)
    _sunlit_qsw(st)
    vp = loaded(VP, cols, cfg)
    vp.set("q_heat", st.q_heat)
    vp.set("sw_net", st.sw_net)
    for _ in range(2):
        st.call("vpo_surface_flux", cfg, DT)
        st.call("vpo_sw_penetration", cfg, DT)
        vp.surface_flux(DT)
        vp.sw_penetration(DT)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    assert_bitwise("heat_budget_surface", vp.get("heat_budget_surface"), st.heat_budget_surface)


@pytest.mark.parametrize("method", [2, 3])
def test_step_with_qsw(VP, oracle, method):
    """Whole steps under sw_source = "q_sw": deposit, penetration, KPP's B0
    charge and the non-local deposit all read q_sw; bitwise."""
    cols = columns(nx=30, ny=18, nz=16, seed=92, thin_frac=0.1)
    cfg = hot_cfg(budgets=1, surface_flux=1, sw_source=1, kpp_sw_method=method, **SW)
    st = oracle_state(oracle, cols, cfg)
    _sunlit_qsw(st)
    vp = loaded(VP, cols, cfg)
    vp.set("q_heat", st.q_heat)
    vp.set("sw_net", st.sw_net)
    assert st.call("vpo_step", cfg, DT, 3) == 0
    vp.step(DT, 3)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    for n in ("kv", "kt", "bl_depth", "b0", "heat_budget", "heat_budget_surface"):
        assert_bitwise(n, vp.get(n), getattr(st, n))


@pytest.mark.parametrize("budgets", [0, 1])
def test_bound_salinity_and_wet_dyn(VP, oracle, budgets):
    """BOUND_SALINITY (the first live layer floored at min_salinity after the
    deposit) and the dynamic wet/dry mask on the deposit, bitwise, standalone
    and through whole steps."""
    cols = columns(nx=33, ny=17, nz=12, seed=93, thin_frac=0.15)
    cols.h[:8, :, -1] = 1.0e-4
    cfg = hot_cfg(budgets=budgets, surface_flux=1, bound_salinity=1, min_salinity=34.9, use_wet_dyn=1)
    st = oracle_state(oracle, cols, cfg)
    st.wet_dyn[...] = ((np.arange(st.nx)[:, None] + 2 * np.arange(st.ny)[None, :]) % 5 != 0).astype(float)
    vp = loaded(VP, cols, cfg)
    vp.set("wet_dyn", st.wet_dyn)
    st.call("vpo_surface_flux", cfg, DT)
    vp.surface_flux(DT)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    assert st.call("vpo_step", cfg, DT, 2) == 0
    vp.step(DT, 2)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    if budgets:
        assert_bitwise("salt_budget_surface", vp.get("salt_budget_surface"), st.salt_budget_surface)


CHL = dict(sw_pen_frac=1.0, sw_chl=1)


def _with_chl(VP, oracle, cols, cfg):
    """Oracle and handle with the same chlorophyll; the band opacities from
    vphys_sw_chl_apply must equal the oracle's bit for bit."""
    st = oracle_state(oracle, cols, cfg)
    st.q_heat[...] = np.abs(st.q_heat) + 60.0
    st.sw_chl[...] = np.abs(np.cos(np.arange(st.nx * st.ny))).reshape((st.nx, st.ny), order="F") * 2.0
    st.sw_chl[0, 0] = 0.0
    st.call("vpo_sw_chl_kappa", cfg)
    vp = loaded(VP, cols, cfg)
    vp.set("q_heat", st.q_heat)
    vp.set("sw_chl", st.sw_chl)
    vp.sw_chl_apply()
    assert_bitwise("sw_kappa", vp.get("sw_kappa")[:, :, :cfg.sw_nbands], st.sw_kappa[:, :, :cfg.sw_nbands])
    return st, vp


@pytest.mark.parametrize("nbands", [3, 5])
def test_chl_penetration_standalone(VP, oracle, nbands):
    """apply_sw_penetration_nb_impl: the whole source moved down the column
    through the N-band transmission, bitwise."""
    cols = columns(nx=40, ny=12, nz=20, seed=94, thin_frac=0.2)
    cols.h[:10, :, -1] = 1.0e-4
    cfg = hot_cfg(budgets=1, surface_flux=1, sw_nbands=nbands, **CHL)
    for n in range(3, nbands):
        cfg.sw_opacity_coef[2 * n], cfg.sw_opacity_coef[2 * n + 1], cfg.sw_chl_power[n] = 0.5 + n, 0.02, 0.4
    st, vp = _with_chl(VP, oracle, cols, cfg)
    for _ in range(2):
        st.call("vpo_surface_flux", cfg, DT)
        st.call("vpo_sw_penetration", cfg, DT)
        vp.surface_flux(DT)
        vp.sw_penetration(DT)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    assert_bitwise("heat_budget_surface", vp.get("heat_budget_surface"), st.heat_budget_surface)


@pytest.mark.parametrize("method", [2, 3])
def test_step_with_chl(VP, oracle, method):
    """Whole steps under the chlorophyll scheme: penetration, KPP's N-band
    charge (both passes and the non-local gamma), bitwise."""
    cols = columns(nx=30, ny=18, nz=16, seed=95, thin_frac=0.1)
    cfg = hot_cfg(budgets=1, surface_flux=1, kpp_sw_method=method, **CHL)
    st, vp = _with_chl(VP, oracle, cols, cfg)
    assert st.call("vpo_step", cfg, DT, 3) == 0
    vp.step(DT, 3)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    for n in ("kv", "kt", "bl_depth", "b0", "heat_budget", "heat_budget_surface"):
        assert_bitwise(n, vp.get(n), getattr(st, n))


@pytest.mark.parametrize("chl", [0, 1])
def test_cover_frac_penetration(VP, oracle, chl):
    """The penetration under a partial ice-shelf cover, two-band and
    chlorophyll forms, bitwise."""
    cols = columns(nx=36, ny=10, nz=14, seed=96, thin_frac=0.1)
    extra = CHL if chl else SW
    cfg = hot_cfg(budgets=1, surface_flux=1, use_cover_frac=1, **extra)
    if chl:
        st, vp = _with_chl(VP, oracle, cols, cfg)
    else:
        st = oracle_state(oracle, cols, cfg)
        vp = loaded(VP, cols, cfg)
    st.cover_frac[...] = np.abs(np.sin(0.7 * np.arange(st.nx * st.ny))).reshape((st.nx, st.ny), order="F")
    st.cover_frac[::4, :] = 1.0
    vp.set("cover_frac", st.cover_frac)
    st.call("vpo_surface_flux", cfg, DT)
    st.call("vpo_sw_penetration", cfg, DT)
    vp.surface_flux(DT)
    vp.sw_penetration(DT)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    assert_bitwise("heat_budget_surface", vp.get("heat_budget_surface"), st.heat_budget_surface)
