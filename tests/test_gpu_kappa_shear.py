"""Parity of kappa-shear (vphys_kappa_shear, and the merge inside the
assembly and vphys_step with kappa_shear = 1) with the CPU oracle.

The column solve is kappa_shear_compute -> kappa_shear_column_kernel
(rdb_ocean_kappa_shear.F90:427-648, solver 953-1909): bitwise on kd_shear
and tke_shear for both EOS variants, non-default knobs, the massless merge of
vanished layers, thin and vanished layers, land, and nz from 1 to 100; the reference's golden column
(test_ocean_kappa_shear.F90:286-393) within its 1e-6 bar; the merge
(kappa_shear_merge_into_kv_kt, :381-421) bitwise through the assembly and
whole steps; the mixed-precision step within its 1e-6 bar.
"""
import math

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


def loaded(VP, cols, cfg, coriolis=None):
    vp = VP(cols.nx, cols.ny, cols.nz, len(cols.tracers), cfg)
    vp.load_columns(cols)
    if coriolis is not None:
        vp.set("coriolis", coriolis)
    return vp


def beta_plane(ny, nx):
    f = (1.0e-4 + 2.0e-11 * 1.0e4 * np.arange(ny))[None, :]
    return np.asfortranarray(np.broadcast_to(f, (nx, ny)))


KNOBS = dict(eos_variant=1, eos_alpha_t=0.2, eos_beta_s=0.77, ks_vel_underflow=1.0e-3, ks_tke_bg=1.0e-12,
             ks_src_max_chg=8.0, ks_lz_rescale=0.5, ks_ri_crit=0.3, ks_max_inner_it=20, ks_max_substep_it=9)
MERGE = dict(ks_massless_merge=1)


@pytest.mark.parametrize("shape,thin", [((24, 20, 12), 0.0), ((30, 18, 40), 0.15), ((16, 12, 75), 0.1),
                                        ((9, 7, 1), 0.0), ((9, 7, 2), 0.0), ((11, 5, 3), 0.2), ((8, 6, 100), 0.1),
                                        ((130, 3, 33), 0.1)])
@pytest.mark.parametrize("knobs", ["default", "knobs", "merge"])
def test_kappa_shear_standalone(VP, oracle, shape, thin, knobs):
    nx, ny, nz = shape
    cols = columns(nx=nx, ny=ny, nz=nz, seed=nx + 7 * nz, thin_frac=thin)
    cols.h[: nx // 4, :, -1] = 1.0e-4       # vanished top layers on part of the domain: floored at H_VANISHED
    over = {"default": {}, "knobs": KNOBS, "merge": MERGE}[knobs]
    cfg = hot_cfg(kappa_shear=1, **over)
    f = beta_plane(ny, nx) * (-1.0 if knobs == "knobs" else 1.0)
    st = oracle_state(oracle, cols, cfg)
    st.coriolis[...] = f
    dt = 1800.0 if knobs == "knobs" else DT
    st.call("vpo_kappa_shear", cfg, dt)
    vp = loaded(VP, cols, cfg, f)
    vp.kappa_shear(dt)
    assert_bitwise("kd_shear", vp.get("kd_shear"), st.kd_shear)
    assert_bitwise("tke_shear", vp.get("tke_shear"), st.tke_shear)
    if nz >= 12:
        assert st.kd_shear.max() > 0.0       # the columns mix somewhere


def test_golden_column_on_the_gpu(VP, oracle):
    """The reference's golden column (nz = 20, linear EOS, f = 1e-4,
    dt = 1800): bitwise with the oracle and within 1e-6 of the golden kd."""
    from tests.test_oracle_kappa_shear import ALPHA, BETA, GOLDEN_SD, RHO0, ks_config, shear_column

    st = shear_column(oracle, 20, 5.0, 0.5, 50.0, 20.0, 3.0e-5)
    cfg = ks_config()
    vp = VP(st.nx, st.ny, st.nz, 2, cfg)
    for n in ("h", "u", "v", "wet", "coriolis"):
        vp.set(n, getattr(st, n))
    vp.set_tracer(0, st.tracers[0])
    vp.set_tracer(1, st.tracers[1])
    vp.kappa_shear(1800.0)
    st.call("vpo_kappa_shear", cfg, 1800.0)
    kd = vp.get("kd_shear")
    assert_bitwise("kd_shear", kd, st.kd_shear)
    worst = max(abs(kd[1, 1, 20 - k] - g) / g for k, g in enumerate(GOLDEN_SD) if g > 1e-10)
    assert worst < 1.0e-6, worst
    assert (ALPHA, BETA, RHO0) == (cfg.eos_alpha_t, cfg.eos_beta_s, cfg.rho0)


def test_assemble_merges_kd(VP, oracle):
    cols = columns(nx=40, ny=24, nz=30, seed=51, thin_frac=0.1)
    cfg = hot_cfg(kappa_shear=1, ks_prandtl_turb=0.8)
    f = beta_plane(cols.ny, cols.nx)
    st = oracle_state(oracle, cols, cfg)
    st.coriolis[...] = f
    st.call("vpo_eos_wright", cfg)
    st.call("vpo_kappa_shear", cfg, DT)
    assert st.call("vpo_build_coefficients", cfg) == 0
    vp = loaded(VP, cols, cfg, f)
    vp.get("gamma_t")        # the gamma fields are written once they exist
    vp.get("gamma_s")
    vp.eos()
    vp.kappa_shear(DT)
    vp.assemble()
    for n in ("kv", "kt", "ks", "bl_depth", "b0", "gamma_t", "kd_shear"):
        assert_bitwise(n, vp.get(n), getattr(st, n))
    # the merge changed the answer
    c0 = hot_cfg()
    s0 = oracle_state(oracle, cols, c0)
    s0.call("vpo_eos_wright", c0)
    s0.call("vpo_build_coefficients", c0)
    assert np.abs(s0.kt - st.kt).max() > 1.0e-3


@pytest.mark.parametrize("budgets", [0, 1])
def test_step_with_kappa_shear(VP, oracle, budgets):
    cols = columns(nx=30, ny=18, nz=24, seed=52, thin_frac=0.1)
    cfg = hot_cfg(kappa_shear=1, budgets=budgets, surface_flux=1)
    f = beta_plane(cols.ny, cols.nx)
    st = oracle_state(oracle, cols, cfg)
    st.coriolis[...] = f
    vp = loaded(VP, cols, cfg, f)
    assert st.call("vpo_step", cfg, DT, 3) == 0
    vp.step(DT, 3)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    for n in ("kv", "kt", "ks", "u", "v", "bl_depth", "kd_shear", "tke_shear"):
        assert_bitwise(n, vp.get(n), getattr(st, n))
    if budgets:
        assert_bitwise("heat_budget", vp.get("heat_budget"), st.heat_budget)


def test_step_graph_with_kappa_shear(VP, oracle):
    cols = columns(nx=40, ny=24, nz=16, seed=53, thin_frac=0.1)
    cfg = hot_cfg(kappa_shear=1)
    f = beta_plane(cols.ny, cols.nx)
    st = oracle_state(oracle, cols, cfg)
    st.coriolis[...] = f
    vp = loaded(VP, cols, cfg, f)
    assert st.call("vpo_step", cfg, DT, 4) == 0
    vp.step_graph(DT, 2)
    vp.step_graph(DT, 2)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    assert_bitwise("kd_shear", vp.get("kd_shear"), st.kd_shear)


@pytest.mark.parametrize("mixed", [1, 2])
def test_mixed_step_with_kappa_shear(VP, oracle, mixed):
    ntr = 6
    cols = columns(nx=48, ny=32, nz=40, seed=54, ntr=ntr, thin_frac=0.15, passive_init="uniform")
    cfg = hot_cfg(ntr=ntr, kappa_shear=1)
    f = beta_plane(cols.ny, cols.nx)
    st = oracle_state(oracle, cols, cfg)
    st.coriolis[...] = f
    vp = loaded(VP, cols, hot_cfg(ntr=ntr, kappa_shear=1, mixed_precision=mixed), f)
    assert st.call("vpo_step", cfg, DT, 1) == 0
    vp.step(DT, 1)
    err = max(float(np.abs(np.asarray(vp.get_tracer(t)) - st.tracers[t]).max()) for t in range(ntr))
    assert err <= 1.0e-6, err
    for n in ("u", "v"):
        assert float(np.abs(vp.get(n) - getattr(st, n)).max()) <= 1.0e-6
    # the column solve itself is FP64 in every form
    assert_bitwise("kd_shear", vp.get("kd_shear"), st.kd_shear)


def test_kappa_shear_without_temperature_is_a_noop(VP):
    cols = columns(nx=8, ny=6, nz=10, seed=55)
    cfg = hot_cfg(kappa_shear=1)
    cfg.idx_temperature = -1
    cfg.eos_in_step = 0
    cfg.use_kpp = 0
    vp = loaded(VP, cols, cfg)
    seed = np.full(vp.shape("kd_shear"), 3.0, order="F")
    vp.set("kd_shear", seed)
    vp.kappa_shear(DT)
    assert (vp.get("kd_shear") == 3.0).all()


def test_uniform_column_domain_is_uniform(VP, oracle):
    """Every column of a horizontally uniform domain is the same column, so
    kd is identical in each (no cross-column state in the kernel)."""
    from tests.test_oracle_kappa_shear import ks_config, shear_column

    st = shear_column(oracle, 40, 5.0, 0.5, 100.0, 20.0, 3.0e-5, nx=70, ny=5)
    cfg = ks_config()
    vp = VP(st.nx, st.ny, st.nz, 2, cfg)
    for n in ("h", "u", "v", "wet", "coriolis"):
        vp.set(n, getattr(st, n))
    vp.set_tracer(0, st.tracers[0])
    vp.set_tracer(1, st.tracers[1])
    vp.kappa_shear(1800.0)
    kd = vp.get("kd_shear")
    assert np.array_equal(kd, np.broadcast_to(kd[:1, :1, :], kd.shape))
    assert kd.max() > 0.0 and math.isfinite(float(kd.max()))
