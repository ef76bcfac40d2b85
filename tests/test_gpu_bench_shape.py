"""Parity at the benchmark's shape: nz = 75, the eddy generator, the default knobs.

The benchmark runs 75 layers through the default-knob kernel instantiations
(PP81 + KPP + Bryan-Lewis; hvel_mom6 z_clear faces; no budgets, remnant or
shortwave) with their level-blocked loads.  These cases run exactly that code
on slices of the same generator (seeded synthetic columns with 30 % land and
geometric layers truncated at the bathymetry) and compare with the oracle:

* plain FP64: every output field bit for bit after 3 whole steps (the lagged
  OBL depth feeding back), at 128x96x75 and at the 360x270x75 slice the
  benchmark's CPU arm times;
* mixed precision (FP32 assembly and Thomas sweeps with the FP64 residual
  correction): within 1e-6 of the oracle after one step in every tracer, on
  the batched configuration's columns (10 tracers, 15 % of the wet columns
  carrying 1 mm layers, uniform passives), at both precision levels.
"""
import numpy as np
import pytest

from roundabout_b200.config import hot_path_config
from roundabout_b200.synthetic import CONFIGS, make_columns
from tests._cases import assert_bitwise, oracle_state

pytestmark = pytest.mark.gpu

DT = 3600.0


@pytest.fixture(scope="module")
def VP():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from roundabout_b200.column import VerticalPhysics

    return VerticalPhysics


def slice_columns(name, nx, ny, seed=1234):
    spec = dict(CONFIGS[name])
    ntr = spec.pop("ntracers")
    spec["nx"], spec["ny"] = nx, ny
    return make_columns(ntracers=ntr, seed=seed, **spec), ntr


@pytest.mark.parametrize("nx,ny", [(128, 96), (360, 270)])
def test_plain_fp64_three_steps_nz75(VP, oracle, nx, ny):
    cols, ntr = slice_columns("eddy_1440x1080x75", nx, ny)
    assert cols.nz == 75 and ntr == 4
    cfg = hot_path_config(ntracers=ntr)
    st = oracle_state(oracle, cols, cfg)
    vp = VP(cols.nx, cols.ny, cols.nz, ntr, cfg)
    vp.load_columns(cols)
    assert st.call("vpo_step", cfg, DT, 3) == 0
    vp.step(DT, 3)
    for n in ("kv", "kt", "ks", "u", "v", "bl_depth", "rho"):
        assert_bitwise(n, vp.get(n), getattr(st, n))
    for t in range(ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    vp.close()


def test_plain_fp64_graph_nz75(VP, oracle):
    """The same code captured as a CUDA graph of 3 steps."""
    cols, ntr = slice_columns("eddy_1440x1080x75", 128, 96, seed=77)
    cfg = hot_path_config(ntracers=ntr)
    st = oracle_state(oracle, cols, cfg)
    vp = VP(cols.nx, cols.ny, cols.nz, ntr, cfg)
    vp.load_columns(cols)
    assert st.call("vpo_step", cfg, DT, 3) == 0
    vp.step_graph(DT, 3)
    for n in ("kv", "kt", "ks", "u", "v", "bl_depth"):
        assert_bitwise(n, vp.get(n), getattr(st, n))
    for t in range(ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    vp.close()


@pytest.mark.parametrize("level", [1, 2])
def test_mixed_one_step_batched_nz75(VP, oracle, level):
    cols, ntr = slice_columns("batched_1440x1080x75", 128, 96)
    assert cols.nz == 75 and ntr == 10
    cfg = hot_path_config(ntracers=ntr)
    st = oracle_state(oracle, cols, cfg)
    mcfg = hot_path_config(ntracers=ntr)
    mcfg.mixed_precision = level
    vp = VP(cols.nx, cols.ny, cols.nz, ntr, mcfg)
    vp.load_columns(cols)
    assert st.call("vpo_step", cfg, DT, 1) == 0
    vp.step(DT, 1)
    errs = [float(np.abs(np.asarray(vp.get_tracer(t)) - st.tracers[t]).max()) for t in range(ntr)]
    du = float(np.abs(np.asarray(vp.get("u")) - st.u).max())
    dv = float(np.abs(np.asarray(vp.get("v")) - st.v).max())
    print(f"mixed_precision={level} at 128x96x75, 10 tracers: max |d tracer| {max(errs):.3e}, "
          f"|du| {du:.3e}, |dv| {dv:.3e}, FP64 re-solved groups {vp.mixed_redo_count()}")
    assert max(errs) <= 1e-6, errs
    assert du <= 1e-6 and dv <= 1e-6
    vp.close()


@pytest.mark.parametrize("level", [0, 2])
def test_fused_tracer_launch_equals_two_calls(VP, level):
    """vphys_vdiff_tracers_nonlocal (the launch the step runs, which the
    benchmark times) gives the same tracers as vphys_vdiff_tracers followed
    by vphys_nonlocal."""
    cols, ntr = slice_columns("eddy_1440x1080x75", 128, 96, seed=5)
    cfg = hot_path_config(ntracers=ntr)
    cfg.mixed_precision = level
    a = VP(cols.nx, cols.ny, cols.nz, ntr, cfg)
    b = VP(cols.nx, cols.ny, cols.nz, ntr, cfg)
    for vp in (a, b):
        vp.load_columns(cols)
        vp.eos()
        vp.assemble()
    a.vdiff_tracers_nonlocal(DT)
    b.vdiff_tracers(DT)
    b.nonlocal_tendencies(DT)
    for t in range(ntr):
        ga, gb = np.asarray(a.get_tracer(t)), np.asarray(b.get_tracer(t))
        if level == 0:
            assert_bitwise(f"tracer{t}", ga, gb)
        else:
            # the mixed solve deposits the non-local term inside its FP32
            # back-substitution, the separate call after it in FP64
            assert float(np.abs(ga - gb).max()) <= 1e-9, t
    a.close()
    b.close()
