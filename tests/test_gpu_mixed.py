"""The mixed-precision forms against the FP64 oracle.

cfg.mixed_precision = 1: FP64 assembly, FP32 Thomas sweeps with the FP64
residual correction.  Bar: max |dT|, |dS| and passive-tracer error <= 1e-6
(absolute: degC, psu, tracer units) against the FP64 result on the same
inputs, per stage and for one whole step, with stiff thin layers (h = 1e-3 m);
velocities <= 1e-6 m/s.  Over 24 steps the bar is the FP64 oracle's own
response to a +-1e-7 perturbation of its initial tracers (thin layers make the
reference's Richardson number amplify such differences far beyond 1e-6).
cfg.mixed_precision = 2: the assembly's interface sweep in FP32 as well: one
step within 2e-5, 24 steps inside the same envelope.
The FP64 path is checked untouched by the switch (bitwise, as everywhere).
"""
import numpy as np
import pytest

from tests._cases import assert_bitwise, columns, hot_cfg, oracle_state

pytestmark = pytest.mark.gpu

DT = 3600.0
TOL_TS = 1.0e-6
TOL_UV = 1.0e-6


@pytest.fixture(scope="module")
def VP():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from roundabout_b200.column import VerticalPhysics

    return VerticalPhysics


def maxabs(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    assert np.isfinite(a).all()
    return float(np.abs(a - b).max()) if a.size else 0.0


TRACER_CASES = {
    "ks_eq_kt": dict(),
    "ks_ne_kt": dict(bkgnd_profile=0, kt_bg=2e-5, ks_bg=7e-6),
    "budgets": dict(budgets=1),
    "use_harmonic": dict(use_harmonic=1),
}


@pytest.mark.parametrize("ntr", [2, 4, 10])
@pytest.mark.parametrize("case", sorted(TRACER_CASES))
def test_tracer_solve_mixed(VP, oracle, case, ntr):
    """Same FP64 coefficients, mixed tracer solve vs the FP64 solve."""
    cols = columns(nx=40, ny=24, nz=30, seed=31, ntr=ntr, thin_frac=0.15, passive_init="uniform")
    cfg = hot_cfg(ntr=ntr, **TRACER_CASES[case])
    st = oracle_state(oracle, cols, cfg)
    vp = VP(cols.nx, cols.ny, cols.nz, ntr, cfg)
    vp.load_columns(cols)
    st.q_heat[...] = -np.abs(st.q_heat)
    vp.set("q_heat", st.q_heat)
    st.call("vpo_eos_wright", cfg)
    st.call("vpo_build_coefficients", cfg)
    vp.eos()
    vp.assemble()
    assert_bitwise("kt", vp.get("kt"), st.kt)
    cfg_mp = hot_cfg(ntr=ntr, mixed_precision=1, **TRACER_CASES[case])
    vp.set_config(cfg_mp)
    st.call("vpo_vdiff_tracers", cfg, DT)
    st.call("vpo_nonlocal", cfg, DT)
    vp.vdiff_tracers(DT)
    vp.nonlocal_tendencies(DT)
    errs = [maxabs(vp.get_tracer(t), st.tracers[t]) for t in range(ntr)]
    assert max(errs) <= TOL_TS, errs
    # a stiff column actually moved: the test is not comparing two copies of the input
    moved = max(float(np.abs(st.tracers[t] - cols.tracers[t]).max()) for t in range(ntr))
    assert moved > 1e-3
    if cfg.budgets:
        for n in ("heat_budget", "salt_budget"):
            want = getattr(st, n)
            assert maxabs(vp.get(n), want) <= 1e-6 * max(1.0, float(np.abs(want).max())), n


def test_momentum_solve_mixed(VP, oracle):
    cols = columns(nx=40, ny=24, nz=30, seed=32, thin_frac=0.2)
    cfg = hot_cfg()
    st = oracle_state(oracle, cols, cfg)
    vp = VP(cols.nx, cols.ny, cols.nz, len(cols.tracers), cfg)
    vp.load_columns(cols)
    st.call("vpo_eos_wright", cfg)
    st.call("vpo_build_coefficients", cfg)
    vp.eos()
    vp.assemble()
    vp.set_config(hot_cfg(mixed_precision=1))
    st.call("vpo_vdiff_momentum", cfg, DT)
    vp.vdiff_momentum(DT)
    assert maxabs(vp.get("u"), st.u) <= TOL_UV
    assert maxabs(vp.get("v"), st.v) <= TOL_UV


@pytest.mark.parametrize("over", [dict(), dict(remnant=1, implicit_stress=1, implicit_drag=1)])
def test_momentum_options_mixed(VP, oracle, over):
    cols = columns(nx=33, ny=17, nz=20, seed=33, thin_frac=0.1)
    cfg = hot_cfg(**over)
    st = oracle_state(oracle, cols, cfg)
    vp = VP(cols.nx, cols.ny, cols.nz, len(cols.tracers), cfg)
    vp.load_columns(cols)
    if cfg.implicit_drag:
        rng = np.random.default_rng(3)
        st.lambda_bot_u[...] = rng.uniform(0, 1e-4, st.lambda_bot_u.shape)
        st.lambda_bot_v[...] = rng.uniform(0, 1e-4, st.lambda_bot_v.shape)
        vp.set("lambda_bot_u", st.lambda_bot_u)
        vp.set("lambda_bot_v", st.lambda_bot_v)
    st.call("vpo_eos_wright", cfg)
    st.call("vpo_build_coefficients", cfg)
    vp.eos()
    vp.assemble()
    vp.set_config(hot_cfg(mixed_precision=1, **over))
    st.call("vpo_vdiff_momentum", cfg, DT)
    vp.vdiff_momentum(DT)
    assert maxabs(vp.get("u"), st.u) <= TOL_UV
    assert maxabs(vp.get("v"), st.v) <= TOL_UV
    if cfg.remnant:
        assert maxabs(vp.get("visc_rem_u"), st.visc_rem_u) <= 1e-5
        assert maxabs(vp.get("visc_rem_v"), st.visc_rem_v) <= 1e-5


@pytest.mark.parametrize("case", ["ks_eq_kt", "ks_ne_kt", "budgets"])
def test_large_increment_resolved_in_fp64(VP, oracle, case):
    """A column group whose one-step increment reaches 2 units (here a 15 K
    cold anomaly in the top layer, mixed down by convection) is re-solved on
    the FP64 path: those groups come out bitwise, every tracer within 1e-6."""
    ntr = 4
    cols = columns(nx=72, ny=12, nz=30, seed=37, ntr=ntr, thin_frac=0.15, passive_init="uniform")
    cols.tracers[1][:8, :, -1] -= 15.0
    cfg = hot_cfg(ntr=ntr, **TRACER_CASES[case])
    st = oracle_state(oracle, cols, cfg)
    vp = VP(cols.nx, cols.ny, cols.nz, ntr, cfg)
    vp.load_columns(cols)
    st.call("vpo_eos_wright", cfg)
    st.call("vpo_build_coefficients", cfg)
    vp.eos()
    vp.assemble()
    vp.set_config(hot_cfg(ntr=ntr, mixed_precision=1, **TRACER_CASES[case]))
    T0 = st.tracers[1].copy()
    st.call("vpo_vdiff_tracers", cfg, DT)
    dT = np.abs(st.tracers[1] - T0)
    st.call("vpo_nonlocal", cfg, DT)
    vp.vdiff_tracers(DT)
    assert vp.mixed_redo_count() > 0
    vp.nonlocal_tendencies(DT)
    errs = [maxabs(vp.get_tracer(t), st.tracers[t]) for t in range(ntr)]
    assert max(errs) <= TOL_TS, errs
    T = np.asarray(vp.get_tracer(1))
    # a column whose own increment passes the bar lies in a re-solved group,
    # whichever way the solve groups its columns
    col_max = dT.max(axis=2)
    sure = np.argwhere(col_max > 2.2)
    assert sure.shape[0] > 0
    for i, j in sure:
        assert_bitwise(f"T, re-solved column ({i}, {j})", T[i, j], st.tracers[1][i, j])
    if cfg.budgets:
        want = st.heat_budget
        assert maxabs(vp.get("heat_budget"), want) <= 1e-6 * max(1.0, float(np.abs(want).max()))


def test_resolve_is_rare_once_mixed(VP, oracle):
    """The first step from the stratified synthetic state homogenises mixed
    layers spanning a few kelvin (|delta| ~ 2 K): a few groups go to FP64.
    Once mixed, the increments stay small and (almost) nothing is re-solved."""
    ntr = 4
    cols = columns(nx=96, ny=32, nz=40, seed=38, ntr=ntr, thin_frac=0.15)
    vp = VP(cols.nx, cols.ny, cols.nz, ntr, hot_cfg(ntr=ntr, mixed_precision=1))
    vp.load_columns(cols)
    groups = 3 * 32 * ntr
    counts = []
    for _ in range(6):
        vp.step(DT, 1)
        counts.append(vp.mixed_redo_count())
    print("re-solved groups per step:", counts, "of", groups)
    assert counts[0] <= 0.1 * groups
    assert counts[-1] <= 0.02 * groups


@pytest.mark.parametrize("level,tol", [(1, TOL_TS), (2, 2e-5)])
def test_mixed_one_step(VP, oracle, level, tol):
    """One whole step (EOS, assembly, momentum, tracers, non-local) from the
    same state: level 1 within 1e-6 of the FP64 oracle in every tracer."""
    ntr = 10
    cols = columns(nx=48, ny=32, nz=40, seed=34, ntr=ntr, thin_frac=0.15, passive_init="uniform")
    cfg = hot_cfg(ntr=ntr)
    st = oracle_state(oracle, cols, cfg)
    vp = VP(cols.nx, cols.ny, cols.nz, ntr, hot_cfg(ntr=ntr, mixed_precision=level))
    vp.load_columns(cols)
    assert st.call("vpo_step", cfg, DT, 1) == 0
    vp.step(DT, 1)
    errs = [maxabs(vp.get_tracer(t), st.tracers[t]) for t in range(ntr)]
    print(f"mixed_precision={level}: 1-step max |d tracer| = {max(errs):.3e}")
    assert max(errs) <= tol, errs
    assert maxabs(vp.get("u"), st.u) <= TOL_UV
    assert maxabs(vp.get("v"), st.v) <= TOL_UV


@pytest.mark.parametrize("level", [1, 2])
def test_mixed_24_steps_within_oracle_envelope(VP, oracle, level):
    """24 steps.  On 1 mm layers under the 1e-10 shear floor, Ri = N^2/S^2
    amplifies density differences by orders of magnitude, so the FP64 oracle
    itself moves by far more than 1e-6 when its initial tracers move by an
    FP32-sized +-1e-7.  The mixed run must stay inside that envelope."""
    ntr = 10
    cols = columns(nx=48, ny=32, nz=40, seed=34, ntr=ntr, thin_frac=0.15, passive_init="uniform")
    cfg = hot_cfg(ntr=ntr)
    st = oracle_state(oracle, cols, cfg)
    pert = oracle_state(oracle, cols, cfg)
    rng = np.random.default_rng(0)
    wet = cols.h > 1.5e-4
    for t in range(ntr):
        pert.tracers[t][...] += rng.uniform(-1e-7, 1e-7, cols.h.shape) * wet
    assert st.call("vpo_step", cfg, DT, 24) == 0
    assert pert.call("vpo_step", cfg, DT, 24) == 0
    envelope = max(float(np.abs(pert.tracers[t] - st.tracers[t]).max()) for t in range(ntr))
    vp = VP(cols.nx, cols.ny, cols.nz, ntr, hot_cfg(ntr=ntr, mixed_precision=level))
    vp.load_columns(cols)
    vp.step(DT, 24)
    errs = [maxabs(vp.get_tracer(t), st.tracers[t]) for t in range(ntr)]
    print(f"mixed_precision={level}: 24-step max |d tracer| = {max(errs):.3e}; "
          f"oracle's own response to +-1e-7: {envelope:.3e}")
    assert max(errs) <= envelope, (errs, envelope)
    bl = np.asarray(vp.get("bl_depth"))
    assert np.abs(bl - st.bl_depth).max() <= 1e-2 * max(1.0, float(np.abs(st.bl_depth).max()))


def test_exact_path_unchanged_after_mixed(VP, oracle):
    """Switching a handle to mixed and back leaves the FP64 path bitwise."""
    cols = columns(nx=24, ny=20, nz=12, seed=35, thin_frac=0.1)
    cfg = hot_cfg()
    st = oracle_state(oracle, cols, cfg)
    vp = VP(cols.nx, cols.ny, cols.nz, len(cols.tracers), hot_cfg(mixed_precision=1))
    vp.load_columns(cols)
    vp.step(DT, 1)
    vp.load_columns(cols)
    vp.set("bl_depth", np.zeros((cols.nx, cols.ny)))   # the lagged OBL depth starts at 0 again
    vp.set_config(cfg)
    assert st.call("vpo_step", cfg, DT, 2) == 0
    vp.step(DT, 2)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    assert_bitwise("u", vp.get("u"), st.u)
    assert_bitwise("kv", vp.get("kv"), st.kv)


@pytest.mark.parametrize("level", [0, 1])
def test_step_graph_equals_steps(VP, level):
    """vphys_step_graph replays the captured launches: the same state as
    vphys_step, bit for bit, and a rebind recaptures."""
    cols = columns(nx=40, ny=24, nz=30, seed=36, ntr=4, thin_frac=0.15)
    a = VP(cols.nx, cols.ny, cols.nz, 4, hot_cfg(ntr=4, mixed_precision=level))
    b = VP(cols.nx, cols.ny, cols.nz, 4, hot_cfg(ntr=4, mixed_precision=level))
    a.load_columns(cols)
    b.load_columns(cols)
    a.step(DT, 6)
    b.step_graph(DT, 3)
    b.step_graph(DT, 3)
    for t in range(4):
        assert_bitwise(f"tracer{t}", b.get_tracer(t), a.get_tracer(t))
    for n in ("u", "v", "kv", "kt", "bl_depth"):
        assert_bitwise(n, b.get(n), a.get(n))
