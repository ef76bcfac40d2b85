"""The in-project autotuner of the mixed-precision solves (vphys_autotune) and
every kernel variant it chooses between.

Each variant of the face solve (registers, TMA-staged ring) and of the tracer
solve (rows in shared memory with 1, 2 or 4 tracers per warp, rows in tensor
memory), pinned with vphys_set_variants, gives a whole mixed step within
1e-6 of the FP64 oracle at the benchmark's depth (nz = 75) on thin-layer
columns (FP64 assembly; with the FP32 assembly too, within its 2e-5 bar).  The autotuner leaves every field of the handle as it found it,
reports a time for every admitted variant and keeps the fastest.
"""
import numpy as np
import pytest

from roundabout_b200.config import hot_path_config
from roundabout_b200.synthetic import make_columns
from tests._cases import oracle_state

pytestmark = pytest.mark.gpu

DT = 3600.0


@pytest.fixture(scope="module")
def VP():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from roundabout_b200.column import VerticalPhysics

    return VerticalPhysics


@pytest.fixture(scope="module")
def case(oracle):
    cols = make_columns(96, 64, 75, ntracers=5, seed=91, land_frac=0.3, thin_frac=0.15, passive_init="uniform")
    cfg = hot_path_config(ntracers=5)
    st = oracle_state(oracle, cols, cfg)
    assert st.call("vpo_step", cfg, DT, 1) == 0
    return cols, st


MOM = ("registers", "tma_ring")
TR = ("smem_1_per_warp", "smem_2_per_warp", "smem_4_per_warp", "tmem_rows")


# the variants change only the solves: level 1 (FP64 assembly) isolates them
# at the 1e-6 bar; level 2 adds the FP32 assembly, held to the bar of its
# own one-step test (tests/test_gpu_mixed.py)
@pytest.mark.parametrize("level,tol", [(1, 1e-6), (2, 2e-5)])
@pytest.mark.parametrize("mom", MOM)
@pytest.mark.parametrize("tr", TR)
def test_every_variant_against_the_oracle(VP, case, mom, tr, level, tol):
    cols, st = case
    cfg = hot_path_config(ntracers=5)
    cfg.mixed_precision = level
    vp = VP(cols.nx, cols.ny, cols.nz, 5, cfg)
    vp.load_columns(cols)
    vp.set_variants(mom, tr)
    vp.step(DT, 1)
    errs = [float(np.abs(np.asarray(vp.get_tracer(t)) - st.tracers[t]).max()) for t in range(5)]
    duv = max(float(np.abs(np.asarray(vp.get(n)) - getattr(st, n)).max()) for n in ("u", "v"))
    print(f"level {level}, {mom}, {tr}: max |d tracer| {max(errs):.3e}, |d u,v| {duv:.3e}")
    assert max(errs) <= tol, (mom, tr, errs)
    assert duv <= tol, (mom, tr, duv)
    vp.close()


def test_autotune_keeps_the_state_and_picks_the_fastest(VP, case):
    cols, st = case
    cfg = hot_path_config(ntracers=5)
    cfg.mixed_precision = 2
    vp = VP(cols.nx, cols.ny, cols.nz, 5, cfg)
    vp.load_columns(cols)
    vp.step(DT, 1)   # a state with every field written
    names = ("h", "u", "v", "kv", "kt", "ks", "bl_depth", "rho", "b0")
    before = {n: np.array(vp.get(n)) for n in names}
    tb = [np.array(vp.get_tracer(t)) for t in range(5)]
    res = vp.autotune(DT, reps=2)
    print(res)
    for n in names:
        assert np.array_equal(np.asarray(vp.get(n)), before[n], equal_nan=True), n
    for t in range(5):
        assert np.array_equal(np.asarray(vp.get_tracer(t)), tb[t]), t
    assert set(res["momentum"]) == set(MOM) and set(res["tracers"]) == set(TR)
    assert res["chosen"]["momentum"] == min(res["momentum"], key=res["momentum"].get)
    assert res["chosen"]["tracers"] == min(res["tracers"], key=res["tracers"].get)
    vp.step(DT, 1)   # the picks run
    vp.close()


def test_autotune_without_mixed_precision_is_a_report(VP, case):
    cols, _ = case
    vp = VP(cols.nx, cols.ny, cols.nz, 5, hot_path_config(ntracers=5))
    vp.load_columns(cols)
    res = vp.autotune(DT)
    assert res["momentum"] == {} and res["tracers"] == {}
    vp.close()
