"""The compensated FP64 column content (cfg.column_integrals).

With the diffusion, the tracer solves write per column and tracer the
Neumaier-compensated content sum_k h_k c_k over the column's live span,
before the solve (terms bottom-up) and after it (top-down, the fused KPP
non-local deposit included).  The exact path's sums equal the oracle's
compensated sums of the same states bit for bit, at the benchmark's depth
(nz = 75), and every column conserves its content to FP64 round-off; the
mixed form's content before the solve is the same exact sum, and its
conservation is stated against the two sums: the FP32 back-substitution
moves a column's content by a few FP32 ulps of its increment, not more.
Switching the diagnostic on leaves the solve's results as they were.
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


def slice_columns(name, nx, ny, seed):
    spec = dict(CONFIGS[name])
    ntr = spec.pop("ntracers")
    spec["nx"], spec["ny"] = nx, ny
    return make_columns(ntracers=ntr, seed=seed, **spec), ntr


@pytest.mark.parametrize("name", ["eddy_1440x1080x75", "batched_1440x1080x75"])
def test_exact_content_matches_the_oracle_and_is_conserved(VP, oracle, name):
    cols, ntr = slice_columns(name, 96, 80, seed=41)
    cfg = hot_path_config(ntracers=ntr)
    st = oracle_state(oracle, cols, cfg)
    old = st.column_content(False)
    assert st.call("vpo_step", cfg, DT, 1) == 0
    new = st.column_content(True)
    cfg_ci = hot_path_config(ntracers=ntr)
    cfg_ci.column_integrals = 1
    vp = VP(cols.nx, cols.ny, cols.nz, ntr, cfg_ci)
    vp.load_columns(cols)
    vp.step(DT, 1)
    assert_bitwise("content_old", vp.get("content_old"), old)
    assert_bitwise("content_new", vp.get("content_new"), new)
    for t in range(ntr):   # the diagnostic does not change the solve
        assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])
    scale = np.maximum(np.abs(old), 1e-300)
    drift = np.abs(new - old) / scale
    live = np.abs(old) > 0
    print(f"{name}: max relative column drift {drift[live].max():.3e}")
    assert drift[live].max() <= 1e-13
    vp.close()


@pytest.mark.parametrize("level", [1, 2])
def test_mixed_content_and_its_conservation(VP, oracle, level):
    cols, ntr = slice_columns("batched_1440x1080x75", 96, 80, seed=42)
    cfg = hot_path_config(ntracers=ntr)
    st = oracle_state(oracle, cols, cfg)
    st.call("vpo_eos_wright", cfg)
    old = st.column_content(False)
    cfg_ci = hot_path_config(ntracers=ntr)
    cfg_ci.column_integrals = 1
    cfg_ci.mixed_precision = level
    vp = VP(cols.nx, cols.ny, cols.nz, ntr, cfg_ci)
    vp.load_columns(cols)
    vp.step(DT, 1)
    assert_bitwise("content_old", vp.get("content_old"), old)
    got_new = np.asarray(vp.get("content_new"))
    # the written new content is the content of the new state
    ref = oracle.OracleState(cols.nx, cols.ny, cols.nz, ntr)
    ref.h[...] = cols.h
    for t in range(ntr):
        ref.tracers[t][...] = vp.get_tracer(t)
    assert_bitwise("content_new", got_new, ref.column_content(True))
    # conservation, per column: the change against the column's increment
    inc = np.stack([np.abs(np.asarray(vp.get_tracer(t)) - cols.tracers[t]) * cols.h[:, :, :]
                    for t in range(ntr)], axis=-1).sum(axis=2)
    drift = np.abs(got_new - old)
    live = np.abs(old) > 0
    ratio = drift[live] / np.maximum(inc[live], 1e-300)
    print(f"mixed_precision={level}: max |content change| / sum h |increment| = {ratio.max():.3e}, "
          f"max relative drift {float((drift[live] / np.abs(old[live])).max()):.3e}")
    assert ratio.max() <= 1e-5
    vp.close()
