"""Size-independent properties at the benchmark's full size, 1440x1080x75
(116.6 M cells, 4 tracers, 30 % land), where the CPU oracle is too slow to run
the whole domain:

* the FP64 tracer solve conserves every column's heat and salt content
  (sum of max(h, H_VANISHED) * c) to round-off, the reference's 1e-12 bar
  (test_ocean_vdiff.F90:270-308);
* with budgets on, the booked heat budget equals the content change;
* two runs of the same step from the same state agree bit for bit
  (no order-dependent reduction anywhere in the step);
* the mixed form stays within 1e-6 (T, S, passives) and 1e-6 m/s (u, v) of
  the FP64 path after one step from the same state.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 3600.0


@pytest.fixture(scope="module")
def setup():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from roundabout_b200.column import VerticalPhysics
    from roundabout_b200.config import hot_path_config
    from roundabout_b200.synthetic import CONFIGS, make_columns

    spec = dict(CONFIGS["eddy_1440x1080x75"])
    ntr = spec.pop("ntracers")
    cols = make_columns(ntracers=ntr, seed=2024, **spec)

    def handle(**over):
        cfg = hot_path_config(ntracers=ntr)
        for k, v in over.items():
            setattr(cfg, k, v)
        vp = VerticalPhysics(cols.nx, cols.ny, cols.nz, ntr, cfg)
        vp.load_columns(cols)
        return vp

    return cols, handle


def column_sums(a, w):
    return (w * a).sum(axis=2), (np.abs(w * a)).sum(axis=2)


def test_fullsize_tracer_solve_conserves_columns(setup):
    cols, handle = setup
    vp = handle(budgets=1)
    vp.eos()
    vp.assemble()
    w = np.maximum(cols.h, 1.5e-4) * (cols.h > 1.5e-4)
    before = [np.asarray(vp.get_tracer(t)) for t in (0, 1)]
    vp.vdiff_tracers(DT)
    for t, b in zip((0, 1), before):
        a = np.asarray(vp.get_tracer(t))
        s0, scale = column_sums(b, w)
        s1, _ = column_sums(a, w)
        rel = np.abs(s1 - s0) / np.maximum(scale, 1e-300)
        assert rel.max() <= 1e-12, (t, rel.max())
        moved = np.abs(a - b).max()
        assert moved > 1e-3
    # the heat budget books h (T_new - T_old) cell by cell
    T1 = np.asarray(vp.get_tracer(1))
    bud = np.asarray(vp.get("heat_budget"))
    booked = bud.sum(axis=2)
    gained = (cols.h * (T1 - before[1])).sum(axis=2)
    scale = np.abs(cols.h * T1).sum(axis=2)
    assert (np.abs(booked - gained) / np.maximum(scale, 1e-300)).max() <= 1e-12
    vp.close()


def test_fullsize_step_is_deterministic(setup):
    cols, handle = setup
    runs = []
    for _ in range(2):
        vp = handle()
        vp.step(DT, 2)
        runs.append([np.asarray(vp.get_tracer(t)) for t in range(4)] + [np.asarray(vp.get(n)) for n in ("u", "kv")])
        vp.close()
    for a, b in zip(*runs):
        assert np.array_equal(a, b)


def test_fullsize_mixed_within_bar_of_fp64(setup):
    cols, handle = setup
    plain, mixed = handle(), handle(mixed_precision=2)
    plain.step(DT, 1)
    mixed.step(DT, 1)
    for t in range(4):
        err = float(np.abs(np.asarray(mixed.get_tracer(t)) - np.asarray(plain.get_tracer(t))).max())
        assert err <= 1e-6, (t, err)
    for n in ("u", "v"):
        err = float(np.abs(np.asarray(mixed.get(n)) - np.asarray(plain.get(n))).max())
        assert err <= 1e-6, (n, err)
    plain.close()
    mixed.close()
