"""Restart through the C ABI (the reference's vmix restart fields,
rdb_ocean_state_restart.F90:214, 248): the state that carries from step to
step -- u, v, the tracers and the lagged KPP boundary-layer depth -- read with
vphys_get_field after n steps and written into a fresh handle continues
exactly as the uninterrupted run."""
import pytest

from tests._cases import assert_bitwise, columns, hot_cfg

pytestmark = pytest.mark.gpu
DT = 3600.0


@pytest.fixture(scope="module")
def VP():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from roundabout_b200.column import VerticalPhysics

    return VerticalPhysics


@pytest.mark.parametrize("level", [0, 1, 2])
def test_restart_continues_bitwise(VP, level):
    cols = columns(nx=40, ny=24, nz=30, seed=51, ntr=4, thin_frac=0.1)
    cfg = hot_cfg(ntr=4, mixed_precision=level)
    a = VP(cols.nx, cols.ny, cols.nz, 4, cfg)
    a.load_columns(cols)
    a.step(DT, 4)
    b = VP(cols.nx, cols.ny, cols.nz, 4, cfg)
    b.load_columns(cols)
    b.step(DT, 2)
    saved = {n: b.get(n) for n in ("u", "v", "bl_depth")}
    saved_tr = [b.get_tracer(t) for t in range(4)]
    b.close()
    c = VP(cols.nx, cols.ny, cols.nz, 4, cfg)
    c.load_columns(cols)
    for n, arr in saved.items():
        c.set(n, arr)
    for t, arr in enumerate(saved_tr):
        c.set_tracer(t, arr)
    c.step(DT, 2)
    for t in range(4):
        assert_bitwise(f"tracer{t}", c.get_tracer(t), a.get_tracer(t))
    for n in ("u", "v", "bl_depth", "kv", "kt"):
        assert_bitwise(n, c.get(n), a.get(n))
