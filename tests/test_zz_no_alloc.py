"""The allocation-free smoothing entry point, for callers that cannot call
cudaMalloc (a host that owns all device memory through its own pool, or code
running where allocating is not allowed): vphys_smooth_121_static keeps its
scratch plane in a fixed device array and must give exactly what the
assembly gate's own smoothing (vphys_assemble with kd_smooth_iterations)
gives, call after call.  Collected last on purpose: a failure here comes after
every other test has run."""
import ctypes

import numpy as np
import pytest

from tests._cases import columns, hot_cfg

pytestmark = pytest.mark.gpu


def test_static_smoothing_matches_the_gate_twice_in_a_row():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from roundabout_b200 import _ffi
    from roundabout_b200.column import VerticalPhysics

    L = _ffi.get_lib()
    cols = columns(nx=70, ny=44, nz=9, seed=17, land_frac=0.3)
    iters = 2
    raw = hot_cfg(kd_smooth_iterations=0)
    vp = VerticalPhysics(cols.nx, cols.ny, cols.nz, len(cols.tracers), raw)
    vp.load_columns(cols)
    vp.eos()
    vp.assemble()
    vp.synchronize()
    unsmoothed = {n: torch.from_numpy(np.ascontiguousarray(vp.get(n).T)).cuda() for n in ("kv", "kt")}
    wet = torch.from_numpy(np.ascontiguousarray(cols.wet.T)).cuda()

    vp.set_config(hot_cfg(kd_smooth_iterations=iters))
    vp.set("bl_depth", np.zeros((cols.nx, cols.ny)))
    vp.eos()
    vp.assemble()
    vp.synchronize()
    want = {n: vp.get(n) for n in ("kv", "kt")}

    for n in ("kv", "kt", "kv"):                 # calls in a row share the scratch array
        fld = unsmoothed[n].clone()
        st = L.vphys_smooth_121_static(ctypes.c_void_p(fld.data_ptr()), ctypes.c_void_p(wet.data_ptr()),
                                       cols.nx, cols.ny, cols.nz, iters, None)
        assert st == _ffi.OK, _ffi.last_error(0)
        torch.cuda.synchronize()
        got = fld.cpu().numpy().T
        assert np.array_equal(got, want[n]), f"{n}: allocation-free smoothing differs from the gate's"

    # beyond the fixed scratch plane: refused before any launch
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = L.vphys_smooth_121_static(ctypes.c_void_p(dummy.data_ptr()), ctypes.c_void_p(dummy.data_ptr()),
                                   4096, 4096, 3, 1, None)
    assert st == _ffi.ERR_TOO_LARGE
    assert "2^23" in _ffi.last_error(0)
    vp.close()
