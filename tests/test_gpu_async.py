"""The asynchronous field copies (vphys_set_field_async / vphys_get_field_async):
a round trip through pinned host memory gives back the same bits, and two
handles on two streams, fed and drained asynchronously in alternation as the
benchmark's end-to-end loop does, end in the same state as the synchronous
copies on one handle."""
import ctypes

import numpy as np
import pytest

from tests._cases import columns, hot_cfg

pytestmark = pytest.mark.gpu

DT = 3600.0


@pytest.fixture(scope="module")
def env():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from roundabout_b200 import _ffi
    from roundabout_b200.column import VerticalPhysics

    return torch, _ffi, VerticalPhysics


def test_async_round_trip(env):
    torch, _ffi, VP = env
    cols = columns(nx=37, ny=21, nz=9, seed=51)
    vp = VP(cols.nx, cols.ny, cols.nz, len(cols.tracers), hot_cfg())
    src = torch.from_numpy(np.ascontiguousarray(cols.u.T)).pin_memory()
    dst = torch.empty_like(src).pin_memory()
    L, h = vp.lib, vp.handle
    _ffi.check(L.vphys_set_field_async(h, _ffi.FIELD_U, ctypes.c_void_p(src.data_ptr()), src.numel()), "set")
    _ffi.check(L.vphys_get_field_async(h, _ffi.FIELD_U, ctypes.c_void_p(dst.data_ptr()), dst.numel()), "get")
    vp.synchronize()
    assert torch.equal(src, dst)
    # a wrong element count is refused before anything is queued
    assert L.vphys_set_field_async(h, _ffi.FIELD_U, ctypes.c_void_p(src.data_ptr()), src.numel() - 1) != 0
    vp.close()


def test_two_handles_pipelined_equal_synchronous(env):
    torch, _ffi, VP = env
    cols = columns(nx=48, ny=30, nz=14, seed=52, thin_frac=0.1)
    ntr = len(cols.tracers)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a.T)).pin_memory()  # noqa: E731
    inputs = {"h": pin(cols.h), "u": pin(cols.u), "v": pin(cols.v), "q_heat": pin(cols.q_heat),
              "q_salt": pin(cols.q_salt), "tau_x": pin(cols.tau_x), "tau_y": pin(cols.tau_y),
              "bl_depth": pin(np.zeros((cols.nx, cols.ny)))}   # the lagged state too: every step starts alike
    tracers = [pin(t) for t in cols.tracers]

    def run(vp, out, asyn):
        L, h = vp.lib, vp.handle
        setf = L.vphys_set_field_async if asyn else L.vphys_set_field
        getf = L.vphys_get_field_async if asyn else L.vphys_get_field
        for n, t in inputs.items():
            _ffi.check(setf(h, _ffi.FIELD_NAMES[n], ctypes.c_void_p(t.data_ptr()), t.numel()), "set")
        for k, t in enumerate(tracers):
            _ffi.check(setf(h, _ffi.FIELD_TRACER0 + k, ctypes.c_void_p(t.data_ptr()), t.numel()), "set")
        _ffi.check(L.vphys_stress_mag(h), "stress")
        _ffi.check(L.vphys_step(h, DT, 1), "step")
        for k, t in enumerate(out):
            _ffi.check(getf(h, _ffi.FIELD_TRACER0 + k, ctypes.c_void_p(t.data_ptr()), t.numel()), "get")

    ref = VP(cols.nx, cols.ny, cols.nz, ntr, hot_cfg())
    ref_out = [torch.empty_like(t).pin_memory() for t in tracers]
    run(ref, ref_out, False)
    pair = []
    for _ in range(2):
        vp = VP(cols.nx, cols.ny, cols.nz, ntr, hot_cfg())
        s = torch.cuda.Stream()
        vp.set_stream(s.cuda_stream)
        pair.append((vp, [torch.empty_like(t).pin_memory() for t in tracers], s))
    for i in range(4):
        vp, out, _ = pair[i % 2]
        run(vp, out, True)
    for vp, out, _ in pair:
        vp.synchronize()
        for a, b in zip(out, ref_out):
            assert torch.equal(a, b)
        vp.set_stream(0)
        vp.close()
    ref.close()
