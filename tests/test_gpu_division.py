"""The kernels' exact-division helpers (zero-guarded quotient, shared
reciprocal with Markstein's correction) against the IEEE quotient a/b, bit for
bit, on seeded operands spanning the exponent ranges the path meets."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("emin,erange", [(-40, 80), (-8, 16), (-499, 998)])
def test_division_helpers_match_ieee(emin, erange):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from roundabout_b200 import _ffi

    L = _ffi.get_lib()
    bad = ctypes.c_ulonglong(123)
    _ffi.check(L.vphys_selftest_division(200_000_000, 20251203 + emin, emin, erange, ctypes.byref(bad)),
               "vphys_selftest_division")
    assert bad.value == 0

