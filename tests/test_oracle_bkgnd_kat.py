"""The oracle's assembly floors against the known-answer tests of
tests/test_ocean_bkgnd_mixing.F90 that tests/test_oracle_kat.py does not
already restate, re-expressed on the oracle (the Fortran tests cannot run
here: no Fortran compiler).  The Henyey cases of that file need a
latitude-dependent background this library refuses.

Bottom-up like the reference: interface k is the bottom of layer k, 1-based.
Checked quantities and tolerances are the reference tests' own:
  with the profile off, coefficients above the scalar floors pass the gate
      bit for bit (test_default_off_bit_identity, :294-326);
  with the Bryan-Lewis profile on (kd 1e-5 at the surface, 1.3e-4 deep,
      z0 1000 m, width 222 m, Prandtl 2) and coefficients of 1e-12: kt and ks
      at the interface 600 m deep take kd_bg(600 m) and kv twice it, to
      1e-15, the bed and surface interfaces stay zero
      (test_profile_floor_applies, :328-381).
"""
import math

import numpy as np

from roundabout_b200.config import default_config


def test_gate_passes_coefficients_above_the_scalar_floors(oracle):
    nz = 5
    c = default_config()
    st = oracle.OracleState(16, 14, nz, 2)
    st.h[...] = 5.0
    for a in (st.kv, st.kt, st.ks):
        a[...] = 0.0
    for k in range(2, nz + 1):
        st.kv[:, :, k - 1] = 1.0e-3 + 1.0e-4 * k
        st.kt[:, :, k - 1] = 2.0e-4 + 1.0e-5 * k
        st.ks[:, :, k - 1] = 3.0e-4 + 1.0e-5 * k
    before = [a.copy() for a in (st.kv, st.kt, st.ks)]
    assert st.call("vpo_assemble_gate", c) == 0
    for a, b in zip((st.kv, st.kt, st.ks), before):
        assert np.array_equal(a, b)


def test_bryan_lewis_floor_applies(oracle):
    NZ, KD_SFC, KD_DEEP, Z0, DELTA, PR, HZ = 30, 1.0e-5, 1.3e-4, 1000.0, 222.0, 2.0, 100.0
    c = default_config()
    c.bkgnd_profile = 1
    c.bkgnd_kd_sfc = KD_SFC
    c.bkgnd_kd_deep = KD_DEEP
    c.bkgnd_z0 = Z0
    c.bkgnd_delta = DELTA
    c.bkgnd_prandtl = PR
    st = oracle.OracleState(16, 14, NZ, 2)
    st.h[...] = HZ
    for a in (st.kv, st.kt, st.ks):
        a[...] = 0.0
        a[:, :, 1:NZ] = 1.0e-12
    assert st.call("vpo_assemble_gate", c) == 0
    i, j, kk = 4, 3, NZ - 5
    depth = (NZ - kk + 1) * HZ
    kd = KD_SFC + (KD_DEEP - KD_SFC) * (0.5 + math.atan((depth - Z0) / DELTA) / math.pi)
    assert abs(st.kt[i, j, kk - 1] - kd) < 1.0e-15
    assert abs(st.ks[i, j, kk - 1] - kd) < 1.0e-15
    assert abs(st.kv[i, j, kk - 1] - PR * kd) < 1.0e-15
    assert abs(st.kv[i, j, 0]) < 1.0e-15 and abs(st.kv[i, j, NZ]) < 1.0e-15
