"""The oracle's surface-band viscosity kv += kv_ml_invz2 (hmix / z)^2 on the
interior interfaces shallower than hmix_fixed against the reference's
known-answer tests (tests/test_ocean_kv_ml_invz2.F90), re-expressed on the
oracle (the Fortran tests cannot run here: no Fortran compiler).

Bottom-up like the reference: interface k lies under layer k, so interface
nz sits h(nz) below the surface.  kv starts at zero on 4 x 4 columns of
uniform layers.  Checked quantities and tolerances are the reference tests'
own:
  kv_ml_invz2 = 0 is a no-op (test_zero_amplitude, :64-81);
  two 100 m layers under hmix = 20 m: nothing augmented
      (test_interface_below_hmix, :83-101);
  50 layers of 1 m: the interface 1 m deep takes more than the one 10 m
      deep, both positive (test_profile_monotone, :103-136);
  10 layers of 5 m: the interface 15 m deep takes 0.01 (20 / 15)^2 to
      1e-14, the walk stopping at the interface that reaches hmix
      (test_value_at_hmix, :138-172).
"""
from roundabout_b200.config import default_config


def augment(oracle, nz, h, amp, hmix):
    c = default_config()
    c.kv_ml_invz2 = amp
    c.hmix_fixed = hmix
    st = oracle.OracleState(4, 4, nz, 2)
    st.h[...] = h
    st.kv[...] = 0.0
    st.call("vpo_kv_ml_invz2", c)
    return st.kv


def test_zero_amplitude_is_a_no_op(oracle):
    assert abs(augment(oracle, 4, 5.0, 0.0, 20.0)).max() < 1.0e-15


def test_interfaces_below_hmix_unchanged(oracle):
    assert abs(augment(oracle, 2, 100.0, 0.01, 20.0)).max() < 1.0e-15


def test_profile_decreases_with_depth(oracle):
    NZ = 50
    kv = augment(oracle, NZ, 1.0, 0.01, 20.0)
    shallow, deep = kv[2, 2, NZ - 1], kv[2, 2, NZ - 10]    # 1-based interfaces nz (1 m) and nz - 9 (10 m)
    assert shallow > deep > 0.0


def test_value_off_the_inverse_square_profile(oracle):
    NZ, KV0, HMIX = 10, 0.01, 20.0
    kv = augment(oracle, NZ, 5.0, KV0, HMIX)
    assert abs(kv[2, 2, NZ - 3] - KV0 * (HMIX / 15.0) ** 2) < 1.0e-14    # 1-based interface nz - 2, 15 m deep
