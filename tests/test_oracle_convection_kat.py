"""The oracle's convective adjustment (kt -> max(kt, kd_conv), kv ->
max(kv, prandtl_conv kd_conv) where the interior N^2 < n2_thresh, strictly
below the boundary-layer depth) against the reference's known-answer tests
(tests/test_ocean_convection.F90), re-expressed on the oracle (the Fortran
tests cannot run here: no Fortran compiler).

Every case runs PP81 -> convection -> assemble (run_conv, :70-90) or the same
chain without the convection (run_no_conv, :92-107) on 8 x 6 columns,
bottom-up (level 1 is the bed).  Checked quantities and tolerances are the
reference tests' own:
  convection off on an inverted column: kv, kt as without it to 1e-15
      (test_disabled_bit_identical, :116-162);
  convection on, stable column: kv, kt as without it to 1e-15
      (test_stable_bit_identical, :164-212);
  inverted column, no boundary layer, prandtl_conv 2: every interior
      interface has kt = kd_conv, kv = 2 kd_conv to 1e-12, the bed and
      surface interfaces zero to 1e-15 (test_unstable_sets_kd_conv, :214-273);
  10 layers of 20 m under a 100 m boundary layer: interfaces shallower than
      100 m keep PP81's Ri < 0 value kappa_bg + nu0, from 100 m down kd_conv,
      to 1e-10 (test_below_bl_only, :275-331);
  N^2 = 5e-6 everywhere: n2_thresh 0 and 1e-6 leave the background, 1e-5
      sets kd_conv, to 1e-9 (test_n2_thresh_live, :333-396);
  a 20-layer inversion (rho = T from 1028 to 1030) diffused 7 x 1200 s with
      the fixed kt: spread below 0.6 with convection, above 1.5 with PP81
      alone, column heat conserved to 1e-9 relative in both
      (test_homogenises_inversion, :398-515);
  two adjacent layers pinched to 1e-6 m across a strong inversion: the
      interface between them keeps PP81's value, finite
      (test_vanished_interface_skipped, :517-585).
"""
import numpy as np

from roundabout_b200.config import default_config

NX, NY = 8, 6
PP81_UNSTABLE_KT = 1.0e-5 + 1.0e-2    # pp81_kappa_bg + pp81_nu0 at Ri < 0
GRAVITY = 9.80665


def cfg(**kw):
    c = default_config()
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def column(oracle, rho, h=10.0, bld=0.0):
    nz = len(rho)
    st = oracle.OracleState(NX, NY, nz, 2)
    if np.isscalar(h):
        st.h[...] = h
    else:
        for k, hk in enumerate(h):
            st.h[:, :, k] = hk
    for k, r in enumerate(rho):
        st.rho[:, :, k] = r
    st.bl_depth[...] = bld
    return st


def run(st, c, conv=True):
    st.call("vpo_pp81", c)
    if conv:
        st.call("vpo_convection", c)
    st.call("vpo_split", c)
    assert st.call("vpo_assemble_gate", c) == 0
    return st


def test_disabled_convection_changes_nothing(oracle):
    rho = [1030.0 + k for k in range(4)]
    a = run(column(oracle, rho), cfg(conv_enable=0, conv_kd=1.0))
    b = run(column(oracle, rho), cfg(), conv=False)
    assert np.abs(a.kv - b.kv).max() < 1.0e-15 and np.abs(a.kt - b.kt).max() < 1.0e-15


def test_stable_column_untouched(oracle):
    rho = [1030.0 - k for k in range(4)]
    a = run(column(oracle, rho), cfg(conv_enable=1, conv_kd=1.0))
    b = run(column(oracle, rho), cfg(), conv=False)
    assert np.abs(a.kv - b.kv).max() < 1.0e-15 and np.abs(a.kt - b.kt).max() < 1.0e-15


def test_inverted_column_takes_kd_conv_and_its_prandtl(oracle):
    KD, PR = 1.0, 2.0
    st = run(column(oracle, [1030.0 + k for k in range(4)]), cfg(conv_enable=1, conv_kd=KD, conv_prandtl=PR))
    assert np.abs(st.kt[4, 3, 1:4] - KD).max() < 1.0e-12
    assert np.abs(st.kv[4, 3, 1:4] - PR * KD).max() < 1.0e-12
    for k in (0, 4):
        assert np.abs(st.kt[:, :, k]).max() < 1.0e-15 and np.abs(st.kv[:, :, k]).max() < 1.0e-15


def test_only_interfaces_below_the_boundary_layer_convect(oracle):
    nz = 10
    st = run(column(oracle, [1028.0 + k for k in range(nz)], h=20.0, bld=100.0), cfg(conv_enable=1, conv_kd=1.0))
    for k in range(7, nz + 1):      # 1-based interfaces 20, 40, 60, 80 m deep
        assert abs(st.kt[4, 3, k - 1] - PP81_UNSTABLE_KT) < 1.0e-10, k
    for k in range(2, 7):           # 100 m (the >= edge) down to 180 m
        assert abs(st.kt[4, 3, k - 1] - 1.0) < 1.0e-10, k


def test_n2_threshold_is_live(oracle):
    H, N2 = 10.0, 5.0e-6
    c0 = cfg()
    drho = N2 * c0.rho0 * H / GRAVITY
    rho = [1030.0 - drho * k for k in range(4)]
    for thresh, expect in ((0.0, c0.pp81_kappa_bg), (1.0e-6, c0.pp81_kappa_bg), (1.0e-5, 1.0)):
        st = run(column(oracle, rho, h=H), cfg(conv_enable=1, conv_kd=1.0, conv_n2_thresh=thresh))
        assert abs(st.kt[4, 3, 1] - expect) < 1.0e-9, thresh


def test_convection_homogenises_an_inversion(oracle):
    NZ, H, DT, NSTEPS = 20, 10.0, 1200.0, 7
    t0 = [1028.0 + 2.0 * k / (NZ - 1) for k in range(NZ)]
    spread, total = [], []
    for conv in (1, 0):
        c = cfg(conv_enable=conv, conv_kd=1.0)
        st = column(oracle, t0, h=H)
        for k in range(NZ):
            st.tracers[c.idx_temperature][:, :, k] = t0[k]
        run(st, c, conv=bool(conv))
        for _ in range(NSTEPS):     # the kt of one build held fixed
            st.call("vpo_vdiff_tracers", c, DT)
        t = st.tracers[c.idx_temperature][4, 3, :]
        spread.append(t.max() - t.min())
        total.append(t.sum() * H)
    assert spread[0] < 0.6
    assert spread[1] > 1.5
    total0 = sum(t0) * H
    assert all(abs(tot - total0) < 1.0e-9 * abs(total0) for tot in total)


def test_pinched_interface_keeps_the_pp81_value(oracle):
    st = run(column(oracle, [1028.0, 1028.0, 1040.0, 1040.0], h=[10.0, 1.0e-6, 1.0e-6, 10.0]),
             cfg(conv_enable=1, conv_kd=1.0))
    kt = st.kt[4, 3, 2]             # 1-based interface 3, between the pinched layers
    assert np.isfinite(kt)
    assert abs(kt - PP81_UNSTABLE_KT) < 1.0e-9
    assert abs(kt - 1.0) > 0.5
