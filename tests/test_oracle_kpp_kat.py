"""The oracle's KPP overlay and non-local term against the known-answer tests
of tests/test_ocean_kpp.F90 and tests/test_ocean_kpp_nonlocal.F90 that
tests/test_oracle_kat.py does not already restate, re-expressed on the
oracle (the Fortran tests cannot run here: no Fortran compiler).

Bottom-up like the reference: level 1 is the bed, nz the surface; the
boundary-layer depth starts at zero (a fresh vmix), so the first overlay's
w* is zero.  Checked quantities and tolerances are the reference tests' own:
  a 75 m mixed layer (u 0.5, rho 1027) over a stratified interior, wind
      0.1 Pa: h_b below the top layer, above the bed, kv above 5 nu_bg
      (test_strat_bl_depth, :152-225);
  6 layers of 5 m, rho = 1030 - 0.2 (k - 1), wind 0.05 Pa and 200 W m^-2 of
      cooling: V_t^2 on (c_vt2 1.8) deepens h_b by more than 1e-6 over off
      (test_vt2_deepens_bl, :374-434);
  the same column unforced: c_vt2 0 and 10 give h_b equal to 1e-13
      (test_vt2_no_forcing_invariant, :436-481);
  wind 0.05 Pa and 150 W m^-2 of cooling: h_b non-decreasing over c_vt2 =
      0, 1.8, 5 and growing by more than 1e-6 (test_vt2_monotonic_in_
      coefficient, :483-546);
  300 W m^-2 of cooling on the west half only, two overlays so the first
      seeds the lagged h_b: the west h_b deeper than the east by more than
      1e-6 (test_half_domain_cooling, :548-609);
  the mixed layer of test_ocean_kpp_nonlocal.F90 (setup_state, :69-105)
      under 500 W m^-2 of cooling and 0.1 Pa of wind: gamma_t negative
      somewhere, and the non-local term alone (dt 100 s) warms the surface
      layer and cools the one below (test_cooling_redistributes, :175-233);
      gamma_t and gamma_s zero (below 1e-15) on every interface at or below
      h_b (test_zero_outside_bl, :271-319).
"""
import numpy as np

from roundabout_b200.config import default_config


def kcfg(**kw):
    c = default_config()
    c.use_kpp = 1
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def stratified(oracle, c, nx=12, ny=10, nz=6, tau=0.05, q_heat=0.0):
    """setup_stratified_column (test_ocean_kpp.F90:358-372)."""
    st = oracle.OracleState(nx, ny, nz, 2)
    st.seed_backgrounds(c)
    st.h[...] = 5.0
    for k in range(1, nz + 1):
        st.rho[:, :, k - 1] = 1030.0 - 0.2 * (k - 1)
    st.stress_mag[...] = tau
    st.q_heat[...] = q_heat
    return st


def pp81_kpp(st, c):
    st.call("vpo_pp81", c)
    st.call("vpo_kpp_overlay", c)
    return st


def mixed_layer(oracle, c, nx=14, ny=12, nz=8, tau=0.1, q_heat=0.0):
    """A 3-layer mixed layer over a stratified interior, 25 m layers."""
    st = oracle.OracleState(nx, ny, nz, 2)
    st.seed_backgrounds(c)
    st.h[...] = 25.0
    for k in range(1, nz + 1):
        if k > nz - 3:
            st.u[:, :, k - 1] = 0.5
            st.rho[:, :, k - 1] = 1027.0
        else:
            st.rho[:, :, k - 1] = 1030.0 - 0.5 * (k - 1)
        st.tracers[c.idx_salinity][:, :, k - 1] = 35.0
        st.tracers[c.idx_temperature][:, :, k - 1] = 18.0
    st.stress_mag[...] = tau
    st.q_heat[...] = q_heat
    return st


def test_stratified_bl_depth_inside_the_column(oracle):
    c = kcfg()
    st = pp81_kpp(mixed_layer(oracle, c), c)
    hb = st.bl_depth[7, 6]
    assert 25.0 < hb < 8 * 25.0
    assert st.kv[7, 6, 1:8].max() > 5.0 * c.pp81_nu_bg


def test_vt2_deepens_the_bl(oracle):
    hb = []
    for cvt2 in (0.0, 1.8):
        c = kcfg(c_vt2=cvt2)
        hb.append(pp81_kpp(stratified(oracle, c, q_heat=-200.0), c).bl_depth[6, 5])
    assert hb[1] >= hb[0]
    assert hb[1] > hb[0] + 1.0e-6


def test_vt2_without_forcing_changes_nothing(oracle):
    out = []
    for cvt2 in (0.0, 10.0):
        c = kcfg(c_vt2=cvt2)
        out.append(pp81_kpp(stratified(oracle, c, tau=0.0, q_heat=0.0), c).bl_depth.copy())
    assert np.abs(out[0] - out[1]).max() < 1.0e-13


def test_vt2_monotonic_in_its_coefficient(oracle):
    hb = []
    for cvt2 in (0.0, 1.8, 5.0):
        c = kcfg(c_vt2=cvt2)
        hb.append(pp81_kpp(stratified(oracle, c, q_heat=-150.0), c).bl_depth[6, 5])
    assert hb[1] >= hb[0] and hb[2] >= hb[1]
    assert hb[2] > hb[0] + 1.0e-6


def test_half_domain_cooling_deepens_the_cooled_half(oracle):
    nx, ny = 16, 12
    c = kcfg()
    st = stratified(oracle, c, nx=nx, ny=ny, q_heat=0.0)
    st.q_heat[: nx // 2, :] = -300.0
    pp81_kpp(st, c)          # seeds the lagged h_b
    pp81_kpp(st, c)          # builds w* from it
    west, east = st.bl_depth[nx // 2 - 2, ny // 2 - 1], st.bl_depth[nx // 2 + 1, ny // 2 - 1]
    assert west > east + 1.0e-6


def test_nonlocal_cooling_warms_the_surface_and_cools_below(oracle):
    c = kcfg()
    st = mixed_layer(oracle, c, q_heat=-500.0)
    t0 = st.tracers[c.idx_temperature].copy()
    st.call("vpo_kpp_overlay", c)
    assert st.gamma_t.min() < 0.0
    st.call("vpo_nonlocal", c, 100.0)
    dt = st.tracers[c.idx_temperature][7, 6, :] - t0[7, 6, :]
    assert dt[7] > 0.0
    assert dt[6] < 0.0


def test_nonlocal_gamma_zero_at_and_below_the_bl(oracle):
    c = kcfg()
    st = mixed_layer(oracle, c, q_heat=-500.0)
    st.call("vpo_kpp_overlay", c)
    worst = 0.0
    nz = st.nz
    for j in range(st.ny):
        for i in range(st.nx):
            hb, d = st.bl_depth[i, j], 0.0
            for k in range(nz, 1, -1):      # 1-based interface k, the bottom of layer k
                d += st.h[i, j, k - 1]
                if d >= hb:
                    worst = max(worst, abs(st.gamma_t[i, j, k - 1]), abs(st.gamma_s[i, j, k - 1]))
    assert worst < 1.0e-15
