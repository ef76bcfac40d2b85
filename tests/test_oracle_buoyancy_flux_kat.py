"""The oracle's KPP surface buoyancy flux B0 = (g / rho0)(alpha_T F_T -
beta_S F_S), with F_T = Q_heat / (rho0 cp) and F_S = Q_salt / rho0 and
dimensional (kg m^-3 per K, per psu) alpha_T and beta_S, against the
reference's known-answer tests (tests/test_ocean_buoyancy_flux.F90),
re-expressed on the oracle (the Fortran tests cannot run here: no Fortran
compiler).

Checked quantities and tolerances are the reference tests' own, with
rho0 = 1035, cp = 3992, alpha_T = 0.2 and beta_S = 0.8:
  8 layers of 20 m, cooling 150 W m^-2 and salting 2e-5 kg m^-2 s^-1: B0 is
      negative and is the documented convention to 1e-14 relative
      (test_kpp_matches_epbl, :172-249; its comparison with EPBL's own B0
      needs that scheme's B0 field, which the oracle state does not hold);
  a neutral resting column of 10 layers of 20 m under 100 W m^-2 of
      cooling and no wind: the boundary layer is the whole 200 m to 1e-10,
      B0 the convention to 1e-13, the kv at the interface 60 m deep
      h_b w* G(0.3) with w* = (-B0 h_b)^(1/3) to 1e-10, and the hand values
      B0 = -4.586480e-8, w* = 0.0209333 to 1e-5 (test_wstar_analytic,
      :251-350).
"""
from roundabout_b200.config import default_config

G = 9.80665
RHO0, CP, ALPHA, BETA = 1035.0, 3992.0, 0.2, 0.8


def kpp_column(oracle, nz, dz, q_heat, q_salt):
    c = default_config()
    c.use_kpp = 1
    c.rho0 = RHO0
    c.cp = CP
    c.alpha_T = ALPHA
    c.beta_S = BETA
    st = oracle.OracleState(8, 6, nz, 2)
    st.h[...] = dz
    st.rho[...] = RHO0
    st.tracers[c.idx_temperature][...] = 12.0
    st.tracers[c.idx_salinity][...] = 35.0
    st.kv[...] = 0.0
    st.kt[...] = 0.0
    st.q_heat[...] = q_heat
    st.q_salt[...] = q_salt
    st.call("vpo_kpp_overlay", c)
    return st


def test_cooling_and_salting_give_the_documented_b0(oracle):
    Q_HEAT, Q_SALT = -150.0, 2.0e-5
    st = kpp_column(oracle, 8, 20.0, Q_HEAT, Q_SALT)
    b0 = st.b0[4, 3]
    assert b0 < 0.0
    want = (G / RHO0) * (ALPHA * (Q_HEAT / (RHO0 * CP)) - BETA * (Q_SALT / RHO0))
    assert abs(b0 - want) <= 1.0e-14 * abs(b0)


def test_convective_wstar_from_the_analytic_b0(oracle):
    NZ, DZ, Q_HEAT, K_PROBE, SIGMA = 10, 20.0, -100.0, 8, 0.3
    H = NZ * DZ
    g_probe = SIGMA * (1.0 - SIGMA) ** 2
    b0_expect = (G / RHO0) * ALPHA * (Q_HEAT / (RHO0 * CP))
    wstar_expect = (-b0_expect * H) ** (1.0 / 3.0)
    kv_expect = H * wstar_expect * g_probe
    assert abs(b0_expect - -4.586480e-8) <= 1.0e-5 * 4.586480e-8
    assert abs(wstar_expect - 0.0209333) <= 1.0e-5 * 0.0209333
    st = kpp_column(oracle, NZ, DZ, Q_HEAT, 0.0)
    assert abs(st.bl_depth[4, 3] - H) <= 1.0e-10 * H
    assert abs(st.b0[4, 3] - b0_expect) <= 1.0e-13 * abs(b0_expect)
    kv = st.kv[4, 3, K_PROBE - 1]
    assert abs(kv - kv_expect) <= 1.0e-10 * kv_expect
    assert abs(kv / (H * g_probe) - wstar_expect) <= 1.0e-10 * wstar_expect
