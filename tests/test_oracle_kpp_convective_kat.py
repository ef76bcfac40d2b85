"""The oracle's KPP overlay with the convective velocity scale against the
reference's known-answer tests (tests/test_ocean_kpp_convective.F90),
re-expressed on the oracle (the Fortran tests cannot run here: no Fortran
compiler).

The column of those tests (setup_state, :53-84): 8 layers of 25 m,
bottom-up; the top three carry u = 0.5 m/s and rho = 1027, the ones below
u = 0 and rho = 1030 - 0.5 (k - 1) for 1-based k; 14 x 12 columns.  The
surface buoyancy flux B0 sets w*^3 = max(0, -B0) h_b, and w_s = sqrt(u*^2 +
w*^2) scales the boundary-layer diffusivity.  Checked quantities and
tolerances are the reference tests' own:
  heating (B0 > 0, w* = 0) changes kv by less than 1e-12 against no flux
      (test_stabilizing_no_op, :130-164);
  cooling without wind lifts the interior kv above 10 x the PP81 background
      (test_cooling_deepens, :166-199);
  wind and cooling together give a larger maximum kv than the wind alone
      (test_combined_exceeds_shear, :201-239).
"""
import numpy as np

from roundabout_b200.config import default_config

NX, NY, NZ = 14, 12, 8


def column(oracle, tau, q_heat):
    st = oracle.OracleState(NX, NY, NZ, 2)
    st.h[...] = 25.0
    for k in range(NZ):
        if k >= NZ - 3:
            st.u[:, :, k] = 0.5
            st.rho[:, :, k] = 1027.0
        else:
            st.rho[:, :, k] = 1030.0 - 0.5 * k
    st.stress_mag[...] = tau
    st.q_heat[...] = q_heat
    return st


def kpp(oracle, tau, q_heat):
    c = default_config()
    c.use_kpp = 1
    st = column(oracle, tau, q_heat)
    st.call("vpo_pp81", c)
    st.call("vpo_kpp_overlay", c)
    return c, st


def test_stabilising_flux_leaves_kv_as_the_shear_only_overlay(oracle):
    _, shear = kpp(oracle, 0.1, 0.0)
    _, heated = kpp(oracle, 0.1, 500.0)
    assert np.abs(heated.kv - shear.kv).max() < 1.0e-12


def test_cooling_without_wind_lifts_kv_above_the_background(oracle):
    c, st = kpp(oracle, 0.0, -500.0)
    assert st.kv[:, :, 1:NZ].max() > 10.0 * c.pp81_nu_bg


def test_wind_and_cooling_exceed_the_wind_alone(oracle):
    _, shear = kpp(oracle, 0.1, 0.0)
    _, both = kpp(oracle, 0.1, -500.0)
    assert both.kv[:, :, 1:NZ].max() > shear.kv[:, :, 1:NZ].max()
