"""The oracle's Wright (1997) equation of state against the known-answer
tests of tests/test_ocean_wright_eos.F90 that tests/test_oracle_kat.py does
not already restate, re-expressed on the oracle (the Fortran tests cannot
run here: no Fortran compiler).  Surface pressure (p_ref = 0) throughout.
Checked quantities and thresholds are the reference tests' own:
  5 K warmer is lighter and 3 psu saltier is denser than (10 C, 35 psu)
      (test_monotonic_ts, :136-173);
  (0 C, 33 psu) and (20 C, 36.5 psu) blended to their mean are denser than
      the mean of their densities by more than 0.05 kg m^-3
      (test_cabbeling, :175-223);
  one pinched cell (h = 0) takes rho0 to 1e-12 while its neighbour stays
      between 1020 and 1035 (test_vanishing_layer, :225-261).
"""
from roundabout_b200.config import default_config


def rho_at(oracle, t, s):
    c = default_config()
    c.eos_p_ref = 0.0
    st = oracle.OracleState(8, 8, 3, 2)
    st.h[...] = 10.0
    st.tracers[c.idx_temperature][...] = t
    st.tracers[c.idx_salinity][...] = s
    st.call("vpo_eos_wright", c)
    return st.rho[0, 0, 0]


def test_warmer_is_lighter_and_saltier_is_denser(oracle):
    base = rho_at(oracle, 10.0, 35.0)
    assert rho_at(oracle, 15.0, 35.0) < base
    assert rho_at(oracle, 10.0, 38.0) > base


def test_cabbeling(oracle):
    ta, sa, tb, sb = 0.0, 33.0, 20.0, 36.5
    mean_of_rho = 0.5 * (rho_at(oracle, ta, sa) + rho_at(oracle, tb, sb))
    assert rho_at(oracle, 0.5 * (ta + tb), 0.5 * (sa + sb)) > mean_of_rho + 0.05


def test_one_pinched_cell_takes_rho0(oracle):
    c = default_config()
    c.eos_p_ref = 0.0
    c.rho0 = 1035.0
    st = oracle.OracleState(8, 8, 3, 2)
    st.h[...] = 10.0
    st.tracers[c.idx_temperature][...] = 10.0
    st.tracers[c.idx_salinity][...] = 35.0
    st.h[0, 0, 0] = 0.0
    st.call("vpo_eos_wright", c)
    assert abs(st.rho[0, 0, 0] - c.rho0) < 1.0e-12
    assert 1020.0 < st.rho[1, 0, 0] < 1035.0
