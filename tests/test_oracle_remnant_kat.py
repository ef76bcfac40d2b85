"""The oracle's viscous remnant (the momentum sweep's gamma = M^-1 1, the
share of a depth-uniform acceleration each layer keeps after the implicit
friction) against the reference's known-answer tests
(tests/test_ocean_visc_rem.F90), re-expressed on the oracle (the Fortran
tests cannot run here: no Fortran compiler).

Bottom-up like the reference: level 1 is the bed, nz the surface.  The
viscosity is a constant on the interior interfaces (the reference's scalar
K_v_momentum); the reference runs these cases with the arithmetic face
thickness (hvel_mom6 off) except the glue's closed form.  Checked quantities
and tolerances are the reference tests' own:
  no drag: gamma = 1 to 1e-12 for any viscosity, thicknesses and dt
      (test_no_drag_remnant_is_one, :120-160);
  near no-slip bed drag, constant viscosity: gamma follows
      1 - exp(-z / sqrt(nu dt)) away from the bed and the surface to 0.03
      (test_analytic_profile, :162-224);
  drag with nu = 0, 0.02, 2: gamma finite, in (0, 1], non-decreasing from
      the bed up, strictly smaller at the bed (test_bounded_and_monotone,
      :226-300);
  asking for the remnant leaves the momentum solve bit for bit unchanged
      (test_absent_is_bit_identical, :302-366);
  gamma equals the finite-difference response of the solve to a uniform
      acceleration to 1e-9 (test_consistent_with_definition, :368-440);
  one layer with linear drag: gamma = 1 / (1 + dt r) to 1e-13
      (test_pr1_single_layer_closed_form, :543-600);
  two layers coupled only by the glue's piston: gamma from the 2x2 system
      by Cramer's rule to 1e-10 (test_pr1_two_layer_bbl_glue_closed_form,
      :602-692).
"""
import math

import numpy as np

from roundabout_b200.config import default_config

RHO0 = 1035.0


def cfg(**kw):
    c = default_config()
    c.rho0 = RHO0
    c.hvel_mom6 = 0
    c.remnant = 1
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def column(oracle, hs, kv, nx=4, ny=4):
    st = oracle.OracleState(nx, ny, len(hs), 1)
    for k, hk in enumerate(hs):
        st.h[:, :, k] = hk
    st.kv[...] = kv
    st.kv[:, :, 0] = 0.0
    st.kv[:, :, -1] = 0.0
    return st


def drag(st, lam):
    st.lambda_bot_u[...] = lam
    st.lambda_bot_v[...] = lam


def test_remnant_is_one_without_drag(oracle):
    st = column(oracle, [17.0 * (k + 1) for k in range(5)], 3.5)
    st.call("vpo_vdiff_momentum", cfg(implicit_drag=0), 900.0)
    dev = max(np.abs(st.visc_rem_u - 1.0).max(), np.abs(st.visc_rem_v - 1.0).max())
    assert dev < 1.0e-12


def test_remnant_follows_the_no_slip_profile(oracle):
    NZ, DZ, NU, DT = 40, 2.0, 0.1, 1000.0
    st = column(oracle, [DZ] * NZ, NU)
    drag(st, 1.0e6)
    st.call("vpo_vdiff_momentum", cfg(implicit_drag=1), DT)
    delta = math.sqrt(NU * DT)
    err = max(abs(st.visc_rem_u[1, 1, k - 1] - (1.0 - math.exp(-((k - 0.5) * DZ) / delta)))
              for k in range(8, NZ))
    assert err < 0.03


def test_remnant_bounded_and_monotone(oracle):
    for nu in (0.0, 0.02, 2.0):
        st = column(oracle, [12.0 * (k + 1) for k in range(6)], nu)
        drag(st, 0.08)
        st.call("vpo_vdiff_momentum", cfg(implicit_drag=1), 450.0)
        g = st.visc_rem_u[1, 1, :]
        assert np.isfinite(g).all() and (g > 0.0).all() and (g <= 1.0 + 1e-12).all(), nu
        assert all(g[k] >= g[k - 1] - 1e-13 for k in range(1, 6)), nu
        assert g[0] < g[-1] - 1e-10, nu


def test_asking_for_the_remnant_leaves_the_solve_unchanged(oracle):
    out = []
    for rem in (0, 1):
        st = column(oracle, [8.0 * (k + 1) for k in range(6)], 2.0e-2)
        for k in range(6):
            st.u[:, :, k] = 0.2 * (k + 1)
            st.v[:, :, k] = -0.1 * (k + 1)
        drag(st, 0.02)
        st.call("vpo_vdiff_momentum", cfg(implicit_drag=1, remnant=rem), 300.0)
        out.append((st.u.copy(), st.v.copy()))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_remnant_is_the_response_to_a_uniform_acceleration(oracle):
    NZ, DT, ABAR = 8, 240.0, 0.37
    du = DT * ABAR
    runs = []
    for shift in (0.0, du):
        st = column(oracle, [9.0 * (k + 1) for k in range(NZ)], 0.15)
        for k in range(NZ):
            st.u[:, :, k] = 0.3 * math.sin(k + 1) + shift
        drag(st, 0.03)
        st.call("vpo_vdiff_momentum", cfg(implicit_drag=1), DT)
        runs.append(st)
    fd = (runs[1].u[1, 1, :] - runs[0].u[1, 1, :]) / du
    assert np.abs(fd - runs[0].visc_rem_u[1, 1, :]).max() < 1.0e-9


def test_single_layer_remnant_closed_form(oracle):
    DT, R = 1800.0, 2.5e-4
    st = column(oracle, [37.0], 0.3)
    drag(st, R)
    st.call("vpo_vdiff_momentum", cfg(implicit_drag=1), DT)
    expect = 1.0 / (1.0 + DT * R)
    assert max(abs(st.visc_rem_u[1, 1, 0] - expect), abs(st.visc_rem_v[1, 1, 0] - expect)) < 1.0e-13


def test_two_layer_glue_remnant_closed_form(oracle):
    DT, H1, H2, HBBL, PISTON, EPS = 1000.0, 8.0, 15.0, 5.0, 2.0e-4, 1.0e-30
    c = cfg(implicit_drag=0, hvel_mom6=1, hvel_harmonic=0, bbl_glue=1, hbbl_visc=HBBL, bbl_piston=PISTON,
            kv_bbl_bg=0.0)
    st = column(oracle, [H1, H2], 0.0)
    st.call("vpo_vdiff_momentum", c, DT)
    # the 2x2 system by Cramer's rule, independently of the Thomas sweep
    kv_bbl = PISTON * HBBL
    zint1 = H1 * (1.0 / (HBBL + EPS))
    botfn = 1.0 / (1.0 + 0.09 * zint1 ** 6)
    nu_eff = max(0.0, kv_bbl * botfn)
    dz = 0.5 * (H1 + H2)
    if dz > HBBL:
        dz = (1.0 - botfn) * dz + botfn * HBBL
    alpha = DT * nu_eff / (H1 * dz)
    beta = DT * nu_eff / (H2 * dz)
    bed = DT * kv_bbl / (H1 * (min(0.5 * H1, HBBL) + EPS))
    b1, c1, a2, b2 = 1.0 + alpha + bed, -alpha, -beta, 1.0 + beta
    det = b1 * b2 - c1 * a2
    g1, g2 = (b2 - c1) / det, (b1 - a2) / det
    for g in (st.visc_rem_u, st.visc_rem_v):
        assert abs(g[1, 1, 0] - g1) < 1.0e-10 and abs(g[1, 1, 1] - g2) < 1.0e-10
