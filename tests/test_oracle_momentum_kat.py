"""The oracle's momentum sweep against the reference's known-answer tests for
the implicit surface stress and bottom drag folded into the vertical-friction
tridiagonal (tests/test_ocean_vdiff_implicit_stress_drag.F90), re-expressed
on the oracle (the Fortran tests cannot run here: no Fortran compiler).

The reference is bottom-up: level 1 is the bed (the drag goes on its
diagonal), level nz the surface (the stress goes into its right-hand side);
the oracle's arrays use the same order.  The viscosity is a constant on the
interior interfaces (the reference's scalar K_v_momentum), zero on the bed and
surface interfaces.  Tolerances and the checked quantities are the reference
tests' own:
  (a) thin bed layer, strong quadratic drag, dt c_d |U| / h = 6 with Picard
      updates of the drag rate over 50 steps: the bed velocity stays in
      (0, U0] and decays monotonically (test_thin_layer_drag_bounded, :83-174);
  (b) thick layers, small drag and stress, no viscosity: the bed matches the
      explicit decay U0 (1 - dt lam) to 1e-6 U0 and the surface matches
      U0 + dt tau / (rho0 h) to 1e-12 (test_well_resolved_equivalence, :176-239);
  (c) the knobs off: large drag rates and stresses in the fields change
      nothing, bit for bit (test_default_off_bit_identity, :241-308);
  (d) eastward stress lands on the surface with the sign of tau, the bed
      untouched without viscosity, and diffuses down with it
      (test_stress_placement_and_sign, :310-389);
  (e) a face touching land takes no stress, an all-wet face the full
      increment (test_stress_land_masked, :391-454);
and from tests/test_ocean_vdiff_bbl.F90 (the harmonic face thickness and the
bottom-boundary-layer glue, with the viscous remnant gamma):
  (f) thickening layers, strong drag, hvel_mom6: gamma finite, in (0, 1],
      non-decreasing from the bed up and strictly smaller at the bed
      (test_hvel_mom6_bounded, :119-185);
  (g) the glue on a thin bed sliver: gamma finite and in (0, 1]
      (test_bbl_glue_finite, :187-252);
  (h) the glue's piston damps the bed velocity harder than the plain drag
      (test_bbl_glue_damps, :254-331);
  (i) an exactly collapsed interior layer with viscosity across it (the
      arithmetic face thickness is 0 there): gamma finite and in (0, 1]
      (test_collapsed_layer_finite, :458-522).
"""
import numpy as np

from roundabout_b200.config import default_config

NZ = 6
RHO0 = 1035.0


def cfg(**kw):
    c = default_config()
    c.rho0 = RHO0
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def state(oracle, h, nx=4, ny=4):
    st = oracle.OracleState(nx, ny, NZ, 1)
    st.h[...] = h
    return st


def interior_kv(st, kv):
    st.kv[...] = kv
    st.kv[:, :, 0] = 0.0
    st.kv[:, :, -1] = 0.0


def test_implicit_drag_thin_bed_layer_bounded_and_monotone(oracle):
    H1, CD, U0, DT = 2.0, 2.5e-3, 8.0, 600.0
    # the explicit forward-Euler factor flips the sign and grows here
    u_explicit = U0 * (1.0 - DT * CD * U0 / H1)
    assert u_explicit < 0.0 and abs(u_explicit) > U0
    c = cfg(implicit_drag=1)
    st = state(oracle, H1)
    interior_kv(st, 0.0)
    st.u[...] = U0
    u_prev = U0
    for _ in range(50):
        st.lambda_bot_u[...] = CD * abs(st.u[1, 1, 0]) / H1   # Picard: the rate from the current bed speed
        st.call("vpo_vdiff_momentum", c, DT)
        u_bed = st.u[1, 1, 0]
        assert np.isfinite(u_bed)
        assert 0.0 <= u_bed <= U0 + 1e-12
        assert u_bed <= u_prev + 1e-12
        u_prev = u_bed
    assert 0.0 < u_prev < U0


def test_implicit_drag_and_stress_match_explicit_when_well_resolved(oracle):
    H0, U0, DT, LAM, TAUX = 100.0, 0.5, 1.0, 1.0e-3, 0.1
    c = cfg(implicit_drag=1, implicit_stress=1)
    st = state(oracle, H0)
    interior_kv(st, 0.0)
    st.u[...] = U0
    st.lambda_bot_u[...] = LAM
    st.lambda_bot_v[...] = LAM
    st.tau_x[...] = TAUX
    st.call("vpo_vdiff_momentum", c, DT)
    assert abs(st.u[1, 1, 0] - U0 * (1.0 - DT * LAM)) < 1.0e-6 * abs(U0)
    assert abs(st.u[1, 1, NZ - 1] - (U0 + DT * TAUX / (RHO0 * H0))) < 1.0e-12


def test_fold_fields_ignored_with_the_knobs_off(oracle):
    H0, DT = 10.0, 60.0
    c = cfg(implicit_drag=0, implicit_stress=0)
    a = state(oracle, H0, nx=6)
    b = state(oracle, H0, nx=6)
    for s in (a, b):
        interior_kv(s, 1.0e-2)
        for k in range(NZ):
            s.u[:, :, k] = 0.1 * (k + 1)
            s.v[:, :, k] = -0.05 * (k + 1)
    b.lambda_bot_u[...] = 5.0   # large drag rates and stresses that must be ignored
    b.lambda_bot_v[...] = 5.0
    b.tau_x[...] = 10.0
    b.tau_y[...] = 10.0
    a.call("vpo_vdiff_momentum", c, DT)
    b.call("vpo_vdiff_momentum", c, DT)
    assert np.array_equal(a.u, b.u) and np.array_equal(a.v, b.v)


def test_implicit_stress_lands_on_the_surface_with_its_sign(oracle):
    H0, DT, TAUX = 10.0, 600.0, 0.2
    c = cfg(implicit_stress=1)
    st = state(oracle, H0)
    interior_kv(st, 0.0)
    st.tau_x[...] = TAUX
    st.call("vpo_vdiff_momentum", c, DT)
    u_surf, u_bed = st.u[1, 1, NZ - 1], st.u[1, 1, 0]
    assert u_surf > 0.0
    assert abs(u_bed) < 1.0e-14
    assert abs(u_surf - DT * TAUX / (RHO0 * H0)) < 1.0e-12
    # with interior viscosity the momentum diffuses down from the surface
    st.u[...] = 0.0
    st.v[...] = 0.0
    interior_kv(st, 1.0e-1)
    st.call("vpo_vdiff_momentum", c, DT)
    u_surf, u_mid, u_bed = st.u[1, 1, NZ - 1], st.u[1, 1, NZ // 2 - 1], st.u[1, 1, 0]
    assert u_surf > u_mid > 0.0 and u_bed > 0.0


def test_implicit_stress_skips_faces_touching_land(oracle):
    H0, TAUX, DT = 50.0, 0.1, 1.0
    c = cfg(implicit_stress=1)
    st = state(oracle, H0)
    interior_kv(st, 0.0)
    st.wet[2, 1] = 0.0          # u face 2 of row 1 lies between cells 1 and 2: a land face
    st.tau_x[...] = TAUX
    st.call("vpo_vdiff_momentum", c, DT)
    assert abs(st.u[2, 1, NZ - 1]) < 1.0e-14
    assert abs(st.u[1, 1, NZ - 1] - DT * TAUX / (RHO0 * H0)) < 1.0e-12


def remnant_ok(g):
    return bool(np.isfinite(g).all() and (g > 0.0).all() and (g <= 1.0 + 1e-12).all())


def test_remnant_with_harmonic_faces_bounded_and_monotone(oracle):
    nz, DT, LAM = 6, 450.0, 0.08
    c = cfg(implicit_drag=1, hvel_mom6=1, remnant=1)
    st = oracle.OracleState(4, 4, nz, 1)
    for k in range(nz):
        st.h[:, :, k] = 12.0 * (k + 1)
    interior_kv(st, 0.2)
    st.lambda_bot_u[...] = LAM
    st.lambda_bot_v[...] = LAM
    st.call("vpo_vdiff_momentum", c, DT)
    g = st.visc_rem_u[1, 1, :]
    assert remnant_ok(g)
    assert all(g[k] >= g[k - 1] - 1e-13 for k in range(1, nz))
    assert g[0] < g[-1] - 1e-10


def test_glue_remnant_finite_on_a_thin_bed_sliver(oracle):
    c = cfg(implicit_drag=1, hvel_mom6=1, bbl_glue=1, remnant=1)
    st = oracle.OracleState(4, 4, 4, 1)
    for k, hk in enumerate((0.05, 1.0, 10.0, 25.0)):
        st.h[:, :, k] = hk
    interior_kv(st, 0.1)
    st.lambda_bot_u[...] = 0.02
    st.lambda_bot_v[...] = 0.02
    st.call("vpo_vdiff_momentum", c, 600.0)
    assert np.isfinite(st.visc_rem_u[1, 1, :]).all() and np.isfinite(st.visc_rem_v[1, 1, :]).all()
    assert remnant_ok(st.visc_rem_u[1, 1, :])


def test_glue_damps_the_bed_harder_than_the_plain_drag(oracle):
    DT, LAM, U0 = 300.0, 0.01, 0.5
    bed = []
    for glue in (0, 1):
        c = cfg(implicit_drag=1, hvel_mom6=1, bbl_glue=glue)
        st = oracle.OracleState(4, 4, 4, 1)
        for k, hk in enumerate((0.2, 5.0, 15.0, 25.0)):
            st.h[:, :, k] = hk
        interior_kv(st, 1.0e-4)   # below the glue's kv_bbl = bbl_piston * hbbl_visc = 3e-3
        st.u[...] = U0
        st.lambda_bot_u[...] = LAM
        st.lambda_bot_v[...] = LAM
        st.call("vpo_vdiff_momentum", c, DT)
        bed.append(st.u[1, 1, 0])
    assert 0.0 < bed[0] < U0
    assert bed[1] < bed[0] - 1e-6


def test_collapsed_interior_layer_keeps_the_remnant_finite(oracle):
    c = cfg(hvel_mom6=0, remnant=1)
    st = oracle.OracleState(4, 4, 4, 1)
    for k, hk in enumerate((10.0, 0.0, 12.0, 20.0)):
        st.h[:, :, k] = hk
    interior_kv(st, 0.2)
    st.call("vpo_vdiff_momentum", c, 450.0)
    assert remnant_ok(st.visc_rem_u[1, 1, :]) and remnant_ok(st.visc_rem_v[1, 1, :])
