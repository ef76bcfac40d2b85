"""The CPU oracle against the reference's own known-answer tests for the path,
re-expressed here (the Fortran tests cannot run: no Fortran compiler).

Cases follow, in order: tests/test_ocean_pp81.F90:42-53, test_ocean_kpp.F90:40-57
(no wind, unstratified h_b, shape function, collapsed top layer),
test_ocean_kpp_nonlocal.F90 (stabilising flux, column heat),
test_ocean_vdiff.F90:42-69 (constancy, K = 0, conservation, vanishing layer,
relax-to-mean, kt = ks), test_ocean_vmix_assembly.F90:39-55 (pass-through,
ceilings, floors), test_ocean_bkgnd_mixing.F90:114-132 (Bryan-Lewis shape),
and test_ocean_wright_eos.F90:87-130 (Wright reference values).  Tolerances are the
reference tests' own.
"""
import numpy as np
import pytest

from roundabout_b200.config import default_config

NZ = 5


def state(oracle, nx=12, ny=10, nz=NZ, ntr=2, h=10.0):
    st = oracle.OracleState(nx, ny, nz, ntr)
    st.h[...] = h
    return st


def cfg_pp81(**kw):
    c = default_config()
    for k, v in kw.items():
        setattr(c, k, v)
    return c


# ---------------------------------------------------------------- PP81 ----
def test_pp81_quiescent_stratified(oracle):
    c = cfg_pp81()
    st = state(oracle)
    for k in range(NZ):
        st.rho[:, :, k] = 1030.0 - 1.0 * k
    st.call("vpo_pp81", c)
    assert np.abs(st.kv[6, 5, 1:NZ] - c.pp81_nu_bg).max() < 1e-6
    assert np.abs(st.kt[6, 5, 1:NZ] - c.pp81_kappa_bg).max() < 1e-6


def test_pp81_shear_without_stratification_is_full_mixing(oracle):
    c = cfg_pp81()
    st = state(oracle)
    st.rho[...] = 1030.0
    for k in range(NZ):
        st.u[:, :, k] = 1.0 * k / (NZ - 1)
    st.call("vpo_pp81", c)
    assert np.abs(st.kv[6, 5, 1:NZ] - (c.pp81_nu_bg + c.pp81_nu0)).max() < 1e-12
    assert np.abs(st.kt[6, 5, 1:NZ] - (c.pp81_kappa_bg + c.pp81_nu0)).max() < 1e-12


def test_pp81_strong_stratification_clamps(oracle):
    c = cfg_pp81()
    st = state(oracle)
    for k in range(NZ):
        st.u[:, :, k] = 1.0e-3 * k / (NZ - 1)
        st.rho[:, :, k] = 1030.0 - 5.0 * k
    st.call("vpo_pp81", c)
    assert st.kv[6, 5, 1:NZ].max() < 0.1 * (c.pp81_nu_bg + c.pp81_nu0)


def test_pp81_unstable_ri_clipped(oracle):
    c = cfg_pp81()
    st = state(oracle)
    for k in range(NZ):
        st.rho[:, :, k] = 1030.0 + 1.0 * k
    st.call("vpo_pp81", c)
    assert np.abs(st.kv[6, 5, 1:NZ] - (c.pp81_nu_bg + c.pp81_nu0)).max() < 1e-12


def test_pp81_boundary_interfaces_zero(oracle):
    c = cfg_pp81()
    st = state(oracle)
    st.u[...] = 0.5
    for k in range(NZ):
        st.rho[:, :, k] = 1030.0 - 0.5 * k
    st.kv[...] = 7.0
    st.kt[...] = 7.0
    st.call("vpo_pp81", c)
    for a in (st.kv, st.kt):
        assert np.abs(a[:, :, 0]).max() < 1e-15 and np.abs(a[:, :, -1]).max() < 1e-15


# ----------------------------------------------------------------- KPP ----
def kpp_state(oracle, nz=10, h=10.0, tau=0.1, strat=0.0):
    st = state(oracle, nz=nz, h=h)
    for k in range(nz):
        st.rho[:, :, k] = 1030.0 - strat * k
    st.stress_mag[...] = tau
    return st


def test_kpp_no_wind_is_no_op(oracle):
    c = cfg_pp81(use_kpp=1)
    st = kpp_state(oracle, nz=NZ, h=5.0, tau=0.0, strat=0.5)
    ref = st.copy()
    ref.call("vpo_pp81", c)
    st.call("vpo_pp81", c)
    st.call("vpo_kpp_overlay", c)
    assert np.abs(st.kv - ref.kv).max() <= 1e-14
    assert np.abs(st.kt - ref.kt).max() <= 1e-14


def test_kpp_unstratified_bl_fills_column(oracle):
    c = cfg_pp81(use_kpp=1)
    nz, h = 8, 10.0
    st = kpp_state(oracle, nz=nz, h=h, tau=0.1, strat=0.0)
    st.call("vpo_pp81", c)
    st.call("vpo_kpp_overlay", c)
    assert np.abs(st.bl_depth - nz * h).max() < 1e-9


def test_kpp_shape_function_matches_closed_form(oracle):
    c = cfg_pp81(use_kpp=1)
    nz, h, tau = 8, 10.0, 0.1
    st = kpp_state(oracle, nz=nz, h=h, tau=tau, strat=0.0)
    st.call("vpo_pp81", c)
    st.call("vpo_kpp_overlay", c)
    hb = nz * h
    u_star = np.sqrt(tau / c.rho0)
    for k in range(1, nz):            # interface k (0-based) is the bottom of layer k
        d = (nz - k) * h              # depth of that interface below the surface
        sig = d / hb
        want = max(c.pp81_nu_bg + c.pp81_nu0, hb * u_star * sig * (1 - sig) ** 2)
        assert abs(st.kv[6, 5, k] - want) < 1e-9


def test_kpp_vt2_never_shallows_the_bl(oracle):
    base = dict(use_kpp=1)
    depths = []
    for cvt2 in (0.0, 1.8, 4.0):
        c = cfg_pp81(c_vt2=cvt2, **base)
        st = kpp_state(oracle, nz=20, h=5.0, tau=0.05, strat=0.02)
        st.q_heat[...] = -200.0
        st.bl_depth[...] = 30.0       # lagged h_b feeds w_s into V_t^2
        st.call("vpo_pp81", c)
        st.call("vpo_kpp_overlay", c)
        depths.append(st.bl_depth[6, 5])
    assert depths[0] <= depths[1] <= depths[2]


def test_kpp_collapsed_top_layer_equals_column_without_it(oracle):
    c = cfg_pp81(use_kpp=1)
    nz = 9
    a = kpp_state(oracle, nz=nz, h=10.0, tau=0.1, strat=0.2)
    b = kpp_state(oracle, nz=nz + 1, h=10.0, tau=0.1, strat=0.2)
    for k in range(nz):
        b.rho[:, :, k] = a.rho[:, :, k]
    b.h[:, :, nz] = 1.0e-4            # a collapsed (vanished) top layer
    b.rho[:, :, nz] = c.rho0
    for s_ in (a, b):
        s_.call("vpo_pp81", c)
        s_.call("vpo_kpp_overlay", c)
    assert abs(a.bl_depth[6, 5] - b.bl_depth[6, 5]) < 1e-9
    np.testing.assert_allclose(b.kv[6, 5, 1:nz], a.kv[6, 5, 1:nz], rtol=0, atol=1e-12)


# -------------------------------------------------------- non-local KPP ----
def test_nonlocal_zero_under_stabilising_flux(oracle):
    c = cfg_pp81(use_kpp=1, alpha_T=0.2, beta_S=0.77)
    st = kpp_state(oracle, nz=10, h=10.0, tau=0.1, strat=0.05)
    st.q_heat[...] = +150.0           # heating: B0 > 0
    st.call("vpo_pp81", c)
    st.call("vpo_kpp_overlay", c)
    assert np.abs(st.gamma_t).max() == 0.0 and np.abs(st.gamma_s).max() == 0.0


def test_nonlocal_conserves_column_heat(oracle):
    c = cfg_pp81(use_kpp=1, alpha_T=0.2, beta_S=0.77)
    st = kpp_state(oracle, nz=12, h=8.0, tau=0.05, strat=0.01)
    st.h[:, :, 0] = 0.0                # a vanished bed filler
    st.q_heat[...] = -300.0            # cooling: B0 < 0
    st.tracers[1][...] = 10.0 + np.arange(12)[None, None, :] * 0.5
    st.call("vpo_pp81", c)
    st.call("vpo_kpp_overlay", c)
    assert np.abs(st.gamma_t).max() > 0.0
    heat0 = (st.h * st.tracers[1]).sum(axis=2)
    st.call("vpo_nonlocal", c, 3600.0)
    heat1 = (st.h * st.tracers[1]).sum(axis=2)
    assert np.abs(heat1 - heat0).max() <= 1e-12 * np.abs(heat0).max()
    assert np.abs(st.gamma_t[:, :, 0]).max() == 0.0 and np.abs(st.gamma_t[:, :, -1]).max() == 0.0


# --------------------------------------------------------------- vdiff ----
def vdiff_state(oracle, nz=8, K=1e-3, h=10.0):
    c = cfg_pp81()
    st = state(oracle, nz=nz, h=h, ntr=2)
    st.kt[...] = K
    st.kt[:, :, 0] = 0.0
    st.kt[:, :, -1] = 0.0
    st.ks[...] = st.kt
    return c, st


def test_vdiff_uniform_tracer_stays_uniform(oracle):
    c, st = vdiff_state(oracle)
    st.tracers[0][...] = 35.0
    st.tracers[1][...] = 12.0
    st.call("vpo_vdiff_tracers", c, 3600.0)
    assert np.abs(st.tracers[0] - 35.0).max() <= 1e-12
    assert np.abs(st.tracers[1] - 12.0).max() <= 1e-12


def test_vdiff_zero_diffusivity_is_no_op(oracle):
    c, st = vdiff_state(oracle, K=0.0)
    rng = np.random.default_rng(0)
    st.tracers[1][...] = rng.uniform(0, 20, st.tracers[1].shape)
    t0 = st.tracers[1].copy()
    st.call("vpo_vdiff_tracers", c, 3600.0)
    assert np.array_equal(st.tracers[1], t0)


def test_vdiff_conserves_column_content(oracle):
    c, st = vdiff_state(oracle, K=5e-2)
    rng = np.random.default_rng(1)
    st.h[...] = rng.uniform(1.0, 50.0, st.h.shape)
    st.tracers[1][...] = rng.uniform(0, 20, st.h.shape)
    c0 = (st.h * st.tracers[1]).sum(axis=2)
    st.call("vpo_vdiff_tracers", c, 3600.0)
    c1 = (st.h * st.tracers[1]).sum(axis=2)
    assert np.abs(c1 - c0).max() <= 1e-12 * np.abs(c0).max()


def test_vdiff_vanishing_layer_is_frozen_and_live_layers_conserve(oracle):
    c, st = vdiff_state(oracle, K=5e-2)
    st.h[:, :, 3] = 1.0e-5              # vanishing (<= H_VANISHED) mid-column layer
    rng = np.random.default_rng(2)
    st.tracers[1][...] = rng.uniform(0, 20, st.h.shape)
    frozen = st.tracers[1][:, :, 3].copy()
    live = st.h > 1.5e-4
    c0 = (st.h * st.tracers[1] * live).sum(axis=2)
    st.call("vpo_vdiff_tracers", c, 3600.0)
    c1 = (st.h * st.tracers[1] * live).sum(axis=2)
    assert np.abs(c1 - c0).max() <= 1e-12 * np.abs(c0).max()
    assert np.abs(st.tracers[1][:, :, 3] - frozen).max() <= 1e-10


def test_vdiff_strong_mixing_relaxes_to_the_mean(oracle):
    # test_ocean_vdiff.F90:310-362: h = 1, dt = 1, K = 1e6
    c, st = vdiff_state(oracle, K=1.0e6, h=1.0)
    st.tracers[1][...] = np.arange(8)[None, None, :] * 1.0
    st.call("vpo_vdiff_tracers", c, 1.0)
    assert np.abs(st.tracers[1] - 3.5).max() < 1e-4


def test_vdiff_kt_equal_ks_gives_identical_tracers(oracle):
    c, st = vdiff_state(oracle, K=2e-3)
    rng = np.random.default_rng(3)
    st.h[...] = rng.uniform(1.0, 50.0, st.h.shape)
    st.tracers[0][...] = rng.uniform(0, 20, st.h.shape)
    st.tracers[1][...] = st.tracers[0]
    st.call("vpo_vdiff_tracers", c, 3600.0)
    assert np.array_equal(st.tracers[0], st.tracers[1])


def test_momentum_uniform_velocity_stays_uniform(oracle):
    c = cfg_pp81()
    st = state(oracle, nz=8, h=10.0)
    st.kv[...] = 1e-2
    st.kv[:, :, 0] = 0.0
    st.kv[:, :, -1] = 0.0
    st.u[...] = 0.3
    st.v[...] = -0.2
    st.call("vpo_vdiff_momentum", c, 3600.0)
    assert np.abs(st.u - 0.3).max() <= 1e-12
    assert np.abs(st.v + 0.2).max() <= 1e-12


# ------------------------------------------------------------- assembly ----
def test_assembly_defaults_pass_pp81_through(oracle):
    c = cfg_pp81()
    st = state(oracle)
    for k in range(NZ):
        st.rho[:, :, k] = 1030.0 - 0.1 * k
        st.u[:, :, k] = 0.01 * k
    st.call("vpo_pp81", c)
    kv0 = st.kv.copy()
    st.call("vpo_split", c)
    assert st.call("vpo_assemble_gate", c) == 0
    assert np.array_equal(st.kv, kv0)
    assert np.array_equal(st.ks, st.kt)


def test_assembly_ceiling_and_floor(oracle):
    c = cfg_pp81(kd_max=2.0e-5, kv_max=3.0e-4, kt_bg=1.5e-5, ks_bg=1.5e-5)
    st = state(oracle)
    st.rho[...] = 1030.0
    for k in range(NZ):
        st.u[:, :, k] = 0.05 * k
    st.call("vpo_pp81", c)
    st.call("vpo_split", c)
    st.call("vpo_assemble_gate", c)
    assert st.kt[:, :, 1:NZ].max() <= 2.0e-5 and st.kv[:, :, 1:NZ].max() <= 3.0e-4
    assert st.kt[:, :, 1:NZ].min() >= 1.5e-5


def test_guard_flags_negative_before_the_clip(oracle):
    c = cfg_pp81(vmix_guard=1)
    st = state(oracle)
    st.kv[:, :, 2] = -1.0
    assert st.call("vpo_assemble_gate", c) == 1
    assert st.kv[:, :, 2].min() >= c.kv_bg        # then floored, as the reference does


def test_bryan_lewis_profile_shape(oracle):
    c = cfg_pp81(bkgnd_profile=1)
    nz = 60
    st = state(oracle, nz=nz, h=100.0)
    st.kv[...] = 0.0
    st.kt[...] = 0.0
    st.ks[...] = 0.0
    st.call("vpo_assemble_gate", c)
    depth = np.array([(nz - k) * 100.0 for k in range(nz + 1)])
    kd = st.kt[6, 5, :]
    assert abs(kd[nz - 1] - c.bkgnd_kd_sfc) < 0.05 * (c.bkgnd_kd_deep - c.bkgnd_kd_sfc)
    assert abs(kd[1] - c.bkgnd_kd_deep) < 0.1 * (c.bkgnd_kd_deep - c.bkgnd_kd_sfc)
    kz = int(np.argmin(np.abs(depth - c.bkgnd_z0)))
    assert abs(kd[kz] - 0.5 * (c.bkgnd_kd_sfc + c.bkgnd_kd_deep)) < 1e-12
    assert np.all(np.diff(kd[1:nz]) <= 0.0)        # deeper -> larger
    np.testing.assert_array_equal(st.kv[6, 5, 1:nz], kd[1:nz])   # kv floor = 1 * kd_bg


def test_wright_eos_reference_value(oracle):
    c = cfg_pp81()
    st = state(oracle, nz=1, ntr=2)
    st.tracers[0][...] = 35.0
    st.tracers[1][...] = 10.0
    st.call("vpo_eos_wright", c)
    # test_ocean_wright_eos.F90:87-107: within 0.5 of 1027 kg/m3 at (10 C, 35 psu, 0 Pa)
    assert abs(st.rho[0, 0, 0] - 1027.0) < 0.5
    st.tracers[0][...] = 0.0
    st.tracers[1][...] = 0.0
    st.call("vpo_eos_wright", c)
    # test_ocean_wright_eos.F90:125-130: pure water at 0 C within 0.5 of 999.7 kg/m3
    assert abs(st.rho[0, 0, 0] - 999.7) < 0.5
    st.h[...] = 0.0
    st.call("vpo_eos_wright", c)
    assert np.all(st.rho == c.rho0)


# ------------------------------------------------------- surface fluxes ----
# test_ocean_surface_flux.F90: zero flux is a no-op (82-117), heat warms the
# top layer by dt*Q/(rho0*cp*h) and leaves the rest (119-169), salt likewise
# with dt*Q/rho0 (171-218), the contributors integrate to the analytic deposit
# (220-300), a non-uniform Q field acts per column (302-364); plus the
# first-live-layer rule (apply_surface_src_2d_impl's k_top walk) and the
# pseudo-salt mirror that books no budget.
def flux_state(oracle, nz=4, h=10.0, ntr=3):
    st = state(oracle, nx=6, ny=4, nz=nz, ntr=ntr, h=h)
    st.tracers[0][...] = 35.0    # salinity
    st.tracers[1][...] = 10.0    # temperature
    return st


def test_surface_flux_zero_is_no_op(oracle):
    c = cfg_pp81(budgets=1)
    st = flux_state(oracle)
    T0, S0 = st.tracers[1].copy(), st.tracers[0].copy()
    for _ in range(5):
        st.call("vpo_surface_flux", c, 3600.0)
    assert np.abs(st.tracers[1] - T0).max() < 1e-14 and np.abs(st.tracers[0] - S0).max() < 1e-14
    assert np.abs(st.heat_budget_surface).max() == 0.0


def test_surface_heat_flux_warms_top(oracle):
    c = cfg_pp81()
    st = flux_state(oracle)
    st.q_heat[...] = 100.0
    st.call("vpo_surface_flux", c, 3600.0)
    dhT = 3600.0 * 100.0 / (c.rho0 * c.cp)
    assert np.abs(st.tracers[1][:, :, -1] - (10.0 + dhT / 10.0)).max() < 1e-10
    assert np.abs(st.tracers[1][:, :, :-1] - 10.0).max() < 1e-14
    assert np.abs(st.tracers[0] - 35.0).max() < 1e-14


def test_surface_salt_flux_salinifies_top(oracle):
    c = cfg_pp81()
    st = flux_state(oracle)
    st.q_salt[...] = 1.0e-3
    st.call("vpo_surface_flux", c, 3600.0)
    dhS = 3600.0 * 1.0e-3 / c.rho0
    assert np.abs(st.tracers[0][:, :, -1] - (35.0 + dhS / 10.0)).max() < 1e-10
    assert np.abs(st.tracers[0][:, :, :-1] - 35.0).max() < 1e-14
    assert np.abs(st.tracers[1] - 10.0).max() < 1e-14


def test_surface_flux_contributors_match_analytic(oracle):
    c = cfg_pp81(budgets=1)
    st = flux_state(oracle)
    st.q_heat[...] = 100.0
    st.q_salt[...] = 1.0e-3
    n = 7
    for _ in range(n):
        st.call("vpo_surface_flux", c, 3600.0)
    cells = st.nx * st.ny
    want_heat = n * 3600.0 * 100.0 / (c.rho0 * c.cp) * cells
    want_salt = n * 3600.0 * 1.0e-3 / c.rho0 * cells
    assert abs(st.heat_budget_surface.sum() - want_heat) < 1e-10 * want_heat
    assert abs(st.salt_budget_surface.sum() - want_salt) < 1e-10 * want_salt
    # the booked content is what the top layer gained
    gained = ((st.tracers[1] - 10.0) * st.h).sum()
    assert abs(gained - want_heat) < 1e-10 * want_heat


def test_surface_flux_nonuniform_field_per_column(oracle):
    c = cfg_pp81()
    st = flux_state(oracle)
    st.q_heat[:3, :] = 100.0       # west half heated, east half not
    st.call("vpo_surface_flux", c, 3600.0)
    dhT = 3600.0 * 100.0 / (c.rho0 * c.cp)
    assert np.abs(st.tracers[1][:3, :, -1] - (10.0 + dhT / 10.0)).max() < 1e-10
    assert np.abs(st.tracers[1][3:, :, -1] - 10.0).max() < 1e-14


def test_surface_flux_lands_on_first_live_layer_and_spares_land(oracle):
    c = cfg_pp81(budgets=1)
    st = flux_state(oracle, nz=6)
    st.h[:, :, -1] = 1.0e-4        # vanished top filler everywhere
    st.h[:2, :, -2] = 0.0          # and a second one on two columns
    st.wet[5, 3] = 0.0             # a land cell
    st.q_heat[...] = 100.0
    st.call("vpo_surface_flux", c, 3600.0)
    T = st.tracers[1]
    assert np.all(T[:, :, -1] == 10.0)                     # the filler takes nothing
    assert np.all(T[2:, :, -2][~(st.wet[2:, :] == 0.0)] > 10.0)
    assert np.all(T[:2, :, -3] > 10.0) and np.all(T[:2, :, -2] == 10.0)
    assert np.all(T[5, 3, :] == 10.0)                      # land: wet = 0
    assert st.heat_budget_surface[5, 3, :].sum() == 0.0
    assert np.all(st.heat_budget_surface[:, :, -1] == 0.0)


def test_surface_flux_pseudo_salt_mirrors_salt_without_budget(oracle):
    c = cfg_pp81(budgets=1, idx_pseudo_salt=2)
    st = flux_state(oracle)
    st.tracers[2][...] = 35.0
    st.q_salt[...] = 1.0e-3
    st.call("vpo_surface_flux", c, 3600.0)
    np.testing.assert_array_equal(st.tracers[2], st.tracers[0])
    dhS = 3600.0 * 1.0e-3 / c.rho0
    assert abs(st.salt_budget_surface.sum() - dhS * st.nx * st.ny) < 1e-10 * dhS * st.nx * st.ny


# ------------------------------------------- buoyancy_coeffs = "eos" ----
# test_ocean_eos_buoyancy.F90: the Wright derivatives against centred
# differences of the EOS itself (points 99-110, steps and tolerances 112-122,
# check 169-201), alpha_T rising with temperature toward 20 C (283-313) and
# with pressure at the freezing point (315-339), and KPP's kv scaling as the
# cube root of the B0 ratio in the closed-form column (462-556).
EOS_PTS = [(-2.0, 33.0, 0.0), (-1.9, 34.5, 0.0), (-1.0, 34.0, 2.5e6), (0.0, 35.0, 5.0e6), (1.0, 33.5, 7.5e6),
           (2.0, 34.5, 1.0e7), (-2.0, 34.5, 1.0e7), (-1.9, 33.0, 5.0e6), (2.0, 35.0, 0.0), (10.0, 35.0, 0.0),
           (18.0, 36.0, 2.0e6), (25.0, 34.0, 4.0e7)]


def eos_rho(oracle, T, S, p):
    c = cfg_pp81(eos_p_ref=p)
    st = state(oracle, nx=1, ny=1, nz=1, ntr=2)
    st.tracers[0][...] = S
    st.tracers[1][...] = T
    st.call("vpo_eos_wright", c)
    return float(st.rho[0, 0, 0])


def test_eos_buoyancy_coeffs_match_finite_differences(oracle):
    eps = 1.0e-4
    for T, S, p in EOS_PTS:
        a, b = oracle.eos_buoyancy_coeffs(T, S, p)
        fd_t = (eos_rho(oracle, T + eps, S, p) - eos_rho(oracle, T - eps, S, p)) / (2.0 * eps)
        fd_s = (eos_rho(oracle, T, S + eps, p) - eos_rho(oracle, T, S - eps, p)) / (2.0 * eps)
        assert abs(-a - fd_t) <= max(1.0e-7 * abs(fd_t), 1.0e-9), (T, S, p, a, fd_t)
        assert abs(b - fd_s) <= max(1.0e-7 * abs(fd_s), 1.0e-9), (T, S, p, b, fd_s)


def test_eos_alpha_grows_with_temperature_and_pressure(oracle):
    a = [oracle.eos_buoyancy_coeffs(-2.0 + n, 34.5, 0.0)[0] for n in range(23)]
    assert all(a[n] > a[n - 1] for n in range(1, 23))
    assert a[12] > 3.0 * a[0] and a[0] > 0.0
    ap = [oracle.eos_buoyancy_coeffs(-1.9, 34.5, n * 1.0e6)[0] for n in range(11)]
    assert all(ap[n] > ap[n - 1] for n in range(1, 11))
    assert ap[10] > 1.5 * ap[0]


def test_kpp_eos_coeffs_scale_kv_as_cube_root_of_b0(oracle):
    nz, H, T0, S0, QH, QS = 8, 40.0, -1.9, 34.5, -200.0, 3.0e-5
    runs = {}
    for mode in (0, 1):
        c = cfg_pp81(use_kpp=1, alpha_T=0.17, beta_S=0.78, buoyancy_coeffs=mode)
        st = state(oracle, nx=6, ny=4, nz=nz, ntr=2, h=H)
        st.tracers[0][...] = S0
        st.tracers[1][...] = T0
        st.rho[...] = 1027.8
        st.q_heat[...] = QH
        st.q_salt[...] = QS
        st.seed_backgrounds(c)
        st.call("vpo_pp81", c)
        st.call("vpo_kpp_overlay", c)
        runs[mode] = st
    a_e, b_e = oracle.eos_buoyancy_coeffs(T0, S0, 0.0)
    qt, qs = QH / (1035.0 * 3992.0), QS / 1035.0
    b0_c = 0.17 * qt - 0.78 * qs
    b0_e = a_e * qt - b_e * qs
    assert b0_c < 0.0 and b0_e < 0.0 and a_e < 0.5 * 0.17
    ratio = (b0_e / b0_c) ** (1.0 / 3.0)
    assert abs(ratio - 1.0) > 0.1
    for k in range(1, nz):
        kv_c, kv_e = runs[0].kv[3, 2, k], runs[1].kv[3, 2, k]
        assert kv_c > 1.0e-3
        assert abs(kv_e / kv_c - ratio) < 1.0e-10 * ratio
    assert runs[1].b0[3, 2] == (9.80665 / 1035.0) * (a_e * qt - b_e * qs)


# ------------------------------------------------- shortwave penetration ----
# test_ocean_sw_penetration.F90: 6 layers of 5 m, Q_heat = 200 W/m2, half of it
# penetrating, two bands R = 0.58, zeta = 0.35 / 23 m (39-47).  The correction
# redistributes (column sum 0, 150-189), follows the two-band closed form
# layer by layer (124-148, 191-218), absorbs most at the top and decays with
# depth (220-268), and is byte-for-byte nothing at sw_pen_frac = 0 (270-290).
SW = dict(sw_pen_frac=0.5, sw_band_ratio=0.58, sw_zeta1=0.35, sw_zeta2=23.0)


def sw_state(oracle, nz=6, h=5.0):
    st = flux_state(oracle, nz=nz, h=h)
    st.q_heat[...] = 200.0
    return st


def sw_closed_form(nz, h, c, dt=3600.0, q=200.0):
    import math

    inv = dt / (c.rho0 * c.cp)
    i0 = c.sw_pen_frac * q
    tr = lambda d: c.sw_band_ratio * math.exp(-d / c.sw_zeta1) + (1 - c.sw_band_ratio) * math.exp(-d / c.sw_zeta2)
    corr = np.zeros(nz)
    d_top = 0.0
    for k in range(nz - 1, -1, -1):
        d_bot = d_top + h
        tb = tr(d_bot) if k > 0 else 0.0
        corr[k] = inv * i0 * (tr(d_top) - tb) - (inv * i0 if k == nz - 1 else 0.0)
        d_top = d_bot
    return corr


def test_sw_penetration_conserves_and_matches_two_band(oracle):
    c = cfg_pp81(**SW)
    st = sw_state(oracle)
    st.call("vpo_sw_penetration", c, 3600.0)
    got = st.h[3, 2, :] * (st.tracers[1][3, 2, :] - 10.0)
    assert abs(got.sum()) < 1e-12
    np.testing.assert_allclose(got, sw_closed_form(6, 5.0, c), rtol=0, atol=1e-12)
    absorbed = got.copy()
    absorbed[-1] += 3600.0 / (c.rho0 * c.cp) * 0.5 * 200.0
    assert np.all(absorbed >= 0.0) and np.all(absorbed[-1] > absorbed[:-1])
    assert np.all(absorbed[2:-1] > absorbed[1:-2])   # interior decays; the opaque bed takes the rest


def test_sw_penetration_off_is_identity(oracle):
    c = cfg_pp81(**dict(SW, sw_pen_frac=0.0))
    st = sw_state(oracle)
    T0 = st.tracers[1].copy()
    st.call("vpo_sw_penetration", c, 3600.0)
    np.testing.assert_array_equal(st.tracers[1], T0)


def test_sw_penetration_skips_vanished_layers_and_books_the_move(oracle):
    """A vanished top filler and a vanished bed layer pass the light on; the
    lump leaves the first live layer; the budget books every move (sum 0)."""
    c = cfg_pp81(budgets=1, **SW)
    st = sw_state(oracle, nz=8)
    st.h[:, :, -1] = 1.0e-4
    st.h[:, :, 0] = 0.0
    st.call("vpo_sw_penetration", c, 3600.0)
    T = st.tracers[1]
    assert np.all(T[:, :, -1] == 10.0) and np.all(T[:, :, 0] == 10.0)
    assert np.all(T[:, :, -2] < 10.0)            # the surface lump left the first live layer
    bud = st.heat_budget_surface
    assert abs(bud.sum()) < 1e-10 and np.abs(bud).max() > 0.0
    np.testing.assert_allclose((st.h * (T - 10.0)).sum(axis=2), bud.sum(axis=2), rtol=0, atol=1e-12)


@pytest.mark.parametrize("method", [1, 2, 3])
def test_kpp_b0_charges_the_absorbed_shortwave(oracle, method):
    """Pass 2's B0 (the stored b0) takes Q_heat minus what passes the new
    boundary layer (MXL) or the surface layer (LV1), all of it with ALL
    (rdb_ocean_vmix.F90:1440-1466)."""
    import math

    c = cfg_pp81(use_kpp=1, alpha_T=0.2, beta_S=0.77, kpp_sw_method=method, **SW)
    st = kpp_state(oracle, nz=10, h=8.0, tau=0.05, strat=0.01)
    st.q_heat[...] = 150.0
    st.call("vpo_pp81", c)
    st.call("vpo_kpp_overlay", c)
    h_b = st.bl_depth[4, 3]
    tr = lambda d: 0.58 * math.exp(-d / 0.35) + 0.42 * math.exp(-d / 23.0)
    q = 150.0 - {1: 0.0, 2: 0.5 * 150.0 * tr(h_b), 3: 0.5 * 150.0 * tr(st.h[4, 3, -1])}[method]
    want = (9.80665 / 1035.0) * (0.2 * q / (1035.0 * 3992.0))
    assert abs(st.b0[4, 3] - want) <= 1e-13 * abs(want)
    c0 = cfg_pp81(use_kpp=1, alpha_T=0.2, beta_S=0.77, kpp_sw_method=method)
    s0 = kpp_state(oracle, nz=10, h=8.0, tau=0.05, strat=0.01)
    s0.q_heat[...] = 150.0
    s0.call("vpo_pp81", c0)
    s0.call("vpo_kpp_overlay", c0)
    if method == 1:
        np.testing.assert_array_equal(st.b0, s0.b0)
    else:
        assert np.all(st.b0 < s0.b0)
