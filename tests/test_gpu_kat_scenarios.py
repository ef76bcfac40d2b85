"""The reference's known-answer scenarios run through the CUDA library (its C
ABI) and compared with the oracle BITWISE.

The oracle files tests/test_oracle_*_kat.py pin the oracle on the
reference's own known answers: thin bed slivers under strong drag, exactly
collapsed and pinched layers, the bottom-boundary-layer glue, the no-slip
remnant profile, inverted and neutral columns, a velocity jump under
kappa-shear, the interior closure "none", Bryan-Lewis floors, smoothing
around a dry column, Manizza opacities.  The same states are loaded here
into the GPU library and into the oracle, one entry point is run on each,
and every output field must agree bit for bit.  The scenarios keep nz >= 3
and at least 8 x 4 columns (the one- and two-layer closed forms stay on the
oracle).
"""
import math

import numpy as np
import pytest

from roundabout_b200.config import INTERIOR_NONE, INTERIOR_PP81, default_config, seed_backgrounds
from tests._cases import assert_bitwise

pytestmark = pytest.mark.gpu

FIELDS = ("h", "u", "v", "rho", "kv", "kt", "ks", "bl_depth", "stress_mag", "q_heat", "q_salt", "wet", "tau_x",
          "tau_y", "lambda_bot_u", "lambda_bot_v", "coriolis")
COEFFS = ("kv", "kt", "ks", "bl_depth", "b0")


@pytest.fixture(scope="module")
def VP():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from roundabout_b200.column import VerticalPhysics

    return VerticalPhysics


def cfg(**kw):
    c = default_config()
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def mirror(VP, st, c, extra=()):
    """A GPU handle holding the oracle state's fields."""
    vp = VP(st.nx, st.ny, st.nz, st.ntr, c)
    for n in FIELDS + tuple(extra):
        vp.set(n, getattr(st, n))
    for t in range(st.ntr):
        vp.set_tracer(t, st.tracers[t])
    return vp


def same(vp, st, names, tracers=False):
    for n in names:
        assert_bitwise(n, vp.get(n), getattr(st, n))
    if tracers:
        for t in range(st.ntr):
            assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])


def interior(a, value):
    a[...] = value
    a[:, :, 0] = 0.0
    a[:, :, -1] = 0.0


# ------------------------------------------------------------- momentum ----
def layered(oracle, hs, nx=8, ny=4, ntr=2):
    st = oracle.OracleState(nx, ny, len(hs), ntr)
    for k, hk in enumerate(hs):
        st.h[:, :, k] = hk
    return st


def momentum_both(VP, oracle, st, c, dt, remnant=False):
    vp = mirror(VP, st, c)
    st.call("vpo_vdiff_momentum", c, dt)
    vp.vdiff_momentum(dt)
    names = ("u", "v") + (("visc_rem_u", "visc_rem_v") if remnant else ())
    same(vp, st, names)
    return vp


def test_thin_bed_drag_picard(VP, oracle):
    H1, CD, U0, DT = 2.0, 2.5e-3, 8.0, 600.0
    c = cfg(rho0=1035.0, implicit_drag=1)
    st = layered(oracle, [H1] * 6)
    interior(st.kv, 0.0)
    st.u[...] = U0
    vp = mirror(VP, st, c)
    for _ in range(5):
        lam_u = CD * np.abs(st.u[:, :, 0]) / H1
        st.lambda_bot_u[...] = lam_u
        vp.set("lambda_bot_u", st.lambda_bot_u)
        st.call("vpo_vdiff_momentum", c, DT)
        vp.vdiff_momentum(DT)
        same(vp, st, ("u", "v"))


def test_resolved_drag_and_stress_with_a_land_face(VP, oracle):
    c = cfg(rho0=1035.0, implicit_drag=1, implicit_stress=1)
    st = layered(oracle, [100.0] * 6)
    interior(st.kv, 1.0e-2)
    st.u[...] = 0.5
    st.lambda_bot_u[...] = 1.0e-3
    st.lambda_bot_v[...] = 1.0e-3
    st.tau_x[...] = 0.1
    st.tau_y[...] = -0.05
    st.wet[2, 1] = 0.0
    momentum_both(VP, oracle, st, c, 600.0)


def test_remnant_with_harmonic_faces(VP, oracle):
    c = cfg(rho0=1035.0, implicit_drag=1, hvel_mom6=1, remnant=1)
    st = layered(oracle, [12.0 * (k + 1) for k in range(6)])
    interior(st.kv, 0.2)
    st.lambda_bot_u[...] = 0.08
    st.lambda_bot_v[...] = 0.08
    momentum_both(VP, oracle, st, c, 450.0, remnant=True)


def test_glue_on_a_thin_bed_sliver(VP, oracle):
    for hs in ((0.05, 1.0, 10.0, 25.0), (0.2, 5.0, 15.0, 25.0)):
        c = cfg(rho0=1035.0, implicit_drag=1, hvel_mom6=1, bbl_glue=1, remnant=1)
        st = layered(oracle, hs)
        interior(st.kv, 1.0e-4)
        st.u[...] = 0.5
        st.lambda_bot_u[...] = 0.02
        st.lambda_bot_v[...] = 0.02
        momentum_both(VP, oracle, st, c, 600.0, remnant=True)


def test_collapsed_interior_layer_remnant(VP, oracle):
    c = cfg(rho0=1035.0, hvel_mom6=0, remnant=1)
    st = layered(oracle, (10.0, 0.0, 12.0, 20.0))
    interior(st.kv, 0.2)
    momentum_both(VP, oracle, st, c, 450.0, remnant=True)


def test_no_slip_remnant_profile(VP, oracle):
    c = cfg(rho0=1035.0, hvel_mom6=0, remnant=1, implicit_drag=1)
    st = layered(oracle, [2.0] * 40)
    interior(st.kv, 0.1)
    st.lambda_bot_u[...] = 1.0e6
    st.lambda_bot_v[...] = 1.0e6
    momentum_both(VP, oracle, st, c, 1000.0, remnant=True)


def test_momentum_stiff_shear(VP, oracle):
    st = layered(oracle, [1.0] * 6)
    interior(st.kv, 1000.0)
    for k in range(6):
        st.u[:, :, k] = 1.0 if k < 3 else -1.0
    momentum_both(VP, oracle, st, cfg(), 1.0)


# ------------------------------------------------------ the build chain ----
def assemble_both(VP, oracle, st, c, extra=(), names=COEFFS):
    vp = mirror(VP, st, c, extra)
    assert st.call("vpo_build_coefficients", c) == 0
    vp.assemble()
    same(vp, st, names)
    return vp


def mixed_layer(oracle, c, tau, q_heat, nx=14, ny=12, nz=8):
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


@pytest.mark.parametrize("tau,q_heat", [(0.1, 0.0), (0.1, 500.0), (0.0, -500.0), (0.1, -500.0)])
def test_kpp_mixed_layer(VP, oracle, tau, q_heat):
    c = cfg(use_kpp=1)
    assemble_both(VP, oracle, mixed_layer(oracle, c, tau, q_heat), c)


def stratified(oracle, c, nx=12, ny=10, nz=6, tau=0.05, q_heat=0.0):
    st = oracle.OracleState(nx, ny, nz, 2)
    st.seed_backgrounds(c)
    st.h[...] = 5.0
    for k in range(1, nz + 1):
        st.rho[:, :, k - 1] = 1030.0 - 0.2 * (k - 1)
    st.stress_mag[...] = tau
    st.q_heat[...] = q_heat
    return st


@pytest.mark.parametrize("cvt2", [0.0, 1.8, 5.0])
def test_kpp_vt2(VP, oracle, cvt2):
    c = cfg(use_kpp=1, c_vt2=cvt2)
    assemble_both(VP, oracle, stratified(oracle, c, q_heat=-150.0), c)


def test_kpp_half_domain_cooling_two_builds(VP, oracle):
    c = cfg(use_kpp=1)
    st = stratified(oracle, c, nx=16, ny=12)
    st.q_heat[:8, :] = -300.0
    vp = assemble_both(VP, oracle, st, c)
    assert st.call("vpo_build_coefficients", c) == 0    # the lagged h_b of the first build feeds w*
    vp.assemble()
    same(vp, st, COEFFS)


def test_kpp_convective_wstar_neutral_column(VP, oracle):
    c = cfg(use_kpp=1, rho0=1035.0, cp=3992.0, alpha_T=0.2, beta_S=0.8)
    st = oracle.OracleState(8, 6, 10, 2)
    st.seed_backgrounds(c)
    st.h[...] = 20.0
    st.rho[...] = 1035.0
    st.q_heat[...] = -100.0
    st.q_salt[...] = 2.0e-5
    assemble_both(VP, oracle, st, c)


@pytest.mark.parametrize("closure,over", [
    (INTERIOR_PP81, {}),
    (INTERIOR_NONE, {}),
    (INTERIOR_NONE, dict(kv_bg=0.0, bkgnd_prandtl=1.0)),
    (INTERIOR_NONE, dict(kv_bg=1.0e-5, bkgnd_prandtl=2.0)),
])
def test_sheared_column_closures(VP, oracle, closure, over):
    c = cfg(rho0=1035.0, use_kpp=0, interior_closure=closure, pp81_nu_bg=2.0e-4, pp81_kappa_bg=3.0e-5)
    seed_backgrounds(c)
    c.ks_bg = 5.0e-5
    for k, v in over.items():
        setattr(c, k, v)
    st = oracle.OracleState(8, 6, 4, 2)
    st.h[...] = 100.0
    for k in range(1, 5):
        st.u[:, :, k - 1] = 0.3 * k
        st.rho[:, :, k - 1] = 1035.0 - 1.7e-4 * (0.05 * (k - 2))
    for a in (st.kv, st.kt, st.ks):
        a[...] = 1.0
    assemble_both(VP, oracle, st, c)


@pytest.mark.parametrize("case", ["inverted", "below_bl", "pinched", "n2_thresh"])
def test_convection(VP, oracle, case):
    if case == "inverted":
        c = cfg(conv_enable=1, conv_kd=1.0, conv_prandtl=2.0)
        rho, h, bld = [1030.0 + k for k in range(4)], [10.0] * 4, 0.0
    elif case == "below_bl":
        c = cfg(conv_enable=1, conv_kd=1.0)
        rho, h, bld = [1028.0 + k for k in range(10)], [20.0] * 10, 100.0
    elif case == "pinched":
        c = cfg(conv_enable=1, conv_kd=1.0)
        rho, h, bld = [1028.0, 1028.0, 1040.0, 1040.0], [10.0, 1.0e-6, 1.0e-6, 10.0], 0.0
    else:
        c = cfg(conv_enable=1, conv_kd=1.0, conv_n2_thresh=1.0e-5)
        drho = 5.0e-6 * c.rho0 * 10.0 / 9.80665
        rho, h, bld = [1030.0 - drho * k for k in range(4)], [10.0] * 4, 0.0
    st = oracle.OracleState(8, 6, len(rho), 2)
    for k in range(len(rho)):
        st.h[:, :, k] = h[k]
        st.rho[:, :, k] = rho[k]
    st.bl_depth[...] = bld
    assemble_both(VP, oracle, st, c)


@pytest.mark.parametrize("nz,h", [(50, 1.0), (10, 5.0)])
def test_kv_ml_invz2(VP, oracle, nz, h):
    c = cfg(kv_ml_invz2=0.01, hmix_fixed=20.0)
    st = oracle.OracleState(8, 4, nz, 2)
    st.h[...] = h
    for k in range(nz):
        st.rho[:, :, k] = 1030.0 - 0.01 * k
    assemble_both(VP, oracle, st, c)


def test_bryan_lewis_floor(VP, oracle):
    c = cfg(bkgnd_profile=1, bkgnd_kd_sfc=1.0e-5, bkgnd_kd_deep=1.3e-4, bkgnd_z0=1000.0, bkgnd_delta=222.0,
            bkgnd_prandtl=2.0)
    st = oracle.OracleState(16, 14, 30, 2)
    st.h[...] = 100.0
    for k in range(30):
        st.rho[:, :, k] = 1030.0 - 0.1 * k
    assemble_both(VP, oracle, st, c)


def test_smoothing_around_a_dry_column(VP, oracle):
    c = cfg(kd_smooth_iterations=2)
    st = oracle.OracleState(16, 14, 4, 2)
    st.h[...] = 5.0
    for j in range(14):
        for i in range(16):
            for k in range(4):
                st.u[i, j, k] = 0.01 * ((i + 2 * j + 3 * k) % 7)
                st.rho[i, j, k] = 1030.0 - 0.05 * k - 0.001 * ((i * j) % 5)
    st.wet[5, 4] = 0.0
    assemble_both(VP, oracle, st, c)


# ------------------------------------------------- kappa-shear and EPBL ----
def shear_jump(oracle, c, du, nx=8, ny=4):
    NZK, KJ, DZ, N2, RHO0 = 12, 6, 5.0, 3.0e-5, 1025.0
    st = oracle.OracleState(nx, ny, NZK, 2)
    dtdz = N2 * RHO0 / (9.80665 * RHO0 * 2.0e-4)
    st.h[...] = DZ
    for k in range(1, NZK + 1):
        st.tracers[c.idx_temperature][:, :, k - 1] = 20.0 + dtdz * DZ * (k - NZK)
        st.tracers[c.idx_salinity][:, :, k - 1] = 35.0
        if k > KJ:
            st.u[:, :, k - 1] = du
    st.coriolis[...] = 1.0e-4
    return st


def shear_cfg(**kw):
    c = cfg(interior_closure=INTERIOR_NONE, pp81_nu_bg=2.0e-4, pp81_kappa_bg=3.0e-5, kappa_shear=1, eos_variant=1,
            eos_alpha_t=1025.0 * 2.0e-4, eos_beta_s=1025.0 * 7.6e-4, rho0=1025.0)
    seed_backgrounds(c)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


@pytest.mark.parametrize("du", [0.0, 0.2])
def test_interior_none_with_kappa_shear(VP, oracle, du):
    c = shear_cfg()
    st = shear_jump(oracle, c, du)
    vp = mirror(VP, st, c)
    st.call("vpo_kappa_shear", c, 1800.0)
    vp.kappa_shear(1800.0)
    same(vp, st, ("kd_shear", "tke_shear"))
    assert st.call("vpo_build_coefficients", c) == 0
    vp.assemble()
    same(vp, st, ("kv", "kt", "ks"))


@pytest.mark.parametrize("combine", [1, 2, 3])
def test_epbl_combines_over_kappa_shear(VP, oracle, combine):
    c = shear_cfg(epbl=1, epbl_prandtl=1.5, epbl_combine=combine)
    st = shear_jump(oracle, c, 0.2)
    st.kd_epbl[...] = 0.0
    st.kd_epbl[:, :, 2] = 0.05
    st.kd_epbl[:, :, 6] = 1.0e-4
    vp = mirror(VP, st, c, extra=("kd_epbl",))
    st.call("vpo_kappa_shear", c, 1800.0)
    vp.kappa_shear(1800.0)
    assert st.call("vpo_build_coefficients", c) == 0
    vp.assemble()
    same(vp, st, ("kv", "kt", "ks"))


# --------------------------------------------------------------- tracers ----
def test_heat_salt_and_passive_with_their_own_diffusivities(VP, oracle):
    for budgets in (0, 1):
        c = cfg(budgets=budgets)
        st = oracle.OracleState(8, 4, 6, 3)
        st.h[...] = 10.0
        for n in range(3):
            for k in range(6):
                st.tracers[n][:, :, k] = 0.0 if k < 3 else 1.0 + n
        interior(st.kt, 1.0e-2)
        interior(st.ks, 4.0e-2)
        vp = mirror(VP, st, c)
        st.call("vpo_vdiff_tracers", c, 60.0)
        vp.vdiff_tracers(60.0)
        same(vp, st, ("heat_budget", "salt_budget") if budgets else (), tracers=True)


def test_harmonic_faces_on_a_thin_layer(VP, oracle):
    for harm in (0, 1):
        c = cfg(use_harmonic=harm)
        st = layered(oracle, (10.0, 0.1, 10.0, 0.1, 5.0))
        interior(st.kt, 1.0e-3)
        st.ks[...] = st.kt
        for k in range(5):
            st.tracers[c.idx_temperature][:, :, k] = float(k)
            st.tracers[c.idx_salinity][:, :, k] = 35.0 - 0.1 * k
        vp = mirror(VP, st, c)
        st.call("vpo_vdiff_tracers", c, 60.0)
        vp.vdiff_tracers(60.0)
        same(vp, st, (), tracers=True)


def test_nonlocal_cooling_on_the_mixed_layer(VP, oracle):
    c = cfg(use_kpp=1)
    st = mixed_layer(oracle, c, 0.1, -500.0)
    vp = assemble_both(VP, oracle, st, c)
    st.call("vpo_nonlocal", c, 100.0)
    vp.nonlocal_tendencies(100.0)
    same(vp, st, (), tracers=True)


# ----------------------------------------------------- shortwave and EOS ----
def chl_cfg():
    c = cfg(sw_chl=1, sw_pen_frac=1.0, sw_nbands=3, sw_blue_frac=0.5, sw_opacity_land=10.0)
    for n, v in enumerate((0.0232, 0.074, 0.225, 0.037, 2.86, 0.0)):
        c.sw_opacity_coef[n] = v
    for n, v in enumerate((0.674, 0.629, 0.0)):
        c.sw_chl_power[n] = v
    return c


def test_manizza_opacities(VP, oracle):
    c = chl_cfg()
    st = oracle.OracleState(8, 4, 3, 2)
    for m, chl in enumerate((0.1, 1.0, 10.0, -1.0e34, 0.5, 3.0, 1.0e-6, 0.02)):
        st.sw_chl[m, :] = chl
    st.wet[4, :] = 0.0
    vp = mirror(VP, st, c, extra=("sw_chl",))
    st.call("vpo_sw_chl_kappa", c)
    vp.sw_chl_apply()
    same(vp, st, ("sw_kappa",))


def test_three_band_absorption(VP, oracle):
    c = chl_cfg()
    st = oracle.OracleState(8, 4, 10, 2)
    st.h[...] = 10.0
    st.q_heat[...] = 300.0
    for n, kap in enumerate((0.0232 + 0.074 * 0.5 ** 0.674, 0.225 + 0.037 * 0.5 ** 0.629, 2.86)):
        st.sw_kappa[:, :, n] = kap
    vp = mirror(VP, st, c, extra=("sw_kappa",))
    st.call("vpo_sw_penetration", c, 1800.0)
    vp.sw_penetration(1800.0)
    same(vp, st, (), tracers=True)


def test_wright_at_the_reference_states(VP, oracle):
    c = cfg(eos_p_ref=0.0, rho0=1035.0)
    st = oracle.OracleState(8, 4, 3, 2)
    st.h[...] = 10.0
    states = ((10.0, 35.0), (0.0, 0.0), (15.0, 35.0), (10.0, 38.0), (0.0, 33.0), (20.0, 36.5), (10.0, 34.75),
              (-1.8, 34.0))
    for m, (t, s) in enumerate(states):
        st.tracers[c.idx_temperature][m, :, :] = t
        st.tracers[c.idx_salinity][m, :, :] = s
    st.h[0, 0, 0] = 0.0
    vp = mirror(VP, st, c)
    st.call("vpo_eos_wright", c)
    vp.eos()
    same(vp, st, ("rho",))
    assert math.isfinite(float(st.rho.max()))
