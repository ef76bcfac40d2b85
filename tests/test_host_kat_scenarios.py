"""The reference's known-answer scenarios (the states of
tests/test_gpu_kat_scenarios.py: thin bed slivers under strong drag,
collapsed and pinched layers, the glue, the no-slip remnant, KPP mixed and
neutral columns, the closure "none", convection, the surface viscosity band,
Bryan-Lewis floors, smoothing around a dry column, tracers with their own
diffusivities, Manizza opacities, Wright states, kappa-shear over the closure
"none" and under the EPBL combines) run through the CUDA source of the
kernels compiled for the host (the plain step's kernels of
tests/test_host_hot_kernels.py, the kappa-shear kernel of
tests/test_host_kernels.py) and compared with the oracle bit for bit, in
every CPU run of the suite."""
import ctypes

import numpy as np
import pytest

from roundabout_b200.config import INTERIOR_NONE, INTERIOR_PP81
from tests import test_gpu_kat_scenarios as K
from tests._cases import assert_bitwise
from tests.test_host_hot_kernels import hot, run  # noqa: F401  (the compiled host kernels)
from tests.test_host_kernels import _ptr, host_libs  # noqa: F401  (the kappa-shear host kernel)

COEFFS = K.COEFFS


def clone(oracle, st):
    """A second oracle state holding the same fields (the host kernels' copy)."""
    c = oracle.OracleState(st.nx, st.ny, st.nz, st.ntr)
    for name, _ in oracle.VpoState._fields_[4:]:
        a = getattr(st, name, None)
        if isinstance(a, np.ndarray):
            getattr(c, name)[...] = a
    for t in range(st.ntr):
        c.tracers[t][...] = st.tracers[t]
    return c


def same(host, ref, names, tracers=False):
    for n in names:
        assert_bitwise(n, getattr(host, n), getattr(ref, n))
    if tracers:
        for t in range(ref.ntr):
            assert_bitwise(f"tracer{t}", host.tracers[t], ref.tracers[t])


def momentum_both(oracle, hot, st, c, dt, remnant=False):
    host = clone(oracle, st)
    st.call("vpo_vdiff_momentum", c, dt)
    run(hot, "host_momentum", c, host, dt, 0)
    same(host, st, ("u", "v") + (("visc_rem_u", "visc_rem_v") if remnant else ()))


def assemble_both(oracle, hot, st, c):
    host = clone(oracle, st)
    assert st.call("vpo_build_coefficients", c) == 0
    assert run(hot, "host_assemble", c, host) == 0
    same(host, st, COEFFS)
    return host


# ------------------------------------------------------------- momentum ----
def test_thin_bed_drag_picard(oracle, hot):
    H1, CD, U0, DT = 2.0, 2.5e-3, 8.0, 600.0
    c = K.cfg(rho0=1035.0, implicit_drag=1)
    st = K.layered(oracle, [H1] * 6)
    K.interior(st.kv, 0.0)
    st.u[...] = U0
    host = clone(oracle, st)
    for _ in range(5):
        for s in (st, host):
            s.lambda_bot_u[...] = CD * np.abs(st.u[:, :, 0]) / H1
        st.call("vpo_vdiff_momentum", c, DT)
        run(hot, "host_momentum", c, host, DT, 0)
        same(host, st, ("u", "v"))


def test_resolved_drag_and_stress_with_a_land_face(oracle, hot):
    c = K.cfg(rho0=1035.0, implicit_drag=1, implicit_stress=1)
    st = K.layered(oracle, [100.0] * 6)
    K.interior(st.kv, 1.0e-2)
    st.u[...] = 0.5
    st.lambda_bot_u[...] = 1.0e-3
    st.lambda_bot_v[...] = 1.0e-3
    st.tau_x[...] = 0.1
    st.tau_y[...] = -0.05
    st.wet[2, 1] = 0.0
    momentum_both(oracle, hot, st, c, 600.0)


@pytest.mark.parametrize("case", ["harmonic", "glue_sliver", "glue_damps", "collapsed", "no_slip", "stiff"])
def test_momentum_scenarios(oracle, hot, case):
    if case == "harmonic":
        c = K.cfg(rho0=1035.0, implicit_drag=1, hvel_mom6=1, remnant=1)
        st, kv, lam, dt = K.layered(oracle, [12.0 * (k + 1) for k in range(6)]), 0.2, 0.08, 450.0
    elif case in ("glue_sliver", "glue_damps"):
        c = K.cfg(rho0=1035.0, implicit_drag=1, hvel_mom6=1, bbl_glue=1, remnant=1)
        hs = (0.05, 1.0, 10.0, 25.0) if case == "glue_sliver" else (0.2, 5.0, 15.0, 25.0)
        st, kv, lam, dt = K.layered(oracle, hs), 1.0e-4, 0.02, 600.0
        st.u[...] = 0.5
    elif case == "collapsed":
        c = K.cfg(rho0=1035.0, hvel_mom6=0, remnant=1)
        st, kv, lam, dt = K.layered(oracle, (10.0, 0.0, 12.0, 20.0)), 0.2, 0.0, 450.0
    elif case == "no_slip":
        c = K.cfg(rho0=1035.0, hvel_mom6=0, remnant=1, implicit_drag=1)
        st, kv, lam, dt = K.layered(oracle, [2.0] * 40), 0.1, 1.0e6, 1000.0
    else:
        c = K.cfg()
        st, kv, lam, dt = K.layered(oracle, [1.0] * 6), 1000.0, 0.0, 1.0
        for k in range(6):
            st.u[:, :, k] = 1.0 if k < 3 else -1.0
    K.interior(st.kv, kv)
    st.lambda_bot_u[...] = lam
    st.lambda_bot_v[...] = lam
    momentum_both(oracle, hot, st, c, dt, remnant=bool(c.remnant))


# ------------------------------------------------------ the build chain ----
@pytest.mark.parametrize("tau,q_heat", [(0.1, 0.0), (0.1, 500.0), (0.0, -500.0), (0.1, -500.0)])
def test_kpp_mixed_layer(oracle, hot, tau, q_heat):
    c = K.cfg(use_kpp=1)
    assemble_both(oracle, hot, K.mixed_layer(oracle, c, tau, q_heat), c)


@pytest.mark.parametrize("cvt2", [0.0, 1.8, 5.0])
def test_kpp_vt2(oracle, hot, cvt2):
    c = K.cfg(use_kpp=1, c_vt2=cvt2)
    assemble_both(oracle, hot, K.stratified(oracle, c, q_heat=-150.0), c)


def test_kpp_half_domain_cooling_two_builds(oracle, hot):
    c = K.cfg(use_kpp=1)
    st = K.stratified(oracle, c, nx=16, ny=12)
    st.q_heat[:8, :] = -300.0
    host = assemble_both(oracle, hot, st, c)
    assert st.call("vpo_build_coefficients", c) == 0
    assert run(hot, "host_assemble", c, host) == 0
    same(host, st, COEFFS)


def test_kpp_convective_wstar_neutral_column(oracle, hot):
    c = K.cfg(use_kpp=1, rho0=1035.0, cp=3992.0, alpha_T=0.2, beta_S=0.8)
    st = oracle.OracleState(8, 6, 10, 2)
    st.seed_backgrounds(c)
    st.h[...] = 20.0
    st.rho[...] = 1035.0
    st.q_heat[...] = -100.0
    st.q_salt[...] = 2.0e-5
    assemble_both(oracle, hot, st, c)


@pytest.mark.parametrize("closure,over", [
    (INTERIOR_PP81, {}),
    (INTERIOR_NONE, {}),
    (INTERIOR_NONE, dict(kv_bg=0.0, bkgnd_prandtl=1.0)),
    (INTERIOR_NONE, dict(kv_bg=1.0e-5, bkgnd_prandtl=2.0)),
])
def test_sheared_column_closures(oracle, hot, closure, over):
    c = K.cfg(rho0=1035.0, use_kpp=0, interior_closure=closure, pp81_nu_bg=2.0e-4, pp81_kappa_bg=3.0e-5)
    K.seed_backgrounds(c)
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
    assemble_both(oracle, hot, st, c)


@pytest.mark.parametrize("case", ["inverted", "below_bl", "pinched", "n2_thresh"])
def test_convection(oracle, hot, case):
    if case == "inverted":
        c = K.cfg(conv_enable=1, conv_kd=1.0, conv_prandtl=2.0)
        rho, h, bld = [1030.0 + k for k in range(4)], [10.0] * 4, 0.0
    elif case == "below_bl":
        c = K.cfg(conv_enable=1, conv_kd=1.0)
        rho, h, bld = [1028.0 + k for k in range(10)], [20.0] * 10, 100.0
    elif case == "pinched":
        c = K.cfg(conv_enable=1, conv_kd=1.0)
        rho, h, bld = [1028.0, 1028.0, 1040.0, 1040.0], [10.0, 1.0e-6, 1.0e-6, 10.0], 0.0
    else:
        c = K.cfg(conv_enable=1, conv_kd=1.0, conv_n2_thresh=1.0e-5)
        drho = 5.0e-6 * c.rho0 * 10.0 / 9.80665
        rho, h, bld = [1030.0 - drho * k for k in range(4)], [10.0] * 4, 0.0
    st = oracle.OracleState(8, 6, len(rho), 2)
    for k in range(len(rho)):
        st.h[:, :, k] = h[k]
        st.rho[:, :, k] = rho[k]
    st.bl_depth[...] = bld
    assemble_both(oracle, hot, st, c)


@pytest.mark.parametrize("nz,h", [(50, 1.0), (10, 5.0)])
def test_kv_ml_invz2(oracle, hot, nz, h):
    c = K.cfg(kv_ml_invz2=0.01, hmix_fixed=20.0)
    st = oracle.OracleState(8, 4, nz, 2)
    st.h[...] = h
    for k in range(nz):
        st.rho[:, :, k] = 1030.0 - 0.01 * k
    assemble_both(oracle, hot, st, c)


def test_bryan_lewis_floor(oracle, hot):
    c = K.cfg(bkgnd_profile=1, bkgnd_kd_sfc=1.0e-5, bkgnd_kd_deep=1.3e-4, bkgnd_z0=1000.0, bkgnd_delta=222.0,
              bkgnd_prandtl=2.0)
    st = oracle.OracleState(16, 14, 30, 2)
    st.h[...] = 100.0
    for k in range(30):
        st.rho[:, :, k] = 1030.0 - 0.1 * k
    assemble_both(oracle, hot, st, c)


def test_smoothing_around_a_dry_column(oracle, hot):
    c = K.cfg(kd_smooth_iterations=2)
    st = oracle.OracleState(16, 14, 4, 2)
    st.h[...] = 5.0
    for j in range(14):
        for i in range(16):
            for k in range(4):
                st.u[i, j, k] = 0.01 * ((i + 2 * j + 3 * k) % 7)
                st.rho[i, j, k] = 1030.0 - 0.05 * k - 0.001 * ((i * j) % 5)
    st.wet[5, 4] = 0.0
    assemble_both(oracle, hot, st, c)


# --------------------------------------------------------------- tracers ----
def test_heat_salt_and_passive_with_their_own_diffusivities(oracle, hot):
    for budgets in (0, 1):
        c = K.cfg(budgets=budgets)
        st = oracle.OracleState(8, 4, 6, 3)
        st.h[...] = 10.0
        for n in range(3):
            for k in range(6):
                st.tracers[n][:, :, k] = 0.0 if k < 3 else 1.0 + n
        K.interior(st.kt, 1.0e-2)
        K.interior(st.ks, 4.0e-2)
        host = clone(oracle, st)
        st.call("vpo_vdiff_tracers", c, 60.0)
        run(hot, "host_tracers", c, host, 60.0, 1, 0, 0)
        same(host, st, ("heat_budget", "salt_budget") if budgets else (), tracers=True)


def test_harmonic_faces_on_a_thin_layer(oracle, hot):
    for harm in (0, 1):
        c = K.cfg(use_harmonic=harm)
        st = K.layered(oracle, (10.0, 0.1, 10.0, 0.1, 5.0))
        K.interior(st.kt, 1.0e-3)
        st.ks[...] = st.kt
        for k in range(5):
            st.tracers[c.idx_temperature][:, :, k] = float(k)
            st.tracers[c.idx_salinity][:, :, k] = 35.0 - 0.1 * k
        host = clone(oracle, st)
        st.call("vpo_vdiff_tracers", c, 60.0)
        run(hot, "host_tracers", c, host, 60.0, 1, 0, 1)
        same(host, st, (), tracers=True)


def test_nonlocal_cooling_on_the_mixed_layer(oracle, hot):
    c = K.cfg(use_kpp=1)
    st = K.mixed_layer(oracle, c, 0.1, -500.0)
    host = assemble_both(oracle, hot, st, c)
    st.call("vpo_nonlocal", c, 100.0)
    run(hot, "host_tracers", c, host, 100.0, 0, 1, 1)
    same(host, st, (), tracers=True)


# ----------------------------------------------------- shortwave and EOS ----
def test_manizza_opacities(oracle, hot):
    c = K.chl_cfg()
    st = oracle.OracleState(8, 4, 3, 2)
    for m, chl in enumerate((0.1, 1.0, 10.0, -1.0e34, 0.5, 3.0, 1.0e-6, 0.02)):
        st.sw_chl[m, :] = chl
    st.wet[4, :] = 0.0
    host = clone(oracle, st)
    st.call("vpo_sw_chl_kappa", c)
    run(hot, "host_sw_chl_kappa", c, host)
    same(host, st, ("sw_kappa",))


def test_three_band_absorption(oracle, hot):
    c = K.chl_cfg()
    st = oracle.OracleState(8, 4, 10, 2)
    st.h[...] = 10.0
    st.q_heat[...] = 300.0
    for n, kap in enumerate((0.0232 + 0.074 * 0.5 ** 0.674, 0.225 + 0.037 * 0.5 ** 0.629, 2.86)):
        st.sw_kappa[:, :, n] = kap
    host = clone(oracle, st)
    st.call("vpo_sw_penetration", c, 1800.0)
    run(hot, "host_sw_penetration", c, host, 1800.0)
    same(host, st, (), tracers=True)


def test_wright_at_the_reference_states(oracle, hot):
    c = K.cfg(eos_p_ref=0.0, rho0=1035.0)
    st = oracle.OracleState(8, 4, 3, 2)
    st.h[...] = 10.0
    for m, (t, s) in enumerate(((10.0, 35.0), (0.0, 0.0), (15.0, 35.0), (10.0, 38.0), (0.0, 33.0), (20.0, 36.5),
                                (10.0, 34.75), (-1.8, 34.0))):
        st.tracers[c.idx_temperature][m, :, :] = t
        st.tracers[c.idx_salinity][m, :, :] = s
    st.h[0, 0, 0] = 0.0
    host = clone(oracle, st)
    st.call("vpo_eos_wright", c)
    run(hot, "host_eos", c, host)
    same(host, st, ("rho",))


# ---------------------------------------- kappa-shear and the EPBL merges ----

def host_kappa_shear(host_libs, c, st, dt):
    host_libs["kshear"].host_kappa_shear(ctypes.byref(c), st.nx, st.ny, st.nz, _ptr(st.h), _ptr(st.u), _ptr(st.v),
                                         _ptr(st.tracers[c.idx_temperature]), _ptr(st.tracers[c.idx_salinity]),
                                         _ptr(st.wet), _ptr(st.coriolis), ctypes.c_double(dt), _ptr(st.kd_shear),
                                         _ptr(st.tke_shear))


@pytest.mark.parametrize("du", [0.0, 0.2])
def test_interior_none_with_kappa_shear(oracle, hot, host_libs, du):
    c = K.shear_cfg()
    st = K.shear_jump(oracle, c, du)
    host = clone(oracle, st)
    st.call("vpo_kappa_shear", c, 1800.0)
    host_kappa_shear(host_libs, c, host, 1800.0)
    same(host, st, ("kd_shear", "tke_shear"))
    assert st.call("vpo_build_coefficients", c) == 0
    assert run(hot, "host_assemble", c, host) == 0
    same(host, st, ("kv", "kt", "ks"))


@pytest.mark.parametrize("combine", [1, 2, 3])
def test_epbl_combines_over_kappa_shear(oracle, hot, host_libs, combine):
    c = K.shear_cfg(epbl=1, epbl_prandtl=1.5, epbl_combine=combine)
    st = K.shear_jump(oracle, c, 0.2)
    st.kd_epbl[...] = 0.0
    st.kd_epbl[:, :, 2] = 0.05
    st.kd_epbl[:, :, 6] = 1.0e-4
    host = clone(oracle, st)
    st.call("vpo_kappa_shear", c, 1800.0)
    host_kappa_shear(host_libs, c, host, 1800.0)
    assert st.call("vpo_build_coefficients", c) == 0
    assert run(hot, "host_assemble", c, host) == 0
    same(host, st, ("kv", "kt", "ks"))
