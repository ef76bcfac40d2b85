"""Known-answer tests of the EPBL oracle (vphys_oracle_epbl.c), re-expressed
from the reference's tests/test_ocean_epbl.F90.  Its driver `run_epbl_steps`
(:117-163) is restated here: per step the surface flux into T, EPBL, then the
implicit tracer diffusion with EPBL's kd as the diffusivity.

* Kraus-Turner wind deepening (:297-357): monotone MLD growth, log-log
  exponent in [0.20, 0.47], prefactor in [0.9, 1.8] of (12 mstar u*^3 t/N^2)^(1/3);
* a stabilising flux shoals the MLD below 95 % of the neutral one (:486-530);
* convective deepening (:532-585): monotone, within [0.5, 1.4] of the
  encroachment depth sqrt(2 B0 t)/N, mixing at the near-surface interface;
* collapsed top layers (:720-790): kd and MLD equal those of the column
  without them, no mixing on the interfaces above the first live layer;
* the OM4 mstar (:243-281) in closed form on a neutral two-layer column,
  including its zero-Ekman-term limit;
* the convective seed of the first cooled step, nstar (-0.5 rho0 h B0)
  (:281-341).
"""
import math

import numpy as np
import pytest

G = 9.80665
RHO0 = 1035.0
ALPHA_LIN = 0.2
BETA_LIN = 0.8
CP = 3992.0


def epbl_config(**over):
    """setup_epbl (test_ocean_epbl.F90:76-97): linear EOS, constant mstar
    1.2, nstar 0.2, f = 0."""
    from roundabout_b200.config import default_config

    c = default_config()
    c.epbl = 1
    c.epbl_mstar_scheme = 1
    c.epbl_mstar_const = 1.2
    c.epbl_nstar = 0.2
    c.eos_variant = 1
    c.eos_alpha_t = ALPHA_LIN
    c.eos_beta_s = BETA_LIN
    c.rho0 = RHO0
    c.cp = CP
    for k, v in over.items():
        setattr(c, k, v)
    return c


def stratified(oracle, nz, dz, t_surf, dtdz, nx=2, ny=1):
    """setup_stratified_T (:99-115)."""
    st = oracle.OracleState(nx, ny, nz, 2)
    st.h[...] = dz
    for k in range(1, nz + 1):
        z = (float(nz - k) + 0.5) * dz
        st.tracers[1][:, :, k - 1] = t_surf - dtdz * z
        st.tracers[0][:, :, k - 1] = 35.0
    return st


def run_steps(st, cfg, dt, n_steps, sample_every, stress=0.0, q_heat=0.0):
    st.stress_mag[...] = stress
    st.q_heat[...] = q_heat
    st.q_salt[...] = 0.0
    mld, t = [], []
    for step in range(1, n_steps + 1):
        st.call("vpo_surface_flux", cfg, dt)
        st.call("vpo_epbl", cfg, dt)
        st.kt[...] = st.kd_epbl
        st.ks[...] = st.kd_epbl
        st.call("vpo_vdiff_tracers", cfg, dt)
        if step % sample_every == 0:
            mld.append(float(st.mld_epbl[0, 0]))
            t.append(step * dt)
    return np.array(mld), np.array(t)


def loglog_slope(t, d):
    x, y = np.log(t), np.log(d)
    x, y = x - x.mean(), y - y.mean()
    return float((x * y).sum() / (x * x).sum())


def test_wind_deepening_kraus_turner(oracle):
    nz, dz, dt, ustar, n2 = 100, 3.0, 1800.0, 0.01, 1.0e-4
    cfg = epbl_config()
    st = stratified(oracle, nz, dz, 15.0, n2 * RHO0 / (G * ALPHA_LIN))
    mld, t = run_steps(st, cfg, dt, 240, 12, stress=RHO0 * ustar ** 2)
    assert (np.diff(mld) >= -1e-9).all(), mld
    slope = loglog_slope(t[len(t) // 2 - 1:], mld[len(mld) // 2 - 1:])
    assert 0.20 < slope < 0.47, slope
    d_analytic = (12.0 * cfg.epbl_mstar_const * ustar ** 3 * t[-1] / n2) ** (1.0 / 3.0)
    assert 0.9 < mld[-1] / d_analytic < 1.8, mld[-1] / d_analytic


def test_stabilising_flux_shoals_the_mld(oracle):
    nz, dz, dt = 60, 3.0, 1800.0
    dtdz = 1.0e-4 * RHO0 / (G * ALPHA_LIN)
    cfg = epbl_config()
    a, _ = run_steps(stratified(oracle, nz, dz, 15.0, dtdz), cfg, dt, 96, 24, stress=RHO0 * 0.01 ** 2)
    b, _ = run_steps(stratified(oracle, nz, dz, 15.0, dtdz), cfg, dt, 96, 24, stress=RHO0 * 0.01 ** 2, q_heat=500.0)
    assert b[-1] < 0.95 * a[-1], (a[-1], b[-1])


def test_convective_deepening(oracle):
    nz, dz, dt, q, n2 = 60, 2.5, 1800.0, -200.0, 1.0e-4
    cfg = epbl_config()
    st = stratified(oracle, nz, dz, 15.0, n2 * RHO0 / (G * ALPHA_LIN))
    mld, t = run_steps(st, cfg, dt, 96, 12, q_heat=q)
    assert (np.diff(mld) >= -1e-9).all(), mld
    b0 = abs(G * ALPHA_LIN * (q / (RHO0 * CP)) / RHO0)
    d_enc = math.sqrt(2.0 * b0 * t[-1]) / math.sqrt(n2)
    assert 0.5 < mld[-1] / d_enc < 1.4, mld[-1] / d_enc
    assert st.kd_epbl[0, 0, nz - 1] > 1.0e-6


@pytest.mark.parametrize("nlive,ndead", [(8, 1), (8, 2), (1, 1)])
def test_collapsed_top_layers(oracle, nlive, ndead):
    dz, dt = 5.0, 1800.0
    cfg = epbl_config()
    ref = stratified(oracle, nlive, dz, 15.0, 0.05)
    dead = oracle.OracleState(2, 1, nlive + ndead, 2)
    dead.h[:, :, :nlive] = ref.h
    dead.tracers[0][:, :, :nlive] = ref.tracers[0]
    dead.tracers[1][:, :, :nlive] = ref.tracers[1]
    dead.h[:, :, nlive:] = 1.0e-5
    dead.tracers[1][:, :, nlive:] = 40.0
    dead.tracers[0][:, :, nlive:] = 35.0
    for st in (ref, dead):
        st.stress_mag[...] = 0.05
        st.q_heat[...] = -200.0
        st.call("vpo_epbl", cfg, dt)
    if nlive >= 2:
        scale = np.abs(ref.kd_epbl[0, 0, 1:nlive]).max()
        assert scale > 0.0
        assert np.abs(dead.kd_epbl[0, 0, 1:nlive] - ref.kd_epbl[0, 0, 1:nlive]).max() < 1e-9 * scale
    assert abs(dead.mld_epbl[0, 0] - ref.mld_epbl[0, 0]) < 1e-6
    assert np.abs(dead.kd_epbl[0, 0, nlive:]).max() == 0.0


def test_om4_mstar_closed_form(oracle):
    """epbl_find_mstar's OM4 branch (:655-662, test_ocean_epbl.F90:243-281)
    through a neutral two-layer column, no fluxes, no TKE decay, no MLD
    iteration: the one interior interface takes the unlimited first-guess
    kd = v* kappa (htot hbs v*)/(f htot hbs + v*) with v* = cbrt(mstar) u*,
    htot = h, hbs = 1/2 and the MLD guess (half the column) in
    mstar = min(1.25, c_ek log(u*/(f BLD))).  When u* <= f BLD the Ekman
    term is 0, so is mstar, and the interface does not mix."""
    dz, dt, f = 10.0, 1800.0, 1.0e-4
    for ustar in (0.01, 0.003, 1.0e-3):
        got = {}
        for scheme in (1, 2):
            cfg = epbl_config(epbl_mstar_scheme=scheme, epbl_mld_iteration=0, epbl_tke_decay=0.0)
            st = stratified(oracle, 2, dz, 15.0, 0.0)
            st.coriolis[...] = f
            st.stress_mag[...] = RHO0 * ustar ** 2
            st.call("vpo_epbl", cfg, dt)
            got[scheme] = float(st.kd_epbl[0, 0, 1])
        bld = 0.5 * (2 * dz + 1e-20)
        ustar_eff = math.sqrt(RHO0 * ustar ** 2 / RHO0)
        for scheme, mstar in ((1, 1.2), (2, 0.085 * math.log(ustar_eff / (f * bld)) if ustar_eff > f * bld else 0.0)):
            mstar = min(1.25, mstar) if scheme == 2 else mstar
            vstar = (mstar * ustar_eff ** 3) ** (1.0 / 3.0)
            want = vstar * 0.41 * (dz * 0.5 * vstar) / (f * dz * 0.5 + vstar) if vstar > 0 else 0.0
            assert abs(got[scheme] - want) <= 1e-12 * max(want, 1e-300), (ustar, scheme, got[scheme], want)
        if ustar <= f * bld:
            assert got[2] == 0.0


def test_shortwave_ledger_limits(oracle):
    """The penetrating-shortwave TKE ledger (rdb_ocean_epbl.F90:1095-1185,
    1373-1425): with no irradiance (Q_heat = 0) it changes nothing, bit for
    bit; under surface heating, charging the penetrating part per layer
    through Phi <= 1 costs less than heating the skin with all of it, so the
    mixed layer is at least as deep."""
    nz, dz, dt = 40, 2.0, 1800.0
    dtdz = 1.0e-5 * RHO0 / (G * ALPHA_LIN)
    out = {}
    for q, frac in ((0.0, 0.0), (0.0, 0.6), (300.0, 0.0), (300.0, 0.6)):
        cfg = epbl_config(sw_pen_frac=frac)
        st = stratified(oracle, nz, dz, 15.0, dtdz)
        st.stress_mag[...] = RHO0 * 0.01 ** 2
        st.q_heat[...] = q
        st.call("vpo_epbl", cfg, dt)
        out[(q, frac)] = (st.kd_epbl.copy(), float(st.mld_epbl[0, 0]))
    assert np.array_equal(out[(0.0, 0.0)][0], out[(0.0, 0.6)][0])
    assert out[(0.0, 0.0)][1] == out[(0.0, 0.6)][1]
    assert out[(300.0, 0.6)][1] >= out[(300.0, 0.0)][1], (out[(300.0, 0.6)][1], out[(300.0, 0.0)][1])
    assert out[(300.0, 0.6)][1] > out[(300.0, 0.0)][1] or not np.array_equal(out[(300.0, 0.6)][0], out[(300.0, 0.0)][0])


def test_rh18_mstar_closed_form(oracle):
    """epbl_find_mstar's RH18 branch (rdb_ocean_epbl.F90:664-670) on the same
    neutral two-layer column: with no buoyancy flux the stabilising term is
    cs1 * 0^cs2 = 0, so mstar = cn1 e/(1 + e) with e = cn2 exp(cn3 BLD f/u*)."""
    dz, dt, f = 10.0, 1800.0, 1.0e-4
    for ustar in (0.01, 0.003):
        cfg = epbl_config(epbl_mstar_scheme=3, epbl_mld_iteration=0, epbl_tke_decay=0.0)
        st = stratified(oracle, 2, dz, 15.0, 0.0)
        st.coriolis[...] = f
        st.stress_mag[...] = RHO0 * ustar ** 2
        st.call("vpo_epbl", cfg, dt)
        ustar_eff = math.sqrt(RHO0 * ustar ** 2 / RHO0)
        bld = 0.5 * (2 * dz + 1e-20)
        e = 8.0 * math.exp(-5.0 * bld * f / ustar_eff)
        mstar = 0.275 * e / (1.0 + e)
        vstar = (mstar * ustar_eff ** 3) ** (1.0 / 3.0)
        want = vstar * 0.41 * (dz * 0.5 * vstar) / (f * dz * 0.5 + vstar)
        got = float(st.kd_epbl[0, 0, 1])
        assert abs(got - want) <= 1e-12 * want, (ustar, got, want)


def test_mixing_length_exponent(oracle):
    """epbl_mixlen_shape (:690-714), shape = ts + (1 - ts) fr^n: at the
    first interface below the surface layer (no energy spent yet, f = 0,
    the first MLD guess half the column) the diffusivity is the unlimited
    first guess v* kappa htot hbs with hbs = the shape, so the exponent-3 /
    exponent-2 ratio of kd there is the ratio of the two shapes; exponent 3
    goes through rdb_sm_pow, exponent 2 through fr * fr."""
    nz, dz, dt = 30, 2.0, 1800.0
    kd_top = {}
    for n in (2.0, 3.0):
        cfg = epbl_config(epbl_mixlen_exponent=n, epbl_mld_iteration=1, epbl_mld_max_its=1)
        st = stratified(oracle, nz, dz, 15.0, 1.0e-5 * RHO0 / (G * ALPHA_LIN))
        st.stress_mag[...] = RHO0 * 0.01 ** 2
        st.call("vpo_epbl", cfg, dt)
        kd_top[n] = float(st.kd_epbl[0, 0, nz - 1])
    fr = (0.5 * nz * dz - dz) / (0.5 * nz * dz)
    want = (0.1 + 0.9 * fr ** 3) / (0.1 + 0.9 * fr ** 2)
    assert kd_top[2.0] > 0.0
    assert abs(kd_top[3.0] / kd_top[2.0] - want) < 1e-12, (kd_top, want)


def test_lf17_spot_values(oracle):
    """epbl_lf17_wave_state + epbl_lf17_la against the reference's prototype
    values (test_ocean_epbl.F90:604-627): U10 within 2 %, La within 1 %."""
    import ctypes

    L = oracle.lib()
    for ustar, bld, la_ref, u10_ref in ((0.005, 20.0, 0.4129, 5.08), (0.01, 20.0, 0.3627, 8.51),
                                        (0.01, 50.0, 0.4372, 8.51), (0.02, 50.0, 0.3947, 14.01)):
        u10, la = ctypes.c_double(), ctypes.c_double()
        L.vpo_epbl_lf17(ustar, RHO0, 0.04 * bld, ctypes.byref(u10), ctypes.byref(la))
        assert abs(u10.value - u10_ref) < 0.02 * u10_ref, (ustar, u10.value)
        assert abs(la.value - la_ref) < 0.01 * la_ref, (ustar, bld, la.value)


def test_lt_enhancement_monotone(oracle):
    """epbl_lt_enhance, rescale scheme (test_ocean_epbl.F90:629-661): a
    smaller La enhances more, the cap holds for a tiny La, and
    1 + 0.447 * 0.3^-1.33 by hand (all lac_i = 0, B0 = 0, f = 0)."""
    import ctypes

    L = oracle.lib()
    cfg = epbl_config(epbl_use_lt=1, epbl_lt_scheme=1, epbl_lt_lac1=0.0, epbl_lt_lac2=0.0, epbl_lt_lac3=0.0,
                      epbl_lt_lac4=0.0, epbl_lt_lac5=0.0)
    m = {la: L.vpo_epbl_lt_enhance(ctypes.byref(cfg), la, 0.0, 0.01, 50.0, 0.0, 1.0) for la in (0.6, 0.3, 0.01)}
    assert m[0.6] > 1.0
    assert m[0.3] > m[0.6]
    assert abs(m[0.01] - 5.0) < 1e-12
    assert abs(m[0.3] - (1.0 + 0.447 * 0.3 ** -1.33)) < 1e-12


def test_lt_deepens_wind_mixing(oracle):
    """Langmuir enhancement deepens the wind-mixed layer by over 10 %, La
    stays in the wind-sea range, and La is 0 with it off
    (test_ocean_epbl.F90:663-716)."""
    nz, dz, dt = 80, 3.0, 1800.0
    dtdz = 1.0e-4 * RHO0 / (G * ALPHA_LIN)
    off = stratified(oracle, nz, dz, 15.0, dtdz)
    a, _ = run_steps(off, epbl_config(), dt, 48, 12, stress=RHO0 * 0.01 ** 2)
    on = stratified(oracle, nz, dz, 15.0, dtdz)
    cfg = epbl_config(epbl_use_lt=1, epbl_lt_scheme=1, epbl_lt_lac1=0.0, epbl_lt_lac4=0.0, epbl_lt_lac5=0.0)
    b, _ = run_steps(on, cfg, dt, 48, 12, stress=RHO0 * 0.01 ** 2)
    assert b[-1] > 1.1 * a[-1], (a[-1], b[-1])
    assert 0.2 < on.la_epbl[0, 0] < 0.6, on.la_epbl[0, 0]
    assert abs(off.la_epbl[0, 0]) < 1e-30


@pytest.mark.parametrize("q_heat,sw", [(-300.0, 0.0), (-300.0, 1.0), (250.0, 1.0), (-50.0, 0.6)])
def test_tke_budget_closes(oracle, q_heat, sw):
    """The column TKE ledger closes to round-off every step
    (test_ocean_epbl.F90:359-484): wind + conv + forcing - mixing -
    mech_decay - conv_decay = 0 within 1e-9 of the sources, on a rotating
    column under wind, a surface heat flux and (sw > 0) penetrating
    shortwave charged per layer -- a heating flux drains the reservoirs
    below the surface (the proportional and the exhausting drain), a cooling
    one releases convective energy."""
    nz, dz, dt = 40, 5.0, 1800.0
    cfg = epbl_config(epbl_tke_diags=1, sw_pen_frac=sw)
    st = stratified(oracle, nz, dz, 15.0, 0.0527, nx=3, ny=2)
    st.coriolis[...] = 1.0e-4
    run_steps(st, cfg, dt, 12, 12, stress=0.1, q_heat=q_heat)
    wind, conv, forcing, mixing, mdecay, cdecay = st.epbl_tke
    residual = wind + conv + forcing - mixing - mdecay - cdecay
    scale = wind + conv + np.abs(forcing) + 1e-30
    assert (np.abs(residual) < 1e-9 * scale).all(), np.abs(residual / scale).max()
    assert (wind > 0.0).all()
    if q_heat < 0.0:
        assert (conv > 0.0).all()
    else:
        assert (forcing < 0.0).all() or (mixing > 0.0).all()


def test_convective_seed(oracle):
    """The convective ledger term of the first step of pure cooling on a
    stable column is nstar (-0.5 rho0 h_sfc B0), B0 = g alpha q_T / rho0 under
    the linear EOS, to 1e-10 relative; the bed and surface interfaces carry
    no diffusivity (test_ocean_epbl.F90:281-341)."""
    nz, dz, dt, q_heat = 8, 5.0, 1800.0, -200.0
    cfg = epbl_config(epbl_tke_diags=1)
    st = stratified(oracle, nz, dz, 15.0, 0.05, nx=6, ny=4)
    run_steps(st, cfg, dt, 1, 1, stress=0.0, q_heat=q_heat)
    b0 = G * ALPHA_LIN * (q_heat / (RHO0 * CP)) / RHO0
    ctke = -0.5 * RHO0 * dz * b0 * dt
    assert ctke > 0.0
    conv_expected = cfg.epbl_nstar * ctke / dt
    assert abs(st.epbl_tke[1][3, 2] - conv_expected) < 1.0e-10 * conv_expected
    assert abs(st.kd_epbl[3, 2, 0]) < 1.0e-30 and abs(st.kd_epbl[3, 2, nz]) < 1.0e-30
