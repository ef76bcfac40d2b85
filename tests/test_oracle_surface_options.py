"""Known-answer tests of the surface-forcing options on the oracle: the
`q_sw` shortwave source (sw_source = 1), BOUND_SALINITY and the dynamic
wet/dry mask (rdb_ocean_surface_flux.F90:959-1091, 1144-1225, 1256-1399;
the KPP charge at rdb_ocean_vmix.F90:1102-1117 and 1321-1348; EPBL's
ledger source at rdb_ocean_epbl.F90:895-920, 1100-1104).

Each option is checked against what the reference's code states: an
identity when the option's input equals the legacy one, the deposit's
conservation, and the clamp or mask in closed form.
"""
import numpy as np

from tests._cases import columns, hot_cfg, oracle_state

DT = 3600.0
SW = dict(sw_pen_frac=0.6, sw_band_ratio=0.58, sw_zeta1=0.35, sw_zeta2=23.0)


def _state(oracle, cfg, seed=81, nx=24, ny=14, nz=18, sunlit=True):
    cols = columns(nx=nx, ny=ny, nz=nz, seed=seed, thin_frac=0.15)
    cols.h[: nx // 4, :, -1] = 1.0e-4          # vanished top fillers: the deposit lands below them
    st = oracle_state(oracle, cols, cfg)
    if sunlit:
        st.q_heat[...] = np.abs(st.q_heat) + 60.0
    return st


def _heat_content(st, cfg):
    return (st.h * st.tracers[cfg.idx_temperature]).sum(axis=2)


def test_qsw_equal_to_net_heat_is_the_legacy_path(oracle):
    """sw_source = "q_sw" with q_sw = Q_heat gives the net_heat answer bit
    for bit: deposit, penetration, KPP's B0 and the whole step."""
    c0 = hot_cfg(budgets=1, surface_flux=1, **SW)
    c1 = hot_cfg(budgets=1, surface_flux=1, sw_source=1, **SW)
    a, b = _state(oracle, c0), _state(oracle, c1)
    b.sw_net[...] = b.q_heat
    assert a.call("vpo_step", c0, DT, 2) == 0
    assert b.call("vpo_step", c1, DT, 2) == 0
    for t in range(a.ntr):
        assert np.array_equal(a.tracers[t], b.tracers[t]), t
    for n in ("kv", "kt", "b0", "bl_depth", "heat_budget_surface"):
        assert np.array_equal(getattr(a, n), getattr(b, n)), n


def test_qsw_penetration_only_moves_heat(oracle):
    """The penetration removes I0 = sw_pen_frac q_sw from the first live
    layer and spreads it down the column: the column's heat content is that
    of the deposit alone to round-off, whatever q_sw is, and the profile
    follows q_sw, not Q_heat."""
    cfg = hot_cfg(surface_flux=1, sw_source=1, **SW)
    st = _state(oracle, cfg)
    st.sw_net[...] = 0.5 * np.abs(st.q_heat) + 200.0 * (np.arange(st.nx)[:, None] % 3 == 0)
    st.call("vpo_surface_flux", cfg, DT)
    before = _heat_content(st, cfg)
    iT = cfg.idx_temperature
    t_dep = st.tracers[iT].copy()
    st.call("vpo_sw_penetration", cfg, DT)
    after = _heat_content(st, cfg)
    scale = np.abs(before).max()
    assert np.abs(after - before).max() <= 1e-12 * scale
    # columns with no shortwave are left alone by the penetration
    ref = _state(oracle, cfg)
    ref.sw_net[...] = 0.0
    ref.call("vpo_surface_flux", cfg, DT)
    ref.call("vpo_sw_penetration", cfg, DT)
    assert np.array_equal(ref.tracers[iT], t_dep)
    assert not np.array_equal(st.tracers[iT], t_dep)


def test_qsw_zero_leaves_kpp_uncharged(oracle):
    """With q_sw = 0 the KPP charge Q_heat - sw_pen_frac q_sw T(d) is Q_heat
    exactly: the assembly equals the one without penetration, bit for bit."""
    for method in (2, 3):
        c_off = hot_cfg()
        c_q = hot_cfg(sw_source=1, kpp_sw_method=method, **SW)
        a, b = _state(oracle, c_off), _state(oracle, c_q)
        b.sw_net[...] = 0.0
        for s, c in ((a, c_off), (b, c_q)):
            s.call("vpo_eos_wright", c)
            assert s.call("vpo_build_coefficients", c) == 0
        for n in ("kv", "kt", "ks", "b0", "bl_depth"):
            assert np.array_equal(getattr(a, n), getattr(b, n)), (method, n)


def test_qsw_charges_kpp_with_the_shortwave(oracle):
    """A q_sw larger than Q_heat's own shortwave share makes B0 more
    stabilising where the boundary layer absorbs less of it (MXL)."""
    c1 = hot_cfg(sw_source=1, kpp_sw_method=2, **SW)
    c0 = hot_cfg(kpp_sw_method=2, **SW)
    a, b = _state(oracle, c0), _state(oracle, c1)
    b.sw_net[...] = 3.0 * b.q_heat
    for s, c in ((a, c0), (b, c1)):
        s.call("vpo_eos_wright", c)
        s.bl_depth[...] = 25.0
        assert s.call("vpo_build_coefficients", c) == 0
    wet = a.wet > 0.5
    # B0 = g/rho0 (alpha_T q_T_kin - ...): a larger penetrating part lowers q_T_kin
    assert (b.b0[wet] <= a.b0[wet]).all() and (b.b0[wet] < a.b0[wet]).any()


def test_bound_salinity_floors_the_first_live_layer(oracle):
    """bound_salinity_top_impl: after the salt deposit, S = max(S, s_min) on
    the first live layer of wet columns only; nothing else moves and the
    budgets do not see it."""
    s_min = 34.9
    c0 = hot_cfg(budgets=1, surface_flux=1)
    c1 = hot_cfg(budgets=1, surface_flux=1, bound_salinity=1, min_salinity=s_min)
    a, b = _state(oracle, c0, seed=82), _state(oracle, c1, seed=82)
    a.call("vpo_surface_flux", c0, DT)
    b.call("vpo_surface_flux", c1, DT)
    iS = c0.idx_salinity
    live = a.h > 1.5e-4
    # first live layer from the top of each column
    kt = a.nz - 1 - np.argmax(live[:, :, ::-1], axis=2)
    ii, jj = np.meshgrid(np.arange(a.nx), np.arange(a.ny), indexing="ij")
    top_a = a.tracers[iS][ii, jj, kt]
    top_b = b.tracers[iS][ii, jj, kt]
    wet = a.wet > 0.5
    assert np.array_equal(top_b[wet], np.maximum(top_a[wet], s_min))
    assert (top_a[wet] < s_min).any() and (top_a[wet] > s_min).any()   # both sides of the floor occur
    assert np.array_equal(top_b[~wet], top_a[~wet])
    mask = np.ones(a.h.shape, bool)
    mask[ii, jj, kt] = False
    assert np.array_equal(a.tracers[iS][mask], b.tracers[iS][mask])
    assert np.array_equal(a.tracers[c0.idx_temperature], b.tracers[c0.idx_temperature])
    assert np.array_equal(a.salt_budget_surface, b.salt_budget_surface)


def test_wet_dyn_masks_the_deposit(oracle):
    """apply_surface_src_2d_dyn_impl: a dynamically dry column takes no
    surface flux (T, S, pseudo-salt and the budgets untouched); an all-wet
    dynamic mask is the static path bit for bit."""
    c0 = hot_cfg(budgets=1, surface_flux=1)
    c1 = hot_cfg(budgets=1, surface_flux=1, use_wet_dyn=1)
    a, b, ref = _state(oracle, c0, seed=83), _state(oracle, c1, seed=83), _state(oracle, c0, seed=83)
    a.call("vpo_surface_flux", c0, DT)
    b.call("vpo_surface_flux", c1, DT)
    for t in range(a.ntr):
        assert np.array_equal(a.tracers[t], b.tracers[t]), t
    dry = (np.arange(ref.nx)[:, None] + np.arange(ref.ny)[None, :]) % 2 == 0
    d = _state(oracle, c1, seed=83)
    d.wet_dyn[...] = np.where(dry, 0.0, 1.0)
    d.call("vpo_surface_flux", c1, DT)
    for t in range(d.ntr):
        assert np.array_equal(d.tracers[t][dry], ref.tracers[t][dry]), t
        assert np.array_equal(d.tracers[t][~dry], a.tracers[t][~dry]), t
    assert (d.heat_budget_surface[dry] == 0.0).all() and (d.salt_budget_surface[dry] == 0.0).all()
    assert np.array_equal(d.heat_budget_surface[~dry], a.heat_budget_surface[~dry])


def test_epbl_ledger_off_is_the_skin_path(oracle):
    """epbl_sw_ctke = .false. (sw_ctke_active, rdb_ocean_epbl.F90:905): the
    whole heat flux is a skin flux, the EPBL answer without penetration."""
    c_off = hot_cfg(epbl=1)
    c_nl = hot_cfg(epbl=1, epbl_sw_ctke=0, **SW)
    c_on = hot_cfg(epbl=1, **SW)
    a, b, c = (_state(oracle, cc, seed=85) for cc in (c_off, c_nl, c_on))
    for s, cc in ((a, c_off), (b, c_nl), (c, c_on)):
        s.call("vpo_epbl", cc, DT)
    assert np.array_equal(a.kd_epbl, b.kd_epbl) and np.array_equal(a.mld_epbl, b.mld_epbl)
    assert not np.array_equal(a.kd_epbl, c.kd_epbl)


def test_shortwave_penetration_closure():
    """The python mirror of forcing.ShortwavePenetration sets the knobs and
    refuses a source the reference does not implement."""
    import pytest

    from roundabout_b200.config import ShortwavePenetration, default_config

    cfg = ShortwavePenetration(fraction=0.4, source="q_sw", epbl_tke_ledger=False).apply(default_config())
    assert cfg.sw_pen_frac == 0.4 and cfg.sw_source == 1 and cfg.epbl_sw_ctke == 0
    assert default_config().epbl_sw_ctke == 1
    with pytest.raises(ValueError):
        ShortwavePenetration(source="chl")


def test_epbl_ledger_reads_qsw(oracle):
    """EPBL's shortwave ledger takes I0 from the selected source: q_sw =
    Q_heat is the net_heat answer bit for bit, a different q_sw moves it."""
    c0 = hot_cfg(epbl=1, **SW)
    c1 = hot_cfg(epbl=1, sw_source=1, **SW)
    a, b, c = _state(oracle, c0, seed=84), _state(oracle, c1, seed=84), _state(oracle, c1, seed=84)
    b.sw_net[...] = b.q_heat
    c.sw_net[...] = 0.0
    a.call("vpo_epbl", c0, DT)
    b.call("vpo_epbl", c1, DT)
    c.call("vpo_epbl", c1, DT)
    assert np.array_equal(a.kd_epbl, b.kd_epbl) and np.array_equal(a.mld_epbl, b.mld_epbl)
    assert not np.array_equal(a.kd_epbl, c.kd_epbl)


# ---- the chlorophyll N-band scheme (Manizza et al. 2005) -------------------
CHL = dict(sw_pen_frac=1.0, sw_chl=1)


def _chl_state(oracle, cfg, seed=86):
    st = _state(oracle, cfg, seed=seed)
    st.sw_chl[...] = np.abs(np.cos(np.arange(st.nx * st.ny))).reshape((st.nx, st.ny), order="F") * 2.0
    st.sw_chl[0, 0] = 0.0                     # below the 1e-4 floor
    st.call("vpo_sw_chl_kappa", cfg)
    return st


def test_chl_band_fractions_sum_to_one(oracle):
    """sw_band_fractions: blue/red split of the visible 0.42, the rest shared
    evenly; the bands sum to 1 for every band count."""
    L = oracle.lib()
    L.vpo_sw_band_frac.restype = __import__("ctypes").c_double
    L.vpo_sw_band_frac.argtypes = [__import__("ctypes").c_int] * 2 + [__import__("ctypes").c_double]
    for nb in range(3, 7):
        fr = [L.vpo_sw_band_frac(n, nb, 0.3) for n in range(1, nb + 1)]
        assert fr[0] == 0.3 * 0.42 and fr[1] == (1.0 - 0.3) * 0.42
        assert abs(sum(fr) - 1.0) <= 4e-16


def test_chl_kappa_in_closed_form(oracle):
    """sw_opacity_manizza: kappa_n = a_n + b_n max(chl, 1e-4)^p_n on wet
    columns (rdb_sm_pow: within 2 ulp of libm's pow), the land value on land."""
    cfg = hot_cfg(**CHL)
    st = _chl_state(oracle, cfg)
    chl = np.maximum(st.sw_chl, 1.0e-4)
    wet = st.wet > 0.5
    for n in range(3):
        a, b, p = cfg.sw_opacity_coef[2 * n], cfg.sw_opacity_coef[2 * n + 1], cfg.sw_chl_power[n]
        want = a + b * chl ** p
        got = st.sw_kappa[:, :, n]
        assert np.allclose(got[wet], want[wet], rtol=4e-16, atol=0.0)
        assert (got[~wet] == cfg.sw_opacity_land).all()
    assert (st.sw_kappa[:, :, 3:] == 1.0).all()     # bands past sw_nbands untouched


def test_chl_penetration_profile_and_conservation(oracle):
    """apply_sw_penetration_nb_impl: all of the source leaves the first live
    layer, each live layer takes I0 (T(d_top) - T(d_bot)) with the N-band T,
    the deepest the rest; the column's heat content is kept to round-off."""
    cfg = hot_cfg(surface_flux=1, **CHL)
    st = _chl_state(oracle, cfg)
    iT = cfg.idx_temperature
    st.call("vpo_surface_flux", cfg, DT)
    before, t0 = _heat_content(st, cfg), st.tracers[iT].copy()
    st.call("vpo_sw_penetration", cfg, DT)
    assert np.abs(_heat_content(st, cfg) - before).max() <= 1e-12 * np.abs(before).max()
    # one wet column with every layer live, against the closed form
    live = (st.h > 1.5e-4).all(axis=2) & (st.wet > 0.5)
    i, j = np.argwhere(live)[0]
    fr = np.array([0.5 * 0.42, 0.5 * 0.42, 0.58])
    kap = st.sw_kappa[i, j, :3]
    d = np.concatenate([[0.0], np.cumsum(st.h[i, j, ::-1])])          # interface depths from the surface
    T = (fr[None, :] * np.exp(-kap[None, :] * d[:, None])).sum(axis=1)
    T[-1] = 0.0                                                       # opaque bed
    absorbed = st.q_heat[i, j] * (T[:-1] - T[1:])                     # surface-down
    absorbed[0] -= st.q_heat[i, j]
    dT = (st.tracers[iT][i, j, ::-1] - t0[i, j, ::-1]) * st.h[i, j, ::-1]
    want = absorbed * DT / (cfg.rho0 * cfg.cp)
    # T_new - T_old cancels: allow a few ulp of T times the layer thickness
    tol = 1e-12 * np.abs(want) + 8 * np.finfo(float).eps * np.abs(t0[i, j, ::-1]) * st.h[i, j, ::-1]
    assert (np.abs(dT - want) <= tol).all()
    assert (want[1:] > 0).any()


def test_chl_opaque_bands_leave_kpp_uncharged(oracle):
    """With every band opaque (kappa 1e6 m-1) nothing passes the boundary
    layer of a wet column: KPP's charge Q - q_sw T(h_b) is Q exactly, the
    assembly of the shortwave-free path bit for bit."""
    c0 = hot_cfg()
    c1 = hot_cfg(kpp_sw_method=2, **CHL)
    a, b = _state(oracle, c0, seed=87), _state(oracle, c1, seed=87)
    b.sw_kappa[...] = 1.0e6
    for s, c in ((a, c0), (b, c1)):
        s.call("vpo_eos_wright", c)
        assert s.call("vpo_build_coefficients", c) == 0
    for n in ("kv", "kt", "bl_depth"):
        assert np.array_equal(getattr(a, n), getattr(b, n)), n
    # on land h_b = 0 and T(0) = 1: the whole source is charged there, as in the two-band form
    wet = a.wet > 0.5
    assert np.array_equal(a.b0[wet], b.b0[wet])


def test_chl_epbl_ledger_with_grey_bands_is_single_band(oracle):
    """The EPBL N-band ledger with every band at one opacity kappa equals a
    two-band ledger of equal e-folding depths 1/kappa, to round-off."""
    kap = 0.08
    c_nb = hot_cfg(epbl=1, epbl_tke_diags=1, **CHL)
    c_2b = hot_cfg(epbl=1, epbl_tke_diags=1, sw_pen_frac=1.0, sw_band_ratio=0.5, sw_zeta1=1.0 / kap,
                   sw_zeta2=1.0 / kap)
    a, b = _state(oracle, c_nb, seed=88), _state(oracle, c_2b, seed=88)
    a.sw_kappa[...] = kap
    a.call("vpo_epbl", c_nb, DT)
    b.call("vpo_epbl", c_2b, DT)
    assert np.allclose(a.mld_epbl, b.mld_epbl, rtol=1e-9, atol=1e-9)
    assert np.allclose(a.kd_epbl, b.kd_epbl, rtol=1e-8, atol=1e-12)


def test_cover_frac_scales_the_penetration(oracle):
    """apply_sw_penetration_cover_impl: I0 scaled by 1 - cover_frac.  No cover
    is the uncovered path bit for bit; a fully covered column takes no light
    (the deposit alone), in both the two-band and the chlorophyll forms."""
    for extra in (SW, CHL):
        c0 = hot_cfg(surface_flux=1, **extra)
        c1 = hot_cfg(surface_flux=1, use_cover_frac=1, **extra)
        a, b, d = (_state(oracle, c, seed=89) for c in (c0, c1, c1))
        d.cover_frac[...] = np.where(np.arange(d.nx)[:, None] % 2 == 0, 1.0, 0.0)
        for s, c in ((a, c0), (b, c1), (d, c1)):
            s.call("vpo_surface_flux", c, DT)
        dep = d.tracers[c1.idx_temperature].copy()
        for s, c in ((a, c0), (b, c1), (d, c1)):
            s.call("vpo_sw_penetration", c, DT)
        iT = c1.idx_temperature
        assert np.array_equal(a.tracers[iT], b.tracers[iT])
        covered = np.arange(d.nx) % 2 == 0
        assert np.array_equal(d.tracers[iT][covered], dep[covered])
        assert np.array_equal(d.tracers[iT][~covered], a.tracers[iT][~covered])
