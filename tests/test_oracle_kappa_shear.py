"""Known-answer tests of the kappa-shear oracle (vphys_oracle_kshear.c),
re-expressed from the reference's tests/test_ocean_kappa_shear.F90:

* golden profile (:286-393): the nz=20 tanh shear column, linear EOS, to the
  reference's golden kd values (its Python prototype's) within 1e-6
  relative;
* no source (:155-208): a strongly stratified resting column gives kd == 0
  exactly and interior TKE below 1e-15;
* activation (:214-280): a mid-column shear layer with Ri ~ 0.1 gives a
  non-negative, interior-peaked kd, exactly 0 on the bed and the surface;
* self-limiting (:399-467): relaxing the shear by 80 % drops max kd > 5x;
* merge (:473-544): kt += kd, kv += prandtl * kd on interior interfaces
  only.
"""
import math

import numpy as np
import pytest

G = 9.80665
RHO0 = 1025.0
ALPHA = RHO0 * 2.0e-4
BETA = RHO0 * 7.6e-4
F_CORIOLIS = 1.0e-4
DT = 1800.0

# kd_int of the golden column, surface-down (local K = 0 is the surface),
# test_ocean_kappa_shear.F90:316-338
GOLDEN_SD = [
    0.0, 5.84500291421640155e-03, 2.55834506759574087e-02, 6.18743388406512718e-02, 1.18040171371964375e-01,
    1.94158207598627230e-01, 2.79264861473862980e-01, 3.75428011380740556e-01, 4.54336837449636988e-01,
    5.06855656580426306e-01, 5.25366868234401263e-01, 5.06855484093826858e-01, 4.54336485854091421e-01,
    3.75427466061297621e-01, 2.79264096140142026e-01, 1.94157172096779573e-01, 1.18038778175938969e-01,
    6.18736389220278515e-02, 2.55832135500080882e-02, 5.84500603701821296e-03, 0.0,
]


def ks_config(**over):
    from roundabout_b200.config import default_config

    c = default_config()
    c.kappa_shear = 1
    c.eos_variant = 1
    c.eos_alpha_t = ALPHA
    c.eos_beta_s = BETA
    c.rho0 = RHO0
    for k, v in over.items():
        setattr(c, k, v)
    return c


def shear_column(oracle, nz, dz, du, depth, width, strat_n2, nx=2, ny=2):
    """setup_shear_column (test_ocean_kappa_shear.F90:123-149): T stable
    with N^2 = strat_n2 under the linear EOS, S = 35, u = du tanh((depth -
    z)/width) on both faces of every cell, v = 0."""
    st = oracle.OracleState(nx, ny, nz, 2)
    dtdm = strat_n2 * RHO0 / (G * ALPHA)
    st.h[...] = dz
    for k in range(1, nz + 1):
        z = (float(nz - k) + 0.5) * dz
        st.tracers[1][:, :, k - 1] = 20.0 - dtdm * z
        st.tracers[0][:, :, k - 1] = 35.0
        st.u[:, :, k - 1] = du * math.tanh((depth - z) / width)
    st.coriolis[...] = F_CORIOLIS
    return st


def test_golden_profile(oracle):
    st = shear_column(oracle, 20, 5.0, 0.5, 50.0, 20.0, 3.0e-5)
    st.call("vpo_kappa_shear", ks_config(), DT)
    kd = st.kd_shear
    assert kd[1, 1, 0] == 0.0 and kd[1, 1, 20] == 0.0
    worst = 0.0
    for k_local, ref in enumerate(GOLDEN_SD):
        got = kd[1, 1, 20 - k_local]
        if ref > 1e-10:
            worst = max(worst, abs(got - ref) / ref)
    assert worst < 1.0e-6, worst
    # every column of the uniform domain is the same column
    assert np.array_equal(kd, np.broadcast_to(kd[:1, :1, :], kd.shape))


def test_no_source(oracle):
    nz, dz = 20, 10.0
    st = oracle.OracleState(2, 2, nz, 2)
    st.h[...] = dz
    for k in range(1, nz + 1):
        st.tracers[1][:, :, k - 1] = 20.0 - 0.05 * ((nz - k) * dz + 0.5 * dz)
        st.tracers[0][:, :, k - 1] = 35.0
    st.coriolis[...] = F_CORIOLIS
    st.call("vpo_kappa_shear", ks_config(), DT)
    assert np.abs(st.kd_shear).max() == 0.0
    assert np.abs(st.tke_shear[:, :, 1:nz]).max() < 1.0e-15


def test_activation(oracle):
    nz = 40
    st = shear_column(oracle, nz, 5.0, 0.5, 100.0, 20.0, 3.0e-5)
    st.call("vpo_kappa_shear", ks_config(), DT)
    kd = st.kd_shear[1, 1, :]
    assert kd[0] == 0.0 and kd[nz] == 0.0
    interior = kd[1:nz]
    assert interior.max() > 0.0
    assert (interior >= 0.0).all()
    k_max = int(np.argmax(interior)) + 2          # 1-based global interface
    assert 2 < k_max < nz


def test_self_limiting(oracle):
    nz = 40
    st = shear_column(oracle, nz, 5.0, 0.5, 100.0, 20.0, 3.0e-5)
    cfg = ks_config()
    st.call("vpo_kappa_shear", cfg, DT)
    kd1 = st.kd_shear[1, 1, 1:nz].max()
    assert kd1 > 0.0
    u_col = st.u[1, 1, :].copy()
    u_mean = u_col.sum() / nz
    for k in range(nz):
        st.u[:, :, k] = u_mean + 0.2 * (u_col[k] - u_mean)
    st.call("vpo_kappa_shear", cfg, DT)
    kd2 = st.kd_shear[1, 1, 1:nz].max()
    assert kd2 < kd1 / 5.0, (kd1, kd2)


def test_merge(oracle):
    nz = 6
    st = oracle.OracleState(4, 4, nz, 2)
    st.kd_shear[...] = 0.0
    for k in range(2, nz + 1):
        st.kd_shear[:, :, k - 1] = k * 1.0e-3
    st.kv[...] = 1.0e-4
    st.kt[...] = 5.0e-5
    st.call("vpo_kappa_shear_merge", ks_config(ks_prandtl_turb=0.8))
    assert (st.kt[:, :, 0] == 5.0e-5).all() and (st.kt[:, :, nz] == 5.0e-5).all()
    assert (st.kv[:, :, 0] == 1.0e-4).all() and (st.kv[:, :, nz] == 1.0e-4).all()
    for k in range(2, nz + 1):
        assert np.abs(st.kt[:, :, k - 1] - (5.0e-5 + k * 1.0e-3)).max() < 1.0e-15
        assert np.abs(st.kv[:, :, k - 1] - (1.0e-4 + 0.8 * k * 1.0e-3)).max() < 1.0e-15


def test_land_and_missing_tracers(oracle):
    st = shear_column(oracle, 12, 5.0, 0.5, 30.0, 10.0, 1.0e-5)
    st.wet[0, :] = 0.0
    st.kd_shear[...] = 7.0
    st.call("vpo_kappa_shear", ks_config(), DT)
    assert (st.kd_shear[0] == 0.0).all() and (st.tke_shear[0] == 0.0).all()
    assert st.kd_shear[1].max() > 0.0
    # no temperature tracer: kappa_shear_compute returns without touching kd
    st.kd_shear[...] = 7.0
    st.call("vpo_kappa_shear", ks_config(idx_temperature=-1), DT)
    assert (st.kd_shear == 7.0).all()


@pytest.mark.parametrize("nz", [1, 2, 3])
def test_shallow_columns(oracle, nz):
    """nz = 1 takes the single-layer pre-step (ks_solve_column :1612-1617);
    every shallow column ends with kd = 0 on its bed and surface."""
    st = shear_column(oracle, nz, 4.0, 0.3, 2.0, 1.0, 1.0e-6)
    st.call("vpo_kappa_shear", ks_config(), DT)
    assert np.isfinite(st.kd_shear).all() and np.isfinite(st.tke_shear).all()
    assert (st.kd_shear[:, :, 0] == 0.0).all() and (st.kd_shear[:, :, nz] == 0.0).all()


# ---- the massless merge (tests/test_ocean_massless.F90) -------------------
H_VANISHED = 1.5e-4


def _maps(oracle, h):
    """vpo_massless_build_maps on a 1-based surface-down column h[1..nz]."""
    import ctypes

    nz = len(h)
    h1 = np.zeros(nz + 2)
    h1[1:nz + 1] = h
    hc, kf = np.zeros(nz + 2), np.zeros(nz + 2)
    kc = np.zeros(nz + 2, dtype=np.int32)
    nzc = ctypes.c_int()
    dp = ctypes.POINTER(ctypes.c_double)
    L = oracle.lib()
    L.vpo_massless_build_maps(h1.ctypes.data_as(dp), nz, ctypes.c_double(H_VANISHED), ctypes.byref(nzc),
                              hc.ctypes.data_as(dp), kc.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                              kf.ctypes.data_as(dp))
    return h1, nzc.value, hc, kc, kf


def _merge(oracle, h1, kc, nzc, fields):
    import ctypes

    dp = ctypes.POINTER(ctypes.c_double)
    nz = len(h1) - 2
    ins = []
    for f in fields:
        a = np.zeros(nz + 2)
        a[1:nz + 1] = f
        ins.append(a)
    outs = [np.zeros(nz + 2) for _ in range(4)]
    oracle.lib().vpo_massless_merge_fields(h1.ctypes.data_as(dp), kc.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                           nz, nzc, *[a.ctypes.data_as(dp) for a in ins],
                                           *[a.ctypes.data_as(dp) for a in outs])
    return outs


def test_massless_golden_maps(oracle):
    """The worked nz = 8 example (test_ocean_massless.F90:63-140)."""
    h = [12.0, 10.0, H_VANISHED * 0.5, 15.0, 8.0, H_VANISHED * 0.5, 6.0, 9.0]
    h1, nzc, hc, kc, kf = _maps(oracle, h)
    assert nzc == 6
    assert list(kc[1:10]) == [1, 2, 2, 3, 4, 4, 5, 6, 7]
    assert hc[1] == 12.0 and hc[3] == 15.0 and hc[5] == 6.0 and hc[6] == 9.0
    assert abs(hc[2] - (10.0 + H_VANISHED * 0.5)) < 1e-15 and abs(hc[4] - (8.0 + H_VANISHED * 0.5)) < 1e-15
    assert abs(kf[3] - 0.99999250005624951) < 1e-14 and abs(kf[6] - 0.99999062508788972) < 1e-14
    assert all(kf[k] == 0.0 for k in (1, 2, 4, 5, 7, 8, 9))
    u = [0.1, 0.2, 0.0, 0.15, 0.05, 0.0, -0.1, -0.05]
    v = [0.0, 0.05, 0.0, -0.1, 0.1, 0.0, 0.08, 0.02]
    t = [22.0, 20.0, 19.5, 18.0, 16.0, 15.5, 14.0, 12.0]
    s = [35.0, 35.2, 35.3, 35.5, 35.6, 35.65, 35.7, 35.8]
    uc, vc, tc, sc = _merge(oracle, h1, kc, nzc, (u, v, t, s))
    assert tc[1] == 22.0 and tc[3] == 18.0 and tc[6] == 12.0
    assert abs(tc[2] - 19.999996250028122) < 1e-12


def test_massless_identity_and_conservation(oracle):
    """I1 (test_ocean_massless.F90:142-205): a healthy column maps onto
    itself bit for bit and interp_back is the identity; I2 (:207-268): the
    merged thickness and thickness-weighted T, S integrals are conserved."""
    import ctypes

    nz = 12
    h = [5.0 + k for k in range(1, nz + 1)]
    h1, nzc, hc, kc, kf = _maps(oracle, h)
    assert nzc == nz and list(kc[1:nz + 2]) == list(range(1, nz + 2))
    assert (kf[1:nz + 2] == 0.0).all() and np.array_equal(hc[1:nz + 1], h1[1:nz + 1])
    qc = np.zeros(nz + 2)
    qc[1:nz + 2] = [1.0e-3 * (k * k - 3 * k) for k in range(1, nz + 2)]
    q = np.zeros(nz + 2)
    dp = ctypes.POINTER(ctypes.c_double)
    oracle.lib().vpo_massless_interp_back(qc.ctypes.data_as(dp), kc.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                          kf.ctypes.data_as(dp), nz, q.ctypes.data_as(dp))
    assert np.array_equal(q[1:nz + 2], qc[1:nz + 2])

    h = [10.0, H_VANISHED * 0.4, 12.0, 8.0, H_VANISHED * 0.6, H_VANISHED * 0.2, 7.0, 9.0, H_VANISHED * 0.3, 5.0, 6.0]
    t = [18.0 - 0.3 * k for k in range(1, 12)]
    s = [34.5 + 0.05 * k for k in range(1, 12)]
    h1, nzc, hc, kc, kf = _maps(oracle, h)
    _, _, tc, sc = _merge(oracle, h1, kc, nzc, ([0.0] * 11, [0.0] * 11, t, s))
    assert abs(sum(hc[1:nzc + 1]) - sum(h)) <= 1e-13 * sum(h)
    assert abs(sum(tc[k] * hc[k] for k in range(1, nzc + 1)) - sum(a * b for a, b in zip(t, h))) <= 1e-12 * 1e3
    assert abs(sum(sc[k] * hc[k] for k in range(1, nzc + 1)) - sum(a * b for a, b in zip(s, h))) <= 1e-12 * 1e4


def _zstar_like(oracle, nz, has_vanish):
    """setup_zstar_like_column (test_ocean_massless.F90:289-326): 10 m layers,
    the three bed-side ones vanished when has_vanish, the golden test's tanh
    shear and stratification."""
    st = oracle.OracleState(2, 2, nz, 2)
    dtdm = 3.0e-5 * RHO0 / (G * ALPHA)
    for k in range(1, nz + 1):
        k_sd = nz + 1 - k
        h = H_VANISHED * 0.5 if (has_vanish and k_sd > nz - 3) else 10.0
        z = (k_sd - 1 + 0.5) * 10.0
        st.h[:, :, k - 1] = h
        st.tracers[1][:, :, k - 1] = 20.0 - dtdm * z
        st.tracers[0][:, :, k - 1] = 35.0
        st.u[:, :, k - 1] = 0.5 * math.tanh((50.0 - z) / 20.0)
    st.coriolis[...] = F_CORIOLIS
    return st


def test_massless_merge_end_to_end(oracle):
    """T4a / T4b (test_ocean_massless.F90:328-430): on a column with vanished
    layers the merge changes kd (and keeps 0 on the bed and surface); on a
    healthy column merge on equals merge off bit for bit."""
    nz = 12
    out = {}
    for vanish in (True, False):
        for merge in (0, 1):
            st = _zstar_like(oracle, nz, vanish)
            st.call("vpo_kappa_shear", ks_config(ks_massless_merge=merge), DT)
            out[(vanish, merge)] = (st.kd_shear.copy(), st.tke_shear.copy())
    on = out[(True, 1)][0]
    assert on[1, 1, 0] == 0.0 and on[1, 1, nz] == 0.0
    assert np.abs(on - out[(True, 0)][0]).max() > 1e-9
    assert np.array_equal(out[(False, 1)][0], out[(False, 0)][0])
    assert np.array_equal(out[(False, 1)][1], out[(False, 0)][1])
