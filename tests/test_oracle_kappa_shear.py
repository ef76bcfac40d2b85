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
