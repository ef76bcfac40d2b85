"""The oracle's interior_closure = "none" seed (scalar backgrounds, the
background Prandtl number, kappa-shear added on top) against the reference's
known-answer tests (tests/test_ocean_vmix_no_pp81.F90), re-expressed on the
oracle (the Fortran tests cannot run here: no Fortran compiler).

The sheared column of those tests (make_sheared_column, :171-204): 8 x 6
columns of 4 layers of 100 m, bottom-up; u = 0.3 k m/s on layer k (1-based),
T = T_ref + 0.05 (k - 2) under the reference's default linear EOS (rho0 1035,
alpha_T 1.7e-4 kg/m^3/K, rdb_eos.F90:532-548), so Ri ~ 1e-4 and PP81 mixes
hard; backgrounds kv_bg = 2e-4, kt_bg = 3e-5 (seeded from the PP81 ones),
ks_bg = 5e-5.  The oracle takes rho directly, so the EOS is written out here.
Checked quantities and tolerances are the reference tests' own:
  PP81 on the column lifts kv above 20 kv_bg, while "none" gives exactly
      kt_bg, kv_bg and ks_bg on every interior interface and zero on the bed
      and the surface (test_none_scalar, :206-247);
  bkgnd_prandtl = 1 with kv_bg = 0 gives kv == kt == kt_bg exactly;
      bkgnd_prandtl = 2 with kv_bg = 1e-5 gives kv = 2 kt_bg + kv_bg to 1e-18
      (test_prandtl, :311-366; its Henyey leg is a latitude-dependent
      background this library refuses);
  "none" with kappa-shear on a uniformly stratified 12-layer column with one
      0.2 m/s velocity jump (ks_pipeline, :368-433): the resting control is
      exactly the background, the jump's interface mixes above 10x the
      background, the merge is additive (background + pure shear to 1e-15
      relative), the peak sits at the jump, every other interface mixes less
      but never below the background, and the boundary interfaces stay zero
      (test_none_kappa_shear, :435-489).
"""
import numpy as np

from roundabout_b200.config import INTERIOR_NONE, INTERIOR_PP81, default_config, seed_backgrounds

NX, NY, NZ, H0 = 8, 6, 4, 100.0
KT_BG, KS_BG, KV_BG = 3.0e-5, 5.0e-5, 2.0e-4
EOS_RHO0, EOS_ALPHA_T = 1035.0, 1.7e-4


def sheared_cfg(closure, **kw):
    c = default_config()
    c.rho0 = EOS_RHO0
    c.use_kpp = 0
    c.interior_closure = closure
    c.pp81_nu_bg = KV_BG
    c.pp81_kappa_bg = KT_BG
    seed_backgrounds(c)
    c.ks_bg = KS_BG
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def sheared_column(oracle):
    st = oracle.OracleState(NX, NY, NZ, 2)
    st.h[...] = H0
    for k in range(1, NZ + 1):
        st.u[:, :, k - 1] = 0.3 * k
        st.rho[:, :, k - 1] = EOS_RHO0 - EOS_ALPHA_T * (0.05 * (k - 2))
    return st


def build(oracle, c):
    st = sheared_column(oracle)
    # stale coefficients from an earlier step, which the seed must overwrite
    st.kv[...] = 1.0
    st.kt[...] = 1.0
    st.ks[...] = 1.0
    assert st.call("vpo_build_coefficients", c) == 0
    return st


def test_none_gives_exactly_the_scalar_backgrounds(oracle):
    witness = build(oracle, sheared_cfg(INTERIOR_PP81))
    assert witness.kv[:, :, 1:NZ].max() > 20.0 * KV_BG
    st = build(oracle, sheared_cfg(INTERIOR_NONE))
    assert (st.kt[:, :, 1:NZ] == KT_BG).all()
    assert (st.kv[:, :, 1:NZ] == KV_BG).all()
    assert (st.ks[:, :, 1:NZ] == KS_BG).all()   # ks follows kt, floored at ks_bg > kt_bg
    assert (st.kv[:, :, 0] == 0.0).all() and (st.kv[:, :, NZ] == 0.0).all()


def test_prandtl_one_ties_kv_to_kt(oracle):
    st = build(oracle, sheared_cfg(INTERIOR_NONE, kv_bg=0.0, bkgnd_prandtl=1.0))
    assert (st.kv[:, :, 1:NZ] == st.kt[:, :, 1:NZ]).all()
    assert (st.kv[:, :, 1:NZ] == KT_BG).all()


def test_prandtl_two_adds_the_momentum_background(oracle):
    st = build(oracle, sheared_cfg(INTERIOR_NONE, kv_bg=1.0e-5, bkgnd_prandtl=2.0))
    assert np.abs(st.kv[:, :, 1:NZ] - (2.0 * KT_BG + 1.0e-5)).max() < 1.0e-18


# ks_pipeline (:368-433): 4 x 4 columns of 12 layers of 5 m, N^2 = 3e-5 under
# a linear EOS, f = 1e-4, dt = 1800 s; u = du on the layers above KJ
NZK, KJ, DZ, N2 = 12, 6, 5.0, 3.0e-5
KS_RHO0, GRAVITY, DT = 1025.0, 9.80665, 1800.0
KS_ALPHA = KS_RHO0 * 2.0e-4


def ks_pipeline(oracle, du, kv_bg, kt_bg):
    c = default_config()
    c.interior_closure = INTERIOR_NONE
    c.pp81_nu_bg = kv_bg
    c.pp81_kappa_bg = kt_bg
    seed_backgrounds(c)
    c.kappa_shear = 1
    c.eos_variant = 1
    c.eos_alpha_t = KS_ALPHA
    c.eos_beta_s = KS_RHO0 * 7.6e-4
    c.rho0 = KS_RHO0
    st = oracle.OracleState(4, 4, NZK, 2)
    dtdz = N2 * KS_RHO0 / (GRAVITY * KS_ALPHA)
    st.h[...] = DZ
    for k in range(1, NZK + 1):
        st.tracers[c.idx_temperature][:, :, k - 1] = 20.0 + dtdz * DZ * (k - NZK)
        st.tracers[c.idx_salinity][:, :, k - 1] = 35.0
        if k > KJ:
            st.u[:, :, k - 1] = du
    st.coriolis[...] = 1.0e-4
    # the production stage order: reset, kappa-shear, merge, split, assemble
    st.call("vpo_seed_interior_none", c)
    st.call("vpo_kappa_shear", c, DT)
    st.call("vpo_kappa_shear_merge", c)
    st.call("vpo_split", c)
    assert st.call("vpo_assemble_gate", c) == 0
    return st.kv[2, 2, :].copy(), st.kt[2, 2, :].copy()


def test_none_with_kappa_shear_adds_to_the_background(oracle):
    assert N2 * DZ * DZ / 0.2 ** 2 < 0.25
    kv0, kt0 = ks_pipeline(oracle, 0.0, KV_BG, KT_BG)
    assert (kv0[1:NZK] == KV_BG).all() and (kt0[1:NZK] == KT_BG).all()
    kv1, kt1 = ks_pipeline(oracle, 0.2, KV_BG, KT_BG)
    kvs, kts = ks_pipeline(oracle, 0.2, 0.0, 0.0)
    jump = KJ   # interface KJ + 1, 1-based
    assert kv1[jump] > 10.0 * KV_BG and kt1[jump] > 10.0 * KT_BG
    assert kts[jump] > 10.0 * KT_BG
    for k in range(1, NZK):
        assert abs(kt1[k] - (KT_BG + kts[k])) <= 1.0e-15 * kt1[k], k
        assert abs(kv1[k] - (KV_BG + kvs[k])) <= 1.0e-15 * kv1[k], k
    assert int(np.argmax(kv1[1:NZK])) + 1 == jump
    for k in range(1, NZK):
        if k == jump:
            continue
        assert kv1[k] < kv1[jump] and kt1[k] < kt1[jump], k
        assert kv1[k] >= KV_BG and kt1[k] >= KT_BG, k
    assert kv1[0] == 0.0 and kv1[NZK] == 0.0
