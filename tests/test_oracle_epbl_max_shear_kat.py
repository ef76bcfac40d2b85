"""The oracle's EPBL combine = "max_shear" (kt = bg + max(kd_shear, kd_epbl),
kv = kv_bg + max(prandtl_turb kd_shear, prandtl_epbl kd_epbl)) against the
reference's known-answer tests (tests/test_ocean_epbl_max_shear.F90),
re-expressed on the oracle (the Fortran tests cannot run here: no Fortran
compiler).

The column of those tests (run_column, :45-134): 4 x 4 columns of 12 layers
of 5 m, bottom-up, N^2 = 3e-5 under a linear EOS (rho0 1025), f = 1e-4,
dt = 1800 s, one 0.2 m/s velocity jump above layer 6, so kappa-shear peaks at
interface B = 7 (1-based); interior closure "none" with kv_bg = 2e-4,
kt_bg = 3e-5; an imposed EPBL kd of 0.05 at interface A = 3 (far above the
local shear) and 1e-4 at B (far below it), prandtl_epbl = 1.5.  Checked
quantities and tolerances are the reference tests' own:
  A takes bg + kd_epbl and kv_bg + 1.5 kd_epbl, B bg + kd_shear and
      kv_bg + prandtl_turb kd_shear, to 1e-15 relative; "add" differs at
      both, "max" at A (test_two_interfaces, :143-169);
  without kappa-shear "max_shear" equals "add" bit for bit and is bg + EPBL
      (test_no_shear_is_add, :171-183).
"""
import numpy as np

from roundabout_b200.config import INTERIOR_NONE, default_config, seed_backgrounds

NZK, KJ, DZ, N2, DU = 12, 6, 5.0, 3.0e-5, 0.2
KA, KB = 3, KJ + 1                      # 1-based interfaces
KT_BG, KV_BG = 3.0e-5, 2.0e-4
PR_EPBL, KD_A, KD_B = 1.5, 0.05, 1.0e-4
RHO0, GRAVITY, DT = 1025.0, 9.80665, 1800.0
ALPHA = RHO0 * 2.0e-4
ADD, MAX, MAX_SHEAR = 1, 2, 3


def run_column(oracle, mode, with_shear):
    c = default_config()
    c.interior_closure = INTERIOR_NONE
    c.pp81_nu_bg = KV_BG
    c.pp81_kappa_bg = KT_BG
    seed_backgrounds(c)
    c.kappa_shear = 1 if with_shear else 0
    c.eos_variant = 1
    c.eos_alpha_t = ALPHA
    c.eos_beta_s = RHO0 * 7.6e-4
    c.rho0 = RHO0
    c.epbl = 1
    c.epbl_prandtl = PR_EPBL
    c.epbl_combine = mode
    st = oracle.OracleState(4, 4, NZK, 2)
    dtdz = N2 * RHO0 / (GRAVITY * ALPHA)
    st.h[...] = DZ
    for k in range(1, NZK + 1):
        st.tracers[c.idx_temperature][:, :, k - 1] = 20.0 + dtdz * DZ * (k - NZK)
        st.tracers[c.idx_salinity][:, :, k - 1] = 35.0
        if k > KJ:
            st.u[:, :, k - 1] = DU
    st.coriolis[...] = 1.0e-4
    st.kd_epbl[...] = 0.0
    st.kd_epbl[:, :, KA - 1] = KD_A
    st.kd_epbl[:, :, KB - 1] = KD_B
    st.call("vpo_seed_interior_none", c)
    if with_shear:
        st.call("vpo_kappa_shear", c, DT)
        if mode != MAX_SHEAR:
            st.call("vpo_kappa_shear_merge", c)
    # with "max_shear" and kappa-shear on, the EPBL merge folds kappa-shear in first
    st.call("vpo_epbl_merge", c)
    return st.kv[2, 2, :].copy(), st.kt[2, 2, :].copy(), st.kd_shear[2, 2, :].copy(), c.ks_prandtl_turb


def close_rel(a, b):
    return abs(a - b) <= 1.0e-15 * abs(b)


def test_max_shear_picks_the_larger_mixing_at_each_interface(oracle):
    kv, kt, kd_s, pt = run_column(oracle, MAX_SHEAR, True)
    a, b = KA - 1, KB - 1
    assert kd_s[a] < 0.2 * KD_A and kd_s[b] > 100.0 * KD_B
    assert close_rel(kt[a], KT_BG + KD_A)
    assert close_rel(kv[a], KV_BG + PR_EPBL * KD_A)
    assert close_rel(kt[b], KT_BG + kd_s[b])
    assert close_rel(kv[b], KV_BG + pt * kd_s[b])
    _, kt_add, _, _ = run_column(oracle, ADD, True)
    _, kt_max, _, _ = run_column(oracle, MAX, True)
    assert not close_rel(kt_add[a], kt[a]) and not close_rel(kt_add[b], kt[b])
    assert not close_rel(kt_max[a], kt[a])


def test_max_shear_without_kappa_shear_is_add(oracle):
    kv1, kt1, _, _ = run_column(oracle, MAX_SHEAR, False)
    kv2, kt2, _, _ = run_column(oracle, ADD, False)
    assert np.array_equal(kt1, kt2) and np.array_equal(kv1, kv2)
    assert close_rel(kt1[KA - 1], KT_BG + KD_A) and close_rel(kv1[KB - 1], KV_BG + PR_EPBL * KD_B)
