"""The oracle's assembly gate (1-2-1 smoothing), the heat/salt split and PP81
against the known-answer tests of tests/test_ocean_vmix_assembly.F90 and
tests/test_ocean_pp81.F90 that tests/test_oracle_kat.py does not already
restate, re-expressed on the oracle (the Fortran tests cannot run here: no
Fortran compiler).

The reference runs these on a 12 x 10 grid with two ghost cells; its
smoothing walks i = 2..nx_total - 1, j = 2..ny_total - 1 of the whole
16 x 14 array, which the oracle's walk over its own 16 x 14 array matches
(indices below are the reference's 1-based ones, minus one).  Checked
quantities and tolerances are the reference tests' own:
  one smoothing pass of a delta of 16 gives 4 / 2 / 1 at the centre, edge
      and corner to 1e-13, kt smoothed like kv, the interior sum kept to
      1e-12 (test_smooth_121, :192-238);
  a uniform 1 with one dry column: the dry value unchanged, no wet value
      above 1 + 1e-13, the wet sum kept to 1e-11 (test_smooth_wetdry,
      :240-310);
  two passes over a non-uniform field with a dry column smooth ks and kt
      to the same bits (test_smooth_ks_matches_kt, :632-671);
  the split overwrites ks with kt on every interface, the boundary ones
      included (test_split_derives_ks, :591-630);
  PP81 at a known Ri: kv = nu_bg + nu0 / (1 + alpha Ri)^2 to 1e-10 for
      alpha 4 and 9 (test_pp81_alpha_changes_answer, :500-590);
  a quiescent stratified column: the edge columns' kv equals their
      neighbours' to 1e-18 (test_ocean_pp81.F90 test_wall_symmetry, :310-374).
The reference's configuration-wiring cases of the same file (knobs reaching
the slot, defaults unchanged) concern its namelist plumbing, which
tests/test_closures_mirror.py mirrors for this library's configuration.
"""
import numpy as np

from roundabout_b200.config import default_config

NX, NY = 16, 14
G = 9.80665


def cfg(**kw):
    c = default_config()
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def floors_off(**kw):
    return cfg(kv_bg=0.0, kt_bg=0.0, ks_bg=0.0, **kw)


def blank(oracle, nz):
    st = oracle.OracleState(NX, NY, nz, 2)
    st.h[...] = 5.0
    st.kv[...] = 0.0
    st.kt[...] = 0.0
    st.ks[...] = 0.0
    return st


def test_one_pass_on_a_delta_is_the_121_stencil(oracle):
    KI = 1                                   # 1-based interface 2
    ic, jc = 5, 4                            # 1-based (6, 5)
    st = blank(oracle, 3)
    st.kv[ic, jc, KI] = 16.0
    st.kt[ic, jc, KI] = 16.0
    before = st.kv[1:NX - 1, 1:NY - 1, KI].sum()
    assert st.call("vpo_assemble_gate", floors_off(kd_smooth_iterations=1)) == 0
    assert abs(st.kv[ic, jc, KI] - 4.0) < 1.0e-13
    assert abs(st.kv[ic - 1, jc, KI] - 2.0) < 1.0e-13
    assert abs(st.kv[ic - 1, jc - 1, KI] - 1.0) < 1.0e-13
    assert abs(st.kt[ic, jc, KI] - 4.0) < 1.0e-13
    assert abs(st.kv[1:NX - 1, 1:NY - 1, KI].sum() - before) < 1.0e-12


def test_smoothing_neither_leaks_into_nor_out_of_a_dry_column(oracle):
    KI = 1
    id_, jd = 5, 4
    st = blank(oracle, 3)
    st.kv[:, :, KI] = 1.0
    st.wet[id_, jd] = 0.0
    interior = np.zeros((NX, NY), dtype=bool)
    interior[1:NX - 1, 1:NY - 1] = True
    wet_interior = interior & (st.wet > 0.0)
    before = st.kv[:, :, KI][wet_interior].sum()
    assert st.call("vpo_assemble_gate", floors_off(kd_smooth_iterations=1)) == 0
    assert st.kv[id_, jd, KI] == 1.0
    assert st.kv[1:NX - 1, 1:NY - 1, KI].max() <= 1.0 + 1.0e-13
    assert abs(st.kv[:, :, KI][wet_interior].sum() - before) < 1.0e-11


def test_smoothing_treats_ks_like_kt(oracle):
    nz = 4
    st = blank(oracle, nz)
    for k in range(2, nz + 1):
        for j in range(1, NY + 1):
            for i in range(1, NX + 1):
                st.kt[i - 1, j - 1, k - 1] = 1.0e-3 + 1.0e-4 * (i + j + k)
    st.ks[...] = st.kt
    st.wet[5, 4] = 0.0
    assert st.call("vpo_assemble_gate", cfg(kd_smooth_iterations=2)) == 0
    assert np.array_equal(st.ks, st.kt)


def test_split_overwrites_ks_with_kt_everywhere(oracle):
    nz = 5
    st = blank(oracle, nz)
    for k in range(1, nz + 2):
        st.kt[:, :, k - 1] = 1.0e-4 + 1.0e-5 * k
    st.ks[...] = -999.0
    st.call("vpo_split", cfg())
    assert np.array_equal(st.ks, st.kt)


def test_pp81_follows_its_alpha(oracle):
    NZ, H, U_STEP, DRHO = 4, 10.0, 0.1, 0.1
    NU0, NU_BG, SHEAR_FLOOR = 1.5e-2, 3.0e-4, 1.0e-12
    got, want = [], []
    for alpha in (4.0, 9.0):
        c = cfg(pp81_nu0=NU0, pp81_nu_bg=NU_BG, shear2_floor=SHEAR_FLOOR, pp81_alpha=alpha)
        st = oracle.OracleState(NX, NY, NZ, 2)
        st.h[...] = H
        for k in range(1, NZ + 1):
            st.u[:, :, k - 1] = U_STEP * (k - 1)
            st.rho[:, :, k - 1] = 1030.0 - DRHO * (k - 1)
        st.call("vpo_pp81", c)
        ri = (G * DRHO / (c.rho0 * H)) / max((U_STEP / H) ** 2, SHEAR_FLOOR)
        got.append(st.kv[NX // 2 - 1, NY // 2 - 1, 1])
        want.append(NU_BG + NU0 / (1.0 + alpha * ri) ** 2)
    assert abs(want[0] - want[1]) > 1.0e-8
    assert all(abs(g - w) < 1.0e-10 for g, w in zip(got, want))


def test_pp81_edge_columns_match_their_neighbours(oracle):
    NZ = 5
    st = oracle.OracleState(NX, NY, NZ, 2)
    st.h[...] = 10.0
    for k in range(1, NZ + 1):
        st.rho[:, :, k - 1] = 1030.0 - (k - 1)
    st.call("vpo_pp81", cfg())
    kv = st.kv[:, :, 1:NZ]
    diff = max(np.abs(kv[0, 4] - kv[1, 4]).max(), np.abs(kv[-1, 4] - kv[-2, 4]).max(),
               np.abs(kv[4, 0] - kv[4, 1]).max(), np.abs(kv[4, -1] - kv[4, -2]).max())
    assert diff < 1.0e-18
