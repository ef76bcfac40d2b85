"""The oracle's backward-Euler solves against the known-answer tests of
tests/test_ocean_vdiff.F90 that tests/test_oracle_kat.py does not already
restate, re-expressed on the oracle (the Fortran tests cannot run here: no
Fortran compiler).

Bottom-up like the reference: level 1 is the bed, nz = 6 the surface; the
diffusivity is a constant on the interior interfaces, zero on the bed and
surface ones.  Checked quantities and tolerances are the reference tests'
own:
  momentum with kv = 0: u and v unchanged to 1e-12 (test_momentum_zero,
      :406-444);
  momentum with kv dt / h^2 = 1000 across a +1 / -1 shear: finite, no
      overshoot past 1 + 1e-6, and damped below half the initial range
      (test_momentum_stab, :446-492);
  the heat and salt budget contributors telescope: their domain sums are
      below 1e-12 of the content and equal the content change to 1e-12 of it
      (test_vdiff_budget_contributor, :494-566);
  harmonic and arithmetic face thickness agree to 1e-14 on uniform layers
      (test_harmonic_uniform, :568-622); on a 10 m / 0.1 m pair the solve
      uses the 2 h_a h_b / (h_a + h_b) face harmonically and the mean
      arithmetically, which the 2 x 2 closed form checks to 1e-14 relative
      (test_harmonic_thin_layer, :624-652, states the face values; here
      they are read off the solve that uses them);
  ks = 4 kt on a step profile: T and S each match an independent Thomas
      solve with their own diffusivity to 1e-13, S moves further than T,
      both columns keep their content to 1e-12 (test_per_tracer_kt_ne_ks,
      :708-819, with host_diffuse_column, :658-706);
  a passive tracer follows ks like salinity, bit for bit, and differs from
      temperature (test_passive_tracer_follows_ks, :890-952).
"""
import numpy as np

from roundabout_b200.config import default_config

NZ = 6


def cfg(**kw):
    c = default_config()
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def interior(a, value):
    a[...] = value
    a[:, :, 0] = 0.0
    a[:, :, -1] = 0.0


def thomas_column(h, K, dt, t_in, harmonic=False):
    """Backward-Euler diffusion of one column, K on nz + 1 interfaces with
    zero at the bed and the surface, solved by the Thomas algorithm."""
    nz = len(h)

    def face(ha, hb):
        return 2.0 * ha * hb / (ha + hb) if harmonic else 0.5 * (ha + hb)

    a, b, c = np.zeros(nz), np.ones(nz), np.zeros(nz)
    for k in range(nz):
        if k > 0:
            beta = dt * K[k] / (h[k] * face(h[k - 1], h[k]))
            a[k] -= beta
            b[k] += beta
        if k < nz - 1:
            alpha = dt * K[k + 1] / (h[k] * face(h[k], h[k + 1]))
            c[k] -= alpha
            b[k] += alpha
    cp, dp = np.zeros(nz), np.zeros(nz)
    cp[0], dp[0] = c[0] / b[0], t_in[0] / b[0]
    for k in range(1, nz):
        den = b[k] - a[k] * cp[k - 1]
        cp[k] = c[k] / den
        dp[k] = (t_in[k] - a[k] * dp[k - 1]) / den
    out = np.zeros(nz)
    out[-1] = dp[-1]
    for k in range(nz - 2, -1, -1):
        out[k] = dp[k] - cp[k] * out[k + 1]
    return out


def test_momentum_zero_viscosity_is_a_no_op(oracle):
    st = oracle.OracleState(6, 4, NZ, 2)
    st.h[...] = 10.0
    interior(st.kv, 0.0)
    for k in range(1, NZ + 1):
        st.u[:, :, k - 1] = 0.1 * k
        st.v[:, :, k - 1] = -0.05 * k
    u0, v0 = st.u.copy(), st.v.copy()
    st.call("vpo_vdiff_momentum", cfg(), 60.0)
    assert np.abs(st.u - u0).max() < 1.0e-12 and np.abs(st.v - v0).max() < 1.0e-12


def test_momentum_implicit_step_is_stable(oracle):
    st = oracle.OracleState(4, 4, NZ, 2)
    st.h[...] = 1.0
    interior(st.kv, 1000.0)
    for k in range(1, NZ + 1):
        st.u[:, :, k - 1] = 1.0 if k <= NZ // 2 else -1.0
    umax, umin = st.u.max(), st.u.min()
    st.call("vpo_vdiff_momentum", cfg(), 1.0)
    u_obs = np.abs(st.u).max()
    assert np.isfinite(u_obs) and u_obs <= umax + 1.0e-6
    assert u_obs < 0.5 * (umax - umin)


def test_budget_contributors_telescope(oracle):
    c = cfg(budgets=1)
    st = oracle.OracleState(6, 4, NZ, 2)
    st.h[...] = 10.0
    interior(st.kt, 1.0e-2)
    st.ks[...] = st.kt
    iT, iS = c.idx_temperature, c.idx_salinity
    for k in range(1, NZ + 1):
        st.tracers[iT][:, :, k - 1] = 5.0 + 2.0 * k
        st.tracers[iS][:, :, k - 1] = 30.0 + 0.5 * k
    st.heat_budget[...] = 0.0
    st.salt_budget[...] = 0.0
    before = [(st.h * st.tracers[n]).sum() for n in (iT, iS)]
    st.call("vpo_vdiff_tracers", c, 60.0)
    after = [(st.h * st.tracers[n]).sum() for n in (iT, iS)]
    for bud, b0, b1 in ((st.heat_budget, before[0], after[0]), (st.salt_budget, before[1], after[1])):
        assert abs(bud.sum()) / abs(b0) < 1.0e-12
        assert abs((b1 - b0) - bud.sum()) < 1.0e-12 * abs(b0)


def test_harmonic_faces_match_arithmetic_on_uniform_layers(oracle):
    out = []
    for harm in (0, 1):
        c = cfg(use_harmonic=harm)
        st = oracle.OracleState(4, 4, NZ, 2)
        st.h[...] = 5.0
        interior(st.kt, 1.0e-3)
        st.ks[...] = st.kt
        for k in range(1, NZ + 1):
            st.tracers[c.idx_temperature][:, :, k - 1] = float(k)
            st.tracers[c.idx_salinity][:, :, k - 1] = 35.0
        st.call("vpo_vdiff_tracers", c, 0.1)
        out.append(st.tracers[c.idx_temperature].copy())
    assert np.abs(out[0] - out[1]).max() < 1.0e-14


def test_thin_layer_face_harmonic_and_arithmetic(oracle):
    H_FAT, H_THIN, K, DT = 10.0, 0.1, 1.0e-3, 60.0
    harm_face = 2.0 * H_FAT * H_THIN / (H_FAT + H_THIN)
    arith_face = 0.5 * (H_FAT + H_THIN)
    assert harm_face < arith_face
    for harm, face in ((0, arith_face), (1, harm_face)):
        c = cfg(use_harmonic=harm)
        st = oracle.OracleState(2, 2, 2, 2)
        st.h[:, :, 0] = H_FAT
        st.h[:, :, 1] = H_THIN
        interior(st.kt, K)
        st.ks[...] = st.kt
        st.tracers[c.idx_temperature][:, :, 0] = 0.0
        st.tracers[c.idx_temperature][:, :, 1] = 1.0
        st.call("vpo_vdiff_tracers", c, DT)
        # the 2 x 2 system by Cramer's rule
        alpha, beta = DT * K / (H_FAT * face), DT * K / (H_THIN * face)
        det = (1.0 + alpha) * (1.0 + beta) - alpha * beta
        want = (alpha / det, (1.0 + alpha) / det)
        got = st.tracers[c.idx_temperature][1, 1, :]
        assert all(abs(g - w) <= 1.0e-14 * max(abs(w), 1e-300) for g, w in zip(got, want)), harm


def test_heat_and_salt_diffuse_with_their_own_diffusivities(oracle):
    H0, DT, KT0 = 10.0, 60.0, 1.0e-2
    KS0 = 4.0 * KT0
    c = cfg()
    st = oracle.OracleState(6, 4, NZ, 2)
    st.h[...] = H0
    profile = np.array([0.0 if k <= NZ // 2 else 1.0 for k in range(1, NZ + 1)])
    iT, iS = c.idx_temperature, c.idx_salinity
    st.tracers[iT][...] = profile
    st.tracers[iS][...] = profile
    interior(st.kt, KT0)
    interior(st.ks, KS0)
    sums0 = [(st.h * st.tracers[n]).sum() for n in (iT, iS)]
    st.call("vpo_vdiff_tracers", c, DT)
    K_T = np.r_[0.0, np.full(NZ - 1, KT0), 0.0]
    K_S = np.r_[0.0, np.full(NZ - 1, KS0), 0.0]
    t_ref = thomas_column(np.full(NZ, H0), K_T, DT, profile)
    s_ref = thomas_column(np.full(NZ, H0), K_S, DT, profile)
    t, s = st.tracers[iT][3, 3, :], st.tracers[iS][3, 3, :]
    assert np.abs(t - t_ref).max() < 1.0e-13
    assert np.abs(s - s_ref).max() < 1.0e-13
    assert ((s - profile) ** 2).sum() > ((t - profile) ** 2).sum()
    sums1 = [(st.h * st.tracers[n]).sum() for n in (iT, iS)]
    assert all(abs(b - a) < 1.0e-12 * abs(a) for a, b in zip(sums0, sums1))


def test_passive_tracer_follows_salinity(oracle):
    c = cfg()
    st = oracle.OracleState(6, 4, NZ, 3)
    st.h[...] = 10.0
    for n in range(3):
        for k in range(1, NZ + 1):
            st.tracers[n][:, :, k - 1] = float(k)
    interior(st.kt, 1.0e-2)
    interior(st.ks, 4.0e-2)
    st.call("vpo_vdiff_tracers", c, 60.0)
    passive = 3 - c.idx_temperature - c.idx_salinity
    age, salt, temp = (st.tracers[n][3, 3, :] for n in (passive, c.idx_salinity, c.idx_temperature))
    assert np.array_equal(age, salt)
    assert (age != temp).any()
