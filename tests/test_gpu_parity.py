"""Parity of the CUDA library (through its C ABI) with the CPU oracle.

Every comparison is BITWISE: the kernels are built without FMA contraction and
follow the reference's operation order, so each FP64 value must equal the
oracle's bit for bit (NaN compared as NaN).  That is stricter than the 1e-12
relative bar of the hot path.
"""
import numpy as np
import pytest

from tests._cases import assert_bitwise, columns, hot_cfg, oracle_state, plain_cfg

pytestmark = pytest.mark.gpu

DT = 3600.0


@pytest.fixture(scope="module")
def VP():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from roundabout_b200.column import VerticalPhysics

    return VerticalPhysics


def gpu_state(VP, cols, cfg):
    vp = VP(cols.nx, cols.ny, cols.nz, len(cols.tracers), cfg)
    vp.load_columns(cols)
    return vp


def compare_all(vp, st, names=("kv", "kt", "ks", "u", "v", "bl_depth", "b0"), tracers=True):
    for n in names:
        assert_bitwise(n, vp.get(n), getattr(st, n))
    if tracers:
        for t in range(st.ntr):
            assert_bitwise(f"tracer{t}", vp.get_tracer(t), st.tracers[t])


def test_stress_mag_and_eos(VP, oracle):
    cols = columns()
    cfg = hot_cfg()
    st = oracle_state(oracle, cols, cfg)
    vp = gpu_state(VP, cols, cfg)
    assert_bitwise("stress_mag", vp.get("stress_mag"), st.stress_mag)
    st.call("vpo_eos_wright", cfg)
    vp.eos()
    assert_bitwise("rho", vp.get("rho"), st.rho)


ASSEMBLE_CASES = {
    "pp81_only": dict(use_kpp=0, bkgnd_profile=0),
    "pp81_kpp": dict(use_kpp=1, bkgnd_profile=0),
    "hot_path": dict(),
    "none_closure_profile": dict(interior_closure=4),
    "none_closure_scalar_prandtl": dict(interior_closure=4, bkgnd_profile=0, bkgnd_prandtl=2.0),
    "scalar_prandtl": dict(bkgnd_profile=0, bkgnd_prandtl=3.0),
    "profile_prandtl": dict(bkgnd_prandtl=5.0),
    "invz2": dict(kv_ml_invz2=1e-2, hmix_fixed=40.0),
    "convection": dict(conv_enable=1, conv_n2_thresh=1e-7),
    "ceilings": dict(kv_max=2e-3, kd_max=5e-4),
    "smoothing": dict(kd_smooth_iterations=2),
    "no_vt2": dict(c_vt2=0.0),
    "eos_buoyancy_coeffs": dict(buoyancy_coeffs=1),
}


@pytest.mark.parametrize("case", sorted(ASSEMBLE_CASES))
def test_assemble(VP, oracle, case):
    cols = columns(seed=11)
    cfg = hot_cfg(**ASSEMBLE_CASES[case])
    st = oracle_state(oracle, cols, cfg)
    st.call("vpo_eos_wright", cfg)
    st.bl_depth[...] = np.abs(np.sin(np.arange(st.bl_depth.size))).reshape(st.bl_depth.shape, order="F") * 80.0
    vp = gpu_state(VP, cols, cfg)
    vp.eos()
    vp.set("bl_depth", st.bl_depth)
    vp.get("gamma_t")   # request the gamma diagnostics
    vp.get("gamma_s")
    assert st.call("vpo_build_coefficients", cfg) == 0
    vp.assemble()
    for n in ("kv", "kt", "ks", "bl_depth", "b0", "gamma_t", "gamma_s"):
        assert_bitwise(n, vp.get(n), getattr(st, n))


MOMENTUM_CASES = {
    "default_zclear": dict(),
    "harmonic_branch": dict(hvel_harmonic=1),
    "harmonic_branch_no_upwind": dict(hvel_harmonic=1, hvel_upwind=0),
    "legacy_arith": dict(hvel_mom6=0),
    "legacy_use_harmonic": dict(hvel_mom6=0, use_harmonic=1),
    "implicit_stress": dict(implicit_stress=1),
    "implicit_drag": dict(implicit_drag=1),
    "remnant": dict(remnant=1),
    "bbl_glue": dict(bbl_glue=1),
    "zlevel_faces": dict(zlevel_faces=1),
}


@pytest.mark.parametrize("case", sorted(MOMENTUM_CASES))
def test_momentum(VP, oracle, case):
    cols = columns(seed=5, thin_frac=0.2)
    cfg = hot_cfg(**MOMENTUM_CASES[case])
    st = oracle_state(oracle, cols, cfg)
    vp = gpu_state(VP, cols, cfg)
    rng = np.random.default_rng(3)
    if cfg.implicit_drag:
        st.lambda_bot_u[...] = rng.uniform(0, 1e-4, st.lambda_bot_u.shape)
        st.lambda_bot_v[...] = rng.uniform(0, 1e-4, st.lambda_bot_v.shape)
        vp.set("lambda_bot_u", st.lambda_bot_u)
        vp.set("lambda_bot_v", st.lambda_bot_v)
    if cfg.zlevel_faces:
        # static first-live indices from the columns (ocean_vcoord_k_bot_from_target rule)
        live = cols.h > 1.5e-4
        kb = np.where(live.any(2), live.argmax(2) + 1, 1)
        ia = np.clip(np.arange(cols.nx + 1) - 1, 0, cols.nx - 1)
        ib = np.clip(np.arange(cols.nx + 1), 0, cols.nx - 1)
        st.k_bot_u[...] = np.maximum(kb[ia, :], kb[ib, :])
        ja = np.clip(np.arange(cols.ny + 1) - 1, 0, cols.ny - 1)
        jb = np.clip(np.arange(cols.ny + 1), 0, cols.ny - 1)
        st.k_bot_v[...] = np.maximum(kb[:, ja], kb[:, jb])
        vp.set("k_bot_u", st.k_bot_u)
        vp.set("k_bot_v", st.k_bot_v)
    st.call("vpo_eos_wright", cfg)
    st.call("vpo_build_coefficients", cfg)
    vp.eos()
    vp.assemble()
    st.call("vpo_vdiff_momentum", cfg, DT)
    vp.vdiff_momentum(DT)
    assert_bitwise("u", vp.get("u"), st.u)
    assert_bitwise("v", vp.get("v"), st.v)
    if cfg.remnant:
        assert_bitwise("visc_rem_u", vp.get("visc_rem_u"), st.visc_rem_u)
        assert_bitwise("visc_rem_v", vp.get("visc_rem_v"), st.visc_rem_v)


TRACER_CASES = {
    "ks_eq_kt": dict(),
    "ks_ne_kt": dict(bkgnd_profile=0, kt_bg=2e-5, ks_bg=7e-6),
    "budgets": dict(budgets=1),
    "use_harmonic": dict(use_harmonic=1),
    "no_kpp": dict(use_kpp=0),
    "eos_buoyancy_coeffs": dict(buoyancy_coeffs=1),
}


@pytest.mark.parametrize("ntr", [1, 2, 4, 7, 10])
@pytest.mark.parametrize("case", sorted(TRACER_CASES))
def test_tracers_and_nonlocal(VP, oracle, case, ntr):
    cols = columns(seed=21, ntr=ntr, thin_frac=0.15, passive_init="uniform")
    over = dict(TRACER_CASES[case])
    if ntr < 2 and over.get("buoyancy_coeffs"):
        pytest.skip("the eos coefficients need T and S")
    cfg = hot_cfg(ntr=ntr, **over)
    if ntr < 2:
        cfg.idx_temperature = -1
        cfg.eos_in_step = 0
    st = oracle_state(oracle, cols, cfg)
    vp = gpu_state(VP, cols, cfg)
    if cfg.eos_in_step:
        st.call("vpo_eos_wright", cfg)
        vp.eos()
    else:
        st.rho[...] = 1030.0 - 0.001 * np.arange(st.rho.size).reshape(st.rho.shape, order="F") % 3
        vp.set("rho", st.rho)
    # a destabilising surface flux everywhere so the non-local term is active
    st.q_heat[...] = -np.abs(st.q_heat)
    vp.set("q_heat", st.q_heat)
    st.call("vpo_build_coefficients", cfg)
    vp.assemble()
    st.call("vpo_vdiff_tracers", cfg, DT)
    vp.vdiff_tracers(DT)
    for t in range(ntr):
        assert_bitwise(f"tracer{t} (diffused)", vp.get_tracer(t), st.tracers[t])
    if cfg.budgets:
        assert_bitwise("heat_budget", vp.get("heat_budget"), st.heat_budget)
        assert_bitwise("salt_budget", vp.get("salt_budget"), st.salt_budget)
    if cfg.use_kpp:
        st.call("vpo_nonlocal", cfg, DT)
        vp.nonlocal_tendencies(DT)
        for t in range(ntr):
            assert_bitwise(f"tracer{t} (non-local)", vp.get_tracer(t), st.tracers[t])


def test_tracers_follow_a_caller_written_ks(VP, oracle):
    """kt diffuses temperature and ks salinity and the passive tracers, also
    when the caller writes ks after an assembly, through vphys_set_field or in
    a bound buffer: the one-factorisation shortcut is only for the gate's
    own ks, which is bitwise kt under the default floors."""
    import torch

    cols = columns(seed=23)
    cfg = hot_cfg()
    st = oracle_state(oracle, cols, cfg)
    vp = gpu_state(VP, cols, cfg)
    st.call("vpo_eos_wright", cfg)
    vp.eos()
    assert st.call("vpo_build_coefficients", cfg) == 0
    vp.assemble()
    st.ks[...] = 3.0 * st.ks
    vp.set("ks", st.ks)
    st.call("vpo_vdiff_tracers", cfg, DT)
    vp.vdiff_tracers(DT)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t} (ks written)", vp.get_tracer(t), st.tracers[t])
    # the gate's coefficients again: one factorisation, the same answer as the oracle
    assert st.call("vpo_build_coefficients", cfg) == 0
    vp.assemble()
    st.call("vpo_vdiff_tracers", cfg, DT)
    vp.vdiff_tracers(DT)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t} (gate's ks)", vp.get_tracer(t), st.tracers[t])
    # a bound ks, scaled in place after the assembly wrote it
    ks_t = torch.zeros(st.ks.size, dtype=torch.float64, device="cuda")
    vp.bind("ks", ks_t)
    assert st.call("vpo_build_coefficients", cfg) == 0
    vp.assemble()
    torch.cuda.synchronize()
    ks_t.mul_(0.5)
    torch.cuda.synchronize()
    st.ks[...] = 0.5 * st.ks
    st.call("vpo_vdiff_tracers", cfg, DT)
    vp.vdiff_tracers(DT)
    for t in range(st.ntr):
        assert_bitwise(f"tracer{t} (bound ks)", vp.get_tracer(t), st.tracers[t])


@pytest.mark.parametrize("shape", [(24, 20, 12), (7, 5, 1), (9, 4, 2), (33, 17, 3), (130, 9, 20)])
def test_full_step(VP, oracle, shape):
    nx, ny, nz = shape
    cols = columns(nx=nx, ny=ny, nz=nz, seed=nx + ny + nz, thin_frac=0.1)
    cfg = hot_cfg(budgets=1)
    st = oracle_state(oracle, cols, cfg)
    vp = gpu_state(VP, cols, cfg)
    assert st.call("vpo_step", cfg, DT, 3) == 0
    vp.step(DT, 3)
    compare_all(vp, st)
    assert_bitwise("rho", vp.get("rho"), st.rho)
    assert_bitwise("heat_budget", vp.get("heat_budget"), st.heat_budget)


def test_full_step_all_land(VP, oracle):
    cols = columns(nx=16, ny=12, nz=8, seed=3, land_frac=0.0)
    cols.h[...] = 0.0
    cols.wet[...] = 0.0
    cols.u[...] = 0.0
    cols.v[...] = 0.0
    cfg = hot_cfg()
    st = oracle_state(oracle, cols, cfg)
    vp = gpu_state(VP, cols, cfg)
    st.call("vpo_step", cfg, DT, 2)
    vp.step(DT, 2)
    compare_all(vp, st)


def test_collapsed_top_layer(VP, oracle):
    cols = columns(nx=20, ny=10, nz=10, seed=9, land_frac=0.0)
    cols.h[:, :, -1] = 1.0e-4      # vanished top layer: KPP starts at the first live one
    cols.h[:5, :, -2] = 0.0        # and two vanished layers in part of the domain
    cfg = hot_cfg()
    st = oracle_state(oracle, cols, cfg)
    vp = gpu_state(VP, cols, cfg)
    st.call("vpo_step", cfg, DT, 2)
    vp.step(DT, 2)
    compare_all(vp, st)


def test_guard_trips_without_fault(VP, oracle):
    """A negative closure value trips vmix_guard: status VPHYS_ERR_GUARD after
    the clip, like the reference's status=1 path -- no trap, handle usable."""
    from roundabout_b200 import _ffi

    cols = columns(nx=12, ny=8, nz=6, seed=2)
    cfg = hot_cfg(vmix_guard=1, pp81_nu_bg=-1.0)
    vp = gpu_state(VP, cols, cfg)
    vp.eos()
    st = vp.assemble_status()
    assert st == _ffi.ERR_GUARD
    assert "negative or NaN" in _ffi.last_error(0)
    cfg2 = hot_cfg(vmix_guard=1)
    vp.set_config(cfg2)
    assert vp.assemble_status() == _ffi.OK
    vp.step(DT, 1)


def test_bind_torch_zero_copy(VP, oracle):
    import torch

    cols = columns(nx=32, ny=16, nz=10, seed=4)
    cfg = hot_cfg()
    st = oracle_state(oracle, cols, cfg)
    vp = gpu_state(VP, cols, cfg)
    u_t = torch.from_numpy(np.ascontiguousarray(cols.u.T)).cuda()
    vp.bind("u", u_t)
    st.call("vpo_step", cfg, DT, 2)
    vp.step(DT, 2)
    vp.synchronize()
    assert_bitwise("u (bound tensor)", u_t.cpu().numpy().T, st.u)
    compare_all(vp, st, names=("kv", "v"))


def test_tracer_solve_conserves_column_content(VP, oracle):
    """Column sum of h~ * T and h~ * S (h~ = max(h, H_VANISHED) as the matrix
    weights rows) before and after the tracer solve: the drift is round-off,
    summed exactly (math.fsum) per column -- the conservation metric of the
    path, on the GPU's own output, with thin stiff layers present."""
    import math

    cols = columns(nx=40, ny=24, nz=30, seed=12, thin_frac=0.15)
    cfg = hot_cfg()
    vp = gpu_state(VP, cols, cfg)
    vp.eos()
    vp.assemble()
    ht = np.maximum(cols.h, 1.5e-4)
    live = cols.h > 1.5e-4
    before = [np.asarray(vp.get_tracer(t)).copy() for t in (0, 1)]
    vp.vdiff_tracers(DT)
    worst = 0.0
    for t, b in zip((0, 1), before):
        a = np.asarray(vp.get_tracer(t))
        for i in range(cols.nx):
            for j in range(cols.ny):
                m = live[i, j]
                if not m.any():
                    continue
                s0 = math.fsum((ht[i, j, m] * b[i, j, m]).tolist())
                s1 = math.fsum((ht[i, j, m] * a[i, j, m]).tolist())
                scale = math.fsum(np.abs(ht[i, j, m] * b[i, j, m]).tolist())
                worst = max(worst, abs(s1 - s0) / scale)
    # the reference's own bar for the column sum is 1e-12 (test_ocean_vdiff.F90:270-308)
    assert worst <= 1e-12, worst


@pytest.mark.parametrize("mixed", [0, 1, 2])
def test_full_step_eos_buoyancy_coeffs(VP, oracle, mixed):
    """KPP's B0 from the Wright derivatives at the surface (T, S): bitwise
    on the FP64 path over 3 steps (assembly, solves, the non-local deposit
    from the stored b0); the mixed forms within their one-step bars."""
    cols = columns(nx=40, ny=24, nz=20, seed=19, thin_frac=0.1)
    cfg = hot_cfg(budgets=1, buoyancy_coeffs=1)
    st = oracle_state(oracle, cols, cfg)
    vp = gpu_state(VP, cols, hot_cfg(budgets=1, buoyancy_coeffs=1, mixed_precision=mixed))
    n = 3 if mixed == 0 else 1
    assert st.call("vpo_step", cfg, DT, n) == 0
    vp.step(DT, n)
    if mixed == 0:
        compare_all(vp, st)
        assert_bitwise("heat_budget", vp.get("heat_budget"), st.heat_budget)
    else:
        tol = 1.0e-6 if mixed == 1 else 2.0e-5
        for t in range(st.ntr):
            assert float(np.abs(np.asarray(vp.get_tracer(t)) - st.tracers[t]).max()) <= tol
    # the eos pair really changed the answer
    c0 = hot_cfg(budgets=1)
    st0 = oracle_state(oracle, cols, c0)
    st0.call("vpo_step", c0, DT, n)
    assert np.abs(st0.b0 - st.b0).max() > 0.0
