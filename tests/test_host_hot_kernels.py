"""The CUDA source of the step's plain FP64 kernels -- the Wright EOS, the
stress magnitude, the surface deposit, the shortwave penetration and the
chlorophyll opacities, the assembly (k_assemble and the 1-2-1 smoothing), the
momentum face solves and the tracer solve with its fused non-local deposit,
and whole steps in the library's launch order -- compiled as host C++ and
run thread by thread on the CPU, against the oracle, bit for bit.

The kernels' arithmetic is plain IEEE FP64 in a fixed order without FMA
contraction (the GPU build uses -fmad=false, g++ here -ffp-contract=off), so
the same source gives the same bits on the host; the L2 residency hints and
read-only loads become plain loads (tests/host_kernels/prelude_hot.h).  This
checks the device code of the hot path itself -- its index arithmetic, the
live-span skipping, the level-blocked loads at every nz, the default-knob
instantiations -- against the oracle in every CPU run of the suite; the GPU
tests (tests/test_gpu_parity.py, tests/test_gpu_bench_shape.py) check the
same source on the B200.  The launchers (the `<<<...>>>` host code) are left
out and restated by tests/host_kernels/hot_driver.inc with the same kernel
choices and pass order.
"""
import ctypes
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from tests._cases import assert_bitwise, columns, hot_cfg, oracle_state

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "roundabout_b200" / "csrc"
HERE = Path(__file__).resolve().parent / "host_kernels"
DT = 3600.0


def device_code(source: str) -> str:
    """The kernels of a .cu file without its includes and its host launch
    code (launch_* functions and the attribute helper)."""
    out, skip = [], False
    for ln in (CSRC / source).read_text().splitlines():
        if skip:
            skip = ln != "}"
            continue
        if ln.startswith("#include"):
            continue
        if re.match(r"^(static )?(void|bool|int) (launch_\w+|redo_attr)\(", ln):
            if out and out[-1].startswith("template <"):
                out.pop()
            skip = not ln.rstrip().endswith(";")
            continue
        out.append(ln.replace("extern __shared__", "extern"))
    return "\n".join(out) + "\n"


@pytest.fixture(scope="module")
def hot(tmp_path_factory, oracle):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    tmp = tmp_path_factory.mktemp("host_hot")
    unit = tmp / "hot_host.cpp"
    unit.write_text('#include "prelude_hot.h"\n' + device_code("vphys_kernels.cu") + device_code("vphys_tracers.cu")
                    + (HERE / "hot_driver.inc").read_text())
    lib = tmp / "hot_host.so"
    cmd = ["g++", "-O2", "-ffp-contract=off", "-fno-fast-math", "-std=c++17", "-fPIC", "-shared", "-w",
           f"-I{HERE}", f"-I{CSRC}", f"-I{ROOT / 'oracle'}", "-o", str(lib), str(unit)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-6000:]
    L = ctypes.CDLL(str(lib))
    S = ctypes.POINTER(oracle.VpoState)
    L.host_eos.argtypes = [ctypes.c_void_p, S]
    L.host_assemble.argtypes = [ctypes.c_void_p, S]
    L.host_assemble.restype = ctypes.c_ulonglong
    L.host_momentum.argtypes = [ctypes.c_void_p, S, ctypes.c_double, ctypes.c_int]
    L.host_tracers.argtypes = [ctypes.c_void_p, S, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    for fn in ("host_stress_mag", "host_sw_chl_kappa"):
        getattr(L, fn).argtypes = [ctypes.c_void_p, S]
    for fn in ("host_surface_flux", "host_sw_penetration"):
        getattr(L, fn).argtypes = [ctypes.c_void_p, S, ctypes.c_double]
    L.host_step.argtypes = [ctypes.c_void_p, S, ctypes.c_double, ctypes.c_int]
    L.host_step.restype = ctypes.c_ulonglong
    return L


def run(L, fn, cfg, st, *args):
    s = st._struct()
    return getattr(L, fn)(ctypes.byref(cfg), ctypes.byref(s), *args)


SHAPES = [(24, 20, 12), (7, 5, 1), (9, 4, 2), (33, 17, 3), (20, 9, 75)]

ASSEMBLE = {
    "hot_path": {},
    "pp81_only": dict(use_kpp=0, bkgnd_profile=0),
    "none_closure_scalar_prandtl": dict(interior_closure=4, bkgnd_profile=0, bkgnd_prandtl=2.0),
    "invz2_convection": dict(kv_ml_invz2=1e-2, hmix_fixed=40.0, conv_enable=1, conv_n2_thresh=1e-7),
    "ceilings_smoothing": dict(kv_max=2e-3, kd_max=5e-4, kd_smooth_iterations=2),
    "eos_buoyancy_coeffs": dict(buoyancy_coeffs=1),
    "shortwave_mxl": dict(sw_pen_frac=0.6, kpp_sw_method=1),
}


def state_pair(oracle, shape, cfg, seed, thin=0.1):
    nx, ny, nz = shape
    cols = columns(nx=nx, ny=ny, nz=nz, seed=seed, thin_frac=thin)
    return oracle_state(oracle, cols, cfg), oracle_state(oracle, cols, cfg)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("case", sorted(ASSEMBLE))
def test_eos_and_assembly_source_matches_oracle(oracle, hot, shape, case):
    cfg = hot_cfg(**ASSEMBLE[case])
    host, ref = state_pair(oracle, shape, cfg, seed=sum(shape) + len(case))
    ref.call("vpo_eos_wright", cfg)
    run(hot, "host_eos", cfg, host)
    assert_bitwise("rho", host.rho, ref.rho)
    lagged = np.abs(np.sin(np.arange(ref.bl_depth.size))).reshape(ref.bl_depth.shape, order="F") * 80.0
    for s in (host, ref):
        s.bl_depth[...] = lagged
    assert ref.call("vpo_build_coefficients", cfg) == 0
    assert run(hot, "host_assemble", cfg, host) == 0
    for n in ("kv", "kt", "ks", "bl_depth", "b0", "gamma_t", "gamma_s"):
        assert_bitwise(n, getattr(host, n), getattr(ref, n))


MOMENTUM = {
    "default_zclear": {},
    "harmonic_branch": dict(hvel_harmonic=1),
    "legacy_arith": dict(hvel_mom6=0),
    "implicit_stress_and_drag": dict(implicit_stress=1, implicit_drag=1),
    "remnant_glue": dict(remnant=1, bbl_glue=1, implicit_drag=1),
}


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("case", sorted(MOMENTUM))
def test_momentum_source_matches_oracle(oracle, hot, shape, case):
    cfg = hot_cfg(**MOMENTUM[case])
    host, ref = state_pair(oracle, shape, cfg, seed=2 * sum(shape) + len(case), thin=0.2)
    rng = np.random.default_rng(sum(shape))
    for n in ("lambda_bot_u", "lambda_bot_v"):
        a = rng.uniform(0.0, 1.0e-4, getattr(ref, n).shape)
        getattr(ref, n)[...] = a
        getattr(host, n)[...] = a
    ref.call("vpo_eos_wright", cfg)
    assert ref.call("vpo_build_coefficients", cfg) == 0
    for n in ("rho", "kv", "kt", "ks", "bl_depth", "b0"):
        getattr(host, n)[...] = getattr(ref, n)
    ref.call("vpo_vdiff_momentum", cfg, DT)
    run(hot, "host_momentum", cfg, host, DT, 0)
    names = ("u", "v") + (("visc_rem_u", "visc_rem_v") if cfg.remnant else ())
    for n in names:
        assert_bitwise(n, getattr(host, n), getattr(ref, n))


TRACERS = {
    "hot_path": {},
    "ks_ne_kt": dict(bkgnd_profile=0, kt_bg=2e-5, ks_bg=7e-6),
    "budgets_harmonic": dict(budgets=1, use_harmonic=1),
    "no_kpp": dict(use_kpp=0),
}


@pytest.mark.parametrize("ntr", [2, 4, 7, 10])
@pytest.mark.parametrize("shape", [(24, 20, 12), (9, 4, 2), (20, 9, 75)])
@pytest.mark.parametrize("case", sorted(TRACERS))
def test_tracer_source_matches_oracle(oracle, hot, shape, case, ntr):
    nx, ny, nz = shape
    cols = columns(nx=nx, ny=ny, nz=nz, ntr=ntr, seed=nx + ntr, thin_frac=0.15, passive_init="uniform")
    cfg = hot_cfg(ntr=ntr, **TRACERS[case])
    ref, host = oracle_state(oracle, cols, cfg), oracle_state(oracle, cols, cfg)
    for s in (host, ref):
        s.q_heat[...] = -np.abs(s.q_heat)      # a destabilising flux: the non-local term is active
    ref.call("vpo_eos_wright", cfg)
    assert ref.call("vpo_build_coefficients", cfg) == 0
    for n in ("rho", "kv", "kt", "ks", "bl_depth", "b0", "gamma_t", "gamma_s"):
        getattr(host, n)[...] = getattr(ref, n)
    ref.call("vpo_vdiff_tracers", cfg, DT)
    run(hot, "host_tracers", cfg, host, DT, 1, 0, 1)
    for t in range(ntr):
        assert_bitwise(f"tracer{t} (diffused)", host.tracers[t], ref.tracers[t])
    if cfg.budgets:
        assert_bitwise("heat_budget", host.heat_budget, ref.heat_budget)
        assert_bitwise("salt_budget", host.salt_budget, ref.salt_budget)
    if cfg.use_kpp:
        ref.call("vpo_nonlocal", cfg, DT)
        run(hot, "host_tracers", cfg, host, DT, 0, 1, 1)
        for t in range(ntr):
            assert_bitwise(f"tracer{t} (non-local)", host.tracers[t], ref.tracers[t])


def test_fused_tracer_launch_and_a_caller_written_ks(oracle, hot):
    """The fused diffusion + non-local launch equals the two calls; with a ks
    that is not the gate's copy of kt the source takes two factorisations and
    still matches the oracle."""
    cols = columns(nx=20, ny=9, nz=30, ntr=4, seed=77, thin_frac=0.15)
    cfg = hot_cfg()
    ref, host = oracle_state(oracle, cols, cfg), oracle_state(oracle, cols, cfg)
    for s in (host, ref):
        s.q_heat[...] = -np.abs(s.q_heat)
    ref.call("vpo_eos_wright", cfg)
    assert ref.call("vpo_build_coefficients", cfg) == 0
    ref.ks[...] = 2.5 * ref.ks
    for n in ("rho", "kv", "kt", "ks", "bl_depth", "b0", "gamma_t", "gamma_s"):
        getattr(host, n)[...] = getattr(ref, n)
    ref.call("vpo_vdiff_tracers", cfg, DT)
    ref.call("vpo_nonlocal", cfg, DT)
    run(hot, "host_tracers", cfg, host, DT, 1, 1, 0)
    for t in range(4):
        assert_bitwise(f"tracer{t}", host.tracers[t], ref.tracers[t])


SW = dict(sw_pen_frac=0.6, sw_band_ratio=0.58, sw_zeta1=0.35, sw_zeta2=23.0)
CHL = dict(sw_pen_frac=1.0, sw_chl=1)
FORCING = {
    "deposit_budgets": dict(budgets=1),
    "two_band": dict(SW),
    "two_band_qsw_wetdyn": dict(SW, sw_source=1, use_wet_dyn=1, budgets=1),
    "chlorophyll": dict(CHL),
    "cover_bound_salinity": dict(SW, use_cover_frac=1, bound_salinity=1, min_salinity=34.5),
}


@pytest.mark.parametrize("shape", [(24, 20, 12), (9, 4, 2), (20, 9, 75)])
@pytest.mark.parametrize("case", sorted(FORCING))
def test_forcing_kernels_source_matches_oracle(oracle, hot, shape, case):
    nx, ny, nz = shape
    cfg = hot_cfg(surface_flux=1, **FORCING[case])
    host, ref = state_pair(oracle, shape, cfg, seed=3 * sum(shape) + len(case), thin=0.15)
    rng = np.random.default_rng(sum(shape))
    extra = {"sw_net": rng.uniform(0.0, 300.0, (nx, ny)), "wet_dyn": (rng.random((nx, ny)) > 0.2) * 1.0,
             "sw_chl": rng.uniform(-1.0, 3.0, (nx, ny)), "cover_frac": rng.uniform(0.0, 1.0, (nx, ny))}
    for s in (host, ref):
        s.q_heat[...] = np.abs(s.q_heat) + 50.0
        for n, a in extra.items():
            getattr(s, n)[...] = a
    ref.stress_mag[...] = 0.0
    ref.stress_mag_from_tau()
    run(hot, "host_stress_mag", cfg, host)
    assert_bitwise("stress_mag", host.stress_mag, ref.stress_mag)
    if cfg.sw_chl:
        ref.call("vpo_sw_chl_kappa", cfg)
        run(hot, "host_sw_chl_kappa", cfg, host)
        assert_bitwise("sw_kappa", host.sw_kappa, ref.sw_kappa)
    ref.call("vpo_surface_flux", cfg, DT)
    run(hot, "host_surface_flux", cfg, host, DT)
    ref.call("vpo_sw_penetration", cfg, DT)
    run(hot, "host_sw_penetration", cfg, host, DT)
    for t in range(ref.ntr):
        assert_bitwise(f"tracer{t}", host.tracers[t], ref.tracers[t])
    if cfg.budgets:
        assert_bitwise("heat_budget_surface", host.heat_budget_surface, ref.heat_budget_surface)
        assert_bitwise("salt_budget_surface", host.salt_budget_surface, ref.salt_budget_surface)


STEP = {
    "hot_path_budgets": dict(budgets=1),
    "surface_two_band": dict(SW, surface_flux=1, budgets=1),
    "none_closure_smoothing": dict(interior_closure=4, kd_smooth_iterations=1),
    "remnant_glue_drag": dict(remnant=1, bbl_glue=1, implicit_drag=1, implicit_stress=1),
}


@pytest.mark.parametrize("shape", [(24, 20, 12), (7, 5, 1), (9, 4, 2), (20, 9, 75)])
@pytest.mark.parametrize("case", sorted(STEP))
def test_three_steps_match_the_oracle_step(oracle, hot, shape, case):
    cfg = hot_cfg(**STEP[case])
    host, ref = state_pair(oracle, shape, cfg, seed=5 * sum(shape) + len(case), thin=0.1)
    rng = np.random.default_rng(len(case))
    for n in ("lambda_bot_u", "lambda_bot_v"):
        a = rng.uniform(0.0, 1.0e-4, getattr(ref, n).shape)
        getattr(ref, n)[...] = a
        getattr(host, n)[...] = a
    assert ref.call("vpo_step", cfg, DT, 3) == 0
    assert run(hot, "host_step", cfg, host, DT, 3) == 0
    for n in ("kv", "kt", "ks", "u", "v", "bl_depth", "b0", "rho"):
        assert_bitwise(n, getattr(host, n), getattr(ref, n))
    for t in range(ref.ntr):
        assert_bitwise(f"tracer{t}", host.tracers[t], ref.tracers[t])
    if cfg.budgets:
        assert_bitwise("heat_budget", host.heat_budget, ref.heat_budget)


@pytest.mark.parametrize("shape", [(24, 20, 12), (9, 4, 3), (20, 9, 75)])
def test_zlevel_faces_source_matches_oracle(oracle, hot, shape):
    """The momentum solve with caller-set first-live indices on the faces
    (the z-level faces: ocean_vcoord_k_bot_from_target's rule, the larger of
    the two cells' first live layers)."""
    cfg = hot_cfg(zlevel_faces=1)
    host, ref = state_pair(oracle, shape, cfg, seed=7 * sum(shape), thin=0.2)
    nx, ny, _ = shape
    live = ref.h > 1.5e-4
    kb = np.where(live.any(2), live.argmax(2) + 1, 1)
    ia, ib = np.clip(np.arange(nx + 1) - 1, 0, nx - 1), np.clip(np.arange(nx + 1), 0, nx - 1)
    ja, jb = np.clip(np.arange(ny + 1) - 1, 0, ny - 1), np.clip(np.arange(ny + 1), 0, ny - 1)
    for s in (host, ref):
        s.k_bot_u[...] = np.maximum(kb[ia, :], kb[ib, :])
        s.k_bot_v[...] = np.maximum(kb[:, ja], kb[:, jb])
    ref.call("vpo_eos_wright", cfg)
    assert ref.call("vpo_build_coefficients", cfg) == 0
    for n in ("rho", "kv", "kt", "ks", "bl_depth", "b0"):
        getattr(host, n)[...] = getattr(ref, n)
    ref.call("vpo_vdiff_momentum", cfg, DT)
    run(hot, "host_momentum", cfg, host, DT, 1)
    for n in ("u", "v"):
        assert_bitwise(n, getattr(host, n), getattr(ref, n))


@pytest.mark.parametrize("shape", [(24, 20, 12), (9, 4, 2), (20, 9, 75)])
@pytest.mark.parametrize("case", sorted(ASSEMBLE))
def test_fp32_assembly_source_within_fp32_of_the_oracle(oracle, hot, shape, case):
    """k_assemble<float> (mixed_precision = 2: the boundary-layer walk in FP64,
    the interface sweep in FP32) against the FP64 oracle: bl_depth and b0 bit
    for bit; kv, kt, ks within 5e-5 relative; gamma within 1e-5 of its
    field's largest value (its shape function cancels to ~0 at the base of
    the layer).  The host stands an exact quotient in for the GPU's fast
    FP32 one, so the GPU tests bound the kernel's own FP32 results."""
    cfg = hot_cfg(**ASSEMBLE[case])
    cfg32 = hot_cfg(mixed_precision=2, **ASSEMBLE[case])
    host, ref = state_pair(oracle, shape, cfg, seed=sum(shape) + 11 * len(case))
    ref.call("vpo_eos_wright", cfg)
    host.rho[...] = ref.rho
    lagged = np.abs(np.sin(np.arange(ref.bl_depth.size))).reshape(ref.bl_depth.shape, order="F") * 80.0
    for s in (host, ref):
        s.bl_depth[...] = lagged
    assert ref.call("vpo_build_coefficients", cfg) == 0
    assert run(hot, "host_assemble", cfg32, host) == 0
    for n in ("bl_depth", "b0"):
        assert_bitwise(n, getattr(host, n), getattr(ref, n))
    for n in ("kv", "kt", "ks"):
        a, b = getattr(host, n), getattr(ref, n)
        assert (np.abs(a - b) <= 5.0e-5 * np.abs(b)).all(), (n, np.abs(a - b).max())
    for n in ("gamma_t", "gamma_s"):
        a, b = getattr(host, n), getattr(ref, n)
        assert np.abs(a - b).max() <= 1.0e-5 * max(np.abs(b).max(), 1e-300), n
