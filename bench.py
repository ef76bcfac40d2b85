"""Benchmark of the vertical-physics hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config eddy_1440x1080x75]

A step is one pass of the path over the whole synthetic domain: Wright EOS ->
coefficient assembly (PP81 + KPP + Bryan-Lewis gate) -> implicit momentum
viscosity (u, v) -> implicit tracer diffusion of every tracer with the KPP
non-local tendency.  The metric is cells/s (nx*ny*nz per step, the
reference's Mcells/s convention, benchmarks/bench_ocean.F90:149-150) on the
1440x1080x75 eddy-permitting configuration with T, S and 2 passives; the
state is FP64 at the interface in every form.

Forms (--form): "mixed" (default) runs the assembly's interface sweep and
the Thomas sweeps in FP32 with the FP64 residual correction
(cfg.mixed_precision = 2; --mixed-level 1 keeps the assembly FP64); "plain"
is FP64 throughout and bitwise the reference's arithmetic.  The line's "forms" object
carries both forms' cells/s and the mixed form's error against the plain FP64
GPU path after one step from the same state, over the whole domain.

One JSON line from rank 0:
  value        device-resident cells/s of the selected form (state in HBM before timing)
  e2e          cells/s through the C ABI with host buffers: every step
               uploads the state (h, u, v, tracers, forcing) from pinned host
               memory with vphys_set_field and downloads the results (u, v,
               tracers, kv, kt, ks, bl_depth) with vphys_get_field
  roofline     dominant stage: algorithmic bytes / its CUDA-event time vs the
               measured HBM copy bandwidth (MEASURED_PEAKS.json), every
               stage's fraction, and the whole path's
  cpu_baseline the CPU restatement (oracle) on the host cores, bounded sample
  gpu_launches the library's kernel launches in the timed region: the
               launches of one untimed step, counted from the CUDA activity
               trace, times the steps
  forms        plain FP64 and mixed on this configuration; the learned-KPP
               form (trained here) with its KPP stage time against the plain
               KPP stage; the batched configuration (10 tracers, 15 % of the
               wet columns with 1 mm layers, 24 graph-captured steps)
  parity_slice the GPU step against the oracle on the CPU arm's slice

Multi-GPU (torchrun): every rank owns an independent full-size domain
(columns shard with no data-path exchange); value = all ranks' cells / the
slowest rank's time (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "vertical-physics cells/s on 1 B200: learned+FP32 vs plain FP64 at stated error"
PEAK_FALLBACK_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="eddy_1440x1080x75")
    ap.add_argument("--e2e-steps", type=int, default=-1,
                    help="steps of the end-to-end timing (0: none; default: the timed steps, 4 to 12)")
    ap.add_argument("--cpu-sample", default="360x270", help="nx x ny of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--form", default="mixed", choices=["mixed", "plain"],
                    help="mixed: FP32 assembly and Thomas sweeps + FP64 residual (cfg.mixed_precision=2); "
                         "plain: FP64 throughout, bitwise the reference's arithmetic")
    ap.add_argument("--mixed-level", type=int, default=2, choices=[1, 2],
                    help="1: FP64 assembly, FP32 sweeps; 2: FP32 assembly too (the default)")
    ap.add_argument("--no-compare", action="store_true", help="skip the plain-FP64 timing and error check")
    ap.add_argument("--learned-cols", type=int, default=4_000_000,
                    help="training columns of the learned-KPP surrogate timed beside the mixed form (0: skip)")
    ap.add_argument("--learned-rounds", type=int, default=2,
                    help="2: a second data round from the network's own trajectories, labelled by the plain KPP")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched configuration (10 tracers, 15%% thin-layer columns, 24-step graph)")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the GPU-vs-oracle comparison on the CPU arm's slice")
    ap.add_argument("--variants", default=None,
                    help="momentum,tracers kernel variants of the mixed solves to pin instead of autotuning "
                         "(e.g. tma_ring,smem_1_per_warp: a profiling run under ncu, whose serialised launches "
                         "would skew the autotuner's timings)")
    return ap.parse_args()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return PEAK_FALLBACK_GBS, "fallback"


def bytes_per_cell(ntr: int, nz: int) -> dict:
    """Algorithmic FP64 bytes per cell (each input read once, each output written once)."""
    ifc = (nz + 1) / nz
    return {
        "eos": 8 * 4.0,                                   # h, T, S -> rho
        "assemble": 8 * 4.0 + 24 * ifc,                   # h, rho, u, v -> kv, kt, ks
        "momentum": 8 * 4.0 + 16.0,                      # h, kv, u, v -> u, v
        "tracers": 8 * 2.0 + 16.0 * ntr,                  # h, kt, c_t -> c_t
        # whole path at the interface (h, rho, u, v, c_t in; u, v, c_t, kv, kt, ks out)
        "path": 8 * (4 + ntr) + 8 * (2 + ntr) + 24 * ifc,
    }


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def traffic_from_profiles(kernel: str):
    """dram bytes per launch of `kernel` ("a+b": the sum over the stage's
    launches) from the committed ncu summary, if every one is there."""
    p = ROOT / "profiles" / "traffic.txt"
    if not p.exists():
        return None
    table = {}
    for line in p.read_text().splitlines():
        parts = line.split()
        if len(parts) >= 2 and not parts[0].startswith("#"):
            try:
                table[parts[0]] = float(parts[1])
            except ValueError:
                pass
    names = kernel.split("+")
    if not all(n in table for n in names):
        return None
    return sum(table[n] for n in names)


# ---------------------------------------------------------------------------
# CPU arm (the oracle: the C restatement of the reference)
# ---------------------------------------------------------------------------
def host_cpu():
    """nproc and the CPU model of this host (/proc/cpuinfo)."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "model": model}


def cpu_run(cfg_name: str, sample: str, steps: int, warmup: int, threads: int = 0):
    from oracle import oracle as o
    from roundabout_b200.config import hot_path_config
    from roundabout_b200.synthetic import CONFIGS, make_columns

    o.build()
    spec = dict(CONFIGS[cfg_name])
    sx, sy = (int(x) for x in sample.lower().split("x"))
    spec["nx"], spec["ny"] = min(sx, spec["nx"]), min(sy, spec["ny"])
    ntr = spec.pop("ntracers")
    cols = make_columns(ntracers=ntr, seed=1234, **spec)
    cfg = hot_path_config(ntracers=ntr)
    st = o.OracleState(cols.nx, cols.ny, cols.nz, ntr)
    st.seed_backgrounds(cfg)
    st.h[...] = cols.h
    st.u[...] = cols.u
    st.v[...] = cols.v
    for t in range(ntr):
        st.tracers[t][...] = cols.tracers[t]
    st.tau_x[...] = cols.tau_x
    st.tau_y[...] = cols.tau_y
    st.q_heat[...] = cols.q_heat
    st.q_salt[...] = cols.q_salt
    st.wet[...] = cols.wet
    st.stress_mag_from_tau()
    threads = threads if threads > 0 else (os.cpu_count() or 1)
    o.set_threads(threads)
    for _ in range(warmup):
        st.call("vpo_step", cfg, 3600.0, 1)
    t0 = time.perf_counter()
    for _ in range(steps):
        st.call("vpo_step", cfg, 3600.0, 1)
    el = time.perf_counter() - t0
    cells = cols.nx * cols.ny * cols.nz
    return {"value": cells * steps / el, "unit": "cells/s", "cores": threads, "kind": "port",
            "sample": f"{cols.nx}x{cols.ny}x{cols.nz} slice of the same generator, {ntr} tracers, {steps} steps "
                      f"(C restatement of the reference, gcc {o.CFLAGS_DESC}, OpenMP)",
            "ms_per_step": el / steps * 1e3}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    from roundabout_b200.synthetic import CONFIGS

    spec = dict(CONFIGS[args.config])
    ntr = spec["ntracers"]
    nx, ny, nz = spec["nx"], spec["ny"], spec["nz"]
    config_out = {"workload": args.config, "nx": nx, "ny": ny, "nz": nz, "tracers": ntr, "dt_s": 3600.0,
                  "closures": "PP81+KPP+Bryan-Lewis, Wright EOS, hvel_mom6 z_clear",
                  "l2": "working set >> 126 MB L2 (no flush needed)", "land_frac": spec["land_frac"]}

    if args.impl == "reference":
        if rank != 0:
            return
        r = cpu_run(args.config, args.cpu_sample, max(1, args.steps), max(0, min(args.warmup, 1)))
        line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": "cells/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config_out,
                "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": r["value"], "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(local)

    from roundabout_b200 import _ffi
    from roundabout_b200.column import VerticalPhysics
    from roundabout_b200.config import hot_path_config
    from roundabout_b200.synthetic import make_columns

    gen_spec = dict(spec)
    gen_spec.pop("ntracers")
    from roundabout_b200.ranks import rank_seed

    cols = make_columns(ntracers=ntr, seed=rank_seed(1234, rank), **gen_spec)
    mixed = args.form == "mixed"
    cfg = hot_path_config(ntracers=ntr)
    cfg.mixed_precision = args.mixed_level if mixed else 0
    vp = VerticalPhysics(nx, ny, nz, ntr, cfg)
    vp.load_columns(cols)
    torch.cuda.synchronize()
    config_out["form"] = args.form

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    from roundabout_b200.ranks import max_over_ranks as _mor, rank_seed, weak_scaling_value

    def max_over_ranks(x):
        return _mor(x, dist)

    dt = 3600.0
    cells = nx * ny * nz

    def timed(handle, steps, warm):
        for _ in range(max(3, warm)):
            handle.step(dt, 1)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        e0.record()
        for _ in range(steps):
            handle.step(dt, 1)
        e1.record()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1))

    # ---- the mixed form against the plain FP64 GPU path: one step from the
    #      same state, max |difference| over the whole domain ----
    forms = {}
    vp_plain = None
    if mixed and not args.no_compare:
        cfg_plain = hot_path_config(ntracers=ntr)
        vp_plain = VerticalPhysics(nx, ny, nz, ntr, cfg_plain)
        vp_plain.load_columns(cols)
        vp.step(dt, 1)
        vp_plain.step(dt, 1)
        torch.cuda.synchronize()
        iT, iS = cfg.idx_temperature, cfg.idx_salinity
        err = {"T": 0.0, "S": 0.0, "passive": 0.0, "u": 0.0, "v": 0.0}
        for t in range(ntr):
            d = float(np.abs(np.asarray(vp.get_tracer(t)) - np.asarray(vp_plain.get_tracer(t))).max())
            key = "T" if t == iT else ("S" if t == iS else "passive")
            err[key] = max(err[key], d)
        for n in ("u", "v"):
            err[n] = float(np.abs(np.asarray(vp.get(n)) - np.asarray(vp_plain.get(n))).max())
        forms["mixed_max_abs_err_vs_plain_fp64_1step"] = {k: float(f"{v:.3e}") for k, v in err.items()}
        forms["fp64_resolved_groups_1step"] = vp.mixed_redo_count()
        forms["error_bar"] = "|dT|, |dS|, tracers <= 1e-6 after one step from the same state"
        ms_plain = timed(vp_plain, args.steps, args.warmup)
        forms["plain_fp64"] = {"cells_per_s": cells * args.steps * world / (ms_plain / 1e3),
                               "ms_per_step": ms_plain / args.steps}
        vp_plain.close()
        vp_plain = None
        vp.load_columns(cols)

    # ---- learned KPP + mixed solves: trained here on the plain KPP's columns ----
    if mixed and not args.no_compare and args.learned_cols > 0:
        forms["learned_kpp_mixed"] = learned_form(args, cols, ntr, nx, ny, nz, timed, cells, world)

    # ---- the in-project autotuner picks the mixed solves' kernel variants on
    #      this handle's state (the state is left as it was) ----
    if mixed and args.variants:
        mv, tv = args.variants.split(",")
        vp.set_variants(mv, tv)
        tune = {"pinned": {"momentum": mv, "tracers": tv}}
    else:
        tune = vp.autotune(dt, reps=3) if mixed else None

    # ---- the timed region: K steps of the selected form; the clocks are
    #      sampled from a second before it to half a second after it, with
    #      untimed steps of the same form keeping the GPU loaded ----
    with ClockSampler(local) as clk:
        keep_busy(vp, dt, 1.0)
        ms = timed(vp, args.steps, args.warmup)
        keep_busy(vp, dt, 0.5)
    value = weak_scaling_value(cells, args.steps, world, ms)
    if mixed:
        forms["mixed"] = {"cells_per_s": value, "ms_per_step": ms / args.steps,
                          "fp64_resolved_groups_last_step": vp.mixed_redo_count(),
                          "groups_per_step": ((nx + 31) // 32) * ny * ntr,
                          "autotune_ms": tune}
        if "plain_fp64" in forms:
            forms["mixed_over_plain"] = round(value / forms["plain_fp64"]["cells_per_s"], 3)

    # ---- kernel launches per step, counted by the CUDA activity trace ----
    per_step, launch_names = count_launches(lambda: vp.step(dt, 1))

    # ---- per-stage device times (same stream, CUDA events) of the launches
    #      the step runs: the EOS, the assembly, the momentum solve (column
    #      depths + face solve) and the fused tracer diffusion + non-local ----
    reps = 5
    stage_ms = {}
    stages = {
        "eos": lambda: vp.eos(),
        "assemble": lambda: vp.assemble(),
        "momentum": lambda: vp.vdiff_momentum(dt),
        "tracers": lambda: vp.vdiff_tracers_nonlocal(dt),
    }
    for name, fn in stages.items():
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        stage_ms[name] = a.elapsed_time(b) / reps
    bpc = bytes_per_cell(ntr, nz)
    kernel_of = {"eos": "k_eos_wright",
                 "assemble": "k_assemble<float>" if (mixed and args.mixed_level >= 2) else "k_assemble<double>",
                 # the stage's launches: the column-depth pass and the face solve
                 "momentum": ("k_column_depth+k_mom_tile_flags+k_momentum_mp_tma"
                              if mixed and (tune or {}).get("chosen", {}).get("momentum") == "tma_ring"
                              else ("k_column_depth+k_momentum_mp" if mixed else "k_column_depth+k_momentum")),
                 "tracers": (("k_spans+k_tracers_mp_tm+k_tracers_redo"
                              if (tune or {}).get("chosen", {}).get("tracers") == "tmem_rows"
                              else "k_spans+k_tracers_mp+k_tracers_redo") if mixed else "k_tracers")}
    dom = max(("assemble", "momentum", "tracers", "eos"), key=lambda k: stage_ms[k])
    peak, peak_kind = peaks()
    achieved = bpc[dom] * cells / (stage_ms[dom] / 1e3) / 1e9
    traffic = traffic_from_profiles(kernel_of[dom])
    roofline = {"bound": "hbm", "kernel": kernel_of[dom], "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
                else "fallback 6.65 TB/s",
                "algorithmic_bytes_per_cell": round(bpc[dom], 2),
                "stage_ms": {k: round(v, 4) for k, v in stage_ms.items()},
                "stage_frac": {k: round(bpc[k] * cells / (v / 1e3) / 1e9 / peak, 4) for k, v in stage_ms.items()},
                "path_bytes_per_cell": round(bpc["path"], 2),
                "path_achieved_gbs": round(bpc["path"] * cells / (ms / args.steps / 1e3) / 1e9, 1),
                "path_frac": round(bpc["path"] * cells / (ms / args.steps / 1e3) / 1e9 / peak, 4)}

    # ---- end to end through the C ABI with host buffers ----
    # Every step uploads its inputs from pinned host memory and downloads its
    # results.  Serial: one handle, synchronous copies, upload -> step ->
    # download.  Pipelined (the reported e2e): two handles on two streams take
    # alternate steps with the asynchronous copies, so one handle's download
    # overlaps the other's upload on the full-duplex host link; each handle
    # has its own pinned result buffers.
    e2e = None
    if args.e2e_steps < 0:
        # the timed steps, bounded: each end-to-end step moves ~15 GB over the host link
        args.e2e_steps = min(max(args.steps, 4), 12)
    if args.e2e_steps > 0:
        import ctypes

        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a.T)).pin_memory()  # noqa: E731
        host_in = {"h": pin(cols.h), "u": pin(cols.u), "v": pin(cols.v), "q_heat": pin(cols.q_heat),
                   "q_salt": pin(cols.q_salt), "tau_x": pin(cols.tau_x), "tau_y": pin(cols.tau_y)}
        host_tr = [pin(t) for t in cols.tracers]
        out_names = ("u", "v", "kv", "kt", "ks", "bl_depth")

        def outputs(h):
            o = {n: torch.empty(tuple(reversed(h.shape(n))), dtype=torch.float64).pin_memory() for n in out_names}
            o["tracers"] = [torch.empty_like(t).pin_memory() for t in host_tr]
            return o

        def e2e_step(h, out, sync):
            lib, hdl = h.lib, h.handle
            setf = lib.vphys_set_field if sync else lib.vphys_set_field_async
            getf = lib.vphys_get_field if sync else lib.vphys_get_field_async
            for n, t in host_in.items():
                _ffi.check(setf(hdl, _ffi.FIELD_NAMES[n], ctypes.c_void_p(t.data_ptr()), t.numel()), "set_field")
            for k, t in enumerate(host_tr):
                _ffi.check(setf(hdl, _ffi.FIELD_TRACER0 + k, ctypes.c_void_p(t.data_ptr()), t.numel()), "set_field")
            _ffi.check(lib.vphys_stress_mag(hdl), "stress_mag")
            _ffi.check(lib.vphys_step(hdl, dt, 1), "step")
            for n in out_names:
                t = out[n]
                _ffi.check(getf(hdl, _ffi.FIELD_NAMES[n], ctypes.c_void_p(t.data_ptr()), t.numel()), "get_field")
            for k, t in enumerate(out["tracers"]):
                _ffi.check(getf(hdl, _ffi.FIELD_TRACER0 + k, ctypes.c_void_p(t.data_ptr()), t.numel()), "get_field")

        h2d = sum(t.numel() * 8 for t in host_in.values()) + sum(t.numel() * 8 for t in host_tr)
        out0 = outputs(vp)
        d2h = sum(out0[n].numel() * 8 for n in out_names) + sum(t.numel() * 8 for t in out0["tracers"])

        # serial, one handle
        e2e_step(vp, out0, True)
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step(vp, out0, True)
        barrier()
        el_serial = max_over_ranks(time.perf_counter() - t0)

        # pipelined, two handles on their own streams
        vp2 = VerticalPhysics(nx, ny, nz, ntr, cfg)
        vp2.load_columns(cols)
        pair = [(vp, out0, torch.cuda.Stream()), (vp2, outputs(vp2), torch.cuda.Stream())]
        for h, _, s in pair:
            h.set_stream(s.cuda_stream)
        for h, o, _ in pair:
            e2e_step(h, o, False)
        for h, _, _ in pair:
            h.synchronize()
        barrier()
        t0 = time.perf_counter()
        for i in range(args.e2e_steps):
            h, o, _ = pair[i % 2]
            e2e_step(h, o, False)
        for h, _, _ in pair:
            h.synchronize()
        barrier()
        el = max_over_ranks(time.perf_counter() - t0)
        vp.set_stream(0)
        vp2.close()
        e2e = {"value": cells * args.e2e_steps * world / el, "unit": "cells/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": el / args.e2e_steps * 1e3,
               "serial_ms_per_step": el_serial / args.e2e_steps * 1e3,
               "serial_cells_per_s": cells * args.e2e_steps * world / el_serial, "steps": args.e2e_steps,
               "what": "C ABI: vphys_set_field_async (pinned host -> HBM) of h, u, v, tracers, forcing; vphys_step; "
                       "vphys_get_field_async of u, v, tracers, kv, kt, ks, bl_depth; two handles on two streams "
                       "take alternate steps so one's download overlaps the other's upload (serial: one handle, "
                       "synchronous vphys_set_field / vphys_get_field)"}

    # ---- conservation of the selected form, stated against the compensated
    #      FP64 column contents (cfg.column_integrals) over one step from the
    #      benchmark's state ----
    if not args.no_compare:
        ci_cfg = hot_path_config(ntracers=ntr)
        ci_cfg.mixed_precision = args.mixed_level if mixed else 0
        ci_cfg.column_integrals = 1
        vp.set_config(ci_cfg)
        vp.load_columns(cols)
        vp.step(dt, 1)
        old, new = np.asarray(vp.get("content_old")), np.asarray(vp.get("content_new"))
        inc = np.zeros_like(old)
        for t in range(ntr):
            inc[:, :, t] = (np.abs(np.asarray(vp.get_tracer(t)) - cols.tracers[t]) * cols.h).sum(axis=2)
        live = np.abs(old) > 0
        forms["column_content_1step"] = {
            "form": args.form, "max_rel_drift": float((np.abs(new - old)[live] / np.abs(old[live])).max()),
            "max_drift_over_sum_h_abs_increment": float(
                (np.abs(new - old)[live] / np.maximum(inc[live], 1e-300)).max()),
            "how": "Neumaier-compensated FP64 sum_k h c over each column's live span before and after the "
                   "tracer solve (with the fused non-local deposit), per column and tracer"}
        cfg.column_integrals = 0
        vp.set_config(cfg)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu = cpu_run(args.config, args.cpu_sample, 2, 1)
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        one = cpu_run(args.config, args.cpu_sample, 1, 1, threads=1)
        cpu["single_thread"] = {"value": one["value"], "unit": "cells/s", "cores": 1}
        cpu["host"] = host_cpu()
    vp.close()

    # ---- the batched configuration (10 tracers, 15 % of the wet columns with
    #      1 mm layers): 24 graph-captured steps of each form ----
    if mixed and not args.no_compare and not args.no_batched:
        forms["batched"] = batched_form(args, dt)

    # ---- the GPU step against the oracle on the CPU arm's slice ----
    parity = None
    if rank == 0 and not args.no_parity:
        parity = parity_slice(args, dt)

    clocks = clk.summary()
    line = {"metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if mixed else "f64", "data": "synthetic",
            "config": config_out, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": per_step * args.steps if per_step else None,
            "gpu_launches_per_step": {"count": per_step, "kernels": launch_names,
                                      "how": "CUDA activity trace (torch.profiler / CUPTI) of one untimed step"},
            "clocks": clocks, "forms": forms, "parity_slice": parity,
            "mode": (f"FP64 state, FP32 assembly and Thomas sweeps with FP64 residual correction "
                     f"(mixed_precision={args.mixed_level})" if mixed
                     else "plain FP64, bit-identical to the CPU restatement")}
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def keep_busy(vp, dt, seconds):
    """Untimed steps for about `seconds` (keeps the GPU under load while the
    clock sampler runs around the timed region)."""
    import torch

    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        vp.step(dt, 1)
        torch.cuda.synchronize()


def count_launches(fn):
    """Kernel launches of `fn` (one untimed step), from the CUDA activity
    trace: (count, {kernel name: launches}).  (None, reason) if the trace is
    unavailable."""
    import torch

    try:
        from torch.profiler import ProfilerActivity, profile

        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            fn()
            torch.cuda.synchronize()
        names = {}
        for e in prof.events():
            if e.device_type != torch.autograd.DeviceType.CUDA:
                continue
            n = e.name
            if "vphys::" in n or n.startswith("k_") or "::k_" in n:
                short = n.split("(")[0].replace("void ", "").replace("vphys::", "")
                names[short] = names.get(short, 0) + 1
        return sum(names.values()), names
    except Exception as exc:  # noqa: BLE001 -- the count is a report, not the measurement
        return None, f"unavailable: {type(exc).__name__}: {exc}"[:200]


def learned_form(args, cols, ntr, nx, ny, nz, timed, cells, world):
    """The learned-KPP form: the surrogate trained here on the plain KPP's
    columns (training size and rounds as the arguments say), its one-step
    OBL-depth error against the plain method over the wet columns, the step
    time with the mixed solves, and the KPP stage's device time, plain
    (bulk-Richardson search inside the assembly) vs learned (features, the
    three tensor-core GEMMs, gate/check and the pass-1-free assembly), each
    net of the assembly without KPP."""
    import torch

    from roundabout_b200 import learned as L
    from roundabout_b200.column import VerticalPhysics
    from roundabout_b200.config import hot_path_config

    dt = 3600.0
    sur, _ = L.train_surrogate(args.learned_cols, nz=nz, seed=100, epochs=4, rounds=args.learned_rounds)

    def handle(learned_kpp, use_kpp=1, level=args.mixed_level):
        cfg = hot_path_config(ntracers=ntr)
        cfg.mixed_precision = level
        cfg.learned_kpp = learned_kpp
        cfg.use_kpp = use_kpp
        vp = VerticalPhysics(nx, ny, nz, ntr, cfg)
        vp.load_columns(cols)
        if learned_kpp:
            sur.attach(vp)
        return vp

    vl, vpp = handle(1), handle(0, level=0)
    vl.step(dt, 1)
    vpp.step(dt, 1)
    torch.cuda.synchronize()
    bl, blp = np.asarray(vl.get("bl_depth")), np.asarray(vpp.get("bl_depth"))
    wetm = np.asarray(cols.wet) > 0
    r = ((bl - blp) / np.maximum(blp, 1.0))[wetm]
    vpp.close()
    ms_l = timed(vl, args.steps, args.warmup)
    out = {"cells_per_s": cells * args.steps * world / (ms_l / 1e3), "ms_per_step": ms_l / args.steps,
           "obl_rms_rel_vs_plain_1step": float(np.sqrt(np.mean(r * r))),
           "train_columns": int(sur.ntrain), "train_rounds": args.learned_rounds,
           "collect_s": round(sur.collect_seconds, 2), "train_s": round(sur.train_seconds, 2),
           "kpp": L.kpp_stats(vl)}
    vl.close()

    def time_assemble(vp, reps=10):
        vp.eos()
        for _ in range(3):
            vp.assemble()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            vp.assemble()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    t = {}
    for name, lk, uk in (("no_kpp", 0, 0), ("plain", 0, 1), ("learned", 1, 1)):
        vp = handle(lk, uk)
        t[name] = time_assemble(vp)
        vp.close()
    plain_stage = t["plain"] - t["no_kpp"]
    learned_stage = t["learned"] - t["no_kpp"]
    out["kpp_stage_ms"] = {"plain": round(plain_stage, 4), "learned": round(learned_stage, 4),
                           "plain_over_learned": round(plain_stage / max(learned_stage, 1e-9), 3),
                           "assemble_without_kpp": round(t["no_kpp"], 4),
                           "how": "assembly with the KPP stage minus the assembly without it (CUDA events, 10 reps)"}
    del sur
    return out


def batched_form(args, dt):
    """The batched configuration: 1440x1080x75, T, S + 8 uniform passives,
    15 % of the wet columns with 1-10 live 1 mm layers.  Each form runs 24
    graph-captured steps (vphys_step_graph) from the same state; the first
    24 give the mixed form's error against the plain FP64 path (which is the
    oracle's arithmetic bit for bit) and, as its yardstick, the plain path's
    own response to a +-1e-7 perturbation of its initial tracers; the second
    24 (the graph replayed) are timed."""
    import torch

    from roundabout_b200.column import VerticalPhysics
    from roundabout_b200.config import hot_path_config
    from roundabout_b200.synthetic import CONFIGS, make_columns

    spec = dict(CONFIGS["batched_1440x1080x75"])
    ntr = spec.pop("ntracers")
    cols = make_columns(ntracers=ntr, seed=4321, **spec)
    nx, ny, nz = cols.nx, cols.ny, cols.nz
    nsteps = 24
    out = {"config": "batched_1440x1080x75", "tracers": ntr, "thin_frac": spec["thin_frac"],
           "steps_per_graph": nsteps}
    finals, times = {}, {}
    for name, level in (("plain_fp64", 0), ("mixed", args.mixed_level)):
        cfg = hot_path_config(ntracers=ntr)
        cfg.mixed_precision = level
        vp = VerticalPhysics(nx, ny, nz, ntr, cfg)
        vp.load_columns(cols)
        if level:
            out["mixed_autotune_ms"] = vp.autotune(dt, reps=2)
        vp.step_graph(dt, nsteps)                 # capture + the first 24 steps
        torch.cuda.synchronize()
        finals[name] = [np.asarray(vp.get_tracer(t)) for t in range(ntr)]
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        vp.step_graph(dt, nsteps)                 # replay: timed
        b.record()
        torch.cuda.synchronize()
        times[name] = a.elapsed_time(b) / nsteps
        out[name] = {"ms_per_step": round(times[name], 4), "cells_per_s": nx * ny * nz / (times[name] / 1e3)}
        if name == "mixed":
            out[name]["fp64_resolved_groups_last_step"] = vp.mixed_redo_count()
        vp.close()
    # the plain path's own sensitivity: +-1e-7 on the initial tracers of live cells
    rng = np.random.default_rng(0)
    live = cols.h > 1.5e-4
    cfg = hot_path_config(ntracers=ntr)
    vp = VerticalPhysics(nx, ny, nz, ntr, cfg)
    vp.load_columns(cols)
    for t in range(ntr):
        vp.set_tracer(t, cols.tracers[t] + rng.uniform(-1e-7, 1e-7, cols.h.shape) * live)
    vp.step_graph(dt, nsteps)
    torch.cuda.synchronize()
    pert = [np.asarray(vp.get_tracer(t)) for t in range(ntr)]
    vp.close()
    iT, iS = 1, 0
    err = [float(np.abs(finals["mixed"][t] - finals["plain_fp64"][t]).max()) for t in range(ntr)]
    env = [float(np.abs(pert[t] - finals["plain_fp64"][t]).max()) for t in range(ntr)]
    out["mixed_over_plain"] = round(times["plain_fp64"] / times["mixed"], 3)
    out["max_abs_err_vs_fp64_24steps"] = {"T": err[iT], "S": err[iS],
                                          "passive": max(e for t, e in enumerate(err) if t not in (iT, iS))}
    out["fp64_response_to_1e-7_perturbation_24steps"] = {
        "T": env[iT], "S": env[iS], "passive": max(e for t, e in enumerate(env) if t not in (iT, iS))}
    return out


def parity_slice(args, dt):
    """The GPU step against the oracle on the CPU arm's 360x270x75 slice of
    the benchmark's generator: plain FP64 after 3 steps (the max relative
    difference over every output field, relative to the field's largest
    magnitude; 0 means bit for bit) and the mixed form after one step (max
    absolute tracer and velocity difference)."""
    from oracle import oracle as o
    from roundabout_b200.column import VerticalPhysics
    from roundabout_b200.config import hot_path_config
    from roundabout_b200.synthetic import CONFIGS, make_columns

    o.build()
    spec = dict(CONFIGS[args.config])
    sx, sy = (int(x) for x in args.cpu_sample.lower().split("x"))
    spec["nx"], spec["ny"] = min(sx, spec["nx"]), min(sy, spec["ny"])
    ntr = spec.pop("ntracers")
    cols = make_columns(ntracers=ntr, seed=1234, **spec)

    def oracle_after(nsteps):
        cfg = hot_path_config(ntracers=ntr)
        st = o.OracleState(cols.nx, cols.ny, cols.nz, ntr)
        st.seed_backgrounds(cfg)
        for n in ("h", "u", "v", "tau_x", "tau_y", "q_heat", "q_salt", "wet"):
            getattr(st, n)[...] = getattr(cols, n)
        for t in range(ntr):
            st.tracers[t][...] = cols.tracers[t]
        st.stress_mag_from_tau()
        st.call("vpo_step", cfg, dt, nsteps)
        return st

    def gpu_after(nsteps, level):
        cfg = hot_path_config(ntracers=ntr)
        cfg.mixed_precision = level
        vp = VerticalPhysics(cols.nx, cols.ny, cols.nz, ntr, cfg)
        vp.load_columns(cols)
        vp.step(dt, nsteps)
        return vp

    o.set_threads(os.cpu_count() or 1)
    st3 = oracle_after(3)
    vp = gpu_after(3, 0)
    rel = 0.0
    for n in ("kv", "kt", "ks", "u", "v", "bl_depth", "rho"):
        want = getattr(st3, n)
        rel = max(rel, float(np.abs(np.asarray(vp.get(n)) - want).max()) / max(float(np.abs(want).max()), 1e-300))
    for t in range(ntr):
        want = st3.tracers[t]
        rel = max(rel, float(np.abs(np.asarray(vp.get_tracer(t)) - want).max()) / float(np.abs(want).max() or 1.0))
    vp.close()
    st1 = oracle_after(1)
    vm = gpu_after(1, args.mixed_level)
    dtr = max(float(np.abs(np.asarray(vm.get_tracer(t)) - st1.tracers[t]).max()) for t in range(ntr))
    duv = max(float(np.abs(np.asarray(vm.get(n)) - getattr(st1, n)).max()) for n in ("u", "v"))
    vm.close()
    return {"slice": f"{cols.nx}x{cols.ny}x{cols.nz}, {ntr} tracers, seed 1234 (the CPU arm's sample)",
            "plain_fp64_3steps_max_rel_diff": rel,
            "mixed_1step_max_abs_diff": {"tracers": dtr, "u_v": duv},
            "bar": "plain <= 1e-12 relative (0: bit for bit); mixed <= 1e-6"}


if __name__ == "__main__":
    main()
