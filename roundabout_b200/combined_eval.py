"""The combined form at the high-resolution shape: 3600x2700x75 (7.29e8
cells), FP32 solves with the FP64 residual correction and the learned KPP,
4 passive tracers, 30 % land, every field resident in HBM, graph-captured
steps.

    python -m roundabout_b200.combined_eval [--steps 48] [--train-cols 2000000] [--mixed-level 2]
                                            [--variants registers,tmem_rows]

The domain is generated on the device (synthetic.make_columns_device) and
bound zero-copy.  The same initial state (regenerated from the seed) is then
run with the plain FP64 path; the line reports both forms' cells/s, the
combined form's HBM GB/s at the path's algorithmic FP64 bytes against the
measured peak, the device memory in use, and the combined form's difference
from the plain FP64 run: T, S, passives (max |d|), SST (mean, RMS, max) and
the OBL depth (RMS relative).
"""
from __future__ import annotations

import argparse
import json
import time
from pathlib import Path


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=48)
    ap.add_argument("--train-cols", type=int, default=2_000_000)
    ap.add_argument("--config", default="combined_3600x2700x75")
    ap.add_argument("--seed", type=int, default=4321)
    ap.add_argument("--mixed-level", type=int, default=2, choices=[1, 2],
                    help="1: FP64 assembly, FP32 solves; 2: FP32 assembly too (the bench's mixed form)")
    ap.add_argument("--variants", default="registers,tmem_rows",
                    help="kernel forms of the mixed solves (the autotuner's copy of the state does not fit "
                         "beside this domain; the default is its pick on 1440x1080x75)")
    args = ap.parse_args()

    import numpy as np
    import torch

    from . import learned as L
    from .column import VerticalPhysics
    from .config import hot_path_config
    from .synthetic import CONFIGS, bind_device_columns, make_columns_device

    spec = CONFIGS[args.config]
    nx, ny, nz, ntr = spec["nx"], spec["ny"], spec["nz"], spec["ntracers"]
    cells = nx * ny * nz
    out = {"config": args.config, "steps": args.steps}

    t0 = time.perf_counter()
    sur, _ = L.train_surrogate(args.train_cols, nz=nz, seed=100, epochs=4)
    out["train"] = {"columns": int(sur.ntrain), "collect_s": round(sur.collect_seconds, 1),
                    "train_s": round(sur.train_seconds, 2)}
    torch.cuda.empty_cache()

    def generate():
        return make_columns_device(nx, ny, nz, ntracers=ntr, seed=args.seed, land_frac=spec["land_frac"],
                                   passive_init=spec.get("passive_init", "uniform"))

    cfg = hot_path_config(ntracers=ntr)
    cfg.mixed_precision = args.mixed_level
    cfg.learned_kpp = 1
    vp = VerticalPhysics(nx, ny, nz, ntr, cfg)
    vp.set_variants(*args.variants.split(","))
    out["mixed_level"], out["variants"] = args.mixed_level, args.variants
    d = generate()
    bind_device_columns(vp, d)
    init = {"u": d["u"].clone(), "v": d["v"].clone(), "tracers": [t.clone() for t in d["tracers"]]}
    torch.cuda.empty_cache()
    sur.attach(vp)
    torch.cuda.synchronize()
    free, total = torch.cuda.mem_get_info()

    def run(label):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        vp.step_graph(3600.0, 1)          # capture of the one-step graph outside the timing
        torch.cuda.synchronize()
        e0.record()
        for _ in range(args.steps - 1):
            vp.step_graph(3600.0, 1)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / max(1, args.steps - 1)
        return {"ms_per_step": ms, "cells_per_s": cells / (ms / 1e3)}

    r = run("combined")
    out["combined"] = r
    out["device_memory_used_GB"] = round((total - free) / 1e9, 1)
    out["device_memory_used_note"] = "includes a copy of the initial u, v and tracers kept for the comparison"
    keep = {0: d["tracers"][0].clone(), 1: d["tracers"][1].clone()}
    bl_c = np.asarray(vp.get("bl_depth"))
    out["kpp"] = L.kpp_stats(vp)
    out["obl_rms_rel_on_own_states"] = float(np.sqrt(out["kpp"]["sum_rel_err2_e6"] / 1e6 /
                                                     max(out["kpp"]["checked"], 1)))

    # the same initial state, plain FP64
    d["u"].copy_(init["u"])
    d["v"].copy_(init["v"])
    for t, a in zip(d["tracers"], init["tracers"]):
        t.copy_(a)
    del init
    torch.cuda.empty_cache()
    vp.set("bl_depth", np.zeros((nx, ny)))
    cfg_p = hot_path_config(ntracers=ntr)
    vp.set_config(cfg_p)
    out["plain_fp64"] = run("plain")
    bl_p = np.asarray(vp.get("bl_depth"))
    wet = d["wet"].bool()
    err = {}
    for k, a in keep.items():
        err[{0: "S", 1: "T"}.get(k, f"passive{k - 2}")] = float((a - d["tracers"][k]).abs().max())
    sst = (keep[1][nz - 1] - d["tracers"][1][nz - 1])[wet]
    wetn = wet.cpu().numpy().T
    r_bl = ((bl_c - bl_p) / np.maximum(bl_p, 1.0))[wetn]
    out["diff_vs_plain_fp64"] = {"max_abs": err, "sst_mean_K": float(sst.mean()),
                                 "sst_rms_K": float(torch.sqrt((sst * sst).mean())),
                                 "sst_max_abs_K": float(sst.abs().max()),
                                 "obl_rms_rel": float(np.sqrt(np.mean(r_bl * r_bl)))}
    peak = json.loads((Path(__file__).resolve().parents[1] / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]
    bpc = 8 * (4 + ntr) + 8 * (2 + ntr) + 24 * (nz + 1) / nz
    gbs = bpc * cells / (r["ms_per_step"] / 1e3) / 1e9
    out["combined_hbm"] = {"path_bytes_per_cell": bpc, "achieved_GBps": round(gbs, 1), "peak_GBps": peak,
                           "frac": round(gbs / peak, 4)}
    out["wall_s"] = round(time.perf_counter() - t0, 1)
    vp.close()
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
