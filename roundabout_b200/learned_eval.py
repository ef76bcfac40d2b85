"""Train the learned KPP surrogate and evaluate it against the plain KPP.

    python -m roundabout_b200.learned_eval [--train-cols 4000000] [--epochs 4] [--days 30]
                                           [--config eddy_1440x1080x75] [--mixed 0|1]

Reports (one JSON line): training-set size and times; the held-out OBL-depth
RMS relative error of the network alone; the KPP stage's device time, plain
(bulk-Richardson search) vs learned (features + MLP on the tensor cores +
gate/check + the pass-1-free assembly), each net of the assembly without KPP;
and a `days`-long run (dt = 3600 s) of the learned form next to the plain
method from the same state: OBL-depth RMS relative error over the wet columns
(time mean and final), SST (top live layer T) difference at the end (mean,
RMS, max), and the surrogate's counters (checked, failed, gated, fallback).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train-cols", type=int, default=4_000_000)
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--days", type=float, default=30.0)
    ap.add_argument("--config", default="eddy_1440x1080x75")
    ap.add_argument("--mixed", type=int, default=0, choices=[0, 1, 2])
    ap.add_argument("--seed", type=int, default=100)
    ap.add_argument("--rounds", type=int, default=2, help="2: a second data round from the network's own trajectories")
    args = ap.parse_args()

    import torch

    from . import learned as L
    from .column import VerticalPhysics
    from .config import hot_path_config
    from .synthetic import CONFIGS, make_columns

    out = {"config": args.config, "mixed_precision": args.mixed}
    log = lambda m: print(m, flush=True)  # noqa: E731

    # ---- training ----
    spec = dict(CONFIGS[args.config])
    nz = spec["nz"]
    s, hist = L.train_surrogate(args.train_cols, nz=nz, seed=args.seed, epochs=args.epochs, batch=args.batch,
                                rounds=args.rounds, log=log)
    out["train"] = {"columns": int(s.ntrain), "rounds": args.rounds, "collect_s": round(s.collect_seconds, 2),
                    "train_s": round(s.train_seconds, 2), "epochs": args.epochs, "batch": args.batch,
                    "sampled_loss_first_last": [hist[0], hist[-1]]}

    # ---- held-out: a domain the network has not seen ----
    raw, T = L.collect(256, 1024, nz, 1, [0, 47, 359], seed=args.seed + 1000)
    X, _, _ = s.standardise(raw)
    hb_true = 10.0 * torch.exp(T[:, 0])
    hb_pred = s.predict_hb(X)
    e = (hb_pred - hb_true) / torch.clamp(hb_true, min=1.0)
    out["held_out"] = {"columns": int(raw.shape[0]), "obl_rms_rel": float(torch.sqrt(torch.mean(e * e))),
                       "obl_mean_abs_rel": float(torch.mean(e.abs()))}
    del raw, T, X

    # ---- stage timing and the long run on the benchmark shape ----
    ntr = spec["ntracers"]
    gen = dict(spec)
    gen.pop("ntracers")
    cols = make_columns(ntracers=ntr, seed=1234, **gen)
    nx, ny = spec["nx"], spec["ny"]

    def handle(learned_kpp, use_kpp=1):
        cfg = hot_path_config(ntracers=ntr)
        cfg.mixed_precision = args.mixed
        cfg.learned_kpp = learned_kpp
        cfg.use_kpp = use_kpp
        vp = VerticalPhysics(nx, ny, nz, ntr, cfg)
        vp.load_columns(cols)
        if learned_kpp:
            s.attach(vp)
        return vp

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
    out["stage_ms"] = {"assemble_without_kpp": round(t["no_kpp"], 4), "assemble_plain_kpp": round(t["plain"], 4),
                       "assemble_learned_kpp": round(t["learned"], 4),
                       "plain_kpp_stage": round(t["plain"] - t["no_kpp"], 4),
                       "learned_kpp_stage": round(t["learned"] - t["no_kpp"], 4),
                       "speedup": round((t["plain"] - t["no_kpp"]) / max(t["learned"] - t["no_kpp"], 1e-9), 3)}
    log(json.dumps(out["stage_ms"]))

    # ---- days-long run, learned vs plain from the same state ----
    steps = int(round(args.days * 24))
    vl, vpn = handle(1), handle(0)
    wet = cols.wet > 0
    iT = 1
    top = nz - 1   # surface layer index (k = nz)
    errs = []
    t0 = time.perf_counter()
    chunk = 24
    done = 0
    while done < steps:
        n = min(chunk, steps - done)
        vl.step(3600.0, n)
        vpn.step(3600.0, n)
        done += n
        bl, blp = np.asarray(vl.get("bl_depth")), np.asarray(vpn.get("bl_depth"))
        r = ((bl - blp) / np.maximum(blp, 1.0))[wet]
        errs.append(float(np.sqrt(np.mean(r * r))))
    torch.cuda.synchronize()
    sst_l = np.asarray(vl.get_tracer(iT))[:, :, top][wet]
    sst_p = np.asarray(vpn.get_tracer(iT))[:, :, top][wet]
    d = sst_l - sst_p
    st = L.kpp_stats(vl)
    out["run"] = {"days": args.days, "steps": steps, "wall_s": round(time.perf_counter() - t0, 1),
                  # the network against the plain pass 1 on the learned run's own states (the 1 % sampled checks)
                  "obl_rms_rel_on_own_states": float(np.sqrt(st["sum_rel_err2_e6"] / 1e6 / max(st["checked"], 1))),
                  # the two runs' OBL depths (includes the divergence of the two trajectories)
                  "obl_rms_rel_final": errs[-1], "obl_rms_rel_time_mean": float(np.mean(errs)),
                  "sst_diff_mean_K": float(d.mean()), "sst_diff_rms_K": float(np.sqrt(np.mean(d * d))),
                  "sst_diff_max_abs_K": float(np.abs(d).max()), "stats": st}
    vl.close()
    vpn.close()
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
