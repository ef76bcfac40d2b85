"""Time each stage of the path on a synthetic domain (CUDA events).

    python -m roundabout_b200.profile_stages --nx 512 --ny 384 --nz 75 --ntr 4 --reps 3
    python -m roundabout_b200.profile_stages --config batched_1440x1080x75 --mixed 1

Prints, per stage, the mean device time and the algorithmic GB/s; used as the
driver of the ncu captures kept under profiles/.
"""
from __future__ import annotations

import argparse
import json


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=512)
    ap.add_argument("--ny", type=int, default=384)
    ap.add_argument("--nz", type=int, default=75)
    ap.add_argument("--ntr", type=int, default=4)
    ap.add_argument("--land", type=float, default=0.3)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--thin", type=float, default=0.0, help="fraction of wet columns with 1 mm layers")
    ap.add_argument("--passive", default="age_ps", choices=["age_ps", "uniform"])
    ap.add_argument("--config", default=None, help="a named synthetic workload (overrides the shape options)")
    ap.add_argument("--mixed", type=int, default=0, choices=[0, 1, 2],
                    help="1: FP32 sweeps + FP64 residual; 2: also the FP32 assembly")
    ap.add_argument("--stages", default="eos,assemble,momentum,tracers,step")
    args = ap.parse_args()

    import torch

    from .column import VerticalPhysics
    from .config import hot_path_config
    from .synthetic import CONFIGS, make_columns

    if args.config:
        w = CONFIGS[args.config]
        args.nx, args.ny, args.nz, args.ntr = w["nx"], w["ny"], w["nz"], w["ntracers"]
        args.land, args.thin = w["land_frac"], w["thin_frac"]
        args.passive = w.get("passive_init", "age_ps")
    cols = make_columns(args.nx, args.ny, args.nz, ntracers=args.ntr, seed=1234, land_frac=args.land,
                        thin_frac=args.thin, passive_init=args.passive)
    cfg = hot_path_config(ntracers=args.ntr)
    cfg.mixed_precision = int(args.mixed)
    vp = VerticalPhysics(args.nx, args.ny, args.nz, args.ntr, cfg)
    vp.load_columns(cols)
    dt = 3600.0
    vp.step(dt, args.warmup)
    torch.cuda.synchronize()
    cells = args.nx * args.ny * args.nz
    ifc = (args.nz + 1) / args.nz
    bpc = {"eos": 32.0, "assemble": 32.0 + 24 * ifc, "momentum": 48.0, "tracers": 16.0 + 16.0 * args.ntr,
           "step": 8 * (4 + args.ntr) + 8 * (2 + args.ntr) + 24 * ifc}
    fns = {"eos": vp.eos, "assemble": vp.assemble, "momentum": lambda: vp.vdiff_momentum(dt),
           "tracers": lambda: vp.vdiff_tracers(dt), "step": lambda: vp.step(dt, 1)}
    out = {}
    for name in args.stages.split(","):
        fn = fns[name]
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / args.reps
        out[name] = {"ms": round(ms, 4), "alg_GBps": round(bpc[name] * cells / ms / 1e6, 1)}
    print(json.dumps({"shape": [args.nx, args.ny, args.nz], "ntr": args.ntr, "thin": args.thin,
                      "mixed": args.mixed, "stages": out}))
    vp.close()


if __name__ == "__main__":
    main()
