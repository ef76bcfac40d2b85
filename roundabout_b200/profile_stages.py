"""Time each stage of the path on a synthetic domain (CUDA events).

    python -m roundabout_b200.profile_stages --nx 512 --ny 384 --nz 75 --ntr 4 --reps 3
    python -m roundabout_b200.profile_stages --config batched_1440x1080x75 --mixed 1
    python -m roundabout_b200.profile_stages --nx 512 --ny 384 --stages features,mlp

Stages: eos, assemble, momentum, tracers (the fused diffusion + non-local
launch the step runs), step (the path), kshear (the
kappa-shear column solve, vphys_kappa_shear, default knobs, Wright EOS), epbl
(the EPBL column solve, vphys_epbl, default knobs: OM4 mstar), and
features, mlp (the learned KPP's feature extraction and its three tensor-core
GEMMs, with untrained weights: the time does not depend on their values).

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
    ap.add_argument("--variants", default=None,
                    help="momentum,tracers kernel variants of the mixed solves (VerticalPhysics.MOM_VARIANTS / "
                         "TRACER_VARIANTS names), e.g. tma_ring,tmem_rows; default: the handle's")
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
    if args.variants:
        mom, trv = args.variants.split(",")
        vp.set_variants(mom, trv)
    dt = 3600.0
    vp.step(dt, args.warmup)
    if "kshear" in args.stages:
        for _ in range(args.warmup):
            vp.kappa_shear(dt)
    if "epbl" in args.stages:
        for _ in range(args.warmup):
            vp.epbl(dt)
    torch.cuda.synchronize()
    cells = args.nx * args.ny * args.nz
    ifc = (args.nz + 1) / args.nz
    bpc = {"eos": 32.0, "assemble": 32.0 + 24 * ifc, "momentum": 48.0, "tracers": 16.0 + 16.0 * args.ntr,
           "step": 8 * (4 + args.ntr) + 8 * (2 + args.ntr) + 24 * ifc,
           "kshear": 8.0 * 7 + 16 * ifc,   # h, u and v (two faces each), T, S in; kd, tke out
           "epbl": 24.0 + 8 * ifc}         # h, T, S in; kd out (the 2-D forcing and MLD ~0.1 B/cell)
    fns = {"eos": vp.eos, "assemble": vp.assemble, "momentum": lambda: vp.vdiff_momentum(dt),
           "tracers": lambda: vp.vdiff_tracers_nonlocal(dt), "step": lambda: vp.step(dt, 1),
           "kshear": lambda: vp.kappa_shear(dt), "epbl": lambda: vp.epbl(dt)}
    ncols = args.nx * args.ny
    if "features" in args.stages or "mlp" in args.stages:   # mlp: three GEMMs; mlp3: the fused network
        import ctypes

        from . import _ffi
        from . import learned as L

        sur = L.KPPSurrogate(seed=1)
        X = torch.empty(ncols, L.NINP, dtype=torch.bfloat16, device="cuda")
        gate = torch.empty(ncols, dtype=torch.uint8, device="cuda")
        colH = torch.empty(ncols, device="cuda")

        def features():
            _ffi.check(vp.lib.vphys_kpp_features(vp.handle, L._p(sur.feat_mean), L._p(sur.feat_istd),
                                                 ctypes.c_float(8.0), None, L._p(X), None, 0, L._p(gate),
                                                 L._p(colH)), "vphys_kpp_features")

        fns["features"] = features
        fns["mlp"] = lambda: sur.forward(X)
        Y3 = torch.empty(ncols, L.NOUTP, device="cuda")
        kerr = torch.zeros(1, dtype=torch.int32, device="cuda")

        def mlp3():
            _ffi.check(vp.lib.vphys_mlp3_bf16(L._p(X), ncols, L._p(sur.Wb[0]), L._p(sur.b[0]), L._p(sur.Wb[1]),
                                               L._p(sur.b[1]), L._p(sur.Wb[2]), L._p(sur.b[2]), L._p(Y3), L._p(kerr),
                                               None), "vphys_mlp3_bf16")

        fns["mlp3"] = mlp3
        bpc["features"] = 40.0 + L.NINP * 2.0 / args.nz   # h, rho, u, v (two faces each) -> X
        bpc["mlp"] = (L.NINP * 2 + 4 * L.NHID * 2 + L.NOUTP * 4) / args.nz   # X in, H1/H2 out+in, Y out
        bpc["mlp3"] = (L.NINP * 2 + L.NOUTP * 4) / args.nz                    # X in, Y out
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
        out[name] = {"ms": round(ms, 4), "alg_GBps": round(bpc[name] * cells / ms / 1e6, 1),
                     "cells_per_s": round(cells / ms * 1e3, 1)}
        if name == "kshear":
            kd = vp.get("kd_shear")
            out[name]["active_columns"] = round(float((kd.max(axis=2) > 0.0).mean()), 4)
    print(json.dumps({"shape": [args.nx, args.ny, args.nz], "ntr": args.ntr, "thin": args.thin,
                      "mixed": args.mixed, "stages": out}))
    vp.close()


if __name__ == "__main__":
    main()
