"""The learned KPP surrogate: an MLP standing in for KPP pass 1's bulk
Richardson search (vmix_kpp_overlay_impl, rdb_ocean_vmix.F90:1288-1426).

    154 standardised features -> 256 GELU -> 256 GELU -> 77 standardised outputs

Features and targets are computed on the GPU by libvphys
(vphys_kpp_features / vphys_kpp_targets: u*, B0, f, the column depth, and the
bulk N^2 and shear^2 of the 75 layers below the surface layer; log h_b, log h_b
w_s and the 75-interface shape G(sigma)).  Every matrix product of training
and inference is the library's tcgen05 BF16 GEMM (vphys_gemm_tn_bf16, FP32
accumulation, GELU and its derivative fused in the epilogue); the loss
gradient, bias sums, standardisation and the Adam step are the library's
kernels too.  torch supplies device memory only.

Training data come from the plain KPP itself: seeded domains of the
benchmark's generators are stepped with the plain FP64 path and every
snapshot contributes (features of the state, h_b that pass 1 then computes).

In a step (cfg.learned_kpp = 1, surrogate attached with attach()), the
library runs features -> MLP -> gate/check and the assembly's pass 1 only for
the gated, sampled or fallback columns.
"""
from __future__ import annotations

import ctypes
import math
import time

import numpy as np

from . import _ffi

NIN, NINP, NHID, NOUT, NOUTP, NLEV = 154, 160, 256, 77, 80, 75


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class KPPSurrogate:
    """Weights (FP32 masters, BF16 copies for the tensor cores), Adam state and
    the standardisation of features and targets."""

    def __init__(self, seed: int = 0):
        import torch

        self.torch = torch
        self.lib = _ffi.get_lib()
        dev = "cuda"
        g = torch.Generator(device="cpu").manual_seed(seed)

        def init(out, inp, fan_in, live_out=None, live_in=None):
            w = (torch.rand(out, inp, generator=g) * 2 - 1) * math.sqrt(3.0 / fan_in)
            if live_in is not None:
                w[:, live_in:] = 0
            if live_out is not None:
                w[live_out:, :] = 0
            return w.to(dev)

        self.W = [init(NHID, NINP, NIN, live_in=NIN), init(NHID, NHID, NHID), init(NOUTP, NHID, NHID, live_out=NOUT)]
        self.b = [torch.zeros(NHID, device=dev), torch.zeros(NHID, device=dev), torch.zeros(NOUTP, device=dev)]
        self.m = [torch.zeros_like(t) for t in self.W + self.b]
        self.v = [torch.zeros_like(t) for t in self.W + self.b]
        self.Wb = [w.to(torch.bfloat16).contiguous() for w in self.W]
        self.WT = [None, self.W[1].T.contiguous().to(torch.bfloat16), self.W[2].T.contiguous().to(torch.bfloat16)]
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        self.feat_mean = torch.zeros(NINP, device=dev)
        self.feat_istd = torch.ones(NINP, device=dev)
        self.tgt_mean = torch.zeros(NOUTP, device=dev)
        self.tgt_std = torch.ones(NOUTP, device=dev)
        w = np.zeros(NOUTP, np.float32)
        w[0], w[1], w[2:NOUT] = 1.0, 0.1, 0.01
        self.loss_w = torch.tensor(w, device=dev)
        self.adam_step = 0
        self._model = None

    # ---- the tensor-core GEMM --------------------------------------------------------
    def gemm(self, A, lda, B, ldb, M, N, K, bias=None, zin=None, act=0, out32=None, outb=None, outbt=None, ld_t=0):
        st = self.lib.vphys_gemm_tn_bf16(_p(A), lda, _p(B), ldb, M, N, K, 1.0, _p(bias), _p(zin), N, act,
                                         _p(out32), N, _p(outb), N, _p(outbt), ld_t, _p(self.err), None)
        _ffi.check(st, "vphys_gemm_tn_bf16")

    def forward(self, X, save: bool = False):
        """X: BF16 [B, 160] standardised features -> FP32 [B, 80] standardised outputs."""
        torch = self.torch
        B = X.shape[0]
        e = lambda *s, dt=torch.bfloat16: torch.empty(*s, dtype=dt, device="cuda")  # noqa: E731
        c = {}
        c["Z1"] = e(B, NHID, dt=torch.float32) if save else None
        c["H1"], c["H1T"] = e(B, NHID), (e(NHID, B) if save else None)
        self.gemm(X, NINP, self.Wb[0], NINP, B, NHID, NINP, bias=self.b[0], act=1, out32=c["Z1"], outb=c["H1"],
                  outbt=c["H1T"], ld_t=B)
        c["Z2"] = e(B, NHID, dt=torch.float32) if save else None
        c["H2"], c["H2T"] = e(B, NHID), (e(NHID, B) if save else None)
        self.gemm(c["H1"], NHID, self.Wb[1], NHID, B, NHID, NHID, bias=self.b[1], act=1, out32=c["Z2"],
                  outb=c["H2"], outbt=c["H2T"], ld_t=B)
        Y = e(B, NOUTP, dt=torch.float32)
        self.gemm(c["H2"], NHID, self.Wb[2], NHID, B, NOUTP, NHID, bias=self.b[2], act=0, out32=Y)
        self._cache = c if save else None
        return Y

    def gradients(self, X, XT, ldxt, T):
        """Loss and parameter gradients of one batch (forward included).  XT is
        the transposed feature matrix slice [160, B] with row stride ldxt."""
        torch = self.torch
        B = X.shape[0]
        Y = self.forward(X, save=True)
        c = self._cache
        L = self.lib
        loss = torch.zeros(1, device="cuda")
        dY32 = torch.empty(B, NOUTP, device="cuda")
        dY = torch.empty(B, NOUTP, dtype=torch.bfloat16, device="cuda")
        dYT = torch.empty(NOUTP, B, dtype=torch.bfloat16, device="cuda")
        _ffi.check(L.vphys_mlp_loss(_p(Y), _p(T), _p(self.loss_w), B, NOUTP, 2.0 / B, _p(dY32), _p(dY), _p(dYT),
                                    _p(loss), None), "vphys_mlp_loss")
        gW = [torch.empty_like(w) for w in self.W]
        gb = [torch.zeros_like(b) for b in self.b]
        # layer 3
        self.gemm(dYT, B, c["H2T"], B, NOUTP, NHID, B, out32=gW[2])
        _ffi.check(L.vphys_mlp_colsum(_p(dY32), B, NOUTP, NOUTP, _p(gb[2]), None), "colsum")
        # layer 2: dZ2 = (dY . W3) * GELU'(Z2)
        dZ2f = torch.empty(B, NHID, device="cuda")
        dZ2 = torch.empty(B, NHID, dtype=torch.bfloat16, device="cuda")
        dZ2T = torch.empty(NHID, B, dtype=torch.bfloat16, device="cuda")
        self.gemm(dY, NOUTP, self.WT[2], NOUTP, B, NHID, NOUTP, zin=c["Z2"], out32=dZ2f, outb=dZ2, outbt=dZ2T,
                  ld_t=B)
        self.gemm(dZ2T, B, c["H1T"], B, NHID, NHID, B, out32=gW[1])
        _ffi.check(L.vphys_mlp_colsum(_p(dZ2f), B, NHID, NHID, _p(gb[1]), None), "colsum")
        # layer 1: dZ1 = (dZ2 . W2) * GELU'(Z1)
        dZ1f = torch.empty(B, NHID, device="cuda")
        dZ1T = torch.empty(NHID, B, dtype=torch.bfloat16, device="cuda")
        self.gemm(dZ2, NHID, self.WT[1], NHID, B, NHID, NHID, zin=c["Z1"], out32=dZ1f, outbt=dZ1T, ld_t=B)
        self.gemm(dZ1T, B, XT, ldxt, NHID, NINP, B, out32=gW[0])
        _ffi.check(L.vphys_mlp_colsum(_p(dZ1f), B, NHID, NHID, _p(gb[0]), None), "colsum")
        return loss, Y, gW, gb

    def adam(self, gW, gb, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.adam_step += 1
        L = self.lib
        params = list(zip(self.W, gW, [self.Wb[0], self.Wb[1], self.Wb[2]], self.WT)) + \
            [(b, g, None, None) for b, g in zip(self.b, gb)]
        for idx, (w, g, wb, wbt) in enumerate(params):
            rows, cols = (w.shape[0], w.shape[1]) if w.dim() == 2 else (1, w.shape[0])
            _ffi.check(L.vphys_mlp_adam(_p(w), _p(self.m[idx]), _p(self.v[idx]), _p(g), rows, cols, lr, b1, b2, eps,
                                        self.adam_step, _p(wb), _p(wbt), None), "vphys_mlp_adam")

    # ---- data -------------------------------------------------------------------------
    def fit_standardisation(self, raw, T):
        """Means and inverse standard deviations of the features (raw [N, 154])
        and targets (T [N, 80]) with the library's column-statistics kernel."""
        torch = self.torch
        L = self.lib
        for arr, ncol, mean_out, scale_out, inv in ((raw, NIN, self.feat_mean, self.feat_istd, True),
                                                   (T, NOUTP, self.tgt_mean, self.tgt_std, False)):
            n = arr.shape[0]
            s = torch.zeros(ncol, dtype=torch.float64, device="cuda")
            q = torch.zeros(ncol, dtype=torch.float64, device="cuda")
            _ffi.check(L.vphys_mlp_colstats(_p(arr), n, ncol, arr.shape[1], _p(s), _p(q), None), "colstats")
            mean = s / n
            std = torch.sqrt(torch.clamp(q / n - mean * mean, min=0.0))
            mean_out.zero_()
            mean_out[:ncol] = mean.float()
            if inv:
                scale_out.zero_()
                scale_out[:ncol] = torch.where(std > 1e-6, 1.0 / std, torch.zeros_like(std)).float()
            else:
                scale_out.fill_(1.0)
                scale_out[:ncol] = torch.where(std > 1e-6, std, torch.ones_like(std)).float()

    def standardise(self, raw, T=None):
        """BF16 X [N, 160], BF16 XT [160, N] and standardised FP32 targets."""
        torch = self.torch
        L = self.lib
        n = raw.shape[0]
        X = torch.empty(n, NINP, dtype=torch.bfloat16, device="cuda")
        XT = torch.empty(NINP, n, dtype=torch.bfloat16, device="cuda")
        _ffi.check(L.vphys_mlp_standardize(_p(raw), n, NIN, NIN, _p(self.feat_mean), _p(self.feat_istd), NINP,
                                           _p(X), _p(XT), n, None, None), "standardize")
        Ts = None
        if T is not None:
            Ts = torch.empty(n, NOUTP, device="cuda")
            inv = torch.where(self.tgt_std > 0, 1.0 / self.tgt_std, torch.zeros_like(self.tgt_std))
            _ffi.check(L.vphys_mlp_standardize(_p(T), n, NOUTP, NOUTP, _p(self.tgt_mean), _p(inv), NOUTP, None, None,
                                               0, _p(Ts), None), "standardize")
        return X, XT, Ts

    def train(self, X, XT, Ts, epochs=4, batch=8192, lr=2e-3, lr_end=1e-4, log=None):
        """Adam over the training set in fixed batches; cosine learning rate."""
        n = (X.shape[0] // batch) * batch
        steps = epochs * (n // batch)
        t0 = time.perf_counter()
        hist = []
        k = 0
        for ep in range(epochs):
            tot = 0.0
            for b0 in range(0, n, batch):
                lr_k = lr_end + 0.5 * (lr - lr_end) * (1 + math.cos(math.pi * k / max(1, steps)))
                XTb = XT[:, b0:]
                loss, _, gW, gb = self.gradients(X[b0:b0 + batch], XTb, XT.shape[1], Ts[b0:b0 + batch])
                self.adam(gW, gb, lr=lr_k)
                tot += float(loss.item()) if (b0 // batch) % 64 == 0 else 0.0
                k += 1
            hist.append(tot)
            if log:
                log(f"epoch {ep}: sampled loss {tot:.4g}")
        self.torch.cuda.synchronize()
        self.train_seconds = time.perf_counter() - t0
        assert int(self.err.item()) == 0
        return hist

    def predict_hb(self, X):
        """OBL depth (m) predicted for the standardised features X."""
        Y = self.forward(X)
        return 10.0 * self.torch.exp(Y[:, 0] * float(self.tgt_std[0]) + float(self.tgt_mean[0]))

    # ---- the library's in-step surrogate -----------------------------------------------
    def model_struct(self, gate_limit=8.0, check_fraction=0.01, check_tolerance=0.25, fail_fraction=0.2):
        m = _ffi.KppModel()
        m.w1, m.w2, m.w3 = (t.data_ptr() for t in self.Wb)
        m.b1, m.b2, m.b3 = (t.data_ptr() for t in self.b)
        m.feat_mean, m.feat_istd = self.feat_mean.data_ptr(), self.feat_istd.data_ptr()
        m.target_mean0, m.target_std0 = float(self.tgt_mean[0]), float(self.tgt_std[0])
        m.gate_limit, m.check_fraction = gate_limit, check_fraction
        m.check_tolerance, m.fail_fraction = check_tolerance, fail_fraction
        self._model = m
        return m

    def attach(self, vp, **kw):
        _ffi.check(self.lib.vphys_kpp_attach(vp.handle, ctypes.byref(self.model_struct(**kw))), "vphys_kpp_attach")


def kpp_stats(vp):
    out = (ctypes.c_ulonglong * 16)()
    _ffi.check(vp.lib.vphys_kpp_stats(vp.handle, out, 16), "vphys_kpp_stats")
    names = ["checked_step", "failed_step", "fallback_step", "gated_step", "checked", "failed", "fallback_steps",
             "gated", "sum_rel_err2_e6", "steps", "gemm_err"]
    return {n: int(out[i]) for i, n in enumerate(names)}


def collect(nx, ny, nz, domains, snapshots, seed=100, dt=3600.0, log=None, surrogate=None):
    """(raw features [N, 154], targets [N, 80]) from trajectories of seeded
    domains (all wet, the benchmark's generators), one sample per column and
    snapshot step.  Without `surrogate` the trajectories are the plain
    KPP's; with one they are the learned form's own (the surrogate attached),
    and each snapshot is still labelled by the plain KPP pass 1 on that state
    (the lagged h_b put back afterwards, so the trajectory is the learned
    one's)."""
    import torch

    from .column import VerticalPhysics
    from .config import hot_path_config
    from .synthetic import make_columns

    lib = _ffi.get_lib()
    raws, tgts = [], []
    ncols = nx * ny
    for d in range(domains):
        cols = make_columns(nx, ny, nz, ntracers=2, seed=seed + d, land_frac=0.0, thin_frac=0.0)
        cfg_plain = hot_path_config(ntracers=2)
        cfg_run = hot_path_config(ntracers=2)
        if surrogate is not None:
            cfg_run.learned_kpp = 1
        vp = VerticalPhysics(nx, ny, nz, 2, cfg_run)
        vp.load_columns(cols)
        if surrogate is not None:
            surrogate.attach(vp)
        step = 0
        for snap in sorted(snapshots):
            if snap > step:
                vp.step(dt, snap - step)
                step = snap
            raw = torch.empty(ncols, NIN, device="cuda")
            T = torch.empty(ncols, NOUTP, device="cuda")
            vp.eos()
            _ffi.check(lib.vphys_kpp_features(vp.handle, None, None, ctypes.c_float(1e30), _p(raw), None, None, 0,
                                              None, None), "vphys_kpp_features")
            lagged = vp.get("bl_depth") if surrogate is not None else None
            if surrogate is not None:
                vp.set_config(cfg_plain)
            vp.assemble()
            _ffi.check(lib.vphys_kpp_targets(vp.handle, _p(T)), "vphys_kpp_targets")
            if surrogate is not None:
                vp.set("bl_depth", lagged)
                vp.set_config(cfg_run)
            raws.append(raw)
            tgts.append(T)
        vp.close()
        if log:
            log(f"domain {d}: {len(snapshots)} snapshots" + (" (learned trajectory)" if surrogate is not None else ""))
    raw = torch.cat(raws)
    T = torch.cat(tgts)
    g = torch.Generator(device="cuda").manual_seed(seed)
    perm = torch.randperm(raw.shape[0], generator=g, device="cuda")
    return raw[perm].contiguous(), T[perm].contiguous()


def train_surrogate(ncols_target=4_000_000, nz=75, seed=100, epochs=4, batch=8192, snaps=(0, 23, 167, 719),
                    domain=(256, 1024), rounds=1, log=None):
    """Collect about `ncols_target` training columns (256 x 1024 domains,
    so that f and the wind stress span the 1080-row benchmark's ranges;
    snapshots after 0, 23, 167 and 719 plain steps) and train a surrogate.
    With rounds = 2 the trained network then runs its own trajectories on
    fresh domains, the plain KPP labels their snapshots, and training goes on
    over both sets (the network learns the states it actually produces)."""
    import torch

    per = domain[0] * domain[1]
    domains = max(1, round(ncols_target / (per * len(snaps))))
    t0 = time.perf_counter()
    raw, T = collect(domain[0], domain[1], nz, domains, list(snaps), seed=seed, log=log)
    t_collect = time.perf_counter() - t0
    s = KPPSurrogate(seed=seed)
    s.fit_standardisation(raw, T)
    X, XT, Ts = s.standardise(raw, T)
    hist = s.train(X, XT, Ts, epochs=epochs, batch=batch, log=log)
    t_train = s.train_seconds
    for r in range(1, rounds):
        del X, XT, Ts
        t0 = time.perf_counter()
        raw2, T2 = collect(domain[0], domain[1], nz, domains, list(snaps), seed=seed + 1000 * r, log=log,
                           surrogate=s)
        t_collect += time.perf_counter() - t0
        raw = torch.cat([raw, raw2])
        T = torch.cat([T, T2])
        g = torch.Generator(device="cuda").manual_seed(seed + r)
        perm = torch.randperm(raw.shape[0], generator=g, device="cuda")
        raw, T = raw[perm].contiguous(), T[perm].contiguous()
        del raw2, T2
        X, XT, Ts = s.standardise(raw, T)   # the first round's standardisation stays
        s.adam_step = 0
        s.m = [torch.zeros_like(t) for t in s.m]
        s.v = [torch.zeros_like(t) for t in s.v]
        hist += s.train(X, XT, Ts, epochs=epochs, batch=batch, lr=1e-3, log=log)
        t_train += s.train_seconds
    s.collect_seconds = t_collect
    s.train_seconds = t_train
    s.ntrain = X.shape[0]
    return s, hist
