"""Seeded synthetic ocean columns with the shapes of the benchmark configurations.

No public dataset is involved: the reference's benchmarks are whole-model
runs on its own namelists, and the hot path is exercised here on seeded
synthetic columns with the stated shapes and value distributions:

* grid: columns (i, j), dx = dy = 10 km; y_j = (j - 1/2) dy, Ly = ny dy;
* bathymetry: 8 seeded Fourier modes with wavelengths >= 1/4 of the domain,
  mapped affinely onto [500, 5000] m;
* land (`land_frac` > 0): a second smooth field thresholded at its
  `land_frac` quantile; land columns have wet = 0 and h = 0 in every layer;
* layers: geometric stretching from the surface (10 m top layer, ratio
  chosen so nz layers sum to 5000 m); a column keeps layers from the surface
  down to its bathymetry, the last one truncated, and the layers below get
  h = 0 (inert fillers, h <= H_VANISHED);
* thin layers (`thin_frac` > 0): that fraction of wet columns gets 1-10 of
  its live layers set to 1e-3 m (live, since 1e-3 > H_VANISHED = 1.5e-4);
* T = 2 + 18 exp(z/500) + N(0, 0.05) degC, S = 35 + N(0, 0.1) psu (z the
  layer-centre depth, negative down); u, v = N(0, 0.1) exp(z/300) m/s on
  faces, zero on faces touching land;
* passives: ideal age = 0, pseudo-salt = S (`passive_init="age_ps"`) or
  U[0, 1] (`passive_init="uniform"`);
* f = 1e-4 + 2e-11 y 1/s (not read by the path; an input of the learned KPP);
* forcing: tau_x = 0.1 sin(pi y / Ly) N/m2, tau_y = 0;
  Q_heat ~ U[-100, 100] W/m2; freshwater F ~ U[-1e-7, 1e-7] m/s turned into
  the reference's salt flux as Q_salt = -rho0 * 35 * F.

Arrays are numpy float64 in Fortran order with the reference's shapes
((nx, ny, nz) cells, (nx+1, ny, nz) u faces, ...), k = 0 the bed.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

DX = 1.0e4


@dataclass
class Columns:
    nx: int
    ny: int
    nz: int
    h: np.ndarray
    u: np.ndarray
    v: np.ndarray
    tracers: list
    tau_x: np.ndarray
    tau_y: np.ndarray
    q_heat: np.ndarray
    q_salt: np.ndarray
    wet: np.ndarray
    kbot: np.ndarray = field(repr=False)   # 1-based index of the deepest live layer (0 on land)
    coriolis: np.ndarray = field(default=None, repr=False)   # f = 1e-4 + 2e-11 y (read by the learned KPP only)

    @property
    def ncells(self) -> int:
        return self.nx * self.ny * self.nz


def _smooth_field(rng, nx, ny, nmodes=8):
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    f = np.zeros((nx, ny))
    for _ in range(nmodes):
        kx = rng.integers(0, 5)   # wavelength >= 1/4 of the domain
        ky = rng.integers(0, 5)
        amp = rng.normal()
        ph = rng.uniform(0, 2 * np.pi)
        f += amp * np.cos(2 * np.pi * (kx * x[:, None] + ky * y[None, :]) + ph)
    return f


def layer_stack(nz, top=10.0, total=5000.0):
    """Geometric layer thicknesses from the surface down summing to `total`."""
    if nz == 1:
        return np.array([total])
    if top * nz >= total:
        return np.full(nz, total / nz)
    lo, hi = 1.0, 2.0
    while top * (hi ** nz - 1) / (hi - 1) < total:
        hi *= 2
    for _ in range(200):
        r = 0.5 * (lo + hi)
        s = top * (r ** nz - 1) / (r - 1)
        if s > total:
            hi = r
        else:
            lo = r
    r = 0.5 * (lo + hi)
    dz = top * r ** np.arange(nz)
    dz *= total / dz.sum()
    return dz


def make_columns(nx, ny, nz, ntracers=2, seed=1234, land_frac=0.0, thin_frac=0.0,
                 passive_init="age_ps", rho0=1035.0) -> Columns:
    rng = np.random.Generator(np.random.Philox(seed))
    F = lambda *s: np.zeros(s, dtype=np.float64, order="F")  # noqa: E731

    bathy = _smooth_field(rng, nx, ny)
    bmin, bmax = bathy.min(), bathy.max()
    bathy = 500.0 + (bathy - bmin) * (4500.0 / max(bmax - bmin, 1e-30))
    wet = np.ones((nx, ny), order="F")
    if land_frac > 0:
        lf = _smooth_field(rng, nx, ny)
        thr = np.quantile(lf, land_frac)
        wet = np.asfortranarray((lf > thr).astype(np.float64))

    dz_top_down = layer_stack(nz)                 # index 0 = surface layer
    edges = np.concatenate([[0.0], np.cumsum(dz_top_down)])
    # per column thickness of each layer counted from the surface
    b = bathy[:, :, None]
    top_edge = edges[None, None, :-1]
    bot_edge = edges[None, None, 1:]
    h_td = np.clip(np.minimum(bot_edge, b) - top_edge, 0.0, None)   # (nx, ny, nz) surface-first
    h_td *= wet[:, :, None]
    if thin_frac > 0:
        wet_idx = np.flatnonzero(wet.ravel(order="F") > 0)
        pick = rng.choice(wet_idx, size=int(thin_frac * wet_idx.size), replace=False)
        nthin = rng.integers(1, 11, size=pick.size)
        h2 = h_td.reshape(nx * ny, nz, order="F")
        for col, n in zip(pick, nthin):
            live = np.flatnonzero(h2[col] > 1.5e-4)
            if live.size == 0:
                continue
            sel = rng.choice(live, size=min(n, live.size), replace=False)
            h2[col, sel] = 1.0e-3
        h_td = h2.reshape(nx, ny, nz, order="F")
    h = np.asfortranarray(h_td[:, :, ::-1])       # bottom-up: k = 0 bed
    live = h > 1.5e-4
    kbot = np.where(live.any(axis=2), np.argmax(live, axis=2) + 1, 0).astype(np.int32)

    # layer-centre depth (negative down), bottom-up
    zc_td = -(edges[:-1] + 0.5 * dz_top_down)
    zc = zc_td[::-1]
    T = 2.0 + 18.0 * np.exp(zc / 500.0)[None, None, :] + rng.normal(0.0, 0.05, size=(nx, ny, nz))
    S = 35.0 + rng.normal(0.0, 0.1, size=(nx, ny, nz))
    T = np.asfortranarray(T)
    S = np.asfortranarray(S)
    decay = np.exp(zc / 300.0)[None, None, :]
    u = np.asfortranarray(rng.normal(0.0, 0.1, size=(nx + 1, ny, nz)) * decay)
    v = np.asfortranarray(rng.normal(0.0, 0.1, size=(nx, ny + 1, nz)) * decay)
    # no flow through faces touching land (or the domain walls)
    wu = np.zeros((nx + 1, ny))
    wu[1:nx] = np.minimum(wet[:-1], wet[1:])
    wv = np.zeros((nx, ny + 1))
    wv[:, 1:ny] = np.minimum(wet[:, :-1], wet[:, 1:])
    u *= wu[:, :, None]
    v *= wv[:, :, None]

    tracers = [S, T]
    for n in range(2, ntracers):
        if passive_init == "uniform":
            tracers.append(np.asfortranarray(rng.uniform(0.0, 1.0, size=(nx, ny, nz))))
        elif n == 2:
            tracers.append(F(nx, ny, nz))          # ideal age
        else:
            tracers.append(S.copy(order="F"))      # pseudo-salt mirror of S
    tracers = tracers[:ntracers]

    y = (np.arange(ny) + 0.5) * DX
    Ly = ny * DX
    tau_x = np.asfortranarray(np.broadcast_to(0.1 * np.sin(np.pi * y / Ly)[None, :], (nx + 1, ny)).copy())
    tau_y = F(nx, ny + 1)
    q_heat = np.asfortranarray(rng.uniform(-100.0, 100.0, size=(nx, ny)))
    fw = rng.uniform(-1.0e-7, 1.0e-7, size=(nx, ny))
    q_salt = np.asfortranarray(-rho0 * 35.0 * fw)
    coriolis = np.asfortranarray(np.broadcast_to((1.0e-4 + 2.0e-11 * y)[None, :], (nx, ny)).copy())
    return Columns(nx, ny, nz, h, u, v, tracers, tau_x, tau_y, q_heat, q_salt, wet, kbot, coriolis)


# Benchmark configurations (shapes of the reference's north-star configs).
CONFIGS = {
    "cpu_64x64x20": dict(nx=64, ny=64, nz=20, ntracers=2, land_frac=0.0, thin_frac=0.0),
    "eddy_1440x1080x75": dict(nx=1440, ny=1080, nz=75, ntracers=4, land_frac=0.3, thin_frac=0.0),
    "batched_1440x1080x75": dict(nx=1440, ny=1080, nz=75, ntracers=10, land_frac=0.3, thin_frac=0.15,
                                 passive_init="uniform"),
    # built on the device (make_columns_device): T, S + 4 passives
    "combined_3600x2700x75": dict(nx=3600, ny=2700, nz=75, ntracers=6, land_frac=0.3, thin_frac=0.0,
                                  passive_init="uniform"),
}


# ---------------------------------------------------------------------------
# Device-side generator for the shapes too large to build on the host
# ---------------------------------------------------------------------------
def make_columns_device(nx, ny, nz, ntracers=6, seed=1234, land_frac=0.3, passive_init="uniform", rho0=1035.0):
    """The same distributions as `make_columns`, drawn on the GPU with torch's
    seeded Philox generator (a different random stream, so not the same
    numbers), returned as contiguous CUDA float64 tensors in the reference's
    layout (torch shape (nz, ny, nx) is Fortran (nx, ny, nz)) ready for
    VerticalPhysics.bind.  For 3600x2700x75 no field ever exists on the host.
    Returns a dict: h, u, v, tracers (list), tau_x, tau_y, q_heat, q_salt,
    wet, coriolis."""
    import math

    import torch

    dev = "cuda"
    g = torch.Generator(device=dev).manual_seed(seed)
    f64 = torch.float64

    def smooth():
        x = (torch.arange(nx, device=dev, dtype=f64) + 0.5) / nx
        y = (torch.arange(ny, device=dev, dtype=f64) + 0.5) / ny
        f = torch.zeros(ny, nx, device=dev, dtype=f64)
        for _ in range(8):
            kx = int(torch.randint(0, 5, (1,), generator=g, device=dev))
            ky = int(torch.randint(0, 5, (1,), generator=g, device=dev))
            amp = float(torch.randn(1, generator=g, device=dev))
            ph = float(torch.rand(1, generator=g, device=dev)) * 2 * math.pi
            f += amp * torch.cos(2 * math.pi * (kx * x[None, :] + ky * y[:, None]) + ph)
        return f

    bathy = smooth()
    bmin, bmax = float(bathy.min()), float(bathy.max())
    bathy = 500.0 + (bathy - bmin) * (4500.0 / max(bmax - bmin, 1e-30))
    wet = torch.ones(ny, nx, device=dev, dtype=f64)
    if land_frac > 0:
        lf = smooth()
        flat = lf.flatten()
        sample = flat[torch.randperm(flat.numel(), generator=g, device=dev)[: min(flat.numel(), 1 << 22)]]
        thr = float(torch.quantile(sample, land_frac))
        wet = (lf > thr).to(f64)

    dz_td = torch.tensor(layer_stack(nz), device=dev, dtype=f64)
    edges = torch.cat([torch.zeros(1, device=dev, dtype=f64), torch.cumsum(dz_td, 0)])
    h = torch.empty(nz, ny, nx, device=dev, dtype=f64)
    for kt in range(nz):   # surface-first index kt -> bottom-up k = nz - 1 - kt
        h[nz - 1 - kt] = torch.clamp(torch.minimum(edges[kt + 1], bathy) - edges[kt], min=0.0) * wet
    zc = -(edges[:-1] + 0.5 * dz_td).flip(0)   # layer-centre depth, bottom-up
    T = 2.0 + 18.0 * torch.exp(zc / 500.0)[:, None, None] + 0.05 * torch.randn(nz, ny, nx, generator=g, device=dev,
                                                                              dtype=f64)
    S = 35.0 + 0.1 * torch.randn(nz, ny, nx, generator=g, device=dev, dtype=f64)
    decay = torch.exp(zc / 300.0)[:, None, None]
    wu = torch.zeros(ny, nx + 1, device=dev, dtype=f64)
    wu[:, 1:nx] = torch.minimum(wet[:, :-1], wet[:, 1:])
    wv = torch.zeros(ny + 1, nx, device=dev, dtype=f64)
    wv[1:ny, :] = torch.minimum(wet[:-1, :], wet[1:, :])
    u = 0.1 * torch.randn(nz, ny, nx + 1, generator=g, device=dev, dtype=f64) * decay * wu[None]
    v = 0.1 * torch.randn(nz, ny + 1, nx, generator=g, device=dev, dtype=f64) * decay * wv[None]
    tracers = [S, T]
    for n in range(2, ntracers):
        if passive_init == "uniform":
            tracers.append(torch.rand(nz, ny, nx, generator=g, device=dev, dtype=f64))
        elif n == 2:
            tracers.append(torch.zeros(nz, ny, nx, device=dev, dtype=f64))
        else:
            tracers.append(S.clone())
    y = (torch.arange(ny, device=dev, dtype=f64) + 0.5) * DX
    Ly = ny * DX
    tau_x = (0.1 * torch.sin(math.pi * y / Ly))[:, None].expand(ny, nx + 1).contiguous()
    tau_y = torch.zeros(ny + 1, nx, device=dev, dtype=f64)
    q_heat = torch.rand(ny, nx, generator=g, device=dev, dtype=f64) * 200.0 - 100.0
    fw = (torch.rand(ny, nx, generator=g, device=dev, dtype=f64) * 2.0 - 1.0) * 1.0e-7
    q_salt = -rho0 * 35.0 * fw
    coriolis = (1.0e-4 + 2.0e-11 * y)[:, None].expand(ny, nx).contiguous()
    return {"h": h.contiguous(), "u": u.contiguous(), "v": v.contiguous(), "tracers": tracers, "tau_x": tau_x,
            "tau_y": tau_y, "q_heat": q_heat.contiguous(), "q_salt": q_salt.contiguous(), "wet": wet.contiguous(),
            "coriolis": coriolis}


def bind_device_columns(vp, d):
    """Bind a `make_columns_device` dict to a VerticalPhysics handle (zero
    copy) and derive the stress magnitude."""
    for name in ("h", "u", "v", "tau_x", "tau_y", "q_heat", "q_salt", "wet", "coriolis"):
        vp.bind(name, d[name])
    for t, a in enumerate(d["tracers"][: vp.ntr]):
        vp.bind(f"tracer{t}", a)
    vp.stress_mag()
