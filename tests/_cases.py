"""Shared builders for the parity tests: one seeded synthetic state, loaded
identically into the CPU oracle (the checker) and into the CUDA library."""
from __future__ import annotations

import numpy as np

from roundabout_b200.config import default_config, hot_path_config
from roundabout_b200.synthetic import make_columns


def columns(nx=24, ny=20, nz=12, ntr=4, seed=7, land_frac=0.3, thin_frac=0.0, passive_init="age_ps"):
    return make_columns(nx, ny, nz, ntracers=ntr, seed=seed, land_frac=land_frac, thin_frac=thin_frac,
                        passive_init=passive_init)


def oracle_state(oracle, cols, cfg):
    st = oracle.OracleState(cols.nx, cols.ny, cols.nz, len(cols.tracers))
    st.seed_backgrounds(cfg)
    st.h[...] = cols.h
    st.u[...] = cols.u
    st.v[...] = cols.v
    for t, a in enumerate(cols.tracers):
        st.tracers[t][...] = a
    st.tau_x[...] = cols.tau_x
    st.tau_y[...] = cols.tau_y
    st.q_heat[...] = cols.q_heat
    st.q_salt[...] = cols.q_salt
    st.wet[...] = cols.wet
    st.stress_mag_from_tau()
    return st


def hot_cfg(ntr=4, **over):
    cfg = hot_path_config(ntracers=ntr, pseudo_salt_index=3 if ntr > 3 else None)
    for k, v in over.items():
        setattr(cfg, k, v)
    return cfg


def plain_cfg(**over):
    cfg = default_config()
    for k, v in over.items():
        setattr(cfg, k, v)
    return cfg


def assert_bitwise(name, got, want):
    got = np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape, (name, got.shape, want.shape)
    # exact FP64 equality (a zero's sign aside: identity rows outside a
    # column's live span are not re-stored), NaN equal to NaN
    eq = (got == want) | (np.isnan(got) & np.isnan(want))
    if not eq.all():
        idx = np.argwhere(~eq)
        i0 = tuple(idx[0])
        diff = np.abs(got - want)
        scale = max(np.abs(want).max(), 1e-300)
        raise AssertionError(f"{name}: {idx.shape[0]} of {got.size} elements differ; first at {i0}: "
                             f"got {got[i0]!r} want {want[i0]!r}; max rel diff {diff.max() / scale:.3e}")
