"""`VerticalPhysics`: the Python driver of libvphys (the CUDA library).

Mirrors the reference's python/rdb model surface for this path
(python/rdb/_model.py:94-96, 703-707: `Model(...).step(n)`, field views such
as `m.kv` / `m.kt`), over the C ABI of include/vphys.h:

    vp = VerticalPhysics(nx, ny, nz, ntracers, config)
    vp.set("h", h); vp.set_tracer(0, S); ...       # host numpy -> HBM
    vp.bind("u", tensor)                             # zero-copy device array
    vp.step(dt, n)                                   # whole chain on the GPU
    kv = vp.get("kv")                                # HBM -> host numpy

Arrays use the reference layout: Fortran order with shape (nx, ny, nz) etc.
(k = 0 the bed).  A torch tensor bound to a field must be a contiguous CUDA
float64 tensor of shape (nz, ny, nx) -- the same bytes as the Fortran
(nx, ny, nz) array.  There is no CPU fallback: a missing library or GPU
raises.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _ffi
from .config import default_config


class VerticalPhysics:
    def __init__(self, nx: int, ny: int, nz: int, ntracers: int, config=None):
        self.lib = _ffi.get_lib()
        self.nx, self.ny, self.nz, self.ntr = int(nx), int(ny), int(nz), int(ntracers)
        self.config = config if config is not None else default_config()
        h = ctypes.c_void_p()
        _ffi.check(self.lib.vphys_create(self.nx, self.ny, self.nz, self.ntr, ctypes.byref(self.config),
                                         ctypes.byref(h)), "vphys_create")
        self._h = h
        self._bound = {}

    # ---- lifecycle ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.vphys_destroy(ctypes.byref(self._h))
        self._h = None
        self._bound = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_config(self, cfg):
        _ffi.check(self.lib.vphys_set_config(self._h, ctypes.byref(cfg)), "vphys_set_config")
        self.config = cfg

    def set_stream(self, stream_ptr: int):
        _ffi.check(self.lib.vphys_set_stream(self._h, ctypes.c_void_p(stream_ptr)), "vphys_set_stream")

    # ---- fields ------------------------------------------------------------
    def _fid(self, name):
        if isinstance(name, int):
            return name
        if name.startswith("tracer"):
            return _ffi.FIELD_TRACER0 + int(name[6:])
        return _ffi.FIELD_NAMES[name]

    def shape(self, name):
        return _ffi.field_shape(self._fid(name), self.nx, self.ny, self.nz, self.ntr)

    def set(self, name, array):
        fid = self._fid(name)
        dtype = np.int32 if fid in _ffi.INT_FIELDS else np.float64
        a = np.asarray(array, dtype=dtype)
        shp = self.shape(fid)
        if a.shape != shp:
            raise ValueError(f"{name}: expected shape {shp}, got {a.shape}")
        a = np.asfortranarray(a)
        _ffi.check(self.lib.vphys_set_field(self._h, fid, a.ctypes.data_as(ctypes.c_void_p), a.size),
                   f"vphys_set_field({name})")

    def get(self, name):
        fid = self._fid(name)
        dtype = np.int32 if fid in _ffi.INT_FIELDS else np.float64
        out = np.empty(self.shape(fid), dtype=dtype, order="F")
        _ffi.check(self.lib.vphys_get_field(self._h, fid, out.ctypes.data_as(ctypes.c_void_p), out.size),
                   f"vphys_get_field({name})")
        return out

    def set_tracer(self, t, array):
        self.set(_ffi.FIELD_TRACER0 + int(t), array)

    def get_tracer(self, t):
        return self.get(_ffi.FIELD_TRACER0 + int(t))

    def device_ptr(self, name):
        ptr = ctypes.c_void_p()
        gen = ctypes.c_int()
        nx, ny, nz = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _ffi.check(self.lib.vphys_get_ptr(self._h, self._fid(name), ctypes.byref(ptr), ctypes.byref(nx),
                                          ctypes.byref(ny), ctypes.byref(nz), ctypes.byref(gen)), "vphys_get_ptr")
        return ptr.value, (nx.value, ny.value, nz.value), gen.value

    def bind(self, name, tensor):
        """Zero-copy: use a CUDA tensor (contiguous, float64/int32) for a field."""
        fid = self._fid(name)
        if tensor is None:
            _ffi.check(self.lib.vphys_bind(self._h, fid, None), f"vphys_bind({name})")
            self._bound.pop(fid, None)
            return
        expect = int(np.prod(self.shape(fid)))
        if not tensor.is_cuda or not tensor.is_contiguous() or tensor.numel() != expect:
            raise ValueError(f"{name}: need a contiguous CUDA tensor with {expect} elements")
        self._bound[fid] = tensor   # keep alive
        _ffi.check(self.lib.vphys_bind(self._h, fid, ctypes.c_void_p(tensor.data_ptr())), f"vphys_bind({name})")

    def load_columns(self, cols):
        """Upload a `synthetic.Columns` (h, u, v, tracers, forcing, wet) and
        derive stress_mag from the face stresses."""
        self.set("h", cols.h)
        self.set("u", cols.u)
        self.set("v", cols.v)
        for t, a in enumerate(cols.tracers[: self.ntr]):
            self.set_tracer(t, a)
        self.set("tau_x", cols.tau_x)
        self.set("tau_y", cols.tau_y)
        self.set("q_heat", cols.q_heat)
        self.set("q_salt", cols.q_salt)
        self.set("wet", cols.wet)
        if getattr(cols, "coriolis", None) is not None:
            self.set("coriolis", cols.coriolis)
        self.stress_mag()

    # ---- the hot path --------------------------------------------------------
    def eos(self):
        _ffi.check(self.lib.vphys_eos_wright(self._h), "vphys_eos_wright")

    def stress_mag(self):
        _ffi.check(self.lib.vphys_stress_mag(self._h), "vphys_stress_mag")

    def surface_flux(self, dt):
        """ocean_surface_flux_apply_tracers (rdb_ocean_surface_flux.F90:959-1070)."""
        _ffi.check(self.lib.vphys_surface_flux(self._h, float(dt)), "vphys_surface_flux")

    def sw_chl_apply(self):
        """sw_chl_fill_kappa (rdb_ocean_sw_chl.F90:160-190): the band opacities from the sw_chl field."""
        _ffi.check(self.lib.vphys_sw_chl_apply(self._h), "vphys_sw_chl_apply")

    def sw_penetration(self, dt):
        """ocean_surface_flux_apply_sw_penetration (rdb_ocean_surface_flux.F90:1255-1370)."""
        _ffi.check(self.lib.vphys_sw_penetration(self._h, float(dt)), "vphys_sw_penetration")

    def kappa_shear(self, dt):
        """kappa_shear_compute, column form (rdb_ocean_kappa_shear.F90:427-648):
        fills the kd_shear / tke_shear fields."""
        _ffi.check(self.lib.vphys_kappa_shear(self._h, float(dt)), "vphys_kappa_shear")

    def epbl(self, dt):
        """epbl_compute, column form (rdb_ocean_epbl.F90:864-1659): fills the
        kd_epbl / mld_epbl fields."""
        _ffi.check(self.lib.vphys_epbl(self._h, float(dt)), "vphys_epbl")

    def assemble(self):
        return _ffi.check(self.lib.vphys_assemble(self._h), "vphys_assemble")

    def assemble_status(self):
        """vphys_assemble returning the status instead of raising (guard path)."""
        return self.lib.vphys_assemble(self._h)

    def vdiff_momentum(self, dt):
        _ffi.check(self.lib.vphys_vdiff_momentum(self._h, float(dt)), "vphys_vdiff_momentum")

    def vdiff_tracers(self, dt):
        """vdiff_apply_tracers (rdb_ocean_vdiff.F90:1107-1414): kt on
        temperature, ks on salinity and the other tracers, as the fields hold
        them (a ks set or bound by the caller is used as written)."""
        _ffi.check(self.lib.vphys_vdiff_tracers(self._h, float(dt)), "vphys_vdiff_tracers")

    def nonlocal_tendencies(self, dt):
        """vmix_apply_nonlocal_tendencies (rdb_ocean_vmix.F90:1605-1714) with the
        gamma of the last assemble(); h, bl_depth, b0 and the forcing must
        still hold what assemble() read."""
        _ffi.check(self.lib.vphys_nonlocal(self._h, float(dt)), "vphys_nonlocal")

    def vdiff_tracers_nonlocal(self, dt):
        """The fused tracer diffusion + non-local launch that step() runs."""
        _ffi.check(self.lib.vphys_vdiff_tracers_nonlocal(self._h, float(dt)), "vphys_vdiff_tracers_nonlocal")

    MOM_VARIANTS = ("registers", "tma_ring")
    TRACER_VARIANTS = ("smem_1_per_warp", "smem_2_per_warp", "smem_4_per_warp", "tmem_rows")

    def autotune(self, dt, reps=3):
        """vphys_autotune: time the kernel variants of the mixed solves on
        this handle's state, keep the fastest, leave the state unchanged.
        Returns {"momentum": {variant: ms}, "tracers": {variant: ms},
        "chosen": {"momentum": name, "tracers": name}} (ms only for the
        variants the configuration admits)."""
        import ctypes as C

        ms = (C.c_double * 6)()
        ch = (C.c_int * 2)()
        _ffi.check(self.lib.vphys_autotune(self._h, float(dt), int(reps), ms, 6, ch), "vphys_autotune")
        mom = {n: ms[i] for i, n in enumerate(self.MOM_VARIANTS) if ms[i] >= 0}
        tr = {n: ms[2 + i] for i, n in enumerate(self.TRACER_VARIANTS) if ms[2 + i] >= 0}
        return {"momentum": mom, "tracers": tr,
                "chosen": {"momentum": self.MOM_VARIANTS[ch[0]], "tracers": self.TRACER_VARIANTS[ch[1]]}}

    def set_variants(self, momentum, tracers):
        """Pin the mixed solves' kernel variants (names of MOM_VARIANTS /
        TRACER_VARIANTS)."""
        _ffi.check(self.lib.vphys_set_variants(self._h, self.MOM_VARIANTS.index(momentum),
                                               self.TRACER_VARIANTS.index(tracers)), "vphys_set_variants")

    def step(self, dt, n_steps=1):
        _ffi.check(self.lib.vphys_step(self._h, float(dt), int(n_steps)), "vphys_step")

    def step_graph(self, dt, n_steps=1):
        """vphys_step_graph: the n steps captured once as a CUDA graph and replayed."""
        _ffi.check(self.lib.vphys_step_graph(self._h, float(dt), int(n_steps)), "vphys_step_graph")

    def mixed_redo_count(self):
        """(32-column group, tracer) pairs of the last mixed tracer solve re-solved in FP64."""
        n = ctypes.c_uint(0)
        _ffi.check(self.lib.vphys_mixed_redo_count(self._h, ctypes.byref(n)), "vphys_mixed_redo_count")
        return int(n.value)

    def step_status(self, dt, n_steps=1):
        return self.lib.vphys_step(self._h, float(dt), int(n_steps))

    def synchronize(self):
        _ffi.check(self.lib.vphys_synchronize(self._h), "vphys_synchronize")
