"""ctypes loader for the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
arm use this module, as the checker; the product (roundabout_b200) never
imports it.  `OracleState` owns numpy arrays in the reference layout (Fortran
order, k = 0 the bed) and exposes the stage functions of vphys_oracle.c.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libvphys_oracle.so"

def _cflags() -> str:
    """The optimisation and floating-point flags the Makefile compiles with."""
    for line in (HERE / "Makefile").read_text().splitlines():
        if line.startswith("CFLAGS"):
            flags = line.split("=", 1)[1].split()
            return " ".join(f for f in flags if f.startswith(("-O", "-ffp", "-fno-fast", "-march")))
    return "unknown"


CFLAGS_DESC = _cflags()

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class VpoState(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("ntr", ctypes.c_int)] + [
        (n, _dp) for n in ("h", "rho", "u", "v", "kv", "kt", "ks", "kd_bg", "bl_depth", "b0", "stress_mag",
                          "q_heat", "q_salt", "wet", "tau_x", "tau_y", "lambda_bot_u", "lambda_bot_v",
                          "visc_rem_u", "visc_rem_v", "gamma_t", "gamma_s", "heat_budget", "salt_budget")
    ] + [(n, _ip) for n in ("k_top_u", "k_top_v", "k_bot_u", "k_bot_v")] + [("tr", ctypes.POINTER(_dp))] + [
        (n, _dp) for n in ("heat_budget_surface", "salt_budget_surface", "coriolis", "kd_shear", "tke_shear", "kd_epbl",
                          "mld_epbl", "la_epbl")] + [("epbl_tke", _dp * 6)] + [(n, _dp) for n in ("sw_net", "wet_dyn", "sw_chl", "sw_kappa", "cover_frac")]


def build(force: bool = False) -> Path:
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    srcs = [HERE / n for n in ("vphys_oracle.c", "vphys_oracle_kshear.c", "vphys_oracle_epbl.c", "vphys_oracle.h",
                               "Makefile")]
    srcs.append(HERE.parent / "include" / "vphys.h")
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < max(p.stat().st_mtime for p in srcs):
        env = dict(os.environ)
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True, env=env)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB_PATH))
        L.vpo_sm_cbrt.restype = ctypes.c_double
        L.vpo_sm_cbrt.argtypes = [ctypes.c_double]
        L.vpo_sm_atan.restype = ctypes.c_double
        L.vpo_sm_atan.argtypes = [ctypes.c_double]
        L.vpo_sm_exp.restype = ctypes.c_double
        L.vpo_sm_exp.argtypes = [ctypes.c_double]
        L.vpo_sm_log.restype = ctypes.c_double
        L.vpo_sm_log.argtypes = [ctypes.c_double]
        L.vpo_sm_erfc.restype = ctypes.c_double
        L.vpo_sm_erfc.argtypes = [ctypes.c_double]
        L.vpo_sm_pow.restype = ctypes.c_double
        L.vpo_sm_pow.argtypes = [ctypes.c_double, ctypes.c_double]
        L.vpo_set_threads.argtypes = [ctypes.c_int]
        L.vpo_get_threads.restype = ctypes.c_int
        for name in ("vpo_eos_wright", "vpo_pp81", "vpo_seed_interior_none", "vpo_kpp_overlay",
                     "vpo_kv_ml_invz2", "vpo_convection", "vpo_split", "vpo_kappa_shear_merge", "vpo_epbl_merge",
                     "vpo_sw_chl_kappa"):
            getattr(L, name).argtypes = [ctypes.c_void_p, ctypes.POINTER(VpoState)]
            getattr(L, name).restype = None
        L.vpo_stress_mag.argtypes = [ctypes.POINTER(VpoState)]
        L.vpo_column_content.argtypes = [ctypes.POINTER(VpoState), ctypes.c_int, _dp]
        for name in ("vpo_assemble_gate", "vpo_build_coefficients"):
            getattr(L, name).argtypes = [ctypes.c_void_p, ctypes.POINTER(VpoState)]
            getattr(L, name).restype = ctypes.c_int
        for name in ("vpo_vdiff_momentum", "vpo_vdiff_tracers", "vpo_nonlocal", "vpo_surface_flux",
                     "vpo_sw_penetration", "vpo_kappa_shear", "vpo_epbl"):
            getattr(L, name).argtypes = [ctypes.c_void_p, ctypes.POINTER(VpoState), ctypes.c_double]
            getattr(L, name).restype = None
        L.vpo_eos_buoyancy_coeffs.argtypes = [ctypes.c_double] * 3 + [ctypes.POINTER(ctypes.c_double)] * 2
        L.vpo_eos_buoyancy_coeffs.restype = None
        L.vpo_epbl_lf17.argtypes = [ctypes.c_double] * 3 + [ctypes.POINTER(ctypes.c_double)] * 2
        L.vpo_epbl_lf17.restype = None
        L.vpo_epbl_lt_enhance.argtypes = [ctypes.c_void_p] + [ctypes.c_double] * 6
        L.vpo_epbl_lt_enhance.restype = ctypes.c_double
        for name in ("vpo_massless_build_maps", "vpo_massless_merge_fields", "vpo_massless_interp_back"):
            getattr(L, name).restype = None
        L.vpo_step.argtypes = [ctypes.c_void_p, ctypes.POINTER(VpoState), ctypes.c_double, ctypes.c_int]
        L.vpo_step.restype = ctypes.c_int
        _lib = L
    return _lib


class OracleState:
    """Column-physics state in the reference layout (numpy, Fortran order).

    Array attributes mirror the vphys field names; tracers is a list of
    (nx, ny, nz) arrays.  Every array is owned here and handed to C by
    pointer, so the oracle updates them in place.
    """

    def __init__(self, nx: int, ny: int, nz: int, ntr: int):
        self.nx, self.ny, self.nz, self.ntr = nx, ny, nz, ntr
        f = lambda *s: np.zeros(s, dtype=np.float64, order="F")  # noqa: E731
        self.h = f(nx, ny, nz)
        self.rho = f(nx, ny, nz)
        self.u = f(nx + 1, ny, nz)
        self.v = f(nx, ny + 1, nz)
        self.kv = f(nx, ny, nz + 1)
        self.kt = f(nx, ny, nz + 1)
        self.ks = f(nx, ny, nz + 1)
        self.kd_bg = f(nx, ny, nz + 1)
        self.bl_depth = f(nx, ny)
        self.b0 = f(nx, ny)
        self.stress_mag = f(nx, ny)
        self.q_heat = f(nx, ny)
        self.q_salt = f(nx, ny)
        self.wet = np.ones((nx, ny), dtype=np.float64, order="F")
        self.tau_x = f(nx + 1, ny)
        self.tau_y = f(nx, ny + 1)
        self.lambda_bot_u = f(nx + 1, ny)
        self.lambda_bot_v = f(nx, ny + 1)
        self.visc_rem_u = f(nx + 1, ny, nz)
        self.visc_rem_v = f(nx, ny + 1, nz)
        self.gamma_t = f(nx, ny, nz + 1)
        self.gamma_s = f(nx, ny, nz + 1)
        self.heat_budget = f(nx, ny, nz)
        self.salt_budget = f(nx, ny, nz)
        self.heat_budget_surface = f(nx, ny, nz)
        self.salt_budget_surface = f(nx, ny, nz)
        self.coriolis = f(nx, ny)
        self.kd_shear = f(nx, ny, nz + 1)
        self.tke_shear = f(nx, ny, nz + 1)
        self.kd_epbl = f(nx, ny, nz + 1)
        self.mld_epbl = f(nx, ny)
        self.la_epbl = f(nx, ny)
        self.epbl_tke = [f(nx, ny) for _ in range(6)]   # wind, conv, forcing, mixing, mech_decay, conv_decay
        self.sw_net = f(nx, ny)
        self.wet_dyn = np.ones((nx, ny), dtype=np.float64, order="F")
        self.sw_chl = np.full((nx, ny), 1.0e-4, dtype=np.float64, order="F")
        self.sw_kappa = np.ones((nx, ny, 6), dtype=np.float64, order="F")
        self.cover_frac = f(nx, ny)
        self.k_top_u = np.full((nx + 1, ny), nz, dtype=np.int32, order="F")
        self.k_top_v = np.full((nx, ny + 1), nz, dtype=np.int32, order="F")
        self.k_bot_u = np.ones((nx + 1, ny), dtype=np.int32, order="F")
        self.k_bot_v = np.ones((nx, ny + 1), dtype=np.int32, order="F")
        self.tracers = [f(nx, ny, nz) for _ in range(ntr)]

    def seed_backgrounds(self, cfg):
        """vmix_seed_backgrounds (rdb_ocean_vmix.F90:843-913)."""
        self.kt[...] = cfg.pp81_kappa_bg
        self.ks[...] = cfg.pp81_kappa_bg
        self.kd_bg[...] = cfg.pp81_kappa_bg
        self.kv[...] = cfg.pp81_nu_bg
        for a in (self.kv, self.ks):
            a[:, :, 0] = 0.0
            a[:, :, -1] = 0.0

    def _struct(self) -> VpoState:
        for t in self.tracers:
            assert t.flags.f_contiguous
        s = VpoState()
        s.nx, s.ny, s.nz, s.ntr = self.nx, self.ny, self.nz, self.ntr
        for name, typ in VpoState._fields_[4:]:
            if typ is _dp or typ is _ip:
                a = getattr(self, name)
                assert a.flags.f_contiguous, name
                setattr(s, name, a.ctypes.data_as(typ))
        s.epbl_tke = (_dp * 6)(*[a.ctypes.data_as(_dp) for a in self.epbl_tke])
        self._trp = (_dp * max(1, self.ntr))(*[t.ctypes.data_as(_dp) for t in self.tracers])
        s.tr = ctypes.cast(self._trp, ctypes.POINTER(_dp))
        return s

    def call(self, name: str, cfg, *args):
        s = self._struct()
        fn = getattr(lib(), name)
        return fn(ctypes.byref(cfg), ctypes.byref(s), *args)

    def stress_mag_from_tau(self):
        s = self._struct()
        lib().vpo_stress_mag(ctypes.byref(s))

    def column_content(self, descending: bool) -> np.ndarray:
        """Compensated sum_k h c over each column's live span, per tracer:
        shape (nx, ny, ntr), Fortran order; the terms added top-down when
        `descending`."""
        out = np.zeros((self.nx, self.ny, max(1, self.ntr)), order="F")
        s = self._struct()
        lib().vpo_column_content(ctypes.byref(s), int(descending), out.ctypes.data_as(_dp))
        return out[:, :, : self.ntr]

    def copy(self) -> "OracleState":
        o = OracleState.__new__(OracleState)
        o.nx, o.ny, o.nz, o.ntr = self.nx, self.ny, self.nz, self.ntr
        for k, v in self.__dict__.items():
            if isinstance(v, np.ndarray):
                setattr(o, k, v.copy(order="F"))
        o.tracers = [t.copy(order="F") for t in self.tracers]
        o.epbl_tke = [t.copy(order="F") for t in self.epbl_tke]
        return o


def set_threads(n: int):
    lib().vpo_set_threads(int(n))


def sm_cbrt(x: float) -> float:
    return lib().vpo_sm_cbrt(float(x))


def sm_atan(x: float) -> float:
    return lib().vpo_sm_atan(float(x))


def sm_exp(x: float) -> float:
    return lib().vpo_sm_exp(float(x))


def sm_log(x: float) -> float:
    return lib().vpo_sm_log(float(x))


def sm_erfc(x: float) -> float:
    return lib().vpo_sm_erfc(float(x))


def sm_pow(x: float, y: float) -> float:
    return lib().vpo_sm_pow(float(x), float(y))


def eos_buoyancy_coeffs(T: float, S: float, p: float):
    """(alpha_T, beta_S) = (-d rho/dT, +d rho/dS) of the Wright EOS at (T, S, p)."""
    a, b = ctypes.c_double(), ctypes.c_double()
    lib().vpo_eos_buoyancy_coeffs(float(T), float(S), float(p), ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value
