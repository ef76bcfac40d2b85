"""Build libvphys.so in-tree for sm_100a (nvcc, no JIT).

    python -m roundabout_b200.build [--verbose]

The exact kernels are compiled with -fmad=false: no a*b+c contraction, so
every column's FP64 result is bit-identical to the CPU restatement of the
reference (which its CPU builds compile with -ffp-contract=off).  The
mixed-precision solves (vphys_mixed.cu) have no bitwise contract and keep
FMA contraction.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

CSRC = Path(__file__).resolve().parent / "csrc"
OUT = CSRC / "_build"
LIB = OUT / "libvphys.so"
SOURCES = ["vphys_api.cu", "vphys_kernels.cu", "vphys_momentum_tma.cu", "vphys_tracers.cu", "vphys_static.cu",
           "vphys_mixed.cu",
           "vphys_gemm.cu", "vphys_learned.cu", "vphys_kshear.cu",
           "vphys_epbl.cu"]
HEADERS = ["vphys_device.cuh", "vphys_faces.cuh", "vphys_kernels.cuh", "vphys_tma.cuh", "vphys_tiles.cuh", "vphys_mom_ring.cuh", "vphys_tmem.cuh",
           "../../include/vphys.h"]
# the mixed-precision solves carry no bitwise contract: FMA contraction allowed
CONTRACT_OK = {"vphys_mixed.cu", "vphys_gemm.cu", "vphys_learned.cu"}

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise FileNotFoundError("nvcc not found")


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any((CSRC / s).stat().st_mtime > t for s in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not stale():
        return LIB
    OUT.mkdir(parents=True, exist_ok=True)
    objs = []
    for s in SOURCES:
        obj = OUT / (Path(s).stem + ".o")
        fmad = "-fmad=true" if s in CONTRACT_OK else "-fmad=false"
        cmd = [nvcc(), *ARCH, *FLAGS, fmad, "-c", str(CSRC / s), "-o", str(obj)]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {s}:\n{r.stderr}")
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(str(obj))
    tmp = OUT / (LIB.name + ".tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose="--verbose" in sys.argv))
