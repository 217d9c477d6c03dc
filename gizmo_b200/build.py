"""Build the sm_100a C-ABI library gizmo_b200/lib/libgizmo_hydro.so with nvcc.

Each translation unit is compiled for sm_100a only. The FP64 pair kernels
(passes_fp64.cu) are compiled with -fmad=false so their products and sums
round like the reference's CPU build; the FP64 re-evaluation of the mixed
form's fragile force pairs (force_refine) lives there too. The FP32 pair
kernels of the mixed form (passes_mixed.cu) keep FMA and use the approximate
FP32 division and square root (a few ulp): the face, Riemann and limiter
arithmetic divides ~25 times per pair, and the IEEE-rounded FP32 sequences
cost several times the approximate ones. Those two flags touch FP32
operations only.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib", "libgizmo_hydro.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-ccbin", "g++"]
UNITS = {
    "grid.cu": [],
    "capi.cu": [],
    "passes_fp64.cu": ["-fmad=false"],
    "passes_mixed.cu": ["-prec-div=false", "-prec-sqrt=false"],
    "noalloc.cu": ["-fmad=false"],
    "kick.cu": ["-fmad=false"],
    "drift.cu": ["-fmad=false"],
    "timestep.cu": ["-fmad=false"],
}


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(HERE, "..", "include", "gizmo_hydro.h"))
    objs = []
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if not ptxas_info and not _newer(obj, [src] + headers + [__file__]):
            continue
        cmd = [NVCC] + ARCH + COMMON + extra + (["-Xptxas", "-v"] if ptxas_info else []) + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {unit}:\n{r.stderr}")
        if ptxas_info:
            sys.stderr.write(r.stderr)
    if _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static" if False else "-cudart=static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc link failed:\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
