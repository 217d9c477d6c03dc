"""One hydro pass to profile: python -m gizmo_b200.profile_case --n1 64 --form mixed

Builds the Plummer-mixture particle set (n1^3 particles), converges the kernel
lengths once in FP64 from the cold seed, seeds the steady state (converged h x
(1 + U(-0.05, 0.05))), and then runs one restage + density + gradients + force
pass of the chosen form inside the NVTX range "steady_pass". A profiler
restricted to that range (ncu --nvtx --nvtx-include "steady_pass/") sees the
kernels of a timed bench step and none of the set-up.
"""
from __future__ import annotations

import argparse

import numpy as np

from . import abi, ics
from .hydro import HydroPass


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n1", type=int, default=64)
    ap.add_argument("--form", choices=["mixed", "fp64"], default="mixed")
    args = ap.parse_args()
    import torch

    wl = ics.plummer_mix(args.n1, seed=4)
    n = wl.n
    with HydroPass(wl.params) as hp:
        hp.upload_workload(wl)
        chunk = 1 << 21
        for a in range(0, n, chunk):
            hp.density(np.arange(a, min(n, a + chunk), dtype=np.int32) if n > chunk else None)
        conv = hp.download(["h", "cond"])
    wl.h = ics.steady_state_seed(conv["h"], 4)
    wl.cond = conv["cond"]
    wl.params.precision = abi.PRECISION_MIXED if args.form == "mixed" else abi.PRECISION_FP64
    with HydroPass(wl.params) as hp:
        hp.upload_workload(wl)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("steady_pass")
        hp.restage()
        hp.full_pass()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        st = hp.status()
    print(f"ok: {n} particles, {st['pairs_symmetric']} symmetric row entries, "
          f"{st['density_iterations']} density iterations")


if __name__ == "__main__":
    main()
