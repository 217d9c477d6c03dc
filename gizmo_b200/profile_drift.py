"""Time the device drift: python -m gizmo_b200.profile_drift --n 16777216 --method mfv

Fills every gz_drift_fields array of n cells in device memory (seeded, all
cells with mass, gravity on), then, in turn, `--warmup` and `--reps` drifts,
each moving every cell on by one step of 2^20 ticks (the target time grows by
one step per drift, so no drift is a no-op). The reps are timed with CUDA
events on the stream the kernel is launched on. Prints one JSON line: the mean
duration of one drift, the algorithmic bytes it moves (each field read or
written once, counted from the arrays it touches) and the bandwidth that
makes. The 3.7 GB working set is ~30x the L2, so every drift streams from
HBM without a flush.
"""
from __future__ import annotations

import argparse
import json
import os

from . import abi, ics
from .hydro import drift

# bytes per cell that one drift reads and writes, every cell drifted, with mass
READ_FIELDS = {"pos": 24, "move": 24, "vel_pred": 24, "grav": 24, "accel": 24, "divvel": 8, "mass": 8, "dtmass": 8,
               "mass_true": 8, "rho": 8, "u_pred": 8, "dudt": 8, "h": 8, "ti_current": 8}
WRITE_FIELDS = {"pos": 24, "vel_pred": 24, "mass": 8, "rho": 8, "u_pred": 8, "h": 8, "pressure": 8, "ti_current": 8}
MFV_ONLY_READS = ("dtmass", "mass_true")


def drift_bytes_per_cell(method: int) -> int:
    mfm = method == abi.METHOD_MFM
    rd = sum(v for k, v in READ_FIELDS.items() if not (mfm and k in MFV_ONLY_READS))
    wr = sum(v for k, v in WRITE_FIELDS.items() if not (mfm and k == "mass"))
    return rd + wr


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1 << 24)
    ap.add_argument("--method", choices=["mfm", "mfv"], default="mfv")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--reps", type=int, default=20)
    args = ap.parse_args()
    import torch

    method = abi.METHOD_MFV if args.method == "mfv" else abi.METHOD_MFM
    params = ics.sedov(4, seed=1).params
    params.method = method
    params.min_kernel_radius, params.max_kernel_radius = 1e-6, 1e6
    n = args.n
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev)
    g.manual_seed(12)

    def f64(*shape, lo=-1.0, hi=1.0):
        return torch.rand(*shape, generator=g, device=dev, dtype=torch.float64) * (hi - lo) + lo

    mass = f64(n, lo=0.5, hi=2.0)
    f = {
        "pos": f64(n, 3, lo=0, hi=1), "vel_pred": f64(n, 3), "grav": f64(n, 3), "accel": f64(n, 3),
        "divvel": f64(n), "mass": mass, "rho": f64(n, lo=0.5, hi=2.0), "u_pred": f64(n, lo=1, hi=10),
        "dudt": f64(n, lo=-1e-3, hi=1e-3), "h": f64(n, lo=0.01, hi=0.02),
        "pressure": torch.zeros(n, dtype=torch.float64, device=dev),
        "ti_current": torch.zeros(n, dtype=torch.int64, device=dev),
        "status": torch.zeros(1, dtype=torch.int32, device=dev),
    }
    if method == abi.METHOD_MFV:
        f.update({"pvel": f64(n, 3), "dtmass": f64(n, lo=-1e-3, hi=1e-3), "mass_true": mass.clone()})
    else:
        f["vel"] = f64(n, 3)
    timebase = 2.0 ** -40
    step = 1 << 20
    stream = torch.cuda.current_stream(dev)
    t = 0
    for _ in range(args.warmup):
        t += step
        drift(params, f, t, timebase, 0.0, stream.cuda_stream)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.reps):
        t += step
        drift(params, f, t, timebase, 0.0, stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    if int(f["status"].item()) != 0:
        raise RuntimeError(f"gz_drift status {int(f['status'].item())}")
    ms = e0.elapsed_time(e1) / args.reps
    bpc = drift_bytes_per_cell(method)
    gbs = bpc * n / (ms * 1e-3) / 1e9
    peak = None
    peaks = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    if os.path.exists(peaks):
        peak = json.load(open(peaks)).get("hbm_gbs")
    print(json.dumps({"kernel": "k_drift", "method": args.method, "n": n, "reps": args.reps, "ms_per_drift": ms,
                      "bytes_per_cell": bpc, "achieved_gbs": gbs, "peak_gbs": peak,
                      "frac": (gbs / peak) if peak else None, "cells_per_s": n / (ms * 1e-3)}))


if __name__ == "__main__":
    main()
