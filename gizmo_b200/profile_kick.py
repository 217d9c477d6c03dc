"""Time the device half-step kick: python -m gizmo_b200.profile_kick --n 16777216 --method mfv

Fills every gz_kick_fields array of n particles in device memory (seeded,
MFV conserved-mass fields with dMass and DtMass of one sign so every cell
takes the mass update on every kick, all particles active, gravity on), runs
`--warmup` second half kicks, then times `--reps` more with CUDA events on
the stream the kernel is launched on, and prints one JSON line: the mean
duration of one kick, the algorithmic bytes one kick moves (each field read
or written once, counted from the arrays it touches) and the bandwidth that
makes. Above ~1M particles the working set exceeds the 126 MB L2, so each kick
streams from HBM without a flush between kicks.
"""
from __future__ import annotations

import argparse
import json
import os

from . import abi, ics
from .hydro import kick

# bytes per particle that one second half kick reads and writes, all active,
# MFV with dMass != 0 and no temperature floor reached
READ_FIELDS = {"mass": 8, "tstart": 8, "tend": 8, "mass_true": 8, "dmass": 8, "dtmass": 8, "active": 4, "grav": 24,
               "gravwork": 24, "u": 8, "dudt": 8, "accel": 24, "vel": 24, "dp": 24}
WRITE_FIELDS = {"mass_true": 8, "dmass": 8, "u": 8, "vel": 24, "vel_pred": 24, "mass": 8, "u_pred": 8, "dp": 24}
MFM_SKIPS = ("mass_true", "dmass", "dtmass", "gravwork")


def kick_bytes_per_particle(method: int) -> int:
    skip = MFM_SKIPS if method == abi.METHOD_MFM else ()
    rd = sum(v for k, v in READ_FIELDS.items() if k not in skip)
    wr = sum(v for k, v in WRITE_FIELDS.items() if k not in skip and not (k == "mass" and skip))
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
    n = args.n
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev)
    g.manual_seed(11)

    def f64(*shape, lo=0.5, hi=2.0):
        return torch.rand(*shape, generator=g, device=dev, dtype=torch.float64) * (hi - lo) + lo

    mass = f64(n)
    timebase = 2.0 ** -40
    f = {
        "vel": f64(n, 3, lo=-1, hi=1), "u": f64(n, lo=1, hi=10), "mass": mass, "mass_true": mass.clone(),
        "dmass": f64(n, lo=1e-6, hi=1e-5), "dtmass": f64(n, lo=1e-9, hi=1e-8), "accel": f64(n, 3, lo=-1, hi=1),
        "dudt": f64(n, lo=-1, hi=1), "grav": f64(n, 3, lo=-1, hi=1), "gravwork": f64(n, 3, lo=-1, hi=1),
        "vel_pred": torch.zeros(n, 3, dtype=torch.float64, device=dev),
        "u_pred": torch.zeros(n, dtype=torch.float64, device=dev),
        "dp": torch.zeros(n, 3, dtype=torch.float64, device=dev),
        "tstart": torch.zeros(n, dtype=torch.int64, device=dev),
        "tend": torch.randint(1 << 20, 1 << 21, (n,), generator=g, device=dev, dtype=torch.int64),
        "active": torch.ones(n, dtype=torch.int32, device=dev),
    }
    if method == abi.METHOD_MFM:
        for k in MFM_SKIPS:
            del f[k]
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        kick(params, f, 1, timebase, 0.0, stream.cuda_stream)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.reps):
        kick(params, f, 1, timebase, 0.0, stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.reps
    bpp = kick_bytes_per_particle(method)
    gbs = bpp * n / (ms * 1e-3) / 1e9
    peak = None
    peaks = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    if os.path.exists(peaks):
        peak = json.load(open(peaks)).get("hbm_gbs")
    print(json.dumps({"kernel": "k_kick", "method": args.method, "n": n, "reps": args.reps, "ms_per_kick": ms,
                      "bytes_per_particle": bpp, "achieved_gbs": gbs, "peak_gbs": peak,
                      "frac": (gbs / peak) if peak else None,
                      "particles_per_s": n / (ms * 1e-3)}))


if __name__ == "__main__":
    main()
