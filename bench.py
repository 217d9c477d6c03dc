"""Benchmark of the meshless hydro pass: particle-updates/s, mixed vs FP64 form.

Workload (default): 256^3 = 16,777,216 gas particles, 90% in 1000 Plummer
spheres + 10% uniform background (seeded synthetic stand-in for the named
configuration), MFV with HLLC, cubic kernel, 32 neighbours, gamma 5/3.
One step = one particle-update of every particle: neighbour grid rebuilt from
the resident inputs, density with kernel-length iteration from the
steady-state seed (converged h x (1 + U(-0.05, 0.05))), gradients, force.

Arms:
  (default)          the sm_100a library through its C ABI, device-resident
                     inputs (`value`), plus the end-to-end rate with pinned host
                     buffers copied in and results copied out every step (`e2e`).
  --impl reference   the reference's own pair bodies (oracle/_ref, compiled from
                     its sources) on the host cores; replicas only for N > 1
                     (rank 0 runs, the others exit).

Multi-GPU: replicas only (one independent particle set per GPU; the pass has
no exchange on one box), weak scaling, timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "hydro particle-updates/s @256^3: mixed-prec vs FP64 GPU at <=1e-5 rel err"
UNIT = "particle-updates/s"

# per-pair FLOP constants (FMA = 2, sqrt/div/exp/log = 1 each), counted by hand
# over the taken MFV ideal-gas branch of the pair bodies (HLLC solved on the
# first try). Density, per accepted pair: separation 8, sqrt 1, u 1, cubic
# kernel and derivative 10, the 17 sums 52 -> 72. Gradient ~60, force ~430.
FLOPS_PER_PAIR = {"density": 72.0, "gradients": 60.0, "force": 430.0}

# DRAM bytes per work unit of a kernel from one ncu capture of the 64^3 case
# (dram__bytes_read.sum + dram__bytes_write.sum over the units of the captured
# launch), scaled to the units of a launch here: density sums per row
# (profiles/density_sums_plummer64.md: 140.1 MB over 262,144 rows), the force
# pair kernel per pair (profiles/force_pairs_plummer64.md: 1313.8 MB over
# 7,841,073 pairs).
DRAM_BYTES_PER_UNIT = {"density_sums": 140.1e6 / 262144, "force": 1313.8e6 / 7841073}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plummer_mix", choices=["plummer_mix", "sedov", "lognormal"])
    ap.add_argument("--n1", type=int, default=None, help="particles per axis (default: 256 plummer_mix)")
    ap.add_argument("--cpu-n1", type=int, default=64, help="size of the CPU-baseline instance")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cold", action="store_true")
    # profiling and kernel timing (no bench line)
    ap.add_argument("--profile-pass", action="store_true",
                    help="one steady-state pass inside the NVTX range 'steady_pass', timing nothing (for ncu)")
    ap.add_argument("--form", choices=["mixed", "fp64"], default="mixed", help="arithmetic form of --profile-pass")
    ap.add_argument("--kernel", choices=["kick", "drift"], default=None,
                    help="time the device half-step kick or drift alone and print one JSON line")
    ap.add_argument("--n", type=int, default=1 << 24, help="particles of --kernel")
    ap.add_argument("--method", choices=["mfm", "mfv"], default="mfv", help="hydro method of --kernel")
    ap.add_argument("--reps", type=int, default=20, help="timed launches of --kernel")
    ap.add_argument("--subsets", action="store_true",
                    help="individual-timestep active subsets of 8,388,608 particles (log-normal, sigma 2.0): "
                         "one JSON line of rates per active fraction, the grid reused across substeps")
    ap.add_argument("--boxes", action="store_true",
                    help="512 independent boxes of 1,024-65,536 particles (shock tubes and Sedov blasts): "
                         "one JSON line of rates, mixed and FP64")
    return ap.parse_args()


def make_workload(name: str, n1: int, precision: int):
    from gizmo_b200 import ics

    if name == "plummer_mix":
        return ics.plummer_mix(n1, seed=4, precision=precision)
    if name == "sedov":
        return ics.sedov(n1, seed=1, precision=precision)
    return ics.lognormal(n1, seed_density=2, seed_velocity=3, precision=precision)


def default_n1(name: str) -> int:
    return {"plummer_mix": 256, "sedov": 32, "lognormal": 128}[name]


def workload_desc(name: str, n1: int) -> str:
    n = n1 ** 3
    return {
        "plummer_mix": f"{n1}^3={n:,} particles: 90% in 1000 Plummer spheres + 10% background, MFV+HLLC, cubic, 32 ngb",
        "sedov": f"{n1}^3={n:,} particles: Sedov lattice+jitter, MFM, cubic, 32 ngb",
        "lognormal": f"{n1}^3={n:,} particles: log-normal field sigma_lnrho=1.5, MFM, Wendland C2, 64 ngb",
    }[name]


# --------------------------------------------------------------- distributed
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if (args.impl == "ours" and torch.cuda.is_available()) else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def dist_max(x: float, world: int, impl: str) -> float:
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if (impl == "ours" and torch.cuda.is_available()) else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def dist_done(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    def __init__(self, device: int):
        self.path = tempfile.mktemp(prefix="gz_clocks_", suffix=".csv")
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--id={device}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------- CPU baseline
def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(n1: int, name: str, kind_pref: str = "reference", steps: int = 1):
    """Full CPU pass (density -> gradients -> force) of a smaller instance of the
    same generator on all host threads; returns (rate, seconds, kind, cores, n)."""
    from oracle import oracle as O

    wl = make_workload(name, n1, 0)
    kind = kind_pref if (kind_pref == "port" or O.ref_available(wl.params)) else "port"
    cores = os.cpu_count() or 1
    orc = O.Oracle(wl.params, kind, n_threads=cores)
    times = []
    for _ in range(steps):
        st = O.new_state(wl.n, wl.inputs())
        t, status = orc.full_pass_seconds(st)
        if status:
            raise RuntimeError(f"CPU pass failed: {status}")
        times.append(t)
    t = float(np.mean(times))
    return wl.n / t, t, kind, cores, wl.n


# ------------------------------------------------------------------ GPU arm
def vector_peaks(torch, n: int = 8192, reps: int = 5) -> dict:
    """Measured non-tensor FP64 and FP32 rates on this GPU, for the roofline of
    the pair kernels (MEASURED_PEAKS.json holds bf16 tensor and HBM figures
    only): cuBLAS DGEMM and SGEMM (TF32 off) at n^3, best of `reps` timed with
    CUDA events, 2 n^3 flop each."""
    out = {}
    tf32 = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for dtype, tag in ((torch.float64, "fp64"), (torch.float32, "fp32")):
            a = torch.randn(n, n, device="cuda", dtype=dtype)
            b = torch.randn(n, n, device="cuda", dtype=dtype)
            torch.matmul(a, b)
            best = None
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                torch.matmul(a, b)
                e1.record()
                torch.cuda.synchronize()
                t = e0.elapsed_time(e1) / 1e3
                best = t if best is None else min(best, t)
            out[tag] = 2.0 * n ** 3 / best / 1e12
            del a, b
    finally:
        torch.backends.cuda.matmul.allow_tf32 = tf32
        torch.cuda.empty_cache()
    return out


def run_ours(args, world, rank, local):
    import torch

    from gizmo_b200 import abi, accuracy, ics
    from gizmo_b200.hydro import HydroPass

    torch.cuda.set_device(local)
    measured = vector_peaks(torch)
    n1 = args.n1 or default_n1(args.workload)
    t_gen = time.time()
    wl = make_workload(args.workload, n1, abi.PRECISION_FP64)
    N = wl.n
    t_gen = time.time() - t_gen
    h_cold = wl.h.copy()  # the generator's seed: octree density estimate
    # steady-state seed: converge once in FP64 from the cold seed
    hp64 = HydroPass(wl.params, device=local)
    hp64.upload_workload(wl)
    # in slices of the particle set: a one-way density row depends on its own
    # target's h only, so slicing changes no result and bounds the rows a
    # cold seed can ask for
    chunk = 1 << 21
    for a in range(0, N, chunk):
        hp64.density(np.arange(a, min(N, a + chunk), dtype=np.int32) if N > chunk else None)
    conv = hp64.download(["h", "cond"])
    wl.h = ics.steady_state_seed(conv["h"], 4)
    wl.cond = conv["cond"]
    hp64.upload_workload(wl)
    from gizmo_b200.ics import make_params

    p = wl.params
    pmix = make_params(p.kernel, p.method, p.gamma, p.des_num_ngb, p.max_num_ngb_dev, abi.PRECISION_MIXED,
                       p.box_size, p.first_step, p.selfgravity_off, p.min_kernel_radius, p.max_kernel_radius)
    hpm = HydroPass(pmix, device=local)
    hpm.upload_workload(wl)

    def run_steps(hp, K, W, record_clock=False, graph=True, timing=False):
        """K timed steps of restage + pass after W untimed ones. graph: the
        restage and the pass as one CUDA graph (gz_hydro_pass with
        GZ_PASS_GRAPH | GZ_PASS_RESTAGE), events around it; otherwise restage
        and the three plain calls with events between them (and, with timing,
        the library's per-kernel timers)."""
        stream = torch.cuda.ExternalStream(hp.stream)
        for _ in range(W):
            if graph:
                hp.hydro_pass(graph=True, restage=True)
            else:
                hp.restage()
                hp.full_pass()
        torch.cuda.synchronize()
        dist_barrier(world)
        torch.cuda.synchronize()
        sampler = ClockSampler(local) if record_clock else None
        if timing:
            hp.kernel_timing(True)
        l0 = hp.status()["kernel_launches"]
        names = ["step"] if graph else ["grid", "density", "gradients", "force"]
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(len(names) + 1)] for _ in range(K)]
        for k in range(K):
            ev[k][0].record(stream)
            if graph:  # the restage and the pass in one graph
                hp.hydro_pass(graph=True, restage=True)
                ev[k][1].record(stream)
            else:
                hp.restage()
                ev[k][1].record(stream)
                hp.density()
                ev[k][2].record(stream)
                hp.hydro_gradient_calc()
                ev[k][3].record(stream)
                hp.hydro_force()
                ev[k][4].record(stream)
        torch.cuda.synchronize()
        dist_barrier(world)
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        launches = hp.status()["kernel_launches"] - l0
        ktimes = None
        if timing:
            ktimes = hp.kernel_times()
            hp.kernel_timing(False)
        total = ev[0][0].elapsed_time(ev[K - 1][len(names)]) / 1e3
        parts = {nm: float(np.mean([ev[k][i].elapsed_time(ev[k][i + 1]) for k in range(K)])) / 1e3
                 for i, nm in enumerate(names)}
        return total, parts, clocks, launches, ktimes

    K, W = args.steps, args.warmup
    # the headline: each step a restage (grid build) and the pass as one CUDA graph
    t_mix, graph_mix, clocks, launches, _ = run_steps(hpm, K, W, record_clock=True)
    st_mix = hpm.status()
    gstats = hpm.graph_stats()
    K64 = max(1, min(K, 3))
    t_64, graph_64, _, _, _ = run_steps(hp64, K64, max(1, min(W, 2)))
    t_mix = dist_max(t_mix, world, "ours")
    t_64 = dist_max(t_64, world, "ours")
    value = world * N * K / t_mix
    value64 = world * N * K64 / t_64
    # stage breakdown and per-kernel timers: plain passes (the graph has no
    # events inside), a few steps of each form
    _, parts_mix, _, _, ktimes = run_steps(hpm, K64, 1, graph=False, timing=True)
    _, parts_64, _, _, _ = run_steps(hp64, K64, 1, graph=False)

    # Accuracy of the mixed form against the FP64 form (same inputs), per
    # particle and field (gizmo_b200/accuracy.py): h, rho, pressure, vsig
    # against |x|; gradients against |g| floored at 1e-6 max |g|; the rates
    # dtmass, accel, dudt against the pair-flux scale of the particle's force
    # row (the bar's denominator) and, reported beside it, against |x| floored
    # at 1e-6 max |x|. The flux scales come from one more FP64 pass with the
    # flux_abs diagnostic on (off in the timed passes; the outputs are the same).
    fields = list(accuracy.FIELDS)
    om = hpm.download(fields + ["iters"])
    refined = hpm.status()["pairs_refined"]
    hp64.set_diagnostics(flux_abs=True)
    hp64.restage()
    hp64.full_pass()
    o64 = hp64.download(fields + ["iters", "flux_abs"])
    mfv = p.method == abi.METHOD_MFV
    scales = accuracy.flux_scales(wl.vel, wl.mass, wl.u, o64["flux_abs"], mfv,
                                  accuracy.sound_speed(p.gamma, o64["pressure"], o64["rho"]))
    err = accuracy.per_particle(om, o64, scales)
    acc = accuracy.summary(err, 1e-5)
    acc["iters_equal_frac"] = float(np.mean(om["iters"] == o64["iters"]))
    acc["particles"] = N
    acc["pairs_refined_fp64"] = int(refined)
    # conservation per pass (both forms)
    cons = {}
    for tag, o in (("mixed", om), ("fp64", o64)):
        m, v = wl.mass, wl.vel
        dtm = o["dtmass"] if p.method == abi.METHOD_MFV else np.zeros(N)
        mom = m[:, None] * o["accel"] + v * dtm[:, None]
        cons[tag] = {"momentum": float(np.abs(mom.sum(0)).max() / np.abs(mom).sum()),
                     "mass": float(abs(dtm.sum()) / (np.abs(dtm).sum() + 1e-300))}

    # Accepted pairs per density row: the one-way rows (r < h at the converged
    # h, the target itself included, as the density sums count it) of a random
    # sample of targets. The density sums' algorithmic work is this count x 72
    # flop per row summed; the candidates the row radius adds are not work.
    sample = np.sort(np.random.default_rng(17).choice(N, min(N, 1 << 16), replace=False)).astype(np.int32)
    off_s, _ = hpm.neighbors(0, sample)
    accepted_per_row = float(off_s[-1]) / len(sample)

    # Cold seed: one mixed-form pass from the generator's h seed (octree density
    # estimate, h0 = (3 DesNumNgb / (4 pi n_local))^(1/3)), timed once after the
    # steady-state runs. Its density runs in slices of 2,097,152 particles (a
    # one-way row depends on its own target's h only, so slicing changes no
    # result and bounds the rows a cold seed can ask for); gradients and force
    # then build their symmetric rows with a tree walk.
    cold = None
    if not args.skip_cold:
        h_steady = wl.h
        wl.h = h_cold
        hpm.upload_workload(wl)
        stream = torch.cuda.ExternalStream(hpm.stream)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        iters = 0
        chunk = 1 << 21
        for a in range(0, N, chunk):
            hpm.density(np.arange(a, min(N, a + chunk), dtype=np.int32) if N > chunk else None)
            iters = max(iters, hpm.status()["density_iterations"])
        ev[1].record(stream)
        hpm.hydro_gradient_calc()
        hpm.hydro_force()
        ev[2].record(stream)
        torch.cuda.synchronize()
        t_cold = ev[0].elapsed_time(ev[2]) / 1e3
        cold = {"value": N / t_cold, "unit": UNIT, "ms_per_pass": 1e3 * t_cold,
                "density_ms": ev[0].elapsed_time(ev[1]), "density_iterations_max": iters,
                "seed": "octree density estimate (3 DesNumNgb / (4 pi n_local))^(1/3)",
                "note": "mixed form; density in slices of 2,097,152 particles; one pass, after the steady-state runs"}
        wl.h = h_steady  # the end-to-end steps below start from the steady-state seed again

    # Roofline of each timed kernel family (CUDA events around its launches on
    # the context's stream, over the timed steps of the mixed form): algorithmic
    # FLOPs / kernel time against the rate of the pipe its arithmetic runs on,
    # measured here as cuBLAS DGEMM / SGEMM (MEASURED_PEAKS.json holds no
    # FP32/FP64 vector figure). None of these kernels is a contraction (no
    # tensor cores) or DRAM-bound (the gathers hit L1/L2: see `traffic`).
    pairs_sym = st_mix["pairs_symmetric"]
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    sm_mhz = float(peaks.get("sm_max_mhz", 1965.0))
    nominal = {"fp32": 148 * 128 * 2 * sm_mhz * 1e6 / 1e12, "fp64": 148 * 64 * 2 * sm_mhz * 1e6 / 1e12}
    fp32_peak = measured.get("fp32") or nominal["fp32"]
    fp64_peak = measured.get("fp64") or nominal["fp64"]
    kernels = {}
    for name, d in (ktimes or {}).items():
        if d["launches"] == 0 or d["ms"] <= 0:
            continue
        e = {"launches_per_step": d["launches"] / K64, "ms_per_step": d["ms"] / K64,
             "ms_per_launch": d["ms"] / d["launches"], "units_per_launch": d["units"] / d["launches"]}
        flops = None
        if name == "density_sums":  # FP64, accepted pairs only
            flops, peak, pipe = FLOPS_PER_PAIR["density"] * accepted_per_row * d["units"], fp64_peak, "fp64"
            e["work"] = (f"{FLOPS_PER_PAIR['density']:.0f} flop x {accepted_per_row:.2f} accepted pairs per row "
                         f"(one-way rows at the converged h of {len(sample)} random targets, self included)")
        elif name == "force":  # FP32 pair arithmetic, each pair evaluated once
            flops, peak, pipe = FLOPS_PER_PAIR["force"] * d["units"], fp32_peak, "fp32"
            e["work"] = f"{FLOPS_PER_PAIR['force']:.0f} flop per pair evaluation"
        elif name == "gradients":  # FP64 pair arithmetic (both forms) over every row entry
            flops, peak, pipe = FLOPS_PER_PAIR["gradients"] * pairs_sym * d["launches"], fp64_peak, "fp64"
            e["work"] = f"{FLOPS_PER_PAIR['gradients']:.0f} flop per row entry"
        if flops is not None:
            ach = flops / (d["ms"] / 1e3) / 1e12
            e.update({"achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak, "pipe": pipe})
        if name in DRAM_BYTES_PER_UNIT:
            e["traffic_bytes_per_launch"] = DRAM_BYTES_PER_UNIT[name] * e["units_per_launch"]
        kernels[name] = e
    dom = max((k for k in kernels if "achieved" in kernels[k]), key=lambda k: kernels[k]["ms_per_step"], default=None)
    kernel_names = {"density_sums": "k_density_sums<double> (FP64 density sums, all h iterations)",
                    "force": "k_force_pairs<float> (MFV pair flux, each pair once)",
                    "gradients": "k_gradients<double> (least-squares gradients, FP64 in both forms)"}
    roofline = None
    if dom:
        d = kernels[dom]
        roofline = {"kernel": kernel_names[dom], "bound": d["pipe"], "achieved": d["achieved"], "peak": d["peak"],
                    "unit": "TFLOP/s", "frac": d["frac"], "work": d["work"],
                    "ms_per_launch": d["ms_per_launch"], "launches_per_step": d["launches_per_step"],
                    "peak_source": (f"measured: cuBLAS {'DGEMM' if d['pipe'] == 'fp64' else 'SGEMM (TF32 off)'} "
                                    "8192^3 on this GPU, best of 5 (MEASURED_PEAKS.json holds no FP32/FP64 vector "
                                    "figure; the pair kernels use no tensor cores)"
                                    if measured.get(d["pipe"]) else "nominal pipe rate (no measurement)"),
                    "peak_nominal": nominal[d["pipe"]],
                    "peaks_measured": measured,
                    "traffic": d.get("traffic_bytes_per_launch"),
                    "traffic_source": "ncu DRAM bytes per unit of the 64^3 capture, scaled to this launch's units"}
    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": 1e3 * t_mix / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 pair / f64 accumulate", "data": "synthetic (seeded generator, no dataset)",
        "config": {"workload": workload_desc(args.workload, n1), "n_particles": N, "precision": "mixed",
                   "h_seed": "steady-state: FP64-converged h x (1+U(-0.05,0.05)), seed 104",
                   "l2": f"inputs larger than L2 (device state {st_mix['device_bytes'] / 1e9:.1f} GB)",
                   "parallelism": f"replicas x{world}", "generate_s": round(t_gen, 1)},
        "fp64_value": value64, "mixed_over_fp64": value / value64,
        "accuracy_mixed_vs_fp64": {
            "bar": 1e-5, "particles_above_bar_any_field": acc["particles_above_bar_any_field"],
            "max_over_fields": acc["max_over_fields"], "pairs_refined_fp64": acc["pairs_refined_fp64"],
            "max": {f: acc[f]["max"] for f in accuracy.FIELDS},
            "rates_vs_value_max": {f: acc[f + ":value"]["max"] for f in accuracy.RATE_FIELDS},
            "denominators": "|x| (h, rho, pressure, vsig); |g| floored at 1e-6 max (gradients); the row's pair-flux "
                            "scale (rates; gizmo_b200/accuracy.py), and |x| floored at 1e-6 max beside it"},
        "gpu_launches": launches, "clocks": clocks, "roofline": roofline,
        "pass_ms": {form: {k: round(1e3 * v, 2) for k, v in parts.items()}
                    for form, parts in (("mixed", parts_mix), ("fp64", parts_64))},
        "graph": {"steps_ms": {form: {k: round(1e3 * v, 2) for k, v in parts.items()}
                               for form, parts in (("mixed", graph_mix), ("fp64", graph_64))},
                  "captures": gstats["captures"], "replays": gstats["replays"], "fallbacks": gstats["fallbacks"],
                  "kernels_per_replay": gstats["kernels_top"] + gstats["kernels_after"]
                  + gstats["kernels_per_iteration"] * st_mix["density_iterations"],
                  "what": "value and fp64_value: gz_hydro_pass(GZ_PASS_GRAPH | GZ_PASS_RESTAGE) per step (the "
                          "restage and the pass in one graph); pass_ms and the kernel rooflines: plain calls with "
                          "events between the stages"},
        "conservation": cons, "density_iterations": st_mix["density_iterations"], "pairs_symmetric": pairs_sym,
    }
    # the long tables go to stderr (the one stdout line stays short)
    details = {"accuracy_mixed_vs_fp64": acc, "kernels": kernels, "cold_seed": cold}

    # end to end: pinned host buffers in, results out, every step. The copies
    # are pipelined: step k+1's inputs go up (gz_upload_async) while step k's
    # pass runs, and step k's results come down (gz_download_async) while step
    # k+1's runs; the timed region holds every step's copies, from the first
    # upload to gz_wait after the last download.
    if not args.skip_e2e:
        pin = {k: torch.from_numpy(np.ascontiguousarray(v, dtype=np.float64)).pin_memory()
               for k, v in wl.inputs().items()}
        outs = {"h": (N,), "rho": (N,), "accel": (N, 3), "dudt": (N,), "vsig": (N,), "dtmass": (N,), "dmass": (N,)}
        pout = {k: torch.empty(s, dtype=torch.float64, pin_memory=True) for k, s in outs.items()}
        stream = torch.cuda.ExternalStream(hpm.stream)
        pin_p = {k: t.data_ptr() for k, t in pin.items()}
        pout_p = {k: t.data_ptr() for k, t in pout.items()}

        def pipelined(steps):
            # the restage stays a call of its own here: it returns with its work
            # queued, so the next step's upload is issued before this pass runs
            hpm.upload_raw_async(N, pin_p)
            for k in range(steps):
                hpm.restage()  # takes step k's inputs
                if k + 1 < steps:
                    hpm.upload_raw_async(N, pin_p)
                hpm.hydro_pass(graph=True)
                hpm.download_raw_async(pout_p)
            hpm.wait()

        pipelined(max(2, min(W, 3)))
        torch.cuda.synchronize()
        dist_barrier(world)
        Ke = max(2, min(K, 5))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        pipelined(Ke)
        e1.record(stream)
        torch.cuda.synchronize()
        te = dist_max(e0.elapsed_time(e1) / 1e3, world, "ours")
        h2d = sum(t.numel() * 8 for t in pin.values())
        d2h = sum(t.numel() * 8 for t in pout.values())
        result["e2e"] = {"value": world * N * Ke / te, "unit": UNIT, "h2d_bytes_per_step": h2d,
                         "d2h_bytes_per_step": d2h, "steps": Ke,
                         "how": "gz_upload_async / gz_restage / gz_hydro_pass(GZ_PASS_GRAPH) / gz_download_async per "
                                "step from pinned host buffers, the next step's upload and the last step's download "
                                "beside the pass; gz_wait after the last"}
    hpm.close()
    hp64.close()

    if rank == 0 and world == 1 and not args.skip_cpu:  # the CPU baseline: one GPU's run only
        rate, secs, kind, cores, ncpu = cpu_baseline(args.cpu_n1, args.workload)
        result["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": kind, "cpu_model": cpu_model(),
                                  "sample": f"one full density->gradients->force pass of a {args.cpu_n1}^3 "
                                            f"({ncpu:,}-particle) instance of the same generator, {secs:.2f} s"}
    if rank == 0:
        print(json.dumps(details), file=sys.stderr, flush=True)
    return result


def run_reference(args, world, rank):
    if rank != 0:
        return None
    n1 = args.cpu_n1
    for _ in range(args.warmup):
        cpu_baseline(n1, args.workload, "reference", 1)
    t0 = time.time()
    rate, secs, kind, cores, ncpu = cpu_baseline(n1, args.workload, "reference", args.steps)
    wall = time.time() - t0
    sample = f"{args.steps} full passes of a {n1}^3 ({ncpu:,}-particle) instance of the same generator"
    return {
        "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * secs, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded generator, no dataset)", "impl": "reference",
        "config": {"workload": workload_desc(args.workload, args.n1 or default_n1(args.workload)),
                   "sample": workload_desc(args.workload, n1), "n_particles_per_sample": ncpu, "precision": "fp64",
                   "parallelism": f"{cores} host threads", "wall_s": round(wall, 1)},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": kind, "cpu_model": cpu_model(),
                         "sample": sample},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# ------------------------------------------------- profiling and kernel timing
def profile_pass(args):
    """One steady-state pass to profile: the workload's particle set, kernel
    lengths converged once in FP64 from the cold seed, the steady-state seed
    (converged h x (1 + U(-0.05, 0.05))), then one restage + density +
    gradients + force pass of ``--form`` inside the NVTX range "steady_pass". A
    profiler restricted to that range (ncu --nvtx --nvtx-include "steady_pass/")
    sees the kernels of a timed bench step and none of the set-up."""
    import torch

    from gizmo_b200 import abi, ics
    from gizmo_b200.hydro import HydroPass

    n1 = args.n1 or default_n1(args.workload)
    wl = make_workload(args.workload, n1, abi.PRECISION_FP64)
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


# bytes per particle one second half kick reads and writes (all active, MFV with
# dMass != 0, no temperature floor reached), and one drift (every cell drifted)
KICK_READ = {"mass": 8, "tstart": 8, "tend": 8, "mass_true": 8, "dmass": 8, "dtmass": 8, "active": 4, "grav": 24,
             "gravwork": 24, "u": 8, "dudt": 8, "accel": 24, "vel": 24, "dp": 24}
KICK_WRITE = {"mass_true": 8, "dmass": 8, "u": 8, "vel": 24, "vel_pred": 24, "mass": 8, "u_pred": 8, "dp": 24}
KICK_MFM_SKIPS = ("mass_true", "dmass", "dtmass", "gravwork")
DRIFT_READ = {"pos": 24, "move": 24, "vel_pred": 24, "grav": 24, "accel": 24, "divvel": 8, "mass": 8, "dtmass": 8,
              "mass_true": 8, "rho": 8, "u_pred": 8, "dudt": 8, "h": 8, "ti_current": 8}
DRIFT_WRITE = {"pos": 24, "vel_pred": 24, "mass": 8, "rho": 8, "u_pred": 8, "h": 8, "pressure": 8, "ti_current": 8}
DRIFT_MFV_ONLY = ("dtmass", "mass_true")


def kernel_bytes_per_particle(kernel: str, mfv: bool) -> int:
    if kernel == "kick":
        skip = () if mfv else KICK_MFM_SKIPS
        return (sum(v for k, v in KICK_READ.items() if k not in skip) +
                sum(v for k, v in KICK_WRITE.items() if k not in skip and not (k == "mass" and skip)))
    return (sum(v for k, v in DRIFT_READ.items() if mfv or k not in DRIFT_MFV_ONLY) +
            sum(v for k, v in DRIFT_WRITE.items() if mfv or k != "mass"))


def time_step_kernel(args):
    """Times ``--reps`` launches of the device kick (second half kicks) or drift
    (each one step of 2^20 ticks further, so none is a no-op) over ``--n``
    seeded particles in device memory, all active, gravity on, with CUDA events
    on the launching stream; prints one JSON line with the mean duration, the
    algorithmic bytes (each field read or written once) and the bandwidth.
    Above ~1M particles the working set exceeds the 126 MB L2, so every launch
    streams from HBM without a flush."""
    import torch

    from gizmo_b200 import abi, ics
    from gizmo_b200.hydro import drift, kick

    mfv = args.method == "mfv"
    params = ics.sedov(4, seed=1).params
    params.method = abi.METHOD_MFV if mfv else abi.METHOD_MFM
    n = args.n
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev)
    g.manual_seed(11 if args.kernel == "kick" else 12)

    def f64(*shape, lo=-1.0, hi=1.0):
        return torch.rand(*shape, generator=g, device=dev, dtype=torch.float64) * (hi - lo) + lo

    timebase = 2.0 ** -40
    stream = torch.cuda.current_stream(dev)
    if args.kernel == "kick":
        mass = f64(n, lo=0.5, hi=2.0)
        f = {"vel": f64(n, 3), "u": f64(n, lo=1, hi=10), "mass": mass, "mass_true": mass.clone(),
             "dmass": f64(n, lo=1e-6, hi=1e-5), "dtmass": f64(n, lo=1e-9, hi=1e-8), "accel": f64(n, 3),
             "dudt": f64(n), "grav": f64(n, 3), "gravwork": f64(n, 3),
             "vel_pred": torch.zeros(n, 3, dtype=torch.float64, device=dev),
             "u_pred": torch.zeros(n, dtype=torch.float64, device=dev),
             "dp": torch.zeros(n, 3, dtype=torch.float64, device=dev),
             "tstart": torch.zeros(n, dtype=torch.int64, device=dev),
             "tend": torch.randint(1 << 20, 1 << 21, (n,), generator=g, device=dev, dtype=torch.int64),
             "active": torch.ones(n, dtype=torch.int32, device=dev)}
        if not mfv:
            for k in KICK_MFM_SKIPS:
                del f[k]

        def launch(_k):
            kick(params, f, 1, timebase, 0.0, stream.cuda_stream)
    else:
        params.min_kernel_radius, params.max_kernel_radius = 1e-6, 1e6
        mass = f64(n, lo=0.5, hi=2.0)
        f = {"pos": f64(n, 3, lo=0, hi=1), "vel_pred": f64(n, 3), "grav": f64(n, 3), "accel": f64(n, 3),
             "divvel": f64(n), "mass": mass, "rho": f64(n, lo=0.5, hi=2.0), "u_pred": f64(n, lo=1, hi=10),
             "dudt": f64(n, lo=-1e-3, hi=1e-3), "h": f64(n, lo=0.01, hi=0.02),
             "pressure": torch.zeros(n, dtype=torch.float64, device=dev),
             "ti_current": torch.zeros(n, dtype=torch.int64, device=dev),
             "status": torch.zeros(1, dtype=torch.int32, device=dev)}
        if mfv:
            f.update({"pvel": f64(n, 3), "dtmass": f64(n, lo=-1e-3, hi=1e-3), "mass_true": mass.clone()})
        else:
            f["vel"] = f64(n, 3)

        def launch(k):
            drift(params, f, (k + 1) << 20, timebase, 0.0, stream.cuda_stream)
    for k in range(args.warmup):
        launch(k)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(args.warmup, args.warmup + args.reps):
        launch(k)
    e1.record(stream)
    torch.cuda.synchronize()
    if args.kernel == "drift" and int(f["status"].item()) != 0:
        raise RuntimeError(f"gz_drift status {int(f['status'].item())}")
    ms = e0.elapsed_time(e1) / args.reps
    bpp = kernel_bytes_per_particle(args.kernel, mfv)
    gbs = bpp * n / (ms * 1e-3) / 1e9
    peak = None
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs")
    except Exception:
        pass
    print(json.dumps({"kernel": f"k_{args.kernel}", "method": args.method, "n": n, "reps": args.reps,
                      "ms_per_launch": ms, "bytes_per_particle": bpp, "achieved_gbs": gbs, "peak_gbs": peak,
                      "frac": (gbs / peak) if peak else None, "particles_per_s": n / (ms * 1e-3)}))


# ------------------------------------------------ active subsets and batched boxes
def run_subsets(args):
    """Individual-timestep substeps: 8,388,608 particles of a log-normal field
    (sigma_lnrho 2.0, Wendland C2, 64 neighbours, MFM). After one full pass the
    active set of each fraction f in {0.001, 0.01, 0.1, 1} is the f N particles
    of smallest h / c_s (the shortest timesteps). The grid (Morton order and
    octree) is built once; each timed substep runs density, gradients and force
    on the active set only, from the kernel lengths of the substep before, with
    no restage, for the mixed and the FP64 form. Rate = active particles / s."""
    import torch

    from gizmo_b200 import abi, ics
    from gizmo_b200.hydro import HydroPass

    n = args.n if args.n != (1 << 24) else (1 << 23)
    t0 = time.time()
    wl = ics.lognormal(203, sigma_lnrho=2.0, seed_density=6, seed_velocity=7, n_particles=n)
    t_gen = time.time() - t0
    res = {"metric": "active particle-updates/s per substep", "unit": "particle-updates/s",
           "config": {"workload": f"log-normal field sigma_lnrho=2.0, {n:,} particles, MFM, Wendland C2, 64 ngb",
                      "active": "the f N particles of smallest h/c_s", "grid": "built once, reused by every substep",
                      "steps": args.steps, "warmup": args.warmup, "generate_s": round(t_gen, 1)},
           "fractions": {}}
    with HydroPass(wl.params) as hp:  # converge once in FP64 (slices bound the cold seed's rows)
        hp.upload_workload(wl)
        chunk = 1 << 21
        for a in range(0, n, chunk):
            hp.density(np.arange(a, min(n, a + chunk), dtype=np.int32))
        hp.hydro_gradient_calc()
        hp.hydro_force()
        conv = hp.download(["h", "cond", "rho", "pressure"])
    wl.h, wl.cond = conv["h"], conv["cond"]
    cs = np.sqrt(wl.params.gamma * conv["pressure"] / conv["rho"])
    order = np.argsort(conv["h"] / cs, kind="stable")
    for precision, tag in ((abi.PRECISION_MIXED, "mixed"), (abi.PRECISION_FP64, "fp64")):
        wl.params.precision = precision
        with HydroPass(wl.params) as hp:
            hp.upload_workload(wl)
            hp.full_pass()
            stream = torch.cuda.ExternalStream(hp.stream)
            for f in (0.001, 0.01, 0.1, 1.0):
                k = max(1, int(round(f * n)))
                act = np.sort(order[:k]).astype(np.int32)
                for _ in range(args.warmup):
                    hp.full_pass(act)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(stream)
                for _ in range(args.steps):
                    hp.full_pass(act)
                e1.record(stream)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / args.steps
                res["fractions"].setdefault(str(f), {})[tag] = {"active": k, "ms_per_substep": ms,
                                                                "value": k / (ms * 1e-3)}
    for f, d in res["fractions"].items():
        d["mixed_over_fp64"] = d["mixed"]["value"] / d["fp64"]["value"]
    print(json.dumps(res), flush=True)


def run_boxes(args):
    """512 independent periodic boxes, log-uniform in [1,024, 65,536] particles
    (seed 5; each a 3-D shock tube or a Sedov blast).
      * set: the boxes as one box set (gz_set_boxes) on one context: every
        kernel of a pass covers all boxes in one launch, and the pass runs as
        one CUDA graph with the restage; K steps, device-resident inputs,
        timed with CUDA events, and the same with the transfers (upload of the
        inputs, download of the rates) every step;
      * per_box: a pass per box on one context (upload, pass, download),
        the launch-bound way, for comparison.
    Rate = particles of all boxes / time, mixed and FP64 forms."""
    import torch

    from gizmo_b200 import abi, ics
    from gizmo_b200.hydro import HydroPass

    t0 = time.time()
    boxes = ics.boxes(512, seed=5)
    t_gen = time.time() - t0
    total = sum(b.n for b in boxes)
    counts = [b.n for b in boxes]
    cat = {k: np.ascontiguousarray(np.concatenate([np.asarray(getattr(b, k)) for b in boxes]), dtype=np.float64)
           for k in ("pos", "vel", "mass", "u", "dt", "h", "cond")}
    K, W = max(args.steps, 3), max(args.warmup, 3)
    res = {"metric": "particle-updates/s over 512 independent boxes", "unit": "particle-updates/s",
           "config": {"workload": f"512 boxes, {total:,} particles, log-uniform 1,024-65,536 per box, shock tubes "
                                  "and Sedov blasts, MFM, cubic, 32 ngb", "generate_s": round(t_gen, 1),
                      "steps": K, "warmup": W}}
    res["set"], res["per_box"] = {}, {}
    for precision, tag in ((abi.PRECISION_MIXED, "mixed"), (abi.PRECISION_FP64, "fp64")):
        params = boxes[0].params
        params.precision = precision
        with HydroPass(params) as hp:
            stream = torch.cuda.ExternalStream(hp.stream)
            hp.set_boxes(counts)
            hp.upload(cat["pos"], cat["vel"], cat["mass"], cat["u"], cat["dt"], cat["h"], cat["cond"])
            hp.full_pass()  # sizes the graph
            for _ in range(W):
                hp.hydro_pass(graph=True, restage=True)
            torch.cuda.synchronize()
            l0 = hp.status()["kernel_launches"]
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(K):
                hp.hydro_pass(graph=True, restage=True)
            e1.record(stream)
            torch.cuda.synchronize()
            sec = e0.elapsed_time(e1) / 1e3 / K
            launches = (hp.status()["kernel_launches"] - l0) / K
            g = hp.graph_stats()
            pin = {k: torch.from_numpy(v).pin_memory() for k, v in cat.items()}
            pout = {k: torch.empty(s, dtype=torch.float64, pin_memory=True)
                    for k, s in (("accel", (total, 3)), ("dudt", (total,)))}
            pin_p = {k: t.data_ptr() for k, t in pin.items()}
            pout_p = {k: t.data_ptr() for k, t in pout.items()}
            torch.cuda.synchronize()
            e0.record(stream)
            hp.upload_raw_async(total, pin_p)
            for k in range(K):
                hp.restage()
                if k + 1 < K:
                    hp.upload_raw_async(total, pin_p)
                hp.hydro_pass(graph=True)
                hp.download_raw_async(pout_p)
            hp.wait()
            e1.record(stream)
            torch.cuda.synchronize()
            sec_e2e = e0.elapsed_time(e1) / 1e3 / K
            res["set"][tag] = {"value": total / sec, "ms_per_pass": 1e3 * sec, "kernel_launches_per_pass": launches,
                               "graph": {"captures": g["captures"], "replays": g["replays"],
                                         "fallbacks": g["fallbacks"]},
                               "e2e": {"value": total / sec_e2e, "ms_per_step": 1e3 * sec_e2e,
                                       "how": "pipelined upload of the inputs and download of accel, dudt every step"}}
        with HydroPass(params) as hp:
            for b in boxes[:8]:  # warm-up
                hp.upload_workload(b)
                hp.full_pass()
            torch.cuda.synchronize()
            stream = torch.cuda.ExternalStream(hp.stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for b in boxes:
                hp.upload_workload(b)
                hp.full_pass()
                hp.download(["accel", "dudt"])
            e1.record(stream)
            torch.cuda.synchronize()
            sec = e0.elapsed_time(e1) / 1e3
        res["per_box"][tag] = {"value": total / sec, "seconds": sec}
    res["mixed_over_fp64"] = res["set"]["mixed"]["value"] / res["set"]["fp64"]["value"]
    print(json.dumps(res), flush=True)


def main():
    args = parse_args()
    if args.subsets:
        run_subsets(args)
        return
    if args.boxes:
        run_boxes(args)
        return
    if args.profile_pass:
        profile_pass(args)
        return
    if args.kernel:
        time_step_kernel(args)
        return
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            res = run_reference(args, world, rank)
        else:
            res = run_ours(args, world, rank, local)
        if rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
    finally:
        dist_done(world)


if __name__ == "__main__":
    main()
