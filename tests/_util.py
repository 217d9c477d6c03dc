"""Shared helpers for the tests (comparison metrics, fixture loading)."""
from __future__ import annotations

import glob
import os

import numpy as np

from gizmo_b200.abi import GzParams
from gizmo_b200.ics import Workload

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

DENSITY_FIELDS = ["h", "num_ngb", "drkern", "divvel", "rho", "pressure", "nvt", "cond", "fce", "pvel"]
GRADIENT_FIELDS = ["grad_rho", "grad_p", "grad_v"]
FORCE_FIELDS = ["accel", "dudt", "vsig", "dtmass", "dmass", "gravwork"]


def rel_err(a, b, floor_frac: float = 1e-6) -> float:
    """max |a-b| / max(|b|, floor_frac * max|b|), element-wise over the field."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if b.size == 0:
        return 0.0
    top = float(np.max(np.abs(b)))
    if top == 0.0:
        return float(np.max(np.abs(a)))
    scale = np.maximum(np.abs(b), floor_frac * top)
    return float(np.max(np.abs(a - b) / scale))


def row_rel_err(a, b, floor_frac: float = 1e-6) -> float:
    """max over rows of |a_row - b_row| / max(|b_row|, floor_frac * max |b_row|),
    with the row the trailing components of a vector or tensor field. The sums
    behind such a field cancel component by component, and their roundoff in
    another summation order scales with the row's magnitude, not with the size
    of one (possibly near-zero) component."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if b.size == 0:
        return 0.0
    a = a.reshape(a.shape[0], -1)
    b = b.reshape(b.shape[0], -1)
    nb = np.linalg.norm(b, axis=1)
    top = float(nb.max())
    if top == 0.0:
        return float(np.linalg.norm(a, axis=1).max())
    return float(np.max(np.linalg.norm(a - b, axis=1) / np.maximum(nb, floor_frac * top)))


def field_err(name: str, a, b, floor_frac: float = 1e-6) -> float:
    """rel_err for a scalar field, row_rel_err for a vector or tensor field."""
    return row_rel_err(a, b, floor_frac) if np.asarray(b).ndim > 1 else rel_err(a, b, floor_frac)


def norm_err(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / (nb if nb > 0 else 1.0)


def golden_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(path: str):
    z = np.load(path)
    p = GzParams()
    p.kernel, p.method, p.precision, p.first_step, p.selfgravity_off = [int(v) for v in z["params"]]
    (p.box_size, p.gamma, p.des_num_ngb, p.max_num_ngb_dev, p.min_kernel_radius,
     p.max_kernel_radius) = [float(v) for v in z["fparams"]]
    inputs = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    outputs = {k[4:]: z[k] for k in z.files if k.startswith("out_")}
    return p, inputs, outputs


def workload_from(params, inputs, name="fixture") -> Workload:
    return Workload(name, params, inputs["pos"], inputs["vel"], inputs["mass"], inputs["u"], inputs["dt"],
                    inputs["h"], inputs["cond"])


def riemann_fallback_case(method: int, seed: int = 0, n1: int = 10, mach: float = 50.0):
    """A Sedov lattice given Gaussian random velocities at rms Mach ~`mach` of
    the background sound speed: so many faces collide or separate supersonically
    that the HLLC star pressure often exceeds the pressure limit, sending those
    faces to the exact iterative Riemann solver (reimann.h:625-664) and through
    the retry with cell-centred states (hydro_core_meshless_functions.h:350-427)."""
    from gizmo_b200 import ics
    wl = ics.sedov(n1, seed=seed)
    wl.params.method = method
    rng = np.random.default_rng(1000 + seed)
    cs = np.sqrt(wl.params.gamma * (wl.params.gamma - 1.0) * np.median(wl.u))
    wl.vel = rng.standard_normal((wl.n, 3)) * mach * cs
    return wl


def riemann_failure_case(method: int):
    """A Sedov set with one particle of NaN internal energy: its pressure is NaN,
    so every face it reaches (and, through the gradients, its neighbours' faces)
    has a NaN star pressure. That is the only way the HLLC stage, whose star
    pressure is clamped at MIN_REAL, hands a face to the Kurganov-Tadmor solver
    (reimann.h:445-477); the exact solver and both retries fail too, and the
    pass stops with 1234 (hydro_core_meshless_functions.h:403-425)."""
    from gizmo_b200 import ics
    wl = ics.sedov(8, seed=1)
    wl.params.method = method
    wl.u = wl.u.copy()
    wl.u[100] = float("nan")
    return wl
