"""Per-particle error of one arithmetic form of the pass against another.

The mixed form is measured against the FP64 form on the same inputs, field by
field and particle by particle (vector and tensor fields by the norm of the
particle's row):

  * h, rho, pressure, vsig: |x - x64| / |x64|;
  * gradients: |g - g64| / max(|g64|, 1e-6 max |g64|);
  * the rates dtmass, accel (dv/dt) and dudt, two ways:
      - "flux": against the scale of the pair fluxes summed into them, from
        the particle's sums over its force row of |mass flux|, |momentum flux|
        and |energy flux| (flux_abs, a diagnostic of the FP64 pass). The rates
        are sums of pair fluxes that cancel, and an FP32 pair carries a
        rounding error in proportion to its flux's natural size: rho c A for
        mass, P A for momentum, P c A for energy (A the face area, c the sound
        speed). Where a pair's mass or energy flux nearly vanishes (a contact
        at rest: F = rho S* A, P S* A with S* ~ 0) the momentum flux still
        carries that size, so the mass and energy scales include the momentum
        sums divided or multiplied by the particle's sound speed;
      - "value": against max(|x64|, 1e-6 max |x64|), reported beside it. Where
        the fluxes of a particle cancel almost exactly (gas at rest in a uniform
        region), this ratio measures the cancellation rather than the pair
        arithmetic.

The bar of the mixed form is the first set: every particle within 1e-5 in
every field (h, rho, pressure, vsig, gradients; the rates on the flux scale).
"""
from __future__ import annotations

import numpy as np

SCALAR_FIELDS = ("h", "rho", "pressure", "vsig")
GRADIENT_FIELDS = ("grad_rho", "grad_p", "grad_v")
RATE_FIELDS = ("accel", "dudt", "dtmass")
FIELDS = SCALAR_FIELDS + GRADIENT_FIELDS + RATE_FIELDS


def _rows(a: np.ndarray, n: int) -> np.ndarray:
    return np.asarray(a, dtype=np.float64).reshape(n, -1)


def flux_scales(vel: np.ndarray, mass: np.ndarray, u: np.ndarray, flux_abs: np.ndarray, mfv: bool,
                cs: np.ndarray) -> dict:
    """The rates' flux scales from flux_abs (sums of |mass flux| M, |momentum
    flux| Pm, |energy flux| E over each force row) and the sound speed cs, in
    the units of each rate: dtmass = sum F_rho -> M + Pm / cs; m accel = sum F_v
    - v dtmass -> Pm + |v| M; m dudt = sum F_E - v.(m accel) - (v^2/2 + u)
    dtmass -> E + (|v| + cs) Pm + (v^2/2 + u) M (the force pass's writeback,
    hydro_toplevel.cc:222-243)."""
    vmag = np.linalg.norm(vel, axis=1)
    fa = flux_abs
    c = np.maximum(cs, 1e-300)
    return {"dtmass": fa[:, 0] + fa[:, 1] / c,
            "accel": (fa[:, 1] + (vmag * fa[:, 0] if mfv else 0.0)) / mass,
            "dudt": (fa[:, 2] + (vmag + c) * fa[:, 1] + ((0.5 * vmag ** 2 + u) * fa[:, 0] if mfv else 0.0)) / mass}


def sound_speed(gamma: float, pressure: np.ndarray, rho: np.ndarray) -> np.ndarray:
    """c = sqrt(gamma P / rho) (effective_soundspeed, cell_data.h:703-713)."""
    return np.sqrt(gamma * np.maximum(pressure, 0.0) / np.maximum(rho, 1e-300))


def per_particle(test: dict, ref: dict, scales: dict, fields=FIELDS) -> dict:
    """{field: per-particle error} under the bar's denominators, plus
    {field + ":value": ...} for the rates against their own values."""
    n = np.asarray(ref["h"]).shape[0]
    out = {}
    for f in fields:
        a, b = _rows(test[f], n), _rows(ref[f], n)
        d = np.linalg.norm(a - b, axis=1)
        nb = np.linalg.norm(b, axis=1)
        top = float(nb.max()) if n else 0.0
        floored = np.maximum(nb, 1e-6 * top)
        if f in RATE_FIELDS:
            out[f] = d / np.maximum(scales[f], 1e-300)
            out[f + ":value"] = d / np.maximum(floored, 1e-300)
        elif f in GRADIENT_FIELDS:
            out[f] = d / np.maximum(floored, 1e-300)
        else:
            out[f] = d / np.maximum(nb, 1e-300)
    return out


def summary(err: dict, bar: float = 1e-5) -> dict:
    """Max / p99.99 / p99 / median per field, the particles above the bar per
    field, and the particles above it in any field of the bar's set."""
    res = {}
    any_bar = None
    for f, e in err.items():
        res[f] = {"max": float(e.max()) if e.size else 0.0,
                  "p99_99": float(np.percentile(e, 99.99)) if e.size else 0.0,
                  "p99": float(np.percentile(e, 99)) if e.size else 0.0,
                  "p50": float(np.median(e)) if e.size else 0.0,
                  "above_bar": int((e > bar).sum())}
        if ":" not in f:
            any_bar = (e > bar) if any_bar is None else (any_bar | (e > bar))
    res["bar"] = bar
    res["max_over_fields"] = max((v["max"] for k, v in res.items() if isinstance(v, dict) and ":" not in k),
                                 default=0.0)
    res["particles_above_bar_any_field"] = int(any_bar.sum()) if any_bar is not None else 0
    return res
