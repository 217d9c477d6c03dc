"""Generate the golden fixtures in tests/golden/step/ from the reference's own
kick, drift, timestep and wake-up code.

The fixtures are the outputs of the reference's do_the_kick (core/kicks.cc),
drift_particle_impl (core/drift_particle_functions.h), get_timestep
(core/timestep.cc) and the force pair body's wake-up (hydro/hydro_functions.h),
compiled from its sources by oracle/build_ref.sh into oracle/_ref/, on small
seeded inputs: the constructed cases of the oracle tests, which reach every
limiter, cap and floor of each update.

Run in a tree that has the reference sources:
    python tests/golden/make_step_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gizmo_b200 import ics  # noqa: E402
from gizmo_b200.abi import METHOD_MFM, METHOD_MFV  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests import test_oracle_drift, test_oracle_kick, test_oracle_timestep  # noqa: E402

OUT = os.path.join(HERE, "step")
TIMEBASE = 2.0 ** -40
METHODS = {"mfm": METHOD_MFM, "mfv": METHOD_MFV}


def _params(method, min_h=None, max_h=None):
    p = ics.sedov(4, seed=1).params
    p.method = method
    if min_h is not None:
        p.min_kernel_radius, p.max_kernel_radius = min_h, max_h
    return p


def _save(name, params, scalars, inputs, outputs):
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"),
                        method=np.array(params.method), min_h=np.array(params.min_kernel_radius),
                        max_h=np.array(params.max_kernel_radius), **{f"s_{k}": np.array(v) for k, v in scalars.items()},
                        **{f"in_{k}": v for k, v in inputs.items()}, **{f"out_{k}": v for k, v in outputs.items()})
    print(name)


def main():
    O.build_reference()
    os.makedirs(OUT, exist_ok=True)
    for tag, method in METHODS.items():
        p = _params(method)
        for mode, floor in ((0, 0.0), (1, 3.0)):
            ks = test_oracle_kick._constructed(256, seed=300 + 10 * mode + method)
            out = {k: v.copy() for k, v in ks.items()}
            assert O.Oracle(p, "reference").kick(out, mode, TIMEBASE, floor) == 0
            _save(f"kick_{tag}_mode{mode}", p, {"mode": mode, "floor": floor}, ks, out)
        p = _params(method, 0.05, 0.5)
        ds, time1 = test_oracle_drift._constructed(256, 400 + method, p)
        out = {k: v.copy() for k, v in ds.items()}
        assert O.Oracle(p, "reference").drift(out, time1, TIMEBASE, 3.0) == 0
        _save(f"drift_{tag}", p, {"time1": time1, "floor": 3.0}, ds, out)
    # timestep (the criterion does not depend on the method)
    p = _params(METHOD_MFV)
    rng = np.random.default_rng(5)
    n = 256
    ts = O.new_timestep_state(n, {
        "grav": rng.normal(size=(n, 3)), "accel": rng.normal(size=(n, 3)) * 10.0 ** rng.uniform(-2, 6, (n, 1)),
        "vsig": 10.0 ** rng.uniform(-1, 3, n), "h": 10.0 ** rng.uniform(-3, -1, n), "num_ngb": rng.uniform(2.5, 4.5, n),
        "divvel": rng.normal(size=n) * 10.0 ** rng.uniform(-1, 4, n), "mass": np.where(rng.random(n) < 0.1, 0.0, 1.0),
        "softening": np.where(rng.random(n) < 0.2, 0.0, 10.0 ** rng.uniform(-5, -2, n)),
        "bin": rng.integers(2, 30, n).astype(np.int32), "ti_begstep": rng.integers(0, 1 << 40, n),
        "dt_step": rng.integers(0, 1 << 20, n)})
    tp = test_oracle_timestep._params(ti_current=1 << 41, active_bins=range(0, 60, 3))
    out = {k: v.copy() for k, v in ts.items()}
    assert O.Oracle(p, "reference").timestep(out, tp) == 0
    _save("timestep", p, {"ti_current": tp.ti_current, "bin_active": np.array(tp.bin_active[:])}, ts, out)
    # wake-up in the force pass
    wl = ics.sedov(8, seed=7)
    wl.params.method = METHOD_MFV
    st = O.new_state(wl.n, wl.inputs())
    orc = O.Oracle(wl.params, "reference", n_threads=1)
    assert orc.density(st) == 0 and orc.gradients(st) == 0 and orc.force(st) == 0
    rng = np.random.default_rng(21)
    st["timebin"][...] = rng.integers(10, 15, wl.n)
    bins = np.zeros(O.TIMEBINS, np.int32)
    bins[[10, 11]] = 1
    st["vsig"][(bins[st["timebin"]] == 0) & (rng.random(wl.n) < 0.5)] *= 0.05
    active = np.nonzero(bins[st["timebin"]])[0].astype(np.int32)
    out = {k: v.copy() for k, v in st.items()}
    assert orc.force_wakeup(out, bins, active) == 0
    _save("wakeup_mfv", wl.params, {"bin_active": bins, "active": active}, st, out)


if __name__ == "__main__":
    main()
