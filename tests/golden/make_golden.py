"""Generate the golden fixtures in tests/golden/ from the reference's own code.

The reference tree has no golden vectors for the hydro pair sums (its tests
download ICs and compare whole runs to analytic profiles), so the fixtures
are produced by running the reference's OWN pair bodies -- compiled from its
sources by oracle/build_ref.sh into oracle/_ref/ -- on small seeded inputs,
through the three passes (density with h-iteration -> gradients -> force).

Run in a tree that has the reference sources:
    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gizmo_b200 import ics  # noqa: E402
from oracle import oracle as O  # noqa: E402

CASES = {
    "sedov_mfm_cubic_8": lambda: ics.sedov(8, seed=1),
    "plummer_mfv_cubic_8": lambda: ics.plummer_mix(8, seed=4, n_spheres=4),
    "lognormal_mfm_wendland_8": lambda: ics.lognormal(8, seed_density=2, seed_velocity=3, grid=16),
}

OUT_FIELDS = ["h", "num_ngb", "drkern", "divvel", "rho", "pressure", "nvt", "cond", "fce", "pvel", "iters",
              "grad_rho", "grad_p", "grad_v", "accel", "dudt", "vsig", "dtmass", "dmass", "gravwork"]


def main():
    O.build_reference()
    for name, make in CASES.items():
        wl = make()
        st = O.new_state(wl.n, wl.inputs())
        ref = O.Oracle(wl.params, "reference", n_threads=1)
        rc = (ref.density(st), ref.gradients(st), ref.force(st))
        assert rc == (0, 0, 0), rc
        p = wl.params
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            params=np.array([p.kernel, p.method, p.precision, p.first_step, p.selfgravity_off]),
            fparams=np.array([p.box_size, p.gamma, p.des_num_ngb, p.max_num_ngb_dev, p.min_kernel_radius,
                              p.max_kernel_radius]),
            **{f"in_{k}": v for k, v in wl.inputs().items()},
            **{f"out_{k}": st[k] for k in OUT_FIELDS})
        print(name, wl.n, "mean iterations", st["iters"].mean())


if __name__ == "__main__":
    main()
