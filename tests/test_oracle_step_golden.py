"""The oracle's kick, drift, timestep and wake-up against golden fixtures
made by the reference's own code (tests/golden/make_step_golden.py): bit-exact
on every field. These pin the restatements without the reference tree or its
compiled libraries."""
import glob
import os

import numpy as np
import pytest

from gizmo_b200 import ics
from oracle import oracle as O

STEP = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "step")
TIMEBASE = 2.0 ** -40
CASES = sorted(glob.glob(os.path.join(STEP, "*.npz")))


def _load(path):
    z = np.load(path)
    p = ics.sedov(4, seed=1).params
    p.method = int(z["method"])
    p.min_kernel_radius, p.max_kernel_radius = float(z["min_h"]), float(z["max_h"])
    pick = lambda pre: {k[len(pre):]: z[k] for k in z.files if k.startswith(pre)}  # noqa: E731
    return p, pick("s_"), pick("in_"), pick("out_")


def test_fixtures_present():
    names = {os.path.basename(c)[:-4] for c in CASES}
    assert {"kick_mfm_mode0", "kick_mfv_mode1", "drift_mfm", "drift_mfv", "timestep", "wakeup_mfv"} <= names


@pytest.mark.parametrize("path", CASES, ids=lambda c: os.path.basename(c)[:-4])
def test_oracle_matches_reference_step_golden(path):
    name = os.path.basename(path)[:-4]
    p, sc, inputs, want = _load(path)
    st = {k: np.ascontiguousarray(v).copy() for k, v in inputs.items()}
    orc = O.Oracle(p, "port", n_threads=1)
    if name.startswith("kick"):
        assert orc.kick(st, int(sc["mode"]), TIMEBASE, float(sc["floor"])) == 0
    elif name.startswith("drift"):
        assert orc.drift(st, int(sc["time1"]), TIMEBASE, float(sc["floor"])) == 0
    elif name == "timestep":
        tp = O.OrcTimestepParams()
        tp.err_tol_int_accuracy, tp.courant_fac = 0.02, 0.2
        tp.max_size_timestep, tp.min_size_timestep, tp.timebase = 1e-2, 0.0, TIMEBASE
        tp.ti_current = int(sc["ti_current"])
        for b in range(O.TIMEBINS):
            tp.bin_active[b] = int(sc["bin_active"][b])
        assert orc.timestep(st, tp) == 0
    else:
        p = ics.sedov(8, seed=7).params
        p.method = int(_load(path)[0].method)
        assert O.Oracle(p, "port", n_threads=1).force_wakeup(st, sc["bin_active"], sc["active"]) == 0
    for k, v in want.items():
        if k == "dmass":
            np.testing.assert_allclose(st[k], v, rtol=0, atol=1e-14 * np.abs(v).max() + 1e-300)
        else:
            np.testing.assert_array_equal(st[k], v, err_msg=k)
