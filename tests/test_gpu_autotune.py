"""The walk's tuning (gz_tuning: octree leaf size and padded row slots) and
its autotuner change what the neighbour walk costs, never a result: the rows
are the exact neighbour sets in ascending order for any tree, so every output
of the pass, in both forms, is the same bit for bit under every setting."""
import numpy as np
import pytest

from gizmo_b200 import abi, ics
from gizmo_b200.hydro import HydroPass

pytestmark = pytest.mark.gpu


def _pass(hp, wl):
    hp.upload_workload(wl)
    hp.full_pass()
    out = hp.download()
    out["rows"] = hp.neighbors(2)
    return out


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_tuning_changes_no_result(precision):
    wl = ics.plummer_mix(32, seed=4, n_spheres=100, precision=precision)
    with HydroPass(wl.params) as hp:
        assert hp.tuning() == {"leaf_max": 96, "row_slots": 2.5}
        ref = _pass(hp, wl)
        results = []
        for leaf, slots in ((32, 1.5), (128, 3.0), (8, 1.0)):
            hp.set_tuning(leaf, slots)
            results.append(_pass(hp, wl))
        hp.upload_workload(wl)
        chosen = hp.autotune()
        assert chosen["leaf_max"] in (32, 64, 96, 128) and chosen["row_slots"] in (1.5, 2.0, 2.5, 3.0)
        assert hp.tuning() == chosen
        hp.full_pass()
        tuned = hp.download()
        tuned["rows"] = hp.neighbors(2)
        results.append(tuned)
    for out in results:
        for k, v in ref.items():
            if k == "rows":
                assert np.array_equal(out[k][0], v[0]) and np.array_equal(out[k][1], v[1])
            else:
                assert np.array_equal(out[k], v), k
    # a second context with the same device, size class, DesNumNgb and kernel takes the tuned setting
    with HydroPass(wl.params) as hp:
        hp.upload_workload(wl)
        assert hp.autotune() == chosen
