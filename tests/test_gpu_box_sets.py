"""Box sets (gz_set_boxes): independent periodic boxes of mixed sizes (shock
tubes and Sedov blasts) as one particle set, each pass one launch per kernel
over all boxes.

Against a pass per box on its own:
  * neighbour sets bit-exact (no pair joins two boxes: every row is the box's
    own, with the box's offset);
  * FP64 outputs within the parity tolerances of tests/test_gpu_parity.py (the
    lanes per row follow the number of rows, so a box's sums run in another
    order inside the set than alone): >= 99.9% of particles on the same
    h-iteration path with h within 1e-10, every other particle within 3e-3,
    the other fields of the same-path particles 1e-10 (force fields against a
    floor of 1e-3 x the field maximum), in boxes whose every particle took the
    same path;
  * momentum conserved per box in both forms;
  * the set as one CUDA graph equal to its plain calls bit for bit.
"""
import numpy as np
import pytest

from gizmo_b200 import abi, ics
from gizmo_b200.hydro import HydroPass
from tests._util import DENSITY_FIELDS, FORCE_FIELDS, GRADIENT_FIELDS, field_err

pytestmark = pytest.mark.gpu

FIELDS = DENSITY_FIELDS + GRADIENT_FIELDS + FORCE_FIELDS + ["iters"]


def _concat(boxes):
    cat = {k: np.concatenate([np.asarray(getattr(b, k)) for b in boxes]) for k in
           ("pos", "vel", "mass", "u", "dt", "h", "cond")}
    return cat


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_box_set_matches_boxes_alone(precision):
    boxes = ics.boxes(12, seed=5, n_min=512, n_max=4096, precision=precision)
    counts = [b.n for b in boxes]
    starts = np.concatenate([[0], np.cumsum(counts)])
    params = boxes[0].params
    alone = []
    with HydroPass(params) as hp:
        for b in boxes:
            hp.upload_workload(b)
            rows = hp.neighbors(1)
            hp.full_pass()
            out = hp.download(FIELDS)
            out["rows"] = rows
            alone.append(out)
    cat = _concat(boxes)
    with HydroPass(params) as hp:
        hp.set_boxes(counts)
        hp.upload(cat["pos"], cat["vel"], cat["mass"], cat["u"], cat["dt"], cat["h"], cat["cond"])
        off, nbr = hp.neighbors(1)
        hp.full_pass()
        got = hp.download(FIELDS)
        launches_plain = hp.status()["kernel_launches"]
        hp.restage()
        hp.hydro_pass(graph=True)  # captured and replayed
        graph = hp.download(FIELDS)
        assert hp.graph_stats()["replays"] == 1
    for f in FIELDS:
        assert np.array_equal(graph[f], got[f]), f
    assert launches_plain > 0
    same_all = []
    for b, (a, s0) in enumerate(zip(alone, starts[:-1])):
        n = counts[b]
        # neighbour rows: the box's own, offset by its start
        bo, bn = a["rows"]
        o = off[s0:s0 + n + 1] - off[s0]
        assert np.array_equal(o, bo), b
        assert np.array_equal(nbr[off[s0]:off[s0 + n]] - s0, bn), b
        sl = slice(s0, s0 + n)
        h_rel = np.abs(got["h"][sl] - a["h"]) / a["h"]
        same = (got["iters"][sl] == a["iters"]) & (h_rel <= 1e-10)
        same_all.append(same)
        assert h_rel.max() <= 3e-3, (b, h_rel.max())
        if precision == abi.PRECISION_FP64 and same.all():
            for f in DENSITY_FIELDS + GRADIENT_FIELDS:
                assert field_err(f, got[f][sl], a[f], 1e-6) < 1e-10, (b, f)
            for f in FORCE_FIELDS:
                assert field_err(f, got[f][sl], a[f], 1e-3) < 1e-10, (b, f)
        # momentum per box
        mom = boxes[b].mass[:, None] * got["accel"][sl]
        assert np.abs(mom.sum(0)).max() <= 1e-12 * np.abs(mom).sum(), b
    assert np.concatenate(same_all).mean() >= 0.999
