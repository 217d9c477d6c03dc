"""Independent boxes of mixed sizes and problems (shock tubes and Sedov blasts,
log-uniform sizes), as a batch of small simulations hands them to the pass:

  * each box's three passes match the oracle pass by pass (FP64 form, the
    tolerances of the other parity tests);
  * mass, momentum and energy are conserved per pass in both forms;
  * one context reused across the boxes (gz_set_params, then gz_upload of a
    set of another size and problem) gives the outputs of a fresh context bit
    for bit, so nothing of one box leaks into the next.
"""
import numpy as np
import pytest

from gizmo_b200 import abi, ics
from gizmo_b200.hydro import HydroPass
from tests.test_gpu_parity import _conservation, check_passwise

pytestmark = pytest.mark.gpu

BOXES = ics.boxes(4, seed=5, n_min=1024, n_max=4096)


def test_batch_holds_both_problems():
    names = {wl.name for wl in BOXES}
    assert names == {"shock_tube", "sedov"}, names
    assert len({wl.n for wl in BOXES}) > 1


@pytest.mark.parametrize("b", range(len(BOXES)))
def test_box_passes_match_oracle(b):
    check_passwise(BOXES[b])


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_box_conservation(precision):
    for wl0 in BOXES:
        wl = ics.boxes(4, seed=5, n_min=1024, n_max=4096, precision=precision)[BOXES.index(wl0)]
        wl.params.max_kernel_radius = 0.45  # no particle reaches the du/dt cap (see test_gpu_parity)
        with HydroPass(wl.params) as hp:
            hp.upload_workload(wl)
            hp.full_pass()
            out = hp.download()
        assert (out["h"] < 0.99 * wl.params.max_kernel_radius).all()
        for k, v in _conservation(wl, out).items():
            assert v <= 1e-12, (wl.name, wl.n, k, v)


def test_one_context_across_boxes():
    fresh = []
    for wl in BOXES:
        with HydroPass(wl.params) as hp:
            hp.upload_workload(wl)
            hp.full_pass()
            fresh.append(hp.download())
    with HydroPass(BOXES[-1].params) as hp:
        for wl, want in zip(BOXES, fresh):
            hp.set_params(wl.params)
            hp.upload_workload(wl)
            hp.full_pass()
            got = hp.download()
            for k in want:
                assert np.array_equal(got[k], want[k]), (wl.name, wl.n, k)
