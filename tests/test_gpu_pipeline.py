"""Pipelined transfers (gz_upload_async / gz_download_async / gz_wait): the
inputs of the next step are copied while a pass runs, the outputs of a step
while the next one runs, and every step's results equal those of the plain
gz_upload -> pass -> gz_download on the same inputs."""
import numpy as np
import pytest
import torch

from gizmo_b200 import abi, ics
from gizmo_b200.hydro import HydroPass

pytestmark = pytest.mark.gpu

OUT = {"h": (1,), "rho": (1,), "accel": (3,), "dudt": (1,), "vsig": (1,), "grad_v": (9,), "iters": (1,)}


def _inputs(wl, vel_scale):
    d = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in wl.inputs().items()}
    d["vel"] = d["vel"] * vel_scale
    return {k: torch.from_numpy(v).pin_memory() for k, v in d.items()}


def _outputs(n):
    return {k: torch.empty((n,) + s if s != (1,) else (n,), dtype=torch.int32 if k == "iters" else torch.float64,
                           pin_memory=True) for k, s in OUT.items()}


def _ptrs(d):
    return {k: t.data_ptr() for k, t in d.items()}


def _plain(wl, inp):
    with HydroPass(wl.params) as hp:
        hp.upload_raw(wl.n, _ptrs(inp))
        hp.full_pass()
        out = _outputs(wl.n)
        hp.download_raw(_ptrs(out))
    return {k: v.numpy().copy() for k, v in out.items()}


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_pipelined_steps_equal_plain(precision):
    wl = ics.plummer_mix(32, seed=4, n_spheres=100, precision=precision)
    steps = [_inputs(wl, s) for s in (1.0, 1.1, 0.9, 1.0)]
    refs = [_plain(wl, inp) for inp in steps[:3]]
    with HydroPass(wl.params) as hp:
        hp.upload_raw(wl.n, _ptrs(steps[0]))
        hp.full_pass()  # sizes the graph
        outs = [_outputs(wl.n) for _ in range(3)]
        hp.upload_raw_async(wl.n, _ptrs(steps[0]))
        for k in range(3):
            hp.restage()  # takes step k's inputs
            hp.upload_raw_async(wl.n, _ptrs(steps[k + 1]))  # the next step's, beside this pass
            hp.hydro_pass(graph=True)
            hp.download_raw_async(_ptrs(outs[k]))  # this step's, beside the next pass
        hp.wait()
        assert hp.graph_stats()["replays"] >= 2
    for k in range(3):
        for f in OUT:
            assert np.array_equal(outs[k][f].numpy(), refs[k][f]), (k, f)


def test_plain_download_groups_fields():
    """The host download scatters the fields into a staging area up to 16
    doubles per particle and copies each group out together: every field of a
    request wider than that still arrives."""
    wl = ics.sedov(12, seed=1)
    with HydroPass(wl.params) as hp:
        hp.upload_workload(wl)
        hp.full_pass()
        every = hp.download()  # 45 doubles and an int per particle
        one = {f: hp.download([f])[f] for f in ("nvt", "grad_v", "accel", "iters", "h")}
    for f, v in one.items():
        assert np.array_equal(every[f], v), f
