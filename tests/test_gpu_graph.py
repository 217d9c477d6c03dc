"""The pass over every particle as one CUDA graph (gz_hydro_pass with
GZ_PASS_GRAPH): the density iteration as a device-driven WHILE node, the
symmetric rows, gradients and force behind IF nodes. Its results equal the
three plain calls' bit for bit, in both forms, on the first replay and on
later ones after a restage; a buffer the graph cannot grow (rows of a seed
far from converged) is answered by the plain pass from the same inputs."""
import numpy as np
import pytest

from gizmo_b200 import abi, ics
from gizmo_b200.hydro import HydroPass

pytestmark = pytest.mark.gpu

CASES = {
    "plummer32_mfv": lambda p: ics.plummer_mix(32, seed=4, n_spheres=100, precision=p),
    "lognormal32_mfm": lambda p: ics.lognormal(32, seed_density=2, seed_velocity=3, precision=p),
    "sedov24_mfm": lambda p: ics.sedov(24, seed=1, precision=p),
}
FIELDS = [f for f, _ in abi.OUTPUT_FIELDS] + ["iters"]


def _plain(wl):
    with HydroPass(wl.params) as hp:
        hp.upload_workload(wl)
        hp.full_pass()
        out = hp.download(FIELDS)
        out["status"] = hp.status()
    return out


def _same(a, b):
    for k in FIELDS:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
@pytest.mark.parametrize("case", list(CASES))
def test_graph_pass_equals_plain_calls(case, precision):
    wl = CASES[case](precision)
    ref = _plain(wl)
    with HydroPass(wl.params) as hp:
        hp.upload_workload(wl)
        hp.hydro_pass(graph=True)  # plain: sizes the graph's buffers
        assert hp.graph_stats()["replays"] == 0
        _same(hp.download(FIELDS), ref)
        for k in range(2):  # capture + replay, then a replay of the same graph
            hp.restage()
            l0 = hp.status()["kernel_launches"]
            hp.hydro_pass(graph=True)
            st = hp.status()
            g = hp.graph_stats()
            assert g["captures"] == 1 and g["replays"] == k + 1 and g["fallbacks"] == 0, g
            _same(hp.download(FIELDS), ref)
            assert st["density_iterations"] == ref["status"]["density_iterations"]
            assert st["pairs_symmetric"] == ref["status"]["pairs_symmetric"]
            assert st["pairs_refined"] == ref["status"]["pairs_refined"]
            # the launches of one replay: the kernels outside the bodies, one
            # iteration's per density iteration, the rows', gradients' and force's
            want = g["kernels_top"] + g["kernels_per_iteration"] * st["density_iterations"] + g["kernels_after"]
            assert st["kernel_launches"] - l0 == want


def test_graph_falls_back_to_plain_pass():
    """DesNumNgb raised from 32 to 64 after the sizing pass: the symmetric rows
    of the next pass hold about twice the entries, past the room the graph
    keeps for them (the last pass's count and a quarter), so the call runs the
    plain pass from the same seeds and gets its results."""
    wl = ics.plummer_mix(32, seed=4, n_spheres=100, precision=abi.PRECISION_MIXED)
    p = wl.params
    p64 = ics.make_params(p.kernel, p.method, p.gamma, 64.0, p.max_num_ngb_dev, p.precision, p.box_size, p.first_step,
                          p.selfgravity_off, p.min_kernel_radius, p.max_kernel_radius)
    with HydroPass(p64) as hp:
        hp.upload_workload(wl)
        hp.full_pass()
        ref = hp.download(FIELDS)
    with HydroPass(wl.params) as hp:
        hp.upload_workload(wl)
        hp.hydro_pass(graph=True)  # plain, at DesNumNgb 32: sizes
        hp.set_params(p64)
        hp.restage()
        hp.hydro_pass(graph=True)
        g = hp.graph_stats()
        assert g["replays"] == 1 and g["fallbacks"] == 1, g
        _same(hp.download(FIELDS), ref)
        hp.restage()  # captured again for the larger rows, and replayed
        hp.hydro_pass(graph=True)
        g = hp.graph_stats()
        assert g["captures"] == 2 and g["replays"] == 2 and g["fallbacks"] == 1, g
        _same(hp.download(FIELDS), ref)


@pytest.mark.parametrize("case", ["plummer32_mfv", "sedov24_mfm"])
def test_graph_with_restage_equals_plain(case):
    """GZ_PASS_RESTAGE: the restage (keys, sort, mirror, octree built on the
    device with nothing read back) captured at the start of the graph: the
    step's results equal restage() + the three plain calls, with box sets too."""
    wl = CASES[case](abi.PRECISION_MIXED)
    ref = _plain(wl)
    with HydroPass(wl.params) as hp:
        hp.upload_workload(wl)
        hp.hydro_pass(graph=True, restage=True)  # plain: sizes
        _same(hp.download(FIELDS), ref)
        for k in range(2):
            hp.hydro_pass(graph=True, restage=True)
            g = hp.graph_stats()
            assert g["captures"] == 1 and g["replays"] == k + 1 and g["fallbacks"] == 0, g
            _same(hp.download(FIELDS), ref)
    # two copies of the set as a box set of two boxes: each box's outputs equal the set's alone
    two = {k: np.concatenate([np.asarray(getattr(wl, k))] * 2) for k in ("pos", "vel", "mass", "u", "dt", "h", "cond")}
    with HydroPass(wl.params) as hp:
        hp.set_boxes([wl.n, wl.n])
        hp.upload(two["pos"], two["vel"], two["mass"], two["u"], two["dt"], two["h"], two["cond"])
        hp.hydro_pass(graph=True, restage=True)
        plain = hp.download(FIELDS)
        hp.hydro_pass(graph=True, restage=True)
        graph = hp.download(FIELDS)
        assert hp.graph_stats()["replays"] == 1
    for f in FIELDS:
        assert np.array_equal(graph[f], plain[f]), f
        assert np.array_equal(plain[f][:wl.n], plain[f][wl.n:]), f
