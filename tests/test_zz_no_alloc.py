"""gz_density_sums_noalloc, the entry point for callers that cannot allocate
device memory (a host code whose own memory pool owns the device, or a loop
that cannot accept the synchronisation cudaMalloc/cudaFree imply).

It is called through the C ABI on particle sets the test holds in device
memory, twice in a row with different sets (different sizes, kernels and
methods), and each result is checked against gz_density_sums -- the context-
based entry point that computes the same sums -- with the tolerance of the
other density-sum parity tests: 1e-10 relative (summation order only).
This file is collected last, so a stop at its first failure has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

from gizmo_b200 import abi, ics
from gizmo_b200.hydro import HydroPass
from tests._util import rel_err

pytestmark = pytest.mark.gpu


def _context_sums(wl):
    with HydroPass(wl.params) as hp:
        hp.upload_workload(wl)
        return hp.density_sums()


def _noalloc_sums(lib, wl, with_pv=True):
    import torch

    dev = torch.device("cuda", 0)

    def on_device(a):
        return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)

    pos, vel, mass, h = on_device(wl.pos), on_device(wl.vel), on_device(wl.mass), on_device(wl.h)
    # outputs start as NaN: every entry must be written by the call
    acc = torch.full((wl.n, 14), float("nan"), dtype=torch.float64, device=dev)
    pv = torch.full((wl.n, 3), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    rc = lib.gz_density_sums_noalloc(C.byref(wl.params), wl.n, pos.data_ptr(), vel.data_ptr(), mass.data_ptr(),
                                     h.data_ptr(), acc.data_ptr(), pv.data_ptr() if with_pv else None,
                                     C.c_void_p(stream.cuda_stream))
    assert rc == abi.OK, rc
    stream.synchronize()
    return acc.cpu().numpy(), (pv.cpu().numpy() if with_pv else None)


def _check(got, want):
    acc_n, pv_n = got
    acc_c, pv_c = want
    assert np.isfinite(acc_n).all()
    for c in range(13):
        assert rel_err(acc_n[:, c], acc_c[:, c], 1e-9) < 1e-10, c
    assert (acc_n[:, 13] == 0).all()
    if pv_n is not None:
        assert np.isfinite(pv_n).all()
        assert rel_err(pv_n, pv_c, 1e-9) < 1e-10


def test_noalloc_matches_context_sums_on_two_calls_in_a_row():
    lib = abi.load_library()
    first = ics.plummer_mix(16, seed=4, n_spheres=12)  # 4096 particles, MFV, cubic kernel
    second = ics.lognormal(12, seed_density=2, seed_velocity=3, grid=24)  # 1728, MFM, Wendland C2
    assert first.params.method != second.params.method and first.params.kernel != second.params.kernel
    got1 = _noalloc_sums(lib, first)
    got2 = _noalloc_sums(lib, second)  # a smaller set right after: nothing of the first may leak in
    _check(got1, _context_sums(first))
    _check(got2, _context_sums(second))


def test_noalloc_ragged_set_without_particle_velocity_and_a_massless_particle():
    """1000 particles (not a multiple of the 128-record tile), pv = NULL, and one
    particle of zero mass: never a candidate, but still a target with its own sums."""
    lib = abi.load_library()
    wl = ics.sedov(10)
    wl.mass = wl.mass.copy()
    wl.mass[123] = 0.0
    got = _noalloc_sums(lib, wl, with_pv=False)
    want = _context_sums(wl)
    _check(got, want)
    assert got[0][123, 0] > 0  # the massless particle's own row was summed


def test_noalloc_rejects_sets_beyond_its_static_scratch():
    lib = abi.load_library()
    wl = ics.sedov(4)
    n = abi.NOALLOC_MAX_PARTICLES + 1
    rc = lib.gz_density_sums_noalloc(C.byref(wl.params), n, None, None, None, None, None, None, None)
    assert rc == abi.ERR_CAPACITY
