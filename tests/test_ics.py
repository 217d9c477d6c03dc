"""Synthetic workload generators: seeded, in the box, exact power-of-two timesteps."""
import numpy as np

from gizmo_b200 import ics


def _check(wl):
    assert wl.pos.shape == (wl.n, 3) and wl.vel.shape == (wl.n, 3)
    assert np.all(wl.pos >= 0) and np.all(wl.pos < 1)
    assert np.all(wl.h > 0) and np.all(wl.mass > 0) and np.all(wl.u > 0)
    k = -np.log2(wl.dt)
    assert np.array_equal(k, np.round(k))


def test_sedov_energy_and_determinism():
    a, b = ics.sedov(8, seed=1), ics.sedov(8, seed=1)
    _check(a)
    assert np.array_equal(a.pos, b.pos) and np.array_equal(a.u, b.u)
    e = (a.mass * (a.u - 1e-5)).sum()
    assert abs(e - 1.0) < 1e-12


def test_plummer_mix_shape():
    wl = ics.plummer_mix(12, seed=4, n_spheres=10)
    _check(wl)
    assert wl.params.method == 1 and wl.params.kernel == 3


def test_lognormal_shape():
    wl = ics.lognormal(10, grid=20)
    _check(wl)
    assert wl.params.kernel == 6 and wl.params.des_num_ngb == 64
