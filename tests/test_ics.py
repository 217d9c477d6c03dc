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


def test_shock_tube_states():
    wl = ics.shock_tube(10, seed=5)
    _check(wl)
    assert wl.params.method == 0 and wl.params.kernel == 3
    n = np.asarray(wl.meta["normal"])
    left = (wl.pos - 0.5) @ n < 0
    rho = wl.mass * wl.n  # equal lattice volumes: the density follows the mass
    rho_l, rho_r = wl.meta["rho"]
    p_l, p_r = wl.meta["p"]
    assert 0.125 <= min(rho_l, rho_r) and max(rho_l, rho_r) <= 1.0
    assert np.allclose(rho[left], rho_l) and np.allclose(rho[~left], rho_r)
    P = (wl.params.gamma - 1.0) * rho * wl.u
    assert np.allclose(P[left], p_l) and np.allclose(P[~left], p_r)
    assert np.all(wl.vel == 0)


def test_boxes_batch():
    a = ics.boxes(6, seed=5, n_min=1024, n_max=4096)
    b = ics.boxes(6, seed=5, n_min=1024, n_max=4096)
    assert [w.name for w in a] == [w.name for w in b]
    for x, y in zip(a, b):
        _check(x)
        assert np.array_equal(x.pos, y.pos) and np.array_equal(x.u, y.u)
        assert 4 ** 3 <= x.n and round(x.n ** (1 / 3)) ** 3 == x.n
    assert {w.name for w in a} == {"shock_tube", "sedov"}
