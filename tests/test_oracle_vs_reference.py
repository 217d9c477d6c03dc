"""The C oracle against the reference's own pair bodies compiled from its
sources (oracle/_ref), on seeded inputs beyond the fixtures: larger sets,
active subsets, the first-step tolerance, and both methods and kernels."""
import numpy as np
import pytest

from gizmo_b200 import abi, ics
from oracle import oracle as O
from tests._util import DENSITY_FIELDS, FORCE_FIELDS, GRADIENT_FIELDS, riemann_fallback_case, riemann_failure_case


def _cases():
    out = []
    for name, make in [("sedov12", lambda: ics.sedov(12, seed=7)),
                       ("plummer12", lambda: ics.plummer_mix(12, seed=8, n_spheres=6)),
                       ("lognormal12", lambda: ics.lognormal(12, seed_density=9, seed_velocity=10, grid=24))]:
        out.append((name, make))
    return out


@pytest.mark.parametrize("name,make", _cases(), ids=[c[0] for c in _cases()])
@pytest.mark.parametrize("subset", [False, True])
def test_port_equals_reference(name, make, subset):
    wl = make()
    if not O.ref_available(wl.params):
        pytest.skip("reference build not present")
    active = None
    if subset:
        rng = np.random.default_rng(11)
        active = np.sort(rng.choice(wl.n, size=wl.n // 3, replace=False)).astype(np.int32)
    res = {}
    for kind in ("port", "reference"):
        st = O.new_state(wl.n, wl.inputs())
        orc = O.Oracle(wl.params, kind, n_threads=1)
        if subset:  # neighbours need a converged state first, as in a running simulation
            assert orc.density(st) == 0 and orc.gradients(st) == 0 and orc.force(st) == 0
        assert orc.density(st, active) == 0
        assert orc.gradients(st, active) == 0
        assert orc.force(st, active) == 0
        res[kind] = st
    for f in DENSITY_FIELDS + GRADIENT_FIELDS + FORCE_FIELDS + ["iters"]:
        a, b = res["port"][f], res["reference"][f]
        if f == "dmass":
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-14 * np.abs(b).max() + 1e-300)
        else:
            assert np.array_equal(a, b), f


def test_first_step_tolerance_reference():
    wl = ics.sedov(10, seed=3)
    wl.params.first_step = 1
    if not O.ref_available(wl.params):
        pytest.skip("reference build not present")
    sts = []
    for kind in ("port", "reference"):
        st = O.new_state(wl.n, wl.inputs())
        assert O.Oracle(wl.params, kind, n_threads=1).density(st) == 0
        sts.append(st)
    for f in DENSITY_FIELDS + ["iters"]:
        assert np.array_equal(sts[0][f], sts[1][f]), f


def test_density_sums_fixed_h_reference():
    wl = ics.plummer_mix(10, seed=5, n_spheres=5)
    if not O.ref_available(wl.params):
        pytest.skip("reference build not present")
    st = O.new_state(wl.n, wl.inputs())
    a1, p1 = O.Oracle(wl.params, "port", n_threads=1).density_sums(st)
    a2, p2 = O.Oracle(wl.params, "reference", n_threads=1).density_sums(st)
    assert np.array_equal(a1, a2) and np.array_equal(p1, p2)


@pytest.mark.parametrize("method", [abi.METHOD_MFM, abi.METHOD_MFV], ids=["mfm", "mfv"])
def test_riemann_fallbacks_port_equals_reference(method):
    """Faces that take the exact iterative Riemann solver and the retry with
    cell-centred states: the port equals the reference bit for bit."""
    wl = riemann_fallback_case(method)
    if not O.ref_available(wl.params):
        pytest.skip("reference build not present")
    res = {}
    for kind in ("port", "reference"):
        st = O.new_state(wl.n, wl.inputs())
        orc = O.Oracle(wl.params, kind, n_threads=1)
        assert orc.density(st) == 0 and orc.gradients(st) == 0 and orc.force(st) == 0
        if kind == "port":
            branches = orc.riemann_branches()
        res[kind] = st
    assert branches["exact"] > 100 and branches["retry_centred"] > 100, branches
    for f in DENSITY_FIELDS + GRADIENT_FIELDS + FORCE_FIELDS:
        a, b = res["port"][f], res["reference"][f]
        if f == "dmass":
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-14 * np.abs(b).max() + 1e-300)
        else:
            assert np.array_equal(a, b), f


@pytest.mark.parametrize("method", [abi.METHOD_MFM, abi.METHOD_MFV], ids=["mfm", "mfv"])
def test_riemann_failure_stops_like_the_reference(method):
    """A NaN star pressure runs the whole cascade -- Kurganov-Tadmor, the exact
    solver, both retries -- and stops the pass with 1234 on both sides."""
    wl = riemann_failure_case(method)
    if not O.ref_available(wl.params):
        pytest.skip("reference build not present")
    for kind in ("port", "reference"):
        st = O.new_state(wl.n, wl.inputs())
        orc = O.Oracle(wl.params, kind, n_threads=1)
        assert orc.density(st) == 0 and orc.gradients(st) == 0
        assert orc.force(st) == abi.ERR_RIEMANN, kind
        if kind == "port":
            b = orc.riemann_branches()
            assert b["kt"] > 0 and b["exact"] > 0 and b["retry_centred"] > 0 and b["retry_at_rest"] > 0, b
