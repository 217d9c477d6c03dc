"""The C restatement of the half-step kick (oracle/gizmo_oracle.c, orc_kick)
against the reference's own do_the_kick (core/kicks.cc:284-545) compiled
from its sources into oracle/_ref: bit-exact on every kicked field, for the
kick that follows a real force pass and for constructed cases that reach
each limiter of the update."""
import numpy as np
import pytest

from gizmo_b200 import ics
from gizmo_b200.abi import METHOD_MFM, METHOD_MFV
from oracle import oracle as O

TIMEBASE = 2.0 ** -40  # physical time per integer tick


def _both(params, st, mode, min_egy_spec=0.0):
    out = {}
    for kind in ("port", "reference"):
        s = {k: v.copy() for k, v in st.items()}
        assert O.Oracle(params, kind).kick(s, mode, TIMEBASE, min_egy_spec) == 0
        out[kind] = s
    return out


def _assert_same(out):
    for name, _, _ in O.KICK_FIELDS:
        np.testing.assert_array_equal(out["port"][name], out["reference"][name], err_msg=name)


def _after_force(method):
    wl = ics.sedov(10, seed=5)
    wl.params.method = method
    if not O.ref_available(wl.params):
        pytest.skip("reference build not present")
    st = O.new_state(wl.n, wl.inputs())
    orc = O.Oracle(wl.params, "port", n_threads=1)
    assert orc.density(st) == 0 and orc.gradients(st) == 0 and orc.force(st) == 0
    steps = np.rint(st["dt"] / TIMEBASE).astype(np.int64)
    rng = np.random.default_rng(17)
    ks = O.new_kick_state(wl.n, {
        "vel": st["vel"], "u": st["u"], "mass": st["mass"], "mass_true": st["mass"],
        "dmass": st["dmass"], "dtmass": st["dtmass"], "accel": st["accel"], "dudt": st["dudt"],
        "grav": rng.normal(scale=0.1, size=(wl.n, 3)), "gravwork": st["gravwork"],
        "vel_pred": st["vel"], "u_pred": st["u"], "tstart": np.zeros(wl.n, np.int64), "tend": steps // 2,
        "active": np.ones(wl.n, np.int32)})
    return wl.params, ks, steps


@pytest.mark.parametrize("method", [METHOD_MFM, METHOD_MFV], ids=["mfm", "mfv"])
def test_kick_after_force_pass(method):
    params, ks, steps = _after_force(method)
    first = _both(params, ks, 0)
    _assert_same(first)
    # the second half kick starts from the first's result, over the other half of the step
    ks2 = first["reference"]
    ks2["tstart"] = steps // 2
    ks2["tend"] = steps
    second = _both(params, ks2, 1)
    _assert_same(second)
    s = second["reference"]
    assert np.array_equal(s["vel_pred"], s["vel"]) and np.array_equal(s["u_pred"], s["u"])
    if method == METHOD_MFV:
        assert np.array_equal(s["mass"], s["mass_true"])


def _constructed(n, seed):
    """Cases for every branch: the MFV mass limiter (opposite signs, overshoot,
    the -0.99 MassTrue floor, dMass = 0), inactive bins, the positivity halving,
    the temperature floor and a zero mass."""
    rng = np.random.default_rng(seed)
    mass = rng.uniform(0.5, 2.0, n)
    mass_true = mass * rng.uniform(0.9, 1.1, n)
    dmass = rng.normal(scale=0.05, size=n) * mass_true
    dtmass = rng.normal(scale=1.0, size=n) * mass_true
    sel = rng.integers(0, 6, n)
    dmass[sel == 0] = 0.0
    dmass[sel == 1] = -2.0 * mass_true[sel == 1]             # below -0.99 MassTrue,
    dtmass[sel == 1] = -1e13 * mass_true[sel == 1]           # in both half kicks
    dtmass[sel == 2] = -np.sign(dmass[sel == 2]) * 50.0       # opposite sign to dMass
    dtmass[sel == 3] = np.sign(dmass[sel == 3]) * 1e6         # overshoots dMass
    u = rng.uniform(0.1, 10.0, n)
    dudt = rng.normal(scale=5.0, size=n)
    steps = rng.integers(1, 2 ** 30, n).astype(np.int64)
    dudt[sel == 4] = -1e3 * u[sel == 4] / (steps[sel == 4] * TIMEBASE)  # below half: the halving catch
    mass[0] = 0.0
    return O.new_kick_state(n, {
        "vel": rng.normal(size=(n, 3)), "u": u, "mass": mass, "mass_true": mass_true, "dmass": dmass,
        "dtmass": dtmass, "accel": rng.normal(scale=1e3, size=(n, 3)), "dudt": dudt,
        "grav": rng.normal(scale=10.0, size=(n, 3)), "gravwork": rng.normal(size=(n, 3)),
        "vel_pred": rng.normal(size=(n, 3)), "u_pred": rng.uniform(0.1, 10.0, n), "dp": rng.normal(size=(n, 3)),
        "tstart": np.zeros(n, np.int64), "tend": steps, "active": (rng.random(n) < 0.8).astype(np.int32)})


@pytest.mark.parametrize("method", [METHOD_MFM, METHOD_MFV], ids=["mfm", "mfv"])
@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("floor", [0.0, 3.0])
def test_kick_constructed_cases(method, mode, floor):
    wl = ics.sedov(4, seed=1)
    wl.params.method = method
    if not O.ref_available(wl.params):
        pytest.skip("reference build not present")
    ks = _constructed(4096, seed=100 + 10 * mode + method)
    out = _both(wl.params, ks, mode, floor)
    _assert_same(out)
    r = out["reference"]
    act = ks["active"] == 1
    # the zero-mass cell is not kicked at all (the kick loops skip it)
    for name, _, _ in O.KICK_FIELDS:
        assert np.array_equal(r[name][0], ks[name][0]), name
    # inactive particles keep their velocity and energy
    assert np.array_equal(r["vel"][~act], ks["vel"][~act]) and np.array_equal(r["u"][~act], ks["u"][~act])
    if floor:
        assert (r["u"][act] >= floor).all()
        floored = act & (r["u"] == floor)
        assert floored.any() and (r["dudt"][floored] == 0).all()
    if method == METHOD_MFV:
        assert (r["mass_true"] > 0).all()
        if mode == 0:  # every kicked cell hands over its whole dMass
            assert (r["dmass"][1:] == 0).all()
