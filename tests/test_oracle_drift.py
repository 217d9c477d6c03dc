"""The C restatement of the drift (oracle/gizmo_oracle.c, orc_drift) against
the reference's own drift_particle_impl (core/drift_particle_functions.h:86-260)
called from oracle/_ref: bit-exact on every drifted field, after a real force
pass and on constructed cases that reach every cap, clamp and floor."""
import numpy as np
import pytest

from gizmo_b200 import abi, ics
from gizmo_b200.abi import METHOD_MFM, METHOD_MFV
from oracle import oracle as O

TIMEBASE = 2.0 ** -40  # physical time per integer tick


def _both(params, st, time1, min_egy_spec=0.0):
    out, codes = {}, {}
    for kind in ("port", "reference"):
        s = {k: v.copy() for k, v in st.items()}
        codes[kind] = O.Oracle(params, kind).drift(s, time1, TIMEBASE, min_egy_spec)
        out[kind] = s
    assert codes["port"] == codes["reference"]
    for name, _, _ in O.DRIFT_FIELDS:
        np.testing.assert_array_equal(out["port"][name], out["reference"][name], err_msg=name)
    return out["reference"], codes["reference"]


@pytest.mark.parametrize("method", [METHOD_MFM, METHOD_MFV], ids=["mfm", "mfv"])
def test_drift_after_force_pass(method):
    wl = ics.sedov(10, seed=5)
    wl.params.method = method
    if not O.ref_available(wl.params):
        pytest.skip("reference build not present")
    st = O.new_state(wl.n, wl.inputs())
    orc = O.Oracle(wl.params, "port", n_threads=1)
    assert orc.density(st) == 0 and orc.gradients(st) == 0 and orc.force(st) == 0
    steps = np.rint(st["dt"] / TIMEBASE).astype(np.int64)
    rng = np.random.default_rng(23)
    time1 = int(steps.max())
    ds = O.new_drift_state(wl.n, {
        "pos": st["pos"], "vel": st["vel"], "pvel": st["pvel"], "vel_pred": st["vel"],
        "grav": rng.normal(scale=0.1, size=(wl.n, 3)), "accel": st["accel"], "divvel": st["divvel"],
        "mass": st["mass"], "dtmass": st["dtmass"], "mass_true": st["mass"], "rho": st["rho"], "u_pred": st["u"],
        "dudt": st["dudt"], "h": st["h"], "pressure": st["pressure"],
        "ti_current": rng.integers(0, time1, wl.n).astype(np.int64)})
    r, code = _both(wl.params, ds, time1)
    assert code == 0
    assert (r["ti_current"] == time1).all()


def _constructed(n, seed, params):
    """Every branch: divv dt beyond both caps, h beyond both clamps, the MFV
    half-MassTrue floor, the positivity halving, the MinEgySpec floor, a zero
    mass (moved, not predicted) and a cell already at time1."""
    rng = np.random.default_rng(seed)
    t0 = rng.integers(0, 1 << 30, n).astype(np.int64)
    time1 = 1 << 30
    dt = (time1 - t0) * TIMEBASE
    sel = rng.integers(0, 6, n)
    divvel = rng.normal(scale=0.1, size=n) / np.maximum(dt, 1e-30)
    divvel[sel == 0] = 2.0 / dt[sel == 0]                            # above +0.3
    divvel[sel == 1] = -2.0 / dt[sel == 1]                           # below -0.3
    h = rng.uniform(0.5 * params.min_kernel_radius, 1.5 * params.max_kernel_radius, n)
    mass = rng.uniform(0.5, 2.0, n)
    mass_true = mass * rng.uniform(0.9, 1.1, n)
    dtmass = rng.normal(scale=0.1, size=n) * mass / np.maximum(dt, 1e-30)
    dtmass[sel == 2] = -3.0 * mass[sel == 2] / dt[sel == 2]         # below half MassTrue
    u = rng.uniform(0.1, 10.0, n)
    dudt = rng.normal(scale=0.1, size=n) * u / np.maximum(dt, 1e-30)
    dudt[sel == 3] = -10.0 * u[sel == 3] / dt[sel == 3]             # below half: the halving catch
    mass[0] = 0.0
    t0[1] = time1
    return O.new_drift_state(n, {
        "pos": rng.uniform(0, 1, (n, 3)), "vel": rng.normal(size=(n, 3)), "pvel": rng.normal(size=(n, 3)),
        "vel_pred": rng.normal(size=(n, 3)), "grav": rng.normal(scale=10.0, size=(n, 3)),
        "accel": rng.normal(scale=1e3, size=(n, 3)), "divvel": divvel, "mass": mass, "dtmass": dtmass,
        "mass_true": mass_true, "rho": rng.uniform(0.1, 10.0, n), "u_pred": u, "dudt": dudt, "h": h,
        "pressure": rng.uniform(0.1, 1.0, n), "ti_current": t0}), time1


@pytest.mark.parametrize("method", [METHOD_MFM, METHOD_MFV], ids=["mfm", "mfv"])
@pytest.mark.parametrize("floor", [0.0, 3.0])
def test_drift_constructed_cases(method, floor):
    params = ics.sedov(4, seed=1).params
    params.method = method
    params.min_kernel_radius, params.max_kernel_radius = 0.05, 0.5
    if not O.ref_available(params):
        pytest.skip("reference build not present")
    ds, time1 = _constructed(4096, 200 + method, params)
    r, code = _both(params, ds, time1, floor)
    assert code == 0
    assert (r["h"][2:] >= params.min_kernel_radius).all() and (r["h"][2:] <= params.max_kernel_radius).all()
    for name in ("h", "rho", "u_pred", "vel_pred", "mass"):  # the zero-mass cell is moved, not predicted
        assert np.array_equal(r[name][0], ds[name][0]), name
    assert not np.array_equal(r["pos"][0], ds["pos"][0])
    for name, _, _ in O.DRIFT_FIELDS:  # the cell already at time1 is left alone
        assert np.array_equal(r[name][1], ds[name][1]), name
    if floor:
        assert (r["u_pred"][2:] >= floor).all()



def test_drift_isothermal_wendland_build():
    """The build of the log-normal workload (MFM, Wendland C2, gamma = 1.0001): the
    pressure of a drifted cell carries gamma - 1 = 1e-4."""
    params = ics.lognormal(8, seed_density=2, seed_velocity=3, grid=16).params
    params.min_kernel_radius, params.max_kernel_radius = 0.05, 0.5
    if not O.ref_available(params):
        pytest.skip("reference build not present")
    ds, time1 = _constructed(2048, 210, params)
    r, code = _both(params, ds, time1, 3.0)
    assert code == 0


def test_drift_into_the_past_is_refused():
    params = ics.sedov(4, seed=1).params
    if not O.ref_available(params):
        pytest.skip("reference build not present")
    ds, time1 = _constructed(64, 9, params)
    ds["ti_current"][5] = time1 + 1
    r, code = _both(params, ds, time1)
    assert code == abi.ERR_NO_PAST_DRIFT
    for name, _, _ in O.DRIFT_FIELDS:
        assert np.array_equal(r[name][5], ds[name][5]), name
