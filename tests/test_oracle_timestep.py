"""The C restatement of the timestep criterion (oracle/gizmo_oracle.c,
orc_timestep) against the reference's own get_timestep (core/timestep.cc:
357-1416) compiled from its sources into oracle/_ref: the physical
acceleration and the wanted integer step bit-exact, for the timesteps that
follow a real force pass and for constructed cells in which each criterion
binds. The binning that follows (a power of two; a larger bin only where it is
synchronised; the end of the timeline) is the per-particle part of
find_timesteps (timestep.cc:176-270), restated on both sides; its outcome is
checked here against the rules themselves."""
import numpy as np
import pytest

from gizmo_b200 import ics
from gizmo_b200.abi import METHOD_MFM, METHOD_MFV
from oracle import oracle as O

TIMEBASE = 2.0 ** -40


def _params(ti_current=0, active_bins=range(O.TIMEBINS), max_dt=1e-2, min_dt=0.0):
    tp = O.OrcTimestepParams()
    tp.err_tol_int_accuracy = 0.02
    tp.courant_fac = 0.2
    tp.max_size_timestep = max_dt
    tp.min_size_timestep = min_dt
    tp.timebase = TIMEBASE
    tp.ti_current = ti_current
    for b in range(O.TIMEBINS):
        tp.bin_active[b] = 1 if b in set(active_bins) else 0
    return tp


def _both(params, st, tp):
    out, codes = {}, {}
    for kind in ("port", "reference"):
        s = {k: v.copy() for k, v in st.items()}
        codes[kind] = O.Oracle(params, kind).timestep(s, tp)
        out[kind] = s
    assert codes["port"] == codes["reference"]
    for name, _, _ in O.TIMESTEP_FIELDS:
        np.testing.assert_array_equal(out["port"][name], out["reference"][name], err_msg=name)
    return out["reference"], codes["reference"]


@pytest.mark.parametrize("method", [METHOD_MFM, METHOD_MFV], ids=["mfm", "mfv"])
def test_timestep_after_force_pass(method):
    wl = ics.sedov(10, seed=5)
    wl.params.method = method
    if not O.ref_available(wl.params):
        pytest.skip("reference build not present")
    st = O.new_state(wl.n, wl.inputs())
    orc = O.Oracle(wl.params, "port", n_threads=1)
    assert orc.density(st) == 0 and orc.gradients(st) == 0 and orc.force(st) == 0
    ts = O.new_timestep_state(wl.n, {
        "accel": st["accel"], "vsig": st["vsig"], "h": st["h"], "num_ngb": st["num_ngb"], "divvel": st["divvel"],
        "mass": st["mass"], "softening": np.full(wl.n, 1e-3), "bin": np.full(wl.n, 20, np.int32)})
    r, code = _both(wl.params, ts, _params())
    assert code == 0
    # the step is a power of two no larger than the wanted one
    assert ((r["dt_step"] & (r["dt_step"] - 1)) == 0).all() and (r["dt_step"] <= r["ti_want"]).all()


@pytest.mark.parametrize("build", ["mfm_cubic", "mfm_wendland_isothermal"])
def test_timestep_constructed_cases(build):
    """Each criterion binds somewhere: acceleration (with and without a
    softening), Courant, divergence, MaxSizeTimestep; zero mass (acceleration
    only); a bin that wants to grow into unsynchronised bins. Against the
    reference compiled for the Sedov build and for the log-normal one."""
    params = (ics.sedov(4, seed=1) if build == "mfm_cubic"
              else ics.lognormal(8, seed_density=2, seed_velocity=3, grid=16)).params
    if not O.ref_available(params):
        pytest.skip("reference build not present")
    n = 4096
    rng = np.random.default_rng(3)
    sel = rng.integers(0, 5, n)
    accel = rng.normal(size=(n, 3)) * 10.0 ** rng.uniform(-2, 6, (n, 1))
    vsig = 10.0 ** rng.uniform(-1, 3, n)
    divvel = rng.normal(size=n) * 10.0 ** rng.uniform(-1, 4, n)
    divvel[sel == 0] = 0.0
    softening = np.where(sel == 1, 0.0, 10.0 ** rng.uniform(-5, -2, n))
    mass = np.where(sel == 2, 0.0, 1.0)
    accel[sel == 3] = 0.0
    ts = O.new_timestep_state(n, {
        "grav": rng.normal(size=(n, 3)), "accel": accel, "vsig": vsig, "h": 10.0 ** rng.uniform(-3, -1, n),
        "num_ngb": rng.uniform(2.5, 4.5, n), "divvel": divvel, "mass": mass, "softening": softening,
        "bin": rng.integers(2, 30, n).astype(np.int32), "ti_begstep": rng.integers(0, 1 << 40, n),
        "dt_step": rng.integers(0, 1 << 20, n)})
    tp = _params(ti_current=1 << 41, active_bins=range(0, 60, 3))
    r, code = _both(params, ts, tp)
    assert code == 0
    grew = r["bin"] > ts["bin"]
    assert grew.any() and (~grew).any()
    assert all(tp.bin_active[b] for b in r["bin"][grew])  # a grown bin is a synchronised one
    assert (r["ti_begstep"] == ts["ti_begstep"] + ts["dt_step"]).all()


def test_timestep_below_the_floor_stops():
    params = ics.sedov(4, seed=1).params
    if not O.ref_available(params):
        pytest.skip("reference build not present")
    ts = O.new_timestep_state(8, {"accel": np.ones((8, 3)), "vsig": np.full(8, 1e12), "h": np.full(8, 1e-3),
                                  "num_ngb": np.full(8, 3.0), "mass": np.ones(8), "softening": np.full(8, 1e-3)})
    r, code = _both(params, ts, _params(min_dt=1e-6))
    assert code == 888
    assert (r["ti_want"] == int(1e-6 / TIMEBASE)).all()
