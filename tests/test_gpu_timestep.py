"""gz_timestep, the timestep criterion on the device (get_timestep,
core/timestep.cc:357-1416, and the per-particle binning of find_timesteps,
timestep.cc:176-270), against the oracle's restatement orc_timestep (itself
pinned to the reference's compiled get_timestep in tests/test_oracle_timestep.py):
the physical acceleration, the wanted integer step, the bin, Ti_begstep and
dt_step bit for bit, and the stop codes, on the cells that follow a real
force pass and on constructed cells in which each criterion binds."""
import ctypes as C

import numpy as np
import pytest

from gizmo_b200 import abi, ics
from gizmo_b200.hydro import timestep
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TIMEBASE = 2.0 ** -40
OUT = ("aphys", "ti_want", "bin", "ti_begstep", "dt_step")


def _params(ti_current=0, active_bins=range(O.TIMEBINS), max_dt=1e-2, min_dt=0.0):
    tp, gp = O.OrcTimestepParams(), abi.GzTimestepParams()
    for t in (tp, gp):
        t.err_tol_int_accuracy = 0.02
        t.courant_fac = 0.2
        t.max_size_timestep = max_dt
        t.min_size_timestep = min_dt
        t.timebase = TIMEBASE
        t.ti_current = ti_current
        for b in range(O.TIMEBINS):
            t.bin_active[b] = 1 if b in set(active_bins) else 0
    return tp, gp


def _both(params, st, tp, gp):
    import torch

    ref = {k: v.copy() for k, v in st.items()}
    code = O.Oracle(params, "port").timestep(ref, tp)
    dev = torch.device("cuda", 0)
    fields = {k: torch.as_tensor(np.ascontiguousarray(v), device=dev) for k, v in st.items()}
    fields["status"] = torch.zeros(1, dtype=torch.int32, device=dev)
    timestep(params, gp, fields, torch.cuda.current_stream(dev).cuda_stream)
    torch.cuda.synchronize()
    got = {k: fields[k].cpu().numpy() for k in OUT}
    for k in OUT:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    assert int(fields["status"].item()) == code
    return got, code


@pytest.mark.parametrize("method", [abi.METHOD_MFM, abi.METHOD_MFV], ids=["mfm", "mfv"])
def test_timestep_after_force_pass(method):
    wl = ics.sedov(10, seed=5)
    wl.params.method = method
    st = O.new_state(wl.n, wl.inputs())
    orc = O.Oracle(wl.params, "port")
    assert orc.density(st) == 0 and orc.gradients(st) == 0 and orc.force(st) == 0
    ts = O.new_timestep_state(wl.n, {
        "accel": st["accel"], "vsig": st["vsig"], "h": st["h"], "num_ngb": st["num_ngb"], "divvel": st["divvel"],
        "mass": st["mass"], "softening": np.full(wl.n, 1e-3), "bin": np.full(wl.n, 20, np.int32)})
    got, code = _both(wl.params, ts, *_params())
    assert code == 0 and ((got["dt_step"] & (got["dt_step"] - 1)) == 0).all()


@pytest.mark.parametrize("build", ["mfm_cubic", "mfm_wendland_isothermal"])
def test_timestep_constructed_cases(build):
    params = (ics.sedov(4, seed=1) if build == "mfm_cubic"
              else ics.lognormal(8, seed_density=2, seed_velocity=3, grid=16)).params
    n = 1 << 16
    rng = np.random.default_rng(3)
    sel = rng.integers(0, 5, n)
    accel = rng.normal(size=(n, 3)) * 10.0 ** rng.uniform(-2, 6, (n, 1))
    divvel = rng.normal(size=n) * 10.0 ** rng.uniform(-1, 4, n)
    divvel[sel == 0] = 0.0
    accel[sel == 3] = 0.0
    ts = O.new_timestep_state(n, {
        "grav": rng.normal(size=(n, 3)), "accel": accel, "vsig": 10.0 ** rng.uniform(-1, 3, n),
        "h": 10.0 ** rng.uniform(-3, -1, n), "num_ngb": rng.uniform(2.5, 4.5, n), "divvel": divvel,
        "mass": np.where(sel == 2, 0.0, 1.0), "softening": np.where(sel == 1, 0.0, 10.0 ** rng.uniform(-5, -2, n)),
        "bin": rng.integers(2, 30, n).astype(np.int32), "ti_begstep": rng.integers(0, 1 << 40, n),
        "dt_step": rng.integers(0, 1 << 20, n)})
    got, code = _both(params, ts, *_params(ti_current=1 << 41, active_bins=range(0, 60, 3)))
    assert code == 0
    grew = got["bin"] > ts["bin"]
    assert grew.any() and (~grew).any()


def test_timestep_stop_codes():
    params = ics.sedov(4, seed=1).params
    ts = O.new_timestep_state(8, {"accel": np.ones((8, 3)), "vsig": np.full(8, 1e12), "h": np.full(8, 1e-3),
                                  "num_ngb": np.full(8, 3.0), "mass": np.ones(8), "softening": np.full(8, 1e-3)})
    _, code = _both(params, ts, *_params(min_dt=1e-6))
    assert code == abi.ERR_MIN_TIMESTEP
    ts = O.new_timestep_state(8, {"accel": np.ones((8, 3)), "vsig": np.full(8, 1.0), "h": np.full(8, 1e-3),
                                  "num_ngb": np.full(8, 3.0), "mass": np.ones(8), "softening": np.full(8, 1e-3)})
    _, code = _both(params, ts, *_params(ti_current=(1 << 60) - 64))
    assert code == abi.ERR_END_OF_TIMELINE
