"""Whole steps of the integration loop on the device (gizmo_b200/step.py:
gz_timestep, gz_kick, gz_drift and the hydro pass through gz_upload_device /
gz_download_device, in the reference's order, core/run.cc:148-489), on the
periodic 3-D shock tube of tests/test_oracle_step_conservation.py, against the
oracle's chain of the same pieces:

  * MFM stays within the bars of the reference's own
    test/shocktube/test_shocktube.py:75-84 (energy 1e-5, momentum 1e-10 in
    units of sqrt(2 M E), mass 1e-12), and MFV conserves the conserved mass
    exactly (with the dMass the last kick still owes);
  * the same integer timeline as the oracle chain, and every cell's position,
    velocity, internal energy and mass within 1e-8 of it after six steps (the
    pass agrees with the oracle to summation order, 1e-10, and the steps carry
    those differences on).
"""
import numpy as np
import pytest

from gizmo_b200 import abi, ics
from gizmo_b200.step import DeviceStep
from tests.test_oracle_step_conservation import TIMEBASE, _errors, _run, _totals

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method", [abi.METHOD_MFM, abi.METHOD_MFV], ids=["mfm", "mfv"])
def test_device_steps_follow_the_oracle_chain(method):
    courant, n_steps = 0.05, 6
    start_o, end_o, ti_o = _run(method, n_steps, courant=courant)
    ref = _run.final
    wl = ics.shock_tube(12, seed=5)
    wl.params.method = method
    tp = abi.GzTimestepParams()
    tp.err_tol_int_accuracy, tp.courant_fac = 0.02, courant
    tp.max_size_timestep, tp.min_size_timestep, tp.timebase = 1e-2, 0.0, TIMEBASE
    for b in range(abi.TIMEBINS):
        tp.bin_active[b] = 1
    ds = DeviceStep(wl.params, tp, wl.pos, wl.vel, wl.mass, wl.u, wl.h)
    try:
        s = ds.state
        start = _totals((s["mass_true"] if method == abi.METHOD_MFV else s["mass"]).cpu().numpy(),
                        s["vel"].cpu().numpy(), s["u"].cpu().numpy())
        for _ in range(n_steps):
            ds.step()
        got = {k: v.cpu().numpy() for k, v in ds.state.items()}
        ti = ds.ti
    finally:
        ds.close()
    assert ti == ti_o
    mass_cons = got["mass_true"] + (got["dmass"] if method == abi.METHOD_MFV else 0.0)
    end = _totals(mass_cons, got["vel"], got["u"])
    energy, momentum, mass = _errors(start, end)
    assert mass < 1e-12
    if method == abi.METHOD_MFM:
        assert energy < 1e-5 and momentum < 1e-10
    for k in ("pos", "vel", "u", "mass"):
        scale = np.abs(ref[k]).max()
        assert np.abs(got[k] - ref[k]).max() <= 1e-8 * scale, (k, np.abs(got[k] - ref[k]).max() / scale)
