"""Whole steps of the integration loop, composed from the oracle's pieces in
the reference's order (core/run.cc:148, 239, 290, 312, 482, 489): an initial
hydro pass; then per step the timestep (orc_timestep), the first half kick
(orc_kick mode 0), the drift (orc_drift), the hydro pass on the predicted
state (orc_density / orc_gradients / orc_force) and the second half kick
(orc_kick mode 1), on a periodic 3-D shock tube with no gravity. This checks
that the kick, drift and timestep restatements compose with the pass the way
the reference's loop composes them.

MFM meets the bars of the reference's own test/shocktube/test_shocktube.py:
75-84: energy 1e-5 relative, momentum 1e-10 in units of sqrt(2 M E), mass
1e-12 relative.

MFV conserves the conserved mass exactly, counting the dMass that the last
second half kick still owes the next first half kick. Its momentum and energy
are conserved only to the integration order. The force pass turns the
momentum flux into an acceleration by subtracting VelPred * DtMass
(src/hydro/hydro_toplevel.cc:225-232), while the kick moves P.Vel, so each
half kick changes the total momentum by sum(dm * (Vel - VelPred)), which is
O(dt^2). The test checks that both errors fall when the step is halved."""
import numpy as np
import pytest

from gizmo_b200 import ics
from gizmo_b200.abi import METHOD_MFM, METHOD_MFV
from oracle import oracle as O

TIMEBASE = 2.0 ** -40
PASS_FIELDS = ("accel", "dudt", "dtmass", "dmass", "gravwork", "vsig", "divvel", "rho", "pressure", "num_ngb",
               "pvel", "h", "cond")


def _hydro_pass(orc, wl, pos, vel_pred, mass, u_pred, dt_phys, h, cond):
    st = O.new_state(wl.n, {"pos": np.mod(pos, wl.params.box_size), "vel": vel_pred, "mass": mass, "u": u_pred,
                            "dt": np.full(wl.n, dt_phys), "h": h, "cond": cond})
    assert orc.density(st) == 0 and orc.gradients(st) == 0 and orc.force(st) == 0
    return {k: st[k] for k in PASS_FIELDS}


def _totals(mass, vel, u):
    return {"mass": mass.sum(), "momentum": (mass[:, None] * vel).sum(0),
            "energy": (mass * (u + 0.5 * (vel * vel).sum(1))).sum()}


def _run(method, n_steps, courant=0.2):
    wl = ics.shock_tube(12, seed=5)
    wl.params.method = method
    orc = O.Oracle(wl.params, "port", n_threads=1)
    n = wl.n
    # P.Vel, CellP.InternalEnergy, P.Mass / CellP.MassTrue and their predictions
    vel, u, mass = wl.vel.copy(), wl.u.copy(), wl.mass.copy()
    mass_true = mass.copy()
    pos, vel_pred, u_pred = wl.pos.copy(), vel.copy(), u.copy()
    h, cond = wl.h.copy(), np.zeros(n)
    tp = O.OrcTimestepParams()
    tp.err_tol_int_accuracy, tp.courant_fac = 0.02, courant
    tp.max_size_timestep, tp.min_size_timestep, tp.timebase = 1e-2, 0.0, TIMEBASE
    for b in range(O.TIMEBINS):
        tp.bin_active[b] = 1
    ti = 0
    # at start-up no step has been assigned yet (dt_step = 0), so the first pass books no dMass
    out = _hydro_pass(orc, wl, pos, vel_pred, mass, u_pred, 0.0, h, cond)
    h, cond = out["h"], out["cond"]
    start = _totals(mass_true if method == METHOD_MFV else mass, vel, u)
    for _ in range(n_steps):
        tp.ti_current = ti
        ts = O.new_timestep_state(n, {"accel": out["accel"], "vsig": out["vsig"], "h": h, "num_ngb": out["num_ngb"],
                                      "divvel": out["divvel"], "mass": mass, "softening": np.zeros(n)})
        assert orc.timestep(ts, tp) == 0
        step = int(ts["dt_step"].min())  # one global step: every cell on the smallest bin
        half = step // 2
        ks = O.new_kick_state(n, {
            "vel": vel, "u": u, "mass": mass, "mass_true": mass_true, "dmass": out["dmass"], "dtmass": out["dtmass"],
            "accel": out["accel"], "dudt": out["dudt"], "gravwork": out["gravwork"], "vel_pred": vel_pred,
            "u_pred": u_pred, "tstart": np.full(n, ti), "tend": np.full(n, ti + half), "active": np.ones(n, np.int32)})
        assert orc.kick(ks, 0, TIMEBASE) == 0
        vel, u, mass, mass_true = ks["vel"], ks["u"], ks["mass"], ks["mass_true"]
        dmass_left = ks["dmass"]
        ds = O.new_drift_state(n, {
            "pos": pos, "vel": vel, "pvel": out["pvel"], "vel_pred": vel_pred, "accel": out["accel"],
            "divvel": out["divvel"], "mass": mass, "dtmass": out["dtmass"], "mass_true": mass_true, "rho": out["rho"],
            "u_pred": u_pred, "dudt": out["dudt"], "h": h, "pressure": out["pressure"], "ti_current": np.full(n, ti)})
        assert orc.drift(ds, ti + step, TIMEBASE) == 0
        pos, vel_pred, mass, u_pred, h = ds["pos"], ds["vel_pred"], ds["mass"], ds["u_pred"], ds["h"]
        out = _hydro_pass(orc, wl, pos, vel_pred, mass, u_pred, step * TIMEBASE, h, cond)
        h, cond = out["h"], out["cond"]
        # the part of last step's dMass the first half kick left (none: mode 0 hands over all of it)
        assert (dmass_left == 0).all()
        ks = O.new_kick_state(n, {
            "vel": vel, "u": u, "mass": mass, "mass_true": mass_true, "dmass": out["dmass"], "dtmass": out["dtmass"],
            "accel": out["accel"], "dudt": out["dudt"], "gravwork": out["gravwork"], "vel_pred": vel_pred,
            "u_pred": u_pred, "tstart": np.full(n, ti + half), "tend": np.full(n, ti + step),
            "active": np.ones(n, np.int32)})
        assert orc.kick(ks, 1, TIMEBASE) == 0
        vel, u, mass, mass_true = ks["vel"], ks["u"], ks["mass"], ks["mass_true"]
        vel_pred, u_pred = ks["vel_pred"], ks["u_pred"]
        out["dmass"] = ks["dmass"]  # what the next first half kick hands over
        ti += step
    # under MFV the conserved mass still owed by the last kick's dMass is part of the total
    end = _totals(mass_true + (out["dmass"] if method == METHOD_MFV else 0.0), vel, u)
    _run.final = {"pos": pos, "vel": vel, "u": u, "mass": mass, "mass_true": mass_true, "h": h,
                  "dmass": out["dmass"]}
    return start, end, ti


def _errors(start, end):
    scale = np.sqrt(2.0 * start["mass"] * abs(start["energy"]))
    return (abs(end["energy"] - start["energy"]) / abs(start["energy"]),
            float(np.linalg.norm(end["momentum"] - start["momentum"]) / scale),
            abs(end["mass"] - start["mass"]) / start["mass"])


def test_mfm_steps_conserve_within_the_reference_bars():
    start, end, ti = _run(METHOD_MFM, 6, courant=0.05)
    assert ti > 0
    energy, momentum, mass = _errors(start, end)
    assert energy < 1e-5 and momentum < 1e-10 and mass < 1e-12


def test_mfv_steps_conserve_mass_and_converge_in_momentum_and_energy():
    coarse = _errors(*_run(METHOD_MFV, 6, courant=0.1)[:2])
    fine = _errors(*_run(METHOD_MFV, 6, courant=0.05)[:2])
    assert coarse[2] < 1e-12 and fine[2] < 1e-12
    assert fine[0] < coarse[0] / 2.5 and fine[1] < coarse[1] / 2.5
    assert fine[0] < 1e-4 and fine[1] < 1e-6
