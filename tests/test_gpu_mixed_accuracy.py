"""The mixed form against the FP64 form, particle by particle, at the north
star's bar: every particle within 1e-5 relative in h, rho, pressure, vsig and
the gradients, and in the rates dm/dt, dv/dt and du/dt on the scale of the pair
fluxes summed into them (gizmo_b200/accuracy.py states the denominators).

The cases are the named generators at sizes a GPU pass takes in milliseconds:
the Plummer mixture (MFV, HLLC, cubic kernel, 32 neighbours, density contrast
~1e5) and the log-normal field (MFM, Wendland C2, 64 neighbours, rms Mach 2)
at 64^3 = 262,144 particles, the Sedov blast at its full 32^3, and the
log-normal field at its full 128^3 from the benchmark's steady-state seed. Both forms
start from the same inputs and converge to bit-identical h (their density sums
and h-iteration are the same FP64 kernels), and their gradients are the same
FP64 sums, so these fields must agree exactly; the force pair is FP32 in the
mixed form, with the pairs whose FP32 branch decisions were too close to call
(or whose arithmetic cancelled beyond FP32's reach) evaluated again in FP64.
"""
import numpy as np
import pytest

from gizmo_b200 import abi, accuracy, ics
from gizmo_b200.hydro import HydroPass

pytestmark = pytest.mark.gpu


def _steady(wl):
    """The timed-pass seed of the benchmark: h converged once in FP64, then
    moved by U(-5%, 5%) (ics.steady_state_seed)."""
    wl.params.precision = abi.PRECISION_FP64
    with HydroPass(wl.params) as hp:
        hp.upload_workload(wl)
        hp.density()
        conv = hp.download(["h", "cond"])
    wl.h = ics.steady_state_seed(conv["h"], 4)
    wl.cond = conv["cond"]
    return wl


CASES = {
    "plummer64": lambda: ics.plummer_mix(64, seed=4),
    "lognormal64": lambda: ics.lognormal(64, seed_density=2, seed_velocity=3),
    "sedov32": lambda: ics.sedov(32, seed=1),
    # the log-normal field's full size (2,097,152 particles, gamma = 1.0001): the near-isothermal
    # exact-solver pairs and the faces at the entropic switch's opening test
    "lognormal128": lambda: _steady(ics.lognormal(128, seed_density=2, seed_velocity=3)),
}


def _pass(wl, precision, flux_abs=False):
    wl.params.precision = precision
    with HydroPass(wl.params) as hp:
        hp.upload_workload(wl)
        if flux_abs:
            hp.set_diagnostics(flux_abs=True)
        hp.full_pass()
        names = list(accuracy.FIELDS) + ["iters", "num_ngb", "nvt", "cond"] + (["flux_abs"] if flux_abs else [])
        out = hp.download(names)
        out["status"] = hp.status()
    return out


@pytest.fixture(scope="module", params=list(CASES))
def forms(request):
    wl = CASES[request.param]()
    o64 = _pass(wl, abi.PRECISION_FP64, flux_abs=True)
    o32 = _pass(wl, abi.PRECISION_MIXED)
    return request.param, wl, o64, o32


def test_density_and_gradients_identical(forms):
    _, _, o64, o32 = forms
    for f in ("h", "rho", "pressure", "iters", "num_ngb", "nvt", "cond", "grad_rho", "grad_p", "grad_v"):
        assert np.array_equal(o32[f], o64[f]), f


def test_every_particle_within_1e5(forms):
    name, wl, o64, o32 = forms
    cs = accuracy.sound_speed(wl.params.gamma, o64["pressure"], o64["rho"])
    scales = accuracy.flux_scales(wl.vel, wl.mass, wl.u, o64["flux_abs"], wl.params.method == abi.METHOD_MFV, cs)
    err = accuracy.per_particle(o32, o64, scales)
    s = accuracy.summary(err, 1e-5)
    worst = {f: s[f]["max"] for f in accuracy.FIELDS}
    assert s["particles_above_bar_any_field"] == 0, (name, worst)
    # the FP64 re-evaluation is the exception, not the rule
    assert o32["status"]["pairs_refined"] < 0.02 * o32["status"]["pairs_symmetric"] / 2, o32["status"]


def test_rates_conserve_in_both_forms(forms):
    _, wl, o64, o32 = forms
    mfv = wl.params.method == abi.METHOD_MFV
    for o in (o64, o32):
        dtm = o["dtmass"] if mfv else np.zeros(wl.n)
        mom = wl.mass[:, None] * o["accel"] + wl.vel * dtm[:, None]
        assert np.abs(mom.sum(0)).max() <= 1e-12 * np.abs(mom).sum()
        if mfv:
            assert abs(dtm.sum()) <= 1e-12 * np.abs(dtm).sum()
