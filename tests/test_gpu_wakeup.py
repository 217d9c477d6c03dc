"""Individual timesteps on the device, through the C ABI, against the oracle:

  * the wake-up of inactive neighbours in a force pass over an active subset
    (hydro_functions.h:534-544; oracle orc_force_wakeup, itself pinned to the
    reference's pair body in tests/test_oracle_wakeup.py): equal flags in both
    arithmetic forms, the oracle fed the GPU's own density and gradient
    outputs (as in test_gpu_parity.passwise) so that both test the same pairs;
  * make_list_of_active_particles (core/run.cc:997-1010): gz_active_list;
  * the bin rule of process_wake_ups (core/timestep.cc:1565-1700):
    gz_wakeup_bins against orc_wakeup_bins on the flags of that pass.
"""
import numpy as np
import pytest

from gizmo_b200 import abi, ics
from gizmo_b200.hydro import HydroPass
from oracle import oracle as O
from tests._util import DENSITY_FIELDS, FORCE_FIELDS, GRADIENT_FIELDS, field_err

pytestmark = pytest.mark.gpu

BUILDS = {
    "sedov_mfm": lambda: ics.sedov(12, seed=7),
    "sedov_mfv": lambda: ics.sedov(12, seed=7),
    "lognormal_mfm_wendland": lambda: ics.lognormal(12, seed_density=2, seed_velocity=3, grid=24),
    "plummer_mfv": lambda: ics.plummer_mix(16, seed=4, n_spheres=12),
}


def _case(build):
    wl = BUILDS[build]()
    if build == "sedov_mfv":
        wl.params.method = abi.METHOD_MFV
    st = O.new_state(wl.n, wl.inputs())
    orc = O.Oracle(wl.params, "port")
    assert orc.density(st) == 0 and orc.gradients(st) == 0 and orc.force(st) == 0
    rng = np.random.default_rng(19)
    timebin = rng.integers(10, 15, wl.n).astype(np.int32)
    bins = np.zeros(O.TIMEBINS, np.int32)
    bins[[10, 11]] = 1  # the short steps end here
    inactive = bins[timebin] == 0
    vsig = st["vsig"].copy()
    slow = inactive & (rng.random(wl.n) < 0.5)
    vsig[slow] *= 0.05  # stored signal speeds too slow for some of their active neighbours
    wl.h = st["h"].copy()  # converged kernel lengths, as a step after the first starts from
    wl.cond = st["cond"].copy()
    return wl, timebin, vsig, bins


@pytest.mark.parametrize("build", list(BUILDS))
def test_wakeup_flags_match_oracle(build):
    wl, timebin, vsig, bins = _case(build)
    active = np.nonzero(bins[timebin])[0].astype(np.int32)
    flags = {}
    for precision in (abi.PRECISION_FP64, abi.PRECISION_MIXED):
        wl.params.precision = precision
        with HydroPass(wl.params) as hp:
            hp.upload(wl.pos, wl.vel, wl.mass, wl.u, wl.dt, wl.h, wl.cond, timebin=timebin, vsig=vsig)
            hp.density()
            hp.hydro_gradient_calc()
            state = hp.download(DENSITY_FIELDS + GRADIENT_FIELDS)
            hp.set_bin_active(bins)
            hp.hydro_force(active)
            out = hp.download(FORCE_FIELDS + ["wakeup"])
        flags[precision] = out["wakeup"]
        if precision == abi.PRECISION_FP64:
            # the oracle's force pass with the wake-up, from the GPU's density and gradients
            st = O.new_state(wl.n, wl.inputs())
            for f in DENSITY_FIELDS + GRADIENT_FIELDS:
                st[f][...] = state[f]
            st["vsig"][...] = vsig
            st["timebin"][...] = timebin
            assert O.Oracle(wl.params, "port").force_wakeup(st, bins, active) == 0
            for f in FORCE_FIELDS:
                assert field_err(f, out[f][active], st[f][active], 1e-3) < 1e-10, f
            want = st["wakeup"]
    assert np.array_equal(flags[abi.PRECISION_FP64], want)
    assert np.array_equal(flags[abi.PRECISION_MIXED], want)
    woke = want > 0
    assert woke.any() and not woke[bins[timebin] == 1].any()
    assert set(np.unique(want[woke])) <= {11, 12}


def test_active_list_and_wakeup_bins():
    wl, timebin, vsig, bins = _case("sedov_mfv")
    wl.mass = wl.mass.copy()
    wl.mass[::97] = 0.0  # cells without mass are never active and never move
    with HydroPass(wl.params) as hp:
        hp.upload(wl.pos, wl.vel, wl.mass, wl.u, wl.dt, wl.h, wl.cond, timebin=timebin, vsig=vsig)
        got = hp.active_list(bins)
        want = O.active_list(timebin, wl.mass, bins)
        assert np.array_equal(got, want) and len(want) > 0
        hp.full_pass()  # every cell's density and gradients, then the force pass of the active cells
        hp.set_bin_active(bins)
        hp.hydro_force(got)
        flags = hp.download(["wakeup"])["wakeup"]
        assert (flags > 0).any()
        for max_active, lowest in ((11, 10), (12, 10), (11, 11)):
            bins_got, moved_got = hp.wakeup_bins(bins, max_active, lowest)
            bins_want, moved_want = O.wakeup_bins(timebin, flags, wl.mass, bins, max_active, lowest)
            assert np.array_equal(bins_got, bins_want) and moved_got == moved_want > 0
        # without a table nothing is woken
        hp.set_bin_active(None)
        hp.hydro_force(got)
        assert (hp.download(["wakeup"])["wakeup"] == 0).all()
