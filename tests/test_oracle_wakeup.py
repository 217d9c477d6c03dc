"""The wake-up of inactive neighbours in the force pass (hydro_functions.h:
534-544), restated in oracle/gizmo_oracle.c (orc_force_wakeup), against the
reference's own pair body compiled into oracle/_ref with a TimeBinActive
table handed to it: equal wake-up flags, and the force outputs unchanged by
the wake-up. An inactive neighbour is flagged with the largest bin + 1 of the
active targets whose pair signal speed exceeds WAKEUP (4.1) times its stored
signal speed."""
import numpy as np
import pytest

from gizmo_b200 import ics
from gizmo_b200.abi import METHOD_MFM, METHOD_MFV
from oracle import oracle as O
from tests._util import FORCE_FIELDS


@pytest.mark.parametrize("build", ["sedov_mfm", "sedov_mfv", "lognormal_mfm_wendland"])
def test_wakeup_port_equals_reference(build):
    if build.startswith("sedov"):
        wl = ics.sedov(12, seed=7)
        wl.params.method = METHOD_MFV if build.endswith("mfv") else METHOD_MFM
    else:
        wl = ics.lognormal(12, seed_density=2, seed_velocity=3, grid=24)
    if not O.ref_available(wl.params):
        pytest.skip("reference build not present")
    base = O.new_state(wl.n, wl.inputs())
    orc = O.Oracle(wl.params, "port", n_threads=1)
    assert orc.density(base) == 0 and orc.gradients(base) == 0 and orc.force(base) == 0
    rng = np.random.default_rng(19)
    base["timebin"][...] = rng.integers(10, 15, wl.n)
    bins = np.zeros(O.TIMEBINS, np.int32)
    bins[[10, 11]] = 1  # the short steps end here
    active = np.nonzero(bins[base["timebin"]])[0].astype(np.int32)
    inactive = bins[base["timebin"]] == 0
    slow = inactive & (rng.random(wl.n) < 0.5)
    base["vsig"][slow] *= 0.05  # stored signal speeds too slow for some of their active neighbours
    res = {}
    for kind in ("port", "reference"):
        st = {k: v.copy() for k, v in base.items()}
        assert O.Oracle(wl.params, kind, n_threads=1).force_wakeup(st, bins, active) == 0
        res[kind] = st
    assert np.array_equal(res["port"]["wakeup"], res["reference"]["wakeup"])
    for f in FORCE_FIELDS:
        a, b = res["port"][f], res["reference"][f]
        if f == "dmass":
            np.testing.assert_allclose(a, b, rtol=0, atol=1e-14 * np.abs(b).max() + 1e-300)
        else:
            assert np.array_equal(a, b), f
    woke = res["reference"]["wakeup"] > 0
    assert woke.any() and not woke[~inactive].any()  # only inactive cells are woken
    assert set(np.unique(res["reference"]["wakeup"][woke])) <= {11, 12}  # an active bin + 1
    # without the table nothing is woken, and the outputs are the same
    st = {k: v.copy() for k, v in base.items()}
    assert O.Oracle(wl.params, "port", n_threads=1).force(st, active) == 0
    assert (st["wakeup"] == 0).all()
    for f in FORCE_FIELDS:
        assert np.array_equal(st[f], res["port"][f]), f
