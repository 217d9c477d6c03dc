"""gz_kick, the half-step kick on the device, against the oracle's orc_kick
(itself pinned bit-exact to the reference's compiled do_the_kick): bit-exact
on every kicked field, for the constructed cases that reach every limiter, a
set of 4M particles (many grid-stride rounds) and the optional fields left
out."""
import numpy as np
import pytest

from gizmo_b200 import hydro, ics
from gizmo_b200.abi import METHOD_MFM, METHOD_MFV
from oracle import oracle as O
from tests.test_oracle_kick import TIMEBASE, _constructed

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _params(method):
    p = ics.sedov(4, seed=1).params
    p.method = method
    return p


def _device_kick(params, ks, mode, floor, drop=()):
    dev = {k: torch.from_numpy(v.copy()).cuda() for k, v in ks.items() if k not in drop}
    hydro.kick(params, dev, mode, TIMEBASE, floor)
    torch.cuda.synchronize()
    out = {k: v.cpu().numpy() for k, v in dev.items()}
    for k in drop:
        out[k] = ks[k].copy()
    return out


def _oracle_kick(params, ks, mode, floor):
    s = {k: v.copy() for k, v in ks.items()}
    assert O.Oracle(params, "port").kick(s, mode, TIMEBASE, floor) == 0
    return s


def _assert_same(got, want):
    for name, _, _ in O.KICK_FIELDS:
        np.testing.assert_array_equal(got[name], want[name], err_msg=name)


@pytest.mark.parametrize("method", [METHOD_MFM, METHOD_MFV], ids=["mfm", "mfv"])
@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("floor", [0.0, 3.0])
def test_device_kick_constructed_cases(method, mode, floor):
    params = _params(method)
    ks = _constructed(4096, seed=100 + 10 * mode + method)
    _assert_same(_device_kick(params, ks, mode, floor), _oracle_kick(params, ks, mode, floor))


@pytest.mark.parametrize("method", [METHOD_MFM, METHOD_MFV], ids=["mfm", "mfv"])
def test_device_kick_large_set_both_half_kicks(method):
    params = _params(method)
    ks = _constructed((1 << 22) + 3, seed=7 + method)
    first_dev = _device_kick(params, ks, 0, 0.0)
    first_orc = _oracle_kick(params, ks, 0, 0.0)
    _assert_same(first_dev, first_orc)
    first_orc["tstart"] = first_orc["tend"].copy()
    first_orc["tend"] = 2 * first_orc["tend"]
    _assert_same(_device_kick(params, first_orc, 1, 0.0), _oracle_kick(params, first_orc, 1, 0.0))


def test_device_kick_optional_fields_left_out():
    """No gravity and no active list: the same as zero gravity, all active."""
    params = _params(METHOD_MFV)
    ks = _constructed(3000, seed=5)
    ks["grav"][...] = 0.0
    ks["gravwork"][...] = 0.0
    ks["active"][...] = 1
    got = _device_kick(params, ks, 1, 0.0, drop=("grav", "gravwork", "active"))
    _assert_same(got, _oracle_kick(params, ks, 1, 0.0))


def test_device_kick_mfm_needs_no_mfv_fields():
    params = _params(METHOD_MFM)
    ks = _constructed(3000, seed=6)
    got = _device_kick(params, ks, 1, 0.0, drop=("mass_true", "dmass", "dtmass"))
    _assert_same(got, _oracle_kick(params, ks, 1, 0.0))
