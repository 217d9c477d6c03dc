"""The two halves of the step either side of the hydro pass, on the device.

gz_kick, the half-step kick on the device, against the oracle's orc_kick
(itself pinned bit-exact to the reference's compiled do_the_kick): bit-exact
on every kicked field, for the constructed cases that reach every limiter, a
set of 4M particles (many grid-stride rounds) and the optional fields left
out.

gz_drift, the drift on the device, against the oracle's orc_drift (itself
pinned bit-exact to the reference's drift_particle_impl). Every field is
bit-exact except three. The density and the kernel radius are products with
an exponential. The device's exp is correctly rounded; the oracle's is the C
library's, which is off by one ulp on ~0.05% of these inputs. A factor one ulp
off moves the exact product by at most 2^-52 of itself, at most 2 ulp of the
product, and the two rounded products stay within 2 ulp. The pressure
multiplies such a density, so a relative gap of up to 2^-51 in its exact
value: within 4 ulp. Cases: the constructed ones that reach every cap, clamp
and floor, a set of 4M cells (many grid-stride rounds), a drift into the
past, and the optional fields left out.

The kick tests come first: they precede the drift tests in a run that stops at
the first failure."""
import numpy as np
import pytest

from gizmo_b200 import abi, hydro, ics
from gizmo_b200.abi import METHOD_MFM, METHOD_MFV
from oracle import oracle as O
from tests.test_oracle_drift import _constructed as drift_cases
from tests.test_oracle_kick import TIMEBASE, _constructed as kick_cases

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _kick_params(method):
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


def _assert_kick_same(got, want):
    for name, _, _ in O.KICK_FIELDS:
        np.testing.assert_array_equal(got[name], want[name], err_msg=name)


@pytest.mark.parametrize("method", [METHOD_MFM, METHOD_MFV], ids=["mfm", "mfv"])
@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("floor", [0.0, 3.0])
def test_device_kick_constructed_cases(method, mode, floor):
    params = _kick_params(method)
    ks = kick_cases(4096, seed=100 + 10 * mode + method)
    _assert_kick_same(_device_kick(params, ks, mode, floor), _oracle_kick(params, ks, mode, floor))


@pytest.mark.parametrize("method", [METHOD_MFM, METHOD_MFV], ids=["mfm", "mfv"])
def test_device_kick_large_set_both_half_kicks(method):
    params = _kick_params(method)
    ks = kick_cases((1 << 22) + 3, seed=7 + method)
    first_dev = _device_kick(params, ks, 0, 0.0)
    first_orc = _oracle_kick(params, ks, 0, 0.0)
    _assert_kick_same(first_dev, first_orc)
    first_orc["tstart"] = first_orc["tend"].copy()
    first_orc["tend"] = 2 * first_orc["tend"]
    _assert_kick_same(_device_kick(params, first_orc, 1, 0.0), _oracle_kick(params, first_orc, 1, 0.0))


def test_device_kick_optional_fields_left_out():
    """No gravity and no active list: the same as zero gravity, all active."""
    params = _kick_params(METHOD_MFV)
    ks = kick_cases(3000, seed=5)
    ks["grav"][...] = 0.0
    ks["gravwork"][...] = 0.0
    ks["active"][...] = 1
    got = _device_kick(params, ks, 1, 0.0, drop=("grav", "gravwork", "active"))
    _assert_kick_same(got, _oracle_kick(params, ks, 1, 0.0))


def test_device_kick_mfm_needs_no_mfv_fields():
    params = _kick_params(METHOD_MFM)
    ks = kick_cases(3000, seed=6)
    got = _device_kick(params, ks, 1, 0.0, drop=("mass_true", "dmass", "dtmass"))
    _assert_kick_same(got, _oracle_kick(params, ks, 1, 0.0))


ULP = {"rho": 2, "h": 2, "pressure": 4}  # fields through exp: bounds derived in the module docstring


def _drift_params(method):
    p = ics.sedov(4, seed=1).params
    p.method = method
    p.min_kernel_radius, p.max_kernel_radius = 0.05, 0.5
    return p


def _device_drift(params, ds, time1, floor, drop=()):
    dev = {k: torch.from_numpy(v.copy()).cuda() for k, v in ds.items() if k not in drop}
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    hydro.drift(params, dict(dev, status=status), time1, TIMEBASE, floor)
    torch.cuda.synchronize()
    out = {k: v.cpu().numpy() for k, v in dev.items()}
    for k in drop:
        out[k] = ds[k].copy()
    return out, int(status.item())


def _oracle_drift(params, ds, time1, floor):
    s = {k: v.copy() for k, v in ds.items()}
    code = O.Oracle(params, "port").drift(s, time1, TIMEBASE, floor)
    return s, code


def _assert_close(got, want):
    for name, _, _ in O.DRIFT_FIELDS:
        if name in ULP:
            np.testing.assert_array_max_ulp(got[name], want[name], maxulp=ULP[name])
        else:
            np.testing.assert_array_equal(got[name], want[name], err_msg=name)


@pytest.mark.parametrize("method", [METHOD_MFM, METHOD_MFV], ids=["mfm", "mfv"])
@pytest.mark.parametrize("floor", [0.0, 3.0])
def test_device_drift_constructed_cases(method, floor):
    params = _drift_params(method)
    ds, time1 = drift_cases(4096, 200 + method, params)
    got, status = _device_drift(params, ds, time1, floor)
    want, code = _oracle_drift(params, ds, time1, floor)
    assert status == code == 0
    _assert_close(got, want)


@pytest.mark.parametrize("method", [METHOD_MFM, METHOD_MFV], ids=["mfm", "mfv"])
def test_device_drift_large_set(method):
    params = _drift_params(method)
    ds, time1 = drift_cases((1 << 22) + 5, 31 + method, params)
    got, status = _device_drift(params, ds, time1, 0.0)
    want, code = _oracle_drift(params, ds, time1, 0.0)
    assert status == code == 0
    _assert_close(got, want)


def test_device_drift_into_the_past_sets_the_status():
    params = _drift_params(METHOD_MFV)
    ds, time1 = drift_cases(1000, 9, params)
    ds["ti_current"][[5, 700]] = time1 + 3
    got, status = _device_drift(params, ds, time1, 0.0)
    want, code = _oracle_drift(params, ds, time1, 0.0)
    assert status == code == abi.ERR_NO_PAST_DRIFT
    _assert_close(got, want)


def test_device_drift_optional_fields_left_out():
    """No gravity, and each method without the other's fields: the same as zero gravity."""
    for method, drop in ((METHOD_MFV, ("grav", "vel")), (METHOD_MFM, ("grav", "pvel", "dtmass", "mass_true"))):
        params = _drift_params(method)
        ds, time1 = drift_cases(3000, 40 + method, params)
        ds["grav"][...] = 0.0
        got, status = _device_drift(params, ds, time1, 0.0, drop=drop)
        want, code = _oracle_drift(params, ds, time1, 0.0)
        assert status == code == 0
        _assert_close(got, want)
