"""Empty inputs, as a GIZMO host meets them: a domain or box holding no gas
cell, and a timestep bin with no active cell. The reference's loops then do
not run; here every call returns GZ_OK without launching a kernel, and no
output changes.
"""
import numpy as np
import pytest

from gizmo_b200 import abi, ics
from gizmo_b200.hydro import HydroPass

pytestmark = pytest.mark.gpu


def test_set_of_no_particles():
    params = ics.sedov(4, seed=1).params
    z3, z1 = np.zeros((0, 3)), np.zeros(0)
    with HydroPass(params) as hp:
        hp.upload(z3, z3, z1, z1, z1, z1, z1)
        hp.full_pass()
        hp.restage()
        hp.hydro_pass(graph=True)
        hp.hydro_pass(graph=True, restage=True)
        out = hp.download()
        assert all(np.asarray(v).shape[0] == 0 for v in out.values())
        st = hp.status()
        assert st["code"] == 0 and st["density_iterations"] == 0


@pytest.mark.parametrize("precision", [abi.PRECISION_FP64, abi.PRECISION_MIXED])
def test_empty_active_list_changes_nothing(precision):
    wl = ics.sedov(8, seed=1, precision=precision)
    none = np.zeros(0, dtype=np.int32)
    with HydroPass(wl.params) as hp:
        hp.upload_workload(wl)
        hp.full_pass()
        before = hp.download()
        hp.density(none)
        hp.hydro_gradient_calc(none)
        hp.hydro_force(none)
        after = hp.download()
        assert hp.status()["code"] == 0
        # the next pass over every particle is the one it would have been
        # without the empty calls (it starts from the last pass's kernel lengths)
        hp.full_pass()
        again = hp.download()
    with HydroPass(wl.params) as hp:
        hp.upload_workload(wl)
        hp.full_pass()
        hp.full_pass()
        control = hp.download()
    for k in before:
        assert np.array_equal(before[k], after[k]), k
        assert np.array_equal(again[k], control[k]), k
