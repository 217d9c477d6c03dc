"""The C oracle against the golden fixtures made by the reference's own pair
bodies (tests/golden/make_golden.py). Pins the oracle: bit-exact, except the
MFV dMass sum whose j-side writes are order-dependent (atomic adds)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests._util import golden_cases, load_golden, DENSITY_FIELDS, GRADIENT_FIELDS, FORCE_FIELDS

CASES = golden_cases()


def test_fixtures_present():
    assert len(CASES) >= 3


@pytest.mark.parametrize("path", CASES, ids=lambda p: p.split("/")[-1][:-4])
def test_oracle_matches_reference_golden(path):
    params, inputs, golden = load_golden(path)
    st = O.new_state(inputs["pos"].shape[0], inputs)
    orc = O.Oracle(params, "port", n_threads=1)
    assert orc.density(st) == 0
    assert orc.gradients(st) == 0
    assert orc.force(st) == 0
    for f in DENSITY_FIELDS + GRADIENT_FIELDS + FORCE_FIELDS + ["iters"]:
        if f == "dmass":
            np.testing.assert_allclose(st[f], golden[f], rtol=0, atol=1e-14 * np.abs(golden[f]).max() + 1e-300)
        else:
            assert np.array_equal(st[f], golden[f]), f
