"""The CPU oracle against the golden fixtures produced by the reference itself."""
import numpy as np
import pytest

from oracle import pyoracle
from tests._cases import golden_cases, load_golden

CASES = golden_cases()


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_fixture(name):
    pb, n = CASES[name]
    g = load_golden(name)
    assert np.array_equal(pb.ic, g["ic"]), "problem setup drifted from the fixture's initial state"
    o = pyoracle.Oracle(pb)
    dts = o.advance(n)
    prim, _ = o.state()
    # bit-exact: the oracle restates the reference's arithmetic in the same order
    assert np.array_equal(prim, g["prim"])
    assert o.t == float(g["t"])
    assert dts[-1] == float(g["dt"])
