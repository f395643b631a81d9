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


def test_oracle_matches_default_maps_fixture():
    """The 1-D fixture on the reference's default build maps (SINH_MODIFIED radius,
    POLYTH theta), kept with the dendritic fixtures: the oracle restates both maps."""
    from tests._cases import golden_cases3d
    pb, n = golden_cases3d()["sph1d_default_sedov_192"]
    g = load_golden("sph1d_default_sedov_192")
    o = pyoracle.Oracle(pb)
    o.advance(n)
    prim, _ = o.state()
    assert np.array_equal(prim, g["prim"])
    assert o.t == float(g["t"])


def test_oracle_refuses_maps_it_does_not_restate():
    from medusa_b200 import problems as P
    pb = P.spherical_1d("sedov", 64, 1.4, dr_min=0.01)
    for bad in (dict(rcoord=4), dict(thcoord=2)):
        with pytest.raises(ValueError):
            pyoracle.Oracle(pb.copy(**bad))
    with pytest.raises(ValueError):
        pyoracle.Oracle(P.sod(64).copy(rcoord=P.RCOORD_SINH, rtrans=0.2))
