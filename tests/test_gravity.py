"""Self-gravity in the monopole approximation (gravity.c:145-425 with GR_MONOPOLE=FALSE)
on the host: the fixtures made by the reference's GRAV=SPHERICAL_MONOPOLE_GRAV builds
against the problem generator and the live reference, and the scope checks of the C ABI
(no device work)."""
import ctypes

import numpy as np
import pytest

from medusa_b200 import problems as P
from medusa_b200 import solver as S
from oracle import pyoracle
from tests._cases import golden_cases_gravity, load_golden

CASES = golden_cases_gravity()


@pytest.mark.parametrize("name", sorted(CASES))
def test_fixture_matches_generator(name):
    pb, n = CASES[name]
    g = load_golden(name)
    assert g["prim"].shape == (pb.ncell, 5) and g["prim1"].shape == (pb.ncell, 5)
    assert int(g["istep"]) == n
    assert np.all(np.isfinite(g["prim"]))
    # the collapse has started: inward radial velocity inside the sphere
    assert g["prim"][:, 2].min() < 0.0


@pytest.mark.parametrize("name", sorted(CASES))
def test_fixture_reproduced_by_live_reference(name):
    pb, n = CASES[name]
    if not pyoracle.ref_available(pb):
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    g = load_golden(name)
    snaps = pyoracle.run_reference(pb, n, every=n)
    assert np.array_equal(snaps[-1][4], g["prim"])


def test_dust_collapse_setup():
    """init_dustcollapse.c: rho0 inside r0, the straddling zone's volume share, the floor
    outside; the SINH radius reaching r_out."""
    pb = P.dust_collapse(200)
    e = P.radial_edges(pb)
    assert abs(e[-1] - 7.0e8) <= 1.0e-6 * 7.0e8 and abs(e[1] - 5.0e4) <= 1.0e-3 * 5.0e4
    rho = pb.ic[:, 0]
    inside = e[1:] < 6.5e8
    assert np.all(rho[inside] == 1.0e9)
    assert np.all(rho[e[:-1] >= 6.5e8] == 1.0e4)
    assert pb.prob_kind == P.PROB_DUST and pb.monopole == 1 and pb.enforce_floors == 1


def _create(pb, precision=0, nprob=1):
    arr = (S.ProblemDesc * nprob)(*[S.desc_of(pb)] * nprob)
    h = ctypes.c_void_p()
    rc = S.library().mdg_create(arr, nprob, precision, 0, ctypes.byref(h))
    assert not h.value
    return rc


@pytest.mark.parametrize("mutate,precision,code", [
    (dict(geom=P.CARTESIAN, rcoord=0, prob_kind=0, bc_hi=(P.OUTFLOW, 0, 0), bc_lo=(P.OUTFLOW, 0, 0)), 0, 1),
    (dict(grav=(0.0, -1.0, 0.0)), 0, 1),        # one gravity switch at a time
    (dict(monopole=2), 0, 1),
    (dict(prob_kind=7), 0, 1),
])
def test_monopole_scope_checked_before_device_work(mutate, precision, code):
    pb = P.dust_collapse(64).copy(**mutate)
    assert _create(pb, precision) == code


def test_dust_hook_only_on_the_outer_boundary():
    pb = P.dust_collapse(64).copy(bc_lo=(P.PROB, 0, 0))
    assert _create(pb) == 5
