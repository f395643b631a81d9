"""GPU parity of the 3-D dendritic spherical sweep against fixtures made by the
reference itself (tests/golden/make_golden.py, cases3d): Sedov blasts on small
dendritic grids, symmetric and with seeded noise (shock tagging, rotation through the
pole rows, restriction of the phi velocity into the Gamma slot), reflecting and
SPHERICAL_ORIGIN boundaries.

Error measure per variable: max |gpu - ref| over the zones divided by the largest
magnitude of that variable (density, internal energy) or of any velocity component
(the three velocities share one scale: in the symmetric blast v^theta and v^phi are
round-off).  Bars as for the 1-D/2-D sweeps: 1e-9 after a whole fixture run, 1e-12
for one step.
"""
import numpy as np
import pytest

from medusa_b200.solver import Solver
from tests._cases import golden_cases3d, load_golden, record

pytestmark = pytest.mark.gpu

CASES3 = golden_cases3d()
FULL_RUN_TOL = 1.0e-9
PER_STEP_TOL = 1.0e-12


def err3(a, b):
    out = 0.0
    vscale = max(np.abs(b[:, 2:5]).max(), 1.0e-300)
    for v in range(5):
        scale = vscale if v >= 2 else max(np.abs(b[:, v]).max(), 1.0e-300)
        out = max(out, float(np.abs(a[:, v] - b[:, v]).max() / scale))
    return out


@pytest.mark.parametrize("name", sorted(CASES3))
def test_3d_full_run_matches_reference_fixture(name):
    pb, n = CASES3[name]
    g = load_golden(name)
    with Solver(pb) as s:
        s.step(n)
        prim = s.update_cpu(0)
        t, dt, istep = s.time(0)
    e = err3(prim, g["prim"])
    record("sweep3d_full_" + name, steps=n, err=e, bit_identical=float(np.mean(prim == g["prim"])))
    assert istep == n
    assert e <= FULL_RUN_TOL
    assert abs(t - float(g["t"])) <= FULL_RUN_TOL * float(g["t"])


@pytest.mark.parametrize("name", sorted(CASES3))
def test_3d_one_step_from_developed_state(name):
    pb, n = CASES3[name]
    g = load_golden(name)
    with Solver(pb.copy(ic=np.array(g["prim"]))) as s:
        s.step(1)
        prim = s.update_cpu(0)
        t, _, _ = s.time(0)
    e = err3(prim, g["prim1"])
    record("sweep3d_step_" + name, err=e, bit_identical=float(np.mean(prim == g["prim1"])))
    assert e <= PER_STEP_TOL
    assert abs(t - float(g["t1"])) <= PER_STEP_TOL * float(g["t1"])


def test_3d_mass_change_is_the_outer_boundary_flux():
    """Reflecting inner and pole boundaries, periodic phi: mass changes only through the
    outer radial face, and the blast has not reached it."""
    pb, n = CASES3["sedov3d_20x16x32"]
    with Solver(pb) as s:
        m0, _ = s.conserved_totals()
        s.step(10)
        m1, _ = s.conserved_totals()
    assert abs(m1[0] - m0[0]) <= 1.0e-13 * m0[0]
