"""The mixed-precision 2-D split sweep (FP32 difference-form reconstruction and HLLC wave
speeds, FP64 fluxes, accumulation, update and dt; declined faces re-solved in FP64)
against the plain FP64 sweep (the reference's arithmetic) at equal physical time.

Bars: volume-weighted relative L1 of rho and u <= 1e-4; mass and total energy equal to
the FP64 run's within 1e-9 relative on periodic grids (both conserve them to round-off);
results independent of the batch (a problem alone equals the same problem in a batch)."""
import numpy as np
import pytest

from medusa_b200 import analytic as A
from medusa_b200 import problems as P
from medusa_b200.solver import PREC_FP64, PREC_MIXED, Solver
from tests._cases import record

pytestmark = pytest.mark.gpu


def _equal_time(pb, n):
    with Solver(pb, precision=PREC_FP64) as s:
        s.step(n)
        ref = s.update_cpu(0)
        t_end = s.time(0)[0]
        m0, e0 = s.conserved_totals()
    with Solver(pb.copy(tmax=t_end), precision=PREC_MIXED) as s:
        k = 0
        while s.time(0)[0] < t_end * (1.0 - 1.0e-12) and k < 4 * n:
            s.step(10)
            k += 10
        mix = s.update_cpu(0)
        t_mix = s.time(0)[0]
        m1, e1 = s.conserved_totals()
    return ref, mix, t_end, t_mix, (m0[0], e0[0], m1[0], e1[0])


@pytest.mark.parametrize("name,pb,n", [
    ("kh_128", P.kelvin_helmholtz(128, 128, seed=4), 120),
    ("rt_64x128", P.rayleigh_taylor_2d(64, 128, g=-0.5, noise=0.05), 120),
    ("blast_96_reflect", P.blast_2d(96, 96, bc=P.REFLECT), 80),
])
def test_mixed_2d_matches_fp64_at_equal_time(name, pb, n):
    ref, mix, t_end, t_mix, (m0, e0, m1, e1) = _equal_time(pb, n)
    assert np.all(np.isfinite(mix))
    assert abs(t_mix - t_end) <= 1.0e-8 * t_end
    l1_rho = A.l1_rel(mix[:, 0], ref[:, 0])
    l1_u = A.l1_rel(mix[:, 1], ref[:, 1])
    record("mixed2d_" + name, steps=n, l1_rho=l1_rho, l1_u=l1_u, dm=abs(m1 - m0) / m0, de=abs(e1 - e0) / e0)
    assert l1_rho <= 1.0e-4 and l1_u <= 1.0e-4
    if pb.bc_lo[0] == P.PERIODIC and pb.bc_lo[1] == P.PERIODIC:
        assert abs(m1 - m0) <= 1.0e-9 * m0 and abs(e1 - e0) <= 1.0e-9 * e0


def test_mixed_2d_batched_equals_alone():
    probs = [P.kelvin_helmholtz(64, 48, seed=5), P.rayleigh_taylor_2d(40, 72, g=-0.5, noise=0.05),
             P.blast_2d(50, 40, bc=P.OUTFLOW)]
    with Solver(probs, precision=PREC_MIXED) as s:
        s.step(25)
        batched = [s.update_cpu(m) for m in range(len(probs))]
    for m, pb in enumerate(probs):
        with Solver(pb, precision=PREC_MIXED) as s:
            s.step(25)
            assert np.array_equal(s.update_cpu(0), batched[m]), pb.name
