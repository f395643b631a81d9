"""Failure detection without a GPU fault: the faults are made on the host (a non-finite
value in an initial state, a dtmin above every possible step), the kernels flag them in
the problem's device time record and the host reads the status (mdg_synchronize,
mdg_server_result) -- the context stays usable, and independent problems in the same
launch or server are unaffected, bit for bit."""
import numpy as np
import pytest

from medusa_b200 import problems as P
from medusa_b200.solver import MdgError, PREC_FP64, PREC_MIXED, Server, Solver

pytestmark = pytest.mark.gpu

NONFINITE = 11


def _poisoned(pb, zone=17):
    ic = np.array(pb.ic)
    ic[zone, 1] = np.nan
    return pb.copy(ic=ic, name=pb.name + "_nan")


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
def test_nonfinite_state_is_reported(precision):
    with Solver(_poisoned(P.spherical_1d("sedov", 200, 1.4, p_ratio=1.0e3, r0=0.1)), precision=precision) as s:
        s.step(5)
        with pytest.raises(MdgError) as e:
            s.synchronize()
        assert e.value.code == NONFINITE
        # the context is still usable
        s.upload(0, P.spherical_1d("sedov", 200, 1.4, p_ratio=1.0e3, r0=0.1).ic)


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
def test_bad_problem_leaves_its_batch_unchanged(precision):
    good = [P.spherical_1d("sod", 300, 1.4, rho_ratio=8.0, p_ratio=50.0), P.sod(257)]
    bad = _poisoned(P.spherical_1d("sedov", 200, 1.4, p_ratio=1.0e3, r0=0.1))
    with Solver([good[0], bad, good[1]], precision=precision) as s:
        s.step(20)
        with pytest.raises(MdgError):
            s.synchronize()
        got = [s.update_cpu(0), s.update_cpu(2)]
    for pb, prim in zip(good, got):
        with Solver(pb, precision=precision) as s:
            s.step(20)
            s.synchronize()
            assert np.array_equal(s.update_cpu(0), prim), pb.name


def test_dt_below_dtmin_is_reported():
    """main.c:229-238 aborts when estimate_dt() drops below dtmin; here the status."""
    with Solver(P.sod(128).copy(dtmin=1.0)) as s:
        s.step(1)
        with pytest.raises(MdgError) as e:
            s.synchronize()
        assert e.value.code == NONFINITE


def test_dendritic_nonfinite_state_is_reported():
    pb = P.sedov_3d(12, 8, 16, r_dep=0.3)
    with Solver(_poisoned(pb, zone=100)) as s:
        s.step(3)
        with pytest.raises(MdgError) as e:
            s.synchronize()
        assert e.value.code == NONFINITE


def test_server_fails_the_bad_request_only():
    good = [P.spherical_1d("sod", 256, 1.4).copy(tmax=0.02), P.sod(300).copy(tmax=0.02)]
    bad = _poisoned(P.spherical_1d("sedov", 200, 1.4, p_ratio=1.0e3, r0=0.1).copy(tmax=0.02))
    with Server(precision=PREC_MIXED, hbm_bytes=64 << 20, max_problems=8, max_zones=4096) as srv:
        ids = [srv.submit(pb) for pb in (good[0], bad, good[1])]
        srv.run(0)
        with pytest.raises(MdgError) as e:
            srv.result(ids[1])
        assert e.value.code == NONFINITE
        for rid, pb in ((ids[0], good[0]), (ids[2], good[1])):
            prim, t, ist, _ = srv.result(rid)
            with Solver(pb, precision=PREC_MIXED) as s:
                for _ in range(10000):
                    s.step(1)
                    if s.time(0)[0] >= pb.tmax:
                        break
                assert np.array_equal(s.update_cpu(0), prim), pb.name
