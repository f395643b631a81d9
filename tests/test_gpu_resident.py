"""The resident 1-D stepper (mdg_launch_config::resident): small plain-FP64 1-D problems
advanced many steps per launch, one thread-block cluster per problem.  It runs the same
tile code and time rules as the per-phase launches, so the two paths must agree bit for
bit -- state, t, dt and step count -- on every boundary kind, map and problem mix; the
golden-fixture tests of test_gpu_parity.py pin the default (resident) path against the
reference itself."""
import numpy as np
import pytest

from medusa_b200 import problems as P
from medusa_b200.solver import MdgError, PREC_FP64, PREC_MIXED, Solver
from oracle import pyoracle
from tests._cases import pointwise_rel_err

pytestmark = pytest.mark.gpu

NONFINITE = 11


def _cases():
    noh = P.spherical_1d("noh", 200, 5.0 / 3.0)
    return [
        P.sod(1024),                                                   # 9 tiles: a 16-CTA cluster
        P.sod(126),                                                    # exactly one tile
        P.sod(127),                                                    # one zone into a second tile
        P.double_rarefaction(2016, v=6.0, rho_floor=1e-6, e_floor=1e-6),   # 16 tiles, floors
        P.spherical_1d("sedov", 300, 1.4, p_ratio=1.0e4, r0=0.05),
        P.spherical_1d("sod", 500, 5.0 / 3.0, dr_min=2.0e-4),           # SINH radius
        P.spherical_1d("sedov", 400, 1.4, p_ratio=1.0e3, r0=0.05, coords="log", r_in=1.0e-3),
        noh,                                                           # PROB boundary
    ]


def _run(pbs, steps, resident, chunks=1):
    with Solver(pbs) as s:
        s.set_launch_config(resident=resident)
        for _ in range(chunks):
            s.step(steps)
        s.synchronize()
        cs = s.resident_cluster()
        out = [(s.update_cpu(m), s.time(m)) for m in range(len(pbs))]
    return cs, out


@pytest.mark.parametrize("pb", _cases(), ids=lambda p: p.name)
def test_resident_equals_per_phase_bit_for_bit(pb):
    cs, res = _run([pb], 300, 1)
    assert cs >= (pb.ncell + 125) // 126
    _, ref = _run([pb], 300, 0)
    assert np.array_equal(res[0][0], ref[0][0], equal_nan=True)
    assert np.array_equal(res[0][1], ref[0][1], equal_nan=True)


def test_resident_batch_of_mixed_sizes_equals_each_alone():
    pbs = _cases()
    cs, res = _run(pbs, 300, 1, chunks=2)     # two calls of 300 steps: two launches each
    assert cs == 16
    for pb, (prim, tm) in zip(pbs, res):
        _, alone = _run([pb], 600, 0)
        assert np.array_equal(prim, alone[0][0], equal_nan=True), pb.name
        assert np.array_equal(tm, alone[0][1], equal_nan=True), pb.name


def test_resident_matches_oracle_to_the_end_time():
    """The Sod tube to t = 0.2 (the whole job, past the end time the steps change
    nothing) against the CPU restatement, which is bit-identical to the reference."""
    pb = P.sod(1024).copy(tmax=0.2)
    with Solver(pb) as s:
        assert s.resident_cluster() == 16
        s.step(700)
        s.synchronize()
        prim = s.update_cpu(0)
        t, dt, istep = s.time(0)
    o = pyoracle.Oracle(pb)
    o.advance(istep)
    assert t >= 0.2 and istep < 700
    assert abs(o.t - t) <= 1.0e-9 * t
    # differences start in the last place of pow() in the wave-speed estimate
    assert pointwise_rel_err(prim, o.state()[0], pb) <= 1.0e-9


def test_resident_not_used_where_it_does_not_apply():
    with Solver(P.sod(2017)) as s:                    # 17 tiles
        assert s.resident_cluster() == 0
    with Solver(P.spherical_1d("sedov", 300, 1.4, p_ratio=1.0e4, r0=0.05), precision=PREC_MIXED) as s:
        assert s.resident_cluster() == 0
    with Solver(P.kelvin_helmholtz(64)) as s:
        assert s.resident_cluster() == 0
    with Solver([P.sod(256), P.sod(4000)]) as s:      # one problem too large: the whole solver
        assert s.resident_cluster() == 0


def test_resident_reports_failures_and_stays_usable():
    pb = P.spherical_1d("sedov", 200, 1.4, p_ratio=1.0e3, r0=0.1)
    ic = np.array(pb.ic)
    ic[17, 1] = np.nan
    with Solver([pb.copy(ic=ic, name="nan"), pb]) as s:
        assert s.resident_cluster() > 0
        s.step(20)
        with pytest.raises(MdgError) as e:
            s.synchronize()
        assert e.value.code == NONFINITE
        good = s.update_cpu(1)
    _, alone = _run([pb], 20, 0)
    assert np.array_equal(good, alone[0][0])
    with Solver(P.sod(128).copy(dtmin=1.0)) as s:
        s.step(3)
        with pytest.raises(MdgError) as e:
            s.synchronize()
        assert e.value.code == NONFINITE


def test_resident_off_with_timers_and_invalid_setting():
    pb = P.sod(512)
    with Solver(pb) as s:
        s.set_timing(True)                            # timers: the per-phase launches
        s.step(10)
        s.synchronize()
        assert s.timers()["stage0"][1] == 10
        with pytest.raises(MdgError):
            s.set_launch_config(resident=2)
