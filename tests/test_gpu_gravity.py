"""GPU parity of the monopole self-gravity (gravity.c:145-425, GR_MONOPOLE=FALSE) against
fixtures made by the reference's GRAV=SPHERICAL_MONOPOLE_GRAV builds: the dust collapse
of problems/init_dustcollapse.c in 1-D (SINH radius with floors and the outer v^r hook;
uniform radius) and on the 2-D and 3-D dendritic grids; and of fixed gravity
(gravity.c:38-64, GRAV=FIXED_GRAV builds) on the dendritic grids.  Bars as for the other sweeps:
1e-9 after a whole fixture run, 1e-12 for one step, on two measures: pointwise
(tests/_cases.py pointwise_rel_err) and per variable relative to its largest magnitude,
the velocities sharing one scale."""
import numpy as np
import pytest

from medusa_b200 import problems as P
from medusa_b200.solver import MdgError, PREC_FP64, PREC_MIXED, Server, Solver
from tests._cases import golden_cases_gravity, load_golden, pointwise_rel_err, record, zone_gcov

pytestmark = pytest.mark.gpu

CASES = golden_cases_gravity()
FULL_RUN_TOL = 1.0e-9
PER_STEP_TOL = 1.0e-12


def err(a, b):
    out = 0.0
    vscale = max(np.abs(b[:, 2:5]).max(), 1.0e-300)
    for v in range(5):
        scale = vscale if v >= 2 else max(np.abs(b[:, v]).max(), 1.0e-300)
        out = max(out, float(np.abs(a[:, v] - b[:, v]).max() / scale))
    return out


@pytest.mark.parametrize("name", sorted(CASES))
def test_gravity_full_run_matches_reference_fixture(name):
    pb, n = CASES[name]
    g = load_golden(name)
    with Solver(pb) as s:
        s.step(n)
        prim = s.update_cpu(0)
        t, _, istep = s.time(0)
    e = err(prim, g["prim"])
    pw = pointwise_rel_err(prim, g["prim"], pb, zone_gcov(pb))
    record("gravity_full_" + name, steps=n, err=e, pointwise=pw, bit_identical=float(np.mean(prim == g["prim"])))
    assert istep == n
    assert e <= FULL_RUN_TOL
    assert pw <= FULL_RUN_TOL
    assert abs(t - float(g["t"])) <= FULL_RUN_TOL * float(g["t"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_gravity_one_step_from_developed_state(name):
    pb, n = CASES[name]
    g = load_golden(name)
    with Solver(pb.copy(ic=np.array(g["prim"]))) as s:
        s.step(1)
        prim = s.update_cpu(0)
    e = err(prim, g["prim1"])
    pw = pointwise_rel_err(prim, g["prim1"], pb, zone_gcov(pb))
    record("gravity_step_" + name, err=e, pointwise=pw, bit_identical=float(np.mean(prim == g["prim1"])))
    assert pw <= PER_STEP_TOL
    assert e <= PER_STEP_TOL


def test_monopole_problem_alone_and_in_a_batch():
    """A 1-D self-gravitating problem batched with problems without gravity: every result
    equals its run alone, bit for bit."""
    dust = P.dust_collapse(200)
    others = [P.spherical_1d("sedov", 300, 1.4, p_ratio=1.0e4, r0=0.05), P.sod(257)]
    with Solver([others[0], dust, others[1]]) as s:
        s.step(40)
        batch = [s.update_cpu(m) for m in range(3)]
    for m, pb in enumerate([others[0], dust, others[1]]):
        with Solver(pb) as s:
            s.step(40)
            alone = s.update_cpu(0)
        assert np.array_equal(alone, batch[m]), pb.name


def test_collapse_accelerates_inwards():
    """Free fall from rest: after a short time the radial velocity inside the sphere is
    close to -g t with g = G M(<r) / r^2 (pressure is 1/gam/mach^2 of the free-fall scale)."""
    pb = P.dust_collapse(200, radius="uniform", floors=False)
    with Solver(pb) as s:
        s.step(40)
        prim = s.update_cpu(0)
        t = s.time(0)[0]
    rc = P.radial_centers(pb)
    i = int(np.searchsorted(rc, 3.0e8))
    m_in = 4.0 / 3.0 * np.pi * rc[i] ** 3 * 1.0e9
    v_ff = -P.GNEWT * m_in / rc[i] ** 2 * t
    record("gravity_freefall", t=t, v=float(prim[i, 2]), v_ff=v_ff)
    assert abs(prim[i, 2] - v_ff) <= 0.05 * abs(v_ff)


def test_dendritic_mixed_matches_fp64():
    """The mixed-precision dendritic sweep with self-gravity: L1 of rho and u against the
    plain FP64 sweep at equal time <= 1e-4."""
    from medusa_b200 import analytic as A
    from medusa_b200.solver import grid3d_zone_volumes
    pb = P.dust_collapse(32, 16, 32, ndim=3, radius="uniform", floors=False)
    with Solver(pb) as s:
        s.step(40)
        ref = s.update_cpu(0)
        t_end = s.time(0)[0]
    with Solver(pb.copy(tmax=t_end), precision=PREC_MIXED) as s:
        for _ in range(40):
            s.step(5)
            if s.time(0)[0] >= t_end * (1.0 - 1.0e-12):
                break
        mix = s.update_cpu(0)
    vol = grid3d_zone_volumes(pb)
    l1_rho = A.l1_rel(mix[:, 0], ref[:, 0], vol)
    l1_u = A.l1_rel(mix[:, 1], ref[:, 1], vol)
    record("gravity_mixed_dust3d_32x16x32", l1_rho=l1_rho, l1_u=l1_u)
    assert l1_rho <= 1.0e-4 and l1_u <= 1.0e-4


def _solver_to_end(pb, precision):
    with Solver(pb, precision=precision) as s:
        for _ in range(100000):
            s.step(1)
            if s.time(0)[0] >= pb.tmax:
                break
        return s.update_cpu(0), s.time(0)


def test_server_runs_monopole_requests():
    """Self-gravitating requests in an FP64 server (1-D with the dust-collapse hook, 3-D
    dendritic) beside plain ones, and the 1-D ones in a mixed server: each result equals
    the solver's, bit for bit."""
    reqs = [P.dust_collapse(200).copy(tmax=2.0e-3),
            P.spherical_1d("sod", 256, 1.4).copy(tmax=0.02),
            P.dust_collapse(16, 8, 16, ndim=3, radius="uniform", floors=False).copy(tmax=1.0e-3)]
    with Server(precision=PREC_FP64, hbm_bytes=128 << 20, max_problems=8, max_zones=4096,
                hbm_bytes_3d=256 << 20) as srv:
        ids = [srv.submit(pb) for pb in reqs]
        srv.run(0)
        for rid, pb in zip(ids, reqs):
            prim, t, ist, _ = srv.result(rid)
            ref, (rt, _, rist) = _solver_to_end(pb, PREC_FP64)
            assert t == rt and ist == rist, pb.name
            assert np.array_equal(prim, ref), pb.name
    # a mixed server: the 1-D requests (one with monopole gravity) equal the mixed solver's
    with Server(precision=PREC_MIXED, hbm_bytes=64 << 20, max_problems=4, max_zones=4096,
                steps_per_round=9) as srv:
        ids = [srv.submit(pb) for pb in reqs[:2]]
        srv.run(0)
        for rid, pb in zip(ids, reqs[:2]):
            prim, t, ist, _ = srv.result(rid)
            ref, (rt, _, rist) = _solver_to_end(pb, PREC_MIXED)
            assert t == rt and ist == rist, pb.name
            assert np.array_equal(prim, ref), pb.name


@pytest.mark.parametrize("radius,floors,n1,nsteps", [("sinh", True, 200, 200), ("uniform", False, 128, 150)])
def test_mixed_1d_monopole_matches_fp64(radius, floors, n1, nsteps):
    """The mixed-precision 1-D sweep with monopole self-gravity (the dust collapse, with its
    outer v^r hook) against the plain FP64 sweep at equal time: volume-weighted L1 of rho
    and u <= 1e-4, mass difference <= 1e-6 relative; batched with problems without
    gravity, its result equals its run alone.  (Without floors the collapse empties the
    zones behind the sphere's edge: both sweeps reach negative density after ~190 steps.)"""
    from medusa_b200 import analytic as A
    pb = P.dust_collapse(n1, radius=radius, floors=floors)
    with Solver(pb) as s:
        s.step(nsteps)
        ref = s.update_cpu(0)
        t_end = s.time(0)[0]
        m_ref, _ = s.conserved_totals()
    with Solver(pb.copy(tmax=t_end), precision=PREC_MIXED) as s:
        for _ in range(100):
            s.step(5)
            if s.time(0)[0] >= t_end * (1.0 - 1.0e-12):
                break
        mix = s.update_cpu(0)
        t_mix = s.time(0)[0]
        m_mix, _ = s.conserved_totals()
    e = P.radial_edges(pb)
    vol = e[1:] ** 3 - e[:-1] ** 3
    l1_rho = A.l1_rel(mix[:, 0], ref[:, 0], vol)
    l1_u = A.l1_rel(mix[:, 1], ref[:, 1], vol)
    l1_v = A.l1_rel(mix[:, 2], ref[:, 2], vol)
    drift_m = abs(m_mix[0] - m_ref[0]) / abs(m_ref[0])
    record("gravity_mixed_dust1d_%s_%d" % (radius, n1), t=t_end, l1_rho=l1_rho, l1_u=l1_u, l1_vr=l1_v,
           mass_drift=drift_m)
    assert abs(t_mix - t_end) <= 1.0e-8 * t_end
    assert l1_rho <= 1.0e-4 and l1_u <= 1.0e-4 and l1_v <= 1.0e-4
    assert drift_m <= 1.0e-6
    others = [P.spherical_1d("sedov", 300, 1.4, p_ratio=1.0e4, r0=0.05), P.sod(257)]
    batch_probs = [others[0], pb, others[1]]
    with Solver(batch_probs, precision=PREC_MIXED) as s:
        s.step(30)
        batch = [s.update_cpu(m) for m in range(3)]
    with Solver(batch_probs, precision=PREC_MIXED) as s:
        s.set_launch_config(lanes=3)   # each problem on a stream of its own
        s.step(30)
        for m in range(3):
            assert np.array_equal(s.update_cpu(m), batch[m])
    for m, q in enumerate(batch_probs):
        with Solver(q, precision=PREC_MIXED) as s:
            s.step(30)
            assert np.array_equal(s.update_cpu(0), batch[m]), q.name
