"""The solve server (mdg_server_*): requests run to their end time, results equal the
solver's, each result is the same alone and in a mix, and admission respects the
device-memory budget.

Equality here is bit-for-bit: the stage kernels do the same arithmetic for a zone whatever
else is in the batch, and a problem that has reached its end time is left unchanged by
later rounds (the main.c loop has ended for it), so neither the company of other problems
nor the round at which a result is collected can change it.
"""
import threading

import numpy as np
import pytest

from medusa_b200 import problems as P
from medusa_b200.solver import (PREC_FP64, PREC_MIXED, REQ_DONE, REQ_QUEUED, REQ_RUNNING, MdgError, Server,
                                Solver)

pytestmark = pytest.mark.gpu


def _req(kind, n1, gam, t_end, **kw):
    return P.spherical_1d(kind, n1, gam, **kw).copy(tmax=t_end)


def _mix():
    """A handful of requests of different kinds, sizes and end times."""
    return [
        _req("sod", 300, 1.4, 0.05, rho_ratio=10.0, p_ratio=100.0),
        _req("noh", 200, 5.0 / 3.0, 0.08),
        _req("sedov", 420, 1.4, 0.02, p_ratio=1.0e4, r0=0.05),
        _req("sod", 150, 4.0 / 3.0, 0.03, rho_ratio=3.0, p_ratio=20.0),
        _req("sedov", 700, 5.0 / 3.0, 0.015, p_ratio=3.0e3, r0=0.08),
        _req("noh", 333, 1.4, 0.05),
    ]


def _solver_result(pb, precision):
    """The same run through the solver: step until the time loop has ended."""
    with Solver(pb, precision=precision) as s:
        for _ in range(2000):
            s.step(25)
            t, _, ist = s.time(0)
            if t >= pb.tmax:
                break
        s.step(5)   # further steps must change nothing
        s.synchronize()
        return s.update_cpu(0), s.time(0)


@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
def test_server_results_equal_solver(precision):
    reqs = _mix()
    with Server(precision=precision, hbm_bytes=256 << 20, max_problems=16, max_zones=4096,
                steps_per_round=17) as srv:
        ids = [srv.submit(pb) for pb in reqs]
        assert srv.run(0) == 0
        st = srv.stats()
        assert st["completed"] == len(reqs) and st["failed"] == 0 and st["queued"] == 0
        for rid, pb in zip(ids, reqs):
            assert srv.poll(rid) == REQ_DONE
            prim, t, ist, lat = srv.result(rid)
            ref, (rt, _, rist) = _solver_result(pb, precision)
            assert t >= pb.tmax and t == rt and ist == rist
            assert np.array_equal(prim, ref)
            assert lat > 0.0


@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
def test_server_nonuniform_radial_maps_equal_solver(precision):
    """Requests on the SINH, LOG and SINH_MODIFIED + POLYTH maps (geometry from the
    Romberg tables built in the submitting thread) next to a uniform-radius one."""
    reqs = [
        _req("sedov", 256, 1.4, 0.01, p_ratio=1.0e4, r0=0.05, dr_min=2.0e-3),
        _req("sedov", 160, 1.4, 0.004, p_ratio=1.0e4, r0=0.02, coords="log", r_in=1.0e-3),
        _req("sod", 200, 1.4, 0.03, rho_ratio=10.0, p_ratio=100.0, dr_min=1.0e-3, coords="default"),
        _req("sod", 300, 1.4, 0.05, rho_ratio=10.0, p_ratio=100.0),
    ]
    with Server(precision=precision, hbm_bytes=256 << 20, max_problems=8, max_zones=4096,
                steps_per_round=13) as srv:
        ids = [srv.submit(pb) for pb in reqs]
        assert srv.run(0) == 0
        for rid, pb in zip(ids, reqs):
            prim, t, ist, _ = srv.result(rid)
            ref, (rt, _, rist) = _solver_result(pb, precision)
            assert t >= pb.tmax and t == rt and ist == rist
            assert np.array_equal(prim, ref)


def test_server_result_same_alone_and_in_mix():
    """Continuous batching: a request's result does not depend on what else is resident,
    nor on when the others arrive."""
    reqs = _mix()
    target = reqs[2]
    with Server(precision=PREC_MIXED, hbm_bytes=256 << 20, max_problems=16, max_zones=4096,
                steps_per_round=13) as srv:
        rid = srv.submit(target)
        srv.run(0)
        alone = srv.result(rid)
    with Server(precision=PREC_MIXED, hbm_bytes=256 << 20, max_problems=16, max_zones=4096,
                steps_per_round=13) as srv:
        others = [srv.submit(pb) for pb in reqs[:2]]
        srv.run(3)                       # the target arrives while two others run
        rid = srv.submit(target)
        srv.run(2)
        late = [srv.submit(pb) for pb in reqs[3:]]   # and more arrive while it runs
        srv.run(0)
        mixed = srv.result(rid)
        for r in others + late:
            srv.result(r)
    assert np.array_equal(alone[0], mixed[0])
    assert alone[1] == mixed[1] and alone[2] == mixed[2]


def test_server_admission_respects_memory_budget():
    """With room for about two problems at a time, the rest wait in the queue and are
    admitted as earlier ones finish; no more memory is ever held than the budget."""
    reqs = [_req("sod", 1000, 1.4, 0.02 + 0.002 * k, rho_ratio=5.0, p_ratio=40.0) for k in range(6)]
    bpu = 2 * 5 * 8 + 22 * 8 + 40 * 8 + 11 * 4
    budget = bpu * (2 * 1004 + 500)
    with Server(precision=PREC_MIXED, hbm_bytes=budget, max_problems=8, max_zones=1000,
                steps_per_round=10) as srv:
        ids = [srv.submit(pb) for pb in reqs]
        srv.run(1)
        st = [srv.poll(r) for r in ids]
        assert st.count(REQ_RUNNING) == 2 and st.count(REQ_QUEUED) == 4
        peak = 0.0
        for _ in range(10000):
            act = srv.run(1)
            s = srv.stats()
            peak = max(peak, s["hbm_in_use"])
            assert s["hbm_in_use"] <= s["hbm_capacity"]
            if act == 0 and s["queued"] == 0:
                break
        assert srv.stats()["completed"] == len(reqs)
        assert 0 < peak <= budget
        for r in ids:
            srv.result(r)


def test_server_request_loop_thread():
    """The loop on the server's own thread while this thread submits and collects."""
    reqs = _mix()
    with Server(precision=PREC_MIXED, hbm_bytes=256 << 20, max_problems=16, max_zones=4096,
                steps_per_round=20) as srv:
        srv.start()
        got = {}

        def client(pbs):
            for pb in pbs:
                got[srv.submit(pb)] = pb

        th = threading.Thread(target=client, args=(reqs,))
        th.start()
        th.join()
        for rid in list(got):
            assert srv.wait(rid, timeout=120.0) == REQ_DONE
        srv.stop()
        s = srv.stats()
        assert s["completed"] == len(reqs) and s["latency_p99"] >= s["latency_p50"] > 0.0
        for rid, pb in got.items():
            prim, t, ist, lat = srv.result(rid)
            assert np.all(np.isfinite(prim)) and t >= pb.tmax


def _mix_2d():
    """2-D requests: Kelvin-Helmholtz and Rayleigh-Taylor of uneven sizes and end times."""
    return [
        P.kelvin_helmholtz(64, 48, seed=5).copy(tmax=0.03, name="kh64x48"),
        P.rayleigh_taylor_2d(40, 72, g=-0.5, noise=0.05).copy(tmax=0.05, name="rt40x72"),
        P.kelvin_helmholtz(96, 130, seed=9).copy(tmax=0.02, name="kh96x130"),
        P.rayleigh_taylor_2d(33, 66, g=-0.1, noise=0.02).copy(tmax=0.04, name="rt33x66"),
    ]


def _server_2d(precision, spr=11):
    return Server(precision=precision, hbm_bytes=256 << 20, max_problems=32, max_zones=4096,
                  steps_per_round=spr, hbm_bytes_2d=64 << 20, max_cells_2d=1 << 16)


@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
def test_server_2d_requests_equal_solver(precision):
    """2-D requests run on the split sweep of the server's precision beside the 1-D lane;
    each result is the solver's run of the same problem, bit for bit, also with 1-D
    requests resident."""
    reqs2 = _mix_2d()
    reqs1 = _mix()[:3]
    with _server_2d(precision) as srv:
        ids2 = [srv.submit(pb) for pb in reqs2]
        ids1 = [srv.submit(pb) for pb in reqs1]
        assert srv.run(0) == 0
        assert srv.stats()["completed"] == len(reqs1) + len(reqs2)
        for rid, pb in zip(ids2, reqs2):
            prim, t, ist, _ = srv.result(rid)
            ref, (rt, _, rist) = _solver_result(pb, precision)
            assert t >= pb.tmax and t == rt and ist == rist, pb.name
            assert np.array_equal(prim, ref), pb.name
        for rid, pb in zip(ids1, reqs1):
            prim, t, ist, _ = srv.result(rid)
            ref, (rt, _, rist) = _solver_result(pb, precision)
            assert t == rt and ist == rist
            assert np.array_equal(prim, ref)


def test_server_2d_slot_reuse_and_graph_recapture():
    """2-D requests arriving and leaving between rounds (the tile lists and the mixed
    round's graph change) and reusing freed cell ranges (shock bits zeroed again)."""
    reqs2 = _mix_2d()
    reqs1 = _mix()
    with _server_2d(PREC_MIXED, spr=7) as srv:
        got = {}
        for k in range(4):
            got[srv.submit(reqs1[k])] = (reqs1[k], PREC_MIXED)
            got[srv.submit(reqs2[k])] = (reqs2[k], PREC_MIXED)
            srv.run(2 + k)
        again = reqs2[0].copy(tmax=0.025)
        got[srv.submit(again)] = (again, PREC_MIXED)
        srv.run(0)
        for rid, (pb, prec) in got.items():
            prim, t, ist, _ = srv.result(rid)
            ref, (rt, _, rist) = _solver_result(pb, prec)
            assert t == rt and ist == rist, pb.name
            assert np.array_equal(prim, ref), pb.name


def _mix_3d():
    # 3-D grids and a 2-D (r, theta) one: all run on the dendritic lane
    return [P.sedov_3d(12, 8, 16, r_dep=0.3).copy(tmax=0.004, name="sedov3d_a"),
            P.sedov_3d(16, 8, 16, r_dep=0.3, noise=0.05).copy(tmax=0.006, name="sedov3d_b"),
            P.sedov_2d_spherical(32, 16, r_dep=0.25, noise=0.05).copy(tmax=0.005, name="sedov2dsph_c")]


@pytest.mark.parametrize("precision", [PREC_MIXED, PREC_FP64])
def test_server_3d_requests_equal_solver(precision):
    """Dendritic-grid requests (3-D, and 2-D in r and theta; each with its own grid, in
    the server's precision) beside 1-D and 2-D Cartesian ones: every result is the
    solver's run of the same problem, bit for bit."""
    reqs3 = _mix_3d()
    reqs = [(pb, precision) for pb in reqs3] + [(pb, precision) for pb in _mix()[:2]] + \
           [(pb, precision) for pb in _mix_2d()[:1]]
    with Server(precision=precision, hbm_bytes=256 << 20, max_problems=32, max_zones=4096, steps_per_round=9,
                hbm_bytes_2d=64 << 20, max_cells_2d=1 << 16, hbm_bytes_3d=512 << 20) as srv:
        ids = []
        for k, (pb, prec) in enumerate(reqs):
            ids.append(srv.submit(pb))
            srv.run(1 + k % 2)           # arrivals between rounds: graph recaptures
        srv.run(0)
        assert srv.stats()["completed"] == len(reqs)
        for rid, (pb, prec) in zip(ids, reqs):
            prim, t, ist, _ = srv.result(rid)
            ref, (rt, _, rist) = _solver_result(pb, prec)
            assert t == rt and ist == rist, pb.name
            assert np.array_equal(prim, ref), pb.name


def test_server_3d_budget_and_refusal():
    pb = _mix_3d()[0]
    with Server(precision=PREC_FP64, hbm_bytes=64 << 20, max_problems=4, max_zones=4096) as srv:
        with pytest.raises(MdgError) as e:
            srv.submit(pb)
        assert e.value.code == 5
    with Server(precision=PREC_FP64, hbm_bytes=64 << 20, max_problems=4, max_zones=4096,
                hbm_bytes_3d=1 << 16) as srv:
        with pytest.raises(MdgError) as e:
            srv.submit(pb)
        assert e.value.code == 6


def test_server_2d_refused_without_arena():
    pb = _mix_2d()[0]
    with Server(precision=PREC_MIXED, hbm_bytes=64 << 20, max_problems=4, max_zones=4096) as srv:
        with pytest.raises(MdgError) as e:
            srv.submit(pb)
        assert e.value.code == 5
    with _server_2d(PREC_MIXED) as srv:
        big = P.kelvin_helmholtz(300, 300, seed=1).copy(tmax=0.01)
        with pytest.raises(MdgError) as e:
            srv.submit(big)
        assert e.value.code == 6


@pytest.mark.parametrize("bad,code", [
    (dict(tmax=1.0e100), 1),                 # no end time
    (dict(n=(5000, 1, 1)), 6),               # larger than max_zones
    (dict(hydro_interp_order=2), 5),         # the mixed sweep is parabolic only
])
def test_server_rejects_requests(bad, code):
    pb = _req("sod", 100, 1.4, 0.01).copy(**bad)
    if "n" in bad:
        pb = pb.copy(ic=np.tile(pb.ic[:1], (bad["n"][0], 1)), dx=(1.0 / bad["n"][0], 2.0, 2.0 * np.pi))
    with Server(precision=PREC_MIXED, hbm_bytes=64 << 20, max_problems=4, max_zones=4096) as srv:
        with pytest.raises(MdgError) as e:
            srv.submit(pb)
        assert e.value.code == code
