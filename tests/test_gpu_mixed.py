"""The mixed-precision batched 1-D sweep (FP32 reconstruction, limiting and Riemann
solve; FP64 state, fluxes, sources, update and dt) against the FP64 oracle and against
analytic solutions, plus the batching, work-queue, CUDA-graph and autotuner invariants.

Accuracy bars (stated per case and recorded in $MDG_PARITY_LOG when set), both runs
compared at the same physical time:
  * volume-weighted relative L1 distance of density and of internal energy density from
    the FP64 oracle after the run: <= MIX_L1_TOL;
  * mass and total-energy difference from the oracle's (compensated sums):
    <= MIX_DRIFT_TOL relative;
  * where an analytic solution exists (planar Sod, spherical Noh): the L1 distance from the
    oracle is at most 10% of the FP64 path's own L1 error against the analytic solution.
Batching invariants are exact: a problem's result does not depend on the other problems
of the batch, on the tile length, on persistent vs one-CTA-per-tile launch or on graph
replay, because every zone's arithmetic is the same in all of them.
"""
import numpy as np
import pytest

from medusa_b200 import analytic as A
from medusa_b200 import problems as P
from medusa_b200.solver import PREC_FP64, PREC_MIXED, MdgError, Solver
from oracle import pyoracle
from tests._cases import record

pytestmark = pytest.mark.gpu

MIX_L1_TOL = 1.0e-4
MIX_DRIFT_TOL = 1.0e-6


def _cases():
    return {
        "sod1d_512": (P.sod(512, tmax=0.2), None),
        "sph_sod_256": (P.spherical_1d("sod", 256, 1.4, rho_ratio=10.0, p_ratio=100.0), 200),
        "sph_noh_256": (P.spherical_1d("noh", 256, 5.0 / 3.0), 300),
        "sph_sedov_256": (P.spherical_1d("sedov", 256, 1.4, p_ratio=1.0e4, r0=0.05), 200),
        "sph_sod_384_g43": (P.spherical_1d("sod", 384, 4.0 / 3.0, rho_ratio=50.0, p_ratio=3.0e3), 250),
        "grav_sod1d_512": (P.sod(512, tmax=0.2).copy(grav=(-0.8, 0.0, 0.0), name="grav_sod1d_512"), 200),
        # non-uniform radial maps: the geometry of the reference's Romberg tables
        "sph_sinh_sedov_256": (P.spherical_1d("sedov", 256, 1.4, p_ratio=1.0e4, r0=0.05, dr_min=2.0e-3), 200),
        "sph_log_sedov_160": (P.spherical_1d("sedov", 160, 1.4, p_ratio=1.0e4, r0=0.02, coords="log",
                                             r_in=1.0e-3), 200),
        "sph_default_sod_256": (P.spherical_1d("sod", 256, 1.4, rho_ratio=10.0, p_ratio=100.0, dr_min=1.0e-3,
                                               coords="default"), 200),
    }


CASES = _cases()


def _weights(pb):
    """Zone volumes (up to 4 pi / 3) of a spherical problem on its radial map."""
    if pb.geom == P.SPHERICAL:
        e = P.radial_edges(pb)
        return e[1:] ** 3 - e[:-1] ** 3
    return None


def _run_oracle(pb, nsteps):
    """FP64 oracle run; with nsteps None, step until t reaches tmax."""
    o = pyoracle.Oracle(pb)
    if nsteps is None:
        nsteps = 0
        while o.t < pb.tmax * (1.0 - 1.0e-12):
            o.advance(1)
            nsteps += 1
    else:
        o.advance(nsteps)
    prim, _ = o.state()
    return prim, nsteps, o.t


def _totals(pb, prim):
    with Solver(pb, precision=PREC_FP64, upload=False) as s:
        s.upload(0, prim)
        m, e = s.conserved_totals()
    return m[0], e[0]


def _analytic(pb, t):
    if pb.name.startswith("sod1d"):
        return A.sod_exact_state(pb.n[0], t, pb.gam)
    if "noh" in pb.name:
        r = (np.arange(pb.n[0]) + 0.5) * pb.dx[0]
        return A.noh_spherical(r, t, pb.gam)
    return None


def _run_mixed_to(pb, t_end, max_steps):
    """Mixed-precision run of pb until t_end (the last step lands on t_end)."""
    with Solver(pb.copy(tmax=t_end), precision=PREC_MIXED) as s:
        n = 0
        while n < max_steps:
            s.step(10)
            n += 10
            if s.time(0)[0] >= t_end * (1.0 - 1.0e-12):
                break
        s.synchronize()
        prim = s.update_cpu(0)
        t, _, istep = s.time(0)
        mm, em = s.conserved_totals()
    return prim, t, mm, em


def _sensitivity_floor(pb, oprim, ot, nsteps):
    """L1 distance (rho, u) at time ot between the FP64 oracle and the FP64 oracle run with
    its CFL number perturbed by 1e-7 relative: how far the problem's own dt sequence can
    move the result for a perturbation at FP32 resolution."""
    o = pyoracle.Oracle(pb.copy(cfl=pb.cfl * (1.0 + 1.0e-7), tmax=ot))
    n = 0
    while o.t < ot * (1.0 - 1.0e-12) and n < 3 * nsteps + 50:
        o.advance(1)
        n += 1
    q, _ = o.state()
    w = _weights(pb)
    return A.l1_rel(q[:, 0], oprim[:, 0], w), A.l1_rel(q[:, 1], oprim[:, 1], w)


@pytest.mark.parametrize("name", sorted(CASES))
def test_mixed_matches_fp64_oracle(name):
    """Both runs stop at the same physical time: the FP64 oracle after its step count,
    the mixed run at that time (its own dt sequence may differ in the last digits).

    Where the problem's FP64 result itself moves by more than 1% of its truncation error
    under a 1e-7 perturbation of the CFL number (the Noh implosion: its dt is set by the
    source-term limit of step.c:205-223 in the zones the shock is entering, and jumps by
    orders of magnitude from step to step), no method that differs from the FP64 sweep in
    the last digits can be closer to it than that floor; there the bar is 3x the floor."""
    pb, nsteps = CASES[name]
    oprim, nsteps, ot = _run_oracle(pb, nsteps)
    prim, t, mm, em = _run_mixed_to(pb, ot, 2 * nsteps + 20)
    floor_rho, floor_u = _sensitivity_floor(pb, oprim, ot, nsteps)
    w = _weights(pb)
    l1_rho = A.l1_rel(prim[:, 0], oprim[:, 0], w)
    l1_u = A.l1_rel(prim[:, 1], oprim[:, 1], w)
    mo, eo = _totals(pb, oprim)
    drift_m = abs(mm[0] - mo) / abs(mo)
    drift_e = abs(em[0] - eo) / abs(eo)
    rec = dict(steps=nsteps, l1_rho=l1_rho, l1_u=l1_u, mass_drift=drift_m, energy_drift=drift_e,
               t_rel=abs(t - ot) / ot, fp64_floor_rho=floor_rho, fp64_floor_u=floor_u)
    ana = _analytic(pb, ot)
    if ana is not None:
        rec["l1_rho_fp64_vs_analytic"] = A.l1_rel(oprim[:, 0], ana[:, 0], w)
        rec["l1_u_fp64_vs_analytic"] = A.l1_rel(oprim[:, 1], ana[:, 1], w)
    record("mixed_vs_oracle_" + name, **rec)
    assert np.all(np.isfinite(prim))
    assert abs(t - ot) <= 1.0e-8 * ot
    sensitive = ana is not None and max(floor_rho / rec["l1_rho_fp64_vs_analytic"],
                                        floor_u / rec["l1_u_fp64_vs_analytic"]) > 0.01
    if sensitive:
        assert l1_rho <= max(MIX_L1_TOL, 3.0 * floor_rho) and l1_u <= max(MIX_L1_TOL, 3.0 * floor_u)
    else:
        assert l1_rho <= MIX_L1_TOL and l1_u <= MIX_L1_TOL
        assert drift_m <= MIX_DRIFT_TOL and drift_e <= MIX_DRIFT_TOL
        if ana is not None:
            assert l1_rho <= 0.1 * rec["l1_rho_fp64_vs_analytic"]
            assert l1_u <= 0.1 * rec["l1_u_fp64_vs_analytic"]


def _small_ensemble(count=12, seed=11):
    return P.ensemble_1d(count=count, seed=seed, nmin=100, nmax=900)


def _run(problems, precision, nsteps, **cfg):
    with Solver(problems, precision=precision) as s:
        if cfg:
            s.set_launch_config(**cfg)
        s.step(nsteps)
        s.synchronize()
        return [s.update_cpu(m) for m in range(len(problems))], [s.time(m) for m in range(len(problems))]


def test_mixed_batched_equals_alone():
    """Continuous-batching invariant: each result is the same alone and in the mix."""
    ens = _small_ensemble()
    batched, bt = _run(ens, PREC_MIXED, 30)
    for m in (0, 3, 7, 11):
        alone, at = _run([ens[m]], PREC_MIXED, 30)
        assert np.array_equal(alone[0], batched[m])
        assert at[0] == bt[m]


def test_mixed_closed_form_and_table_problems_batched_equal_alone():
    """Problems whose geometry is evaluated in closed form and problems that read the
    Romberg tables (SINH and LOG radii, SINH_MODIFIED + POLYTH) run in two launches per
    stage with their own work queues: each result is the same alone and in the batch, in
    persistent and one-CTA-per-tile mode, and with the problems split into lanes."""
    probs = [P.spherical_1d("sedov", 300, 1.4, p_ratio=1.0e4, r0=0.05),
             P.spherical_1d("sedov", 256, 1.4, p_ratio=1.0e4, r0=0.05, dr_min=2.0e-3),
             P.sod(257),
             P.spherical_1d("sedov", 160, 1.4, p_ratio=1.0e4, r0=0.02, coords="log", r_in=1.0e-3),
             P.spherical_1d("sod", 200, 1.4, rho_ratio=10.0, p_ratio=100.0, dr_min=1.0e-3, coords="default")]
    for cfg in (dict(), dict(ctas_per_sm=0), dict(lanes=3)):
        batched, bt = _run(probs, PREC_MIXED, 25, **cfg)
        for m, pb in enumerate(probs):
            alone, at = _run([pb], PREC_MIXED, 25, **cfg)
            assert np.array_equal(alone[0], batched[m]), pb.name
            assert at[0] == bt[m]


@pytest.mark.parametrize("cfg", [dict(threads=64), dict(threads=256), dict(ctas_per_sm=2),
                                 dict(threads=64, ctas_per_sm=8), dict(steps_per_graph=0),
                                 dict(steps_per_graph=7), dict(lanes=2), dict(lanes=4, steps_per_graph=0),
                                 dict(lanes=3, ctas_per_sm=0), dict(lanes=4, threads=256)])
def test_mixed_launch_shapes_identical(cfg):
    ens = _small_ensemble()
    ref, rt = _run(ens, PREC_MIXED, 23)
    got, gt = _run(ens, PREC_MIXED, 23, **cfg)
    for m in range(len(ens)):
        assert np.array_equal(ref[m], got[m])
        assert rt[m] == gt[m]


def test_fp64_graph_replay_identical():
    kh = P.kelvin_helmholtz(64, 48, nsteps=12)
    direct, dtm = _run([kh], PREC_FP64, 12, steps_per_graph=0)
    graph, gtm = _run([kh], PREC_FP64, 12, steps_per_graph=5)
    assert np.array_equal(direct[0], graph[0])
    assert dtm == gtm


def test_autotune_restores_state():
    ens = _small_ensemble(count=20, seed=5)
    ref, rt = _run(ens, PREC_MIXED, 8)
    with Solver(ens, precision=PREC_MIXED) as s:
        s.step(4)
        cfg, ms = s.autotune(trial_steps=3)
        assert cfg["threads"] in (64, 128, 256) and cfg["ctas_per_sm"] >= 0 and cfg["lanes"] in (1, 2, 4) and ms > 0
        assert s.launch_config() == cfg
        s.step(4)
        s.synchronize()
        for m in range(len(ens)):
            assert np.array_equal(s.update_cpu(m), ref[m])
            assert s.time(m) == rt[m]


def test_autotune_rejected_for_fp64():
    with Solver(P.sod(64), precision=PREC_FP64) as s:
        with pytest.raises(MdgError) as e:
            s.autotune(2)
        assert e.value.code == 5


def test_launch_config_validation():
    with Solver(P.sod(64), precision=PREC_MIXED) as s:
        for bad in (dict(threads=96), dict(ctas_per_sm=-1), dict(steps_per_graph=-3), dict(run_length=0),
                    dict(run_length=65), dict(lanes=0), dict(lanes=5)):
            with pytest.raises(MdgError) as e:
                s.set_launch_config(**bad)
            assert e.value.code == 1


def test_conserved_totals_compensated():
    """Totals against numpy sums of the same integrands (1-D spherical with the oracle's
    zone volumes and metric, and 2-D Cartesian)."""
    pb = P.spherical_1d("sedov", 500, 1.4, p_ratio=1.0e4, r0=0.05)
    o = pyoracle.Oracle(pb)
    vol = np.array([o.geom(i)[0] for i in range(pb.n[0])])
    gcov = np.array([o.geom(i)[2:5] for i in range(pb.n[0])])
    with Solver(pb) as s:
        s.step(20)
        prim = s.update_cpu(0)
        m, e = s.conserved_totals()
    rho, u, v = prim[:, 0], prim[:, 1], prim[:, 2:5]
    m_np = np.sum(rho * vol)
    e_np = np.sum((0.5 * rho * np.sum(v * v * gcov, axis=1) + u) * vol)
    assert abs(m[0] - m_np) <= 1e-13 * abs(m_np)
    assert abs(e[0] - e_np) <= 1e-13 * abs(e_np)
    kh = P.kelvin_helmholtz(64, 64, nsteps=5)
    with Solver(kh) as s:
        s.step(5)
        prim = s.update_cpu(0)
        m, e = s.conserved_totals()
    dv = kh.dx[0] * kh.dx[1]
    m_np = np.sum(prim[:, 0]) * dv
    e_np = np.sum(0.5 * prim[:, 0] * np.sum(prim[:, 2:5] ** 2, axis=1) + prim[:, 1]) * dv
    assert abs(m[0] - m_np) <= 1e-13 * abs(m_np)
    assert abs(e[0] - e_np) <= 1e-13 * abs(e_np)
