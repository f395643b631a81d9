"""GPU parity of the dendritic spherical sweep against fixtures made by the reference
itself (tests/golden/make_golden.py, cases3d): Sedov blasts on small 3-D dendritic
grids and on 2-D (r, theta) ones, symmetric and with seeded noise (shock tagging,
rotation through the pole rows, restriction of the phi velocity into the Gamma slot),
reflecting and SPHERICAL_ORIGIN boundaries.

Error measures: pointwise (tests/_cases.py pointwise_rel_err: density and internal
energy relative at every zone, each physical velocity component over the zone's own
speed scale max(|v|, c_s), with the library's zone metric), and field-relative per
variable (max |gpu - ref| over the zones divided by the largest magnitude of that
variable, or of any velocity component: the three velocities share one scale, since in
the symmetric blast v^theta and v^phi are round-off).  Bars as for the 1-D/2-D sweeps,
both measures: 1e-9 after a whole fixture run, 1e-12 for one step.
"""
import numpy as np
import pytest

from medusa_b200 import problems as P
from medusa_b200.solver import PREC_FP64, PREC_MIXED, Solver
from tests._cases import golden_cases3d, load_golden, pointwise_rel_err, record, zone_gcov

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
    pw = pointwise_rel_err(prim, g["prim"], pb, zone_gcov(pb))
    record("sweep3d_full_" + name, steps=n, err=e, pointwise=pw, bit_identical=float(np.mean(prim == g["prim"])))
    assert istep == n
    assert e <= FULL_RUN_TOL
    assert pw <= FULL_RUN_TOL
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
    pw = pointwise_rel_err(prim, g["prim1"], pb, zone_gcov(pb))
    record("sweep3d_step_" + name, err=e, pointwise=pw, bit_identical=float(np.mean(prim == g["prim1"])))
    assert pw <= PER_STEP_TOL
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


def test_2d_spherical_mass_change_is_the_outer_boundary_flux():
    pb, n = CASES3["sedov2dsph_24x16"]
    with Solver(pb) as s:
        m0, _ = s.conserved_totals()
        s.step(10)
        m1, _ = s.conserved_totals()
    assert abs(m1[0] - m0[0]) <= 1.0e-13 * m0[0]


# ---------------------------------------------------------------- mixed precision
def _shock_radius(pb, prim):
    """Radius of the largest radial-row mean density (zone centre on the grid's radial map)
    and the width of that zone."""
    from medusa_b200.solver import grid3d_radial_mean
    i = int(np.argmax(grid3d_radial_mean(pb, prim[:, 0])))
    e = P.radial_edges(pb)
    return P.radial_centers(pb)[i], e[i + 1] - e[i]


@pytest.mark.parametrize("dr_min", [None, 0.004], ids=["uniform", "sinh"])
def test_3d_mixed_matches_fp64_at_equal_time(dr_min):
    """FP32 reconstruction and wave speeds, FP64 state, fluxes, sources and dt: volume-
    weighted relative L1 of rho and u against the plain FP64 sweep (the reference's
    arithmetic) at the same physical time <= 1e-4; mass and energy within 1e-6 of the
    FP64 run's; the blast radius equal to the FP64 run's within one zone, both near
    Sedov's R_s = xi0 (E t^2/rho)^(1/5); on the uniform radius and on the SINH map."""
    from medusa_b200 import analytic as A
    from medusa_b200.solver import PREC_MIXED
    pb = P.sedov_3d(48, 32, 64, r_dep=0.1 if dr_min is None else 0.04, dr_min=dr_min)
    n = 60
    with Solver(pb) as s:
        s.step(n)
        ref = s.update_cpu(0)
        t_end = s.time(0)[0]
        m0, e0 = s.conserved_totals()
    with Solver(pb.copy(tmax=t_end), precision=PREC_MIXED) as s:
        for _ in range(40):
            s.step(5)
            if s.time(0)[0] >= t_end * (1.0 - 1.0e-12):
                break
        mix = s.update_cpu(0)
        t_mix = s.time(0)[0]
        m1, e1 = s.conserved_totals()
    assert abs(t_mix - t_end) <= 1.0e-8 * t_end
    from medusa_b200.solver import grid3d_zone_volumes
    vol = grid3d_zone_volumes(pb)
    l1_rho = A.l1_rel(mix[:, 0], ref[:, 0], vol)
    l1_u = A.l1_rel(mix[:, 1], ref[:, 1], vol)
    drift_m = abs(m1[0] - m0[0]) / m0[0]
    drift_e = abs(e1[0] - e0[0]) / e0[0]
    (r_ref, w_ref), (r_mix, _) = _shock_radius(pb, ref), _shock_radius(pb, mix)
    r_sedov = A.sedov_shock_radius(1.0, t_end, 1.0, 1.4)
    record("sweep3d_mixed_" + pb.name, l1_rho=l1_rho, l1_u=l1_u, drift_mass=drift_m, drift_energy=drift_e,
           r_fp64=r_ref, r_mixed=r_mix, r_sedov=r_sedov, t=t_end)
    assert np.all(np.isfinite(mix))
    assert l1_rho <= 1.0e-4 and l1_u <= 1.0e-4
    assert drift_m <= 1.0e-6 and drift_e <= 1.0e-6
    assert abs(r_mix - r_ref) <= w_ref
    if dr_min is None:   # 60 steps of the fine central zones leave the SINH blast near its deposit
        assert abs(r_ref - r_sedov) <= 4 * w_ref


def test_2d_spherical_mixed_matches_fp64_at_equal_time():
    """The mixed-precision dendritic sweep on a 2-D (r, theta) Sedov blast: the same bars
    as in 3-D against the plain FP64 sweep at the same time."""
    from medusa_b200 import analytic as A
    from medusa_b200.solver import PREC_MIXED, grid3d_zone_volumes
    pb = P.sedov_2d_spherical(96, 64, r_dep=0.06, noise=0.02)
    n = 80
    with Solver(pb) as s:
        s.step(n)
        ref = s.update_cpu(0)
        t_end = s.time(0)[0]
        m0, e0 = s.conserved_totals()
    with Solver(pb.copy(tmax=t_end), precision=PREC_MIXED) as s:
        for _ in range(40):
            s.step(5)
            if s.time(0)[0] >= t_end * (1.0 - 1.0e-12):
                break
        mix = s.update_cpu(0)
        t_mix = s.time(0)[0]
        m1, e1 = s.conserved_totals()
    assert abs(t_mix - t_end) <= 1.0e-8 * t_end
    vol = grid3d_zone_volumes(pb)
    l1_rho = A.l1_rel(mix[:, 0], ref[:, 0], vol)
    l1_u = A.l1_rel(mix[:, 1], ref[:, 1], vol)
    drift_m = abs(m1[0] - m0[0]) / m0[0]
    drift_e = abs(e1[0] - e0[0]) / e0[0]
    record("sweep2dsph_mixed_sedov_96x64", l1_rho=l1_rho, l1_u=l1_u, drift_mass=drift_m, drift_energy=drift_e, t=t_end)
    assert np.all(np.isfinite(mix))
    assert l1_rho <= 1.0e-4 and l1_u <= 1.0e-4
    assert drift_m <= 1.0e-6 and drift_e <= 1.0e-6
    (r_ref, w_ref), (r_mix, _) = _shock_radius(pb, ref), _shock_radius(pb, mix)
    assert abs(r_mix - r_ref) <= w_ref


def test_c3_full_size_invariants():
    """The measured workload itself (384 x 128 x 256, zones log-spaced from r = 1e-3 to 1
    on the SINH map with rtrans = 1e-3, 8.49 M zones), where the reference cannot run per
    step: size-independent properties after 10 steps.  The blast is symmetric in phi, so
    the zones of a row (i, j) must hold the same state and v^phi must stay zero -- up to
    the round-off of the polar-axis fix, which rotates the phi-face states of the last
    theta row through Cartesian components (the reference does the same).  Velocities are
    compared as physical components (sqrt(g_kk) v^k) over the zone's own speed scale
    max(|v|, c_s), density and internal energy over their values at the row's first zone:
    bar 1e-10.  Mass changes only through the outer face, which the blast has not
    reached."""
    import bench
    from medusa_b200.solver import grid3d_counts, grid3d_zone_gcov
    pb = bench.sedov3d_problem((384, 128, 256))
    nj, nk, n = grid3d_counts(pb)
    with Solver(pb) as s:
        m0, _ = s.conserved_totals()
        s.step(10)
        m1, _ = s.conserved_totals()
        prim = s.update_cpu(0)
    assert np.all(np.isfinite(prim))
    drift = abs(m1[0] - m0[0]) / m0[0]
    sq = np.sqrt(grid3d_zone_gcov(pb))
    vphys = prim[:, 2:5] * sq
    cs = np.sqrt(pb.gam * (pb.gam - 1.0) * prim[:, 1] / prim[:, 0])
    vscale = np.maximum(np.sqrt(np.sum(vphys ** 2, axis=1)), cs)
    vphi = float(np.max(np.abs(vphys[:, 2]) / vscale))
    rows = np.repeat(np.arange(len(nk)), nk)
    first = np.concatenate([[0], np.cumsum(nk)[:-1]])[rows]
    asym = [float(np.max(np.abs(prim[:, v] - prim[first, v]) / np.abs(prim[first, v]))) for v in (0, 1)]
    asym += [float(np.max(np.abs(vphys[:, k] - vphys[first, k]) / vscale[first])) for k in (0, 1)]
    record("sweep3d_c3_full_size_invariants", zones=n, mass_change=drift, vphi_rel=vphi, phi_asymmetry=asym)
    assert drift <= 1.0e-13
    assert vphi <= 1.0e-10
    assert max(asym) <= 1.0e-10


@pytest.mark.parametrize("precision", [PREC_FP64, PREC_MIXED])
def test_3d_run_length_does_not_change_results(precision):
    """The radial and theta run kernels give the same bits for every run length (each
    face's pencil entries and reconstructions are the same whichever work item computes
    them); the autotuner picks a run length and leaves the state as it was."""
    pb = P.sedov_3d(24, 16, 32, r_dep=0.2, noise=0.05, dr_min=0.02)
    out = {}
    for run in (1, 3, 16, 64):
        with Solver(pb, precision=precision) as s:
            s.set_launch_config(run_length=run)
            assert s.launch_config()["run_length"] == run
            s.step(12)
            out[run] = (s.update_cpu(0), s.time(0))
    for run in (1, 3, 64):
        assert np.array_equal(out[run][0], out[16][0])
        assert out[run][1] == out[16][1]
    with Solver(pb, precision=precision) as s:
        s.step(4)
        cfg, ms = s.autotune(trial_steps=2)
        assert cfg["run_length"] in (4, 8, 16, 32) and ms > 0
        assert s.launch_config()["run_length"] == cfg["run_length"]
        s.step(8)
        assert np.array_equal(s.update_cpu(0), out[16][0])
        assert s.time(0) == out[16][1]
