"""The output path: asynchronous snapshots of a problem's state and EOS records, and the
reference's 1-D ASCII dump (dump_ascii1, io.c:111-220) written from them.  The dump is
compared character by character with the same format restated here, from the solver's
own download and the reference geometry (the oracle's, pinned to the reference build)."""
import numpy as np
import pytest

from medusa_b200 import problems as P
from medusa_b200.solver import MdgError, Solver
from oracle import pyoracle

pytestmark = pytest.mark.gpu


def _dump_text(pb, prim, eos, t):
    o = pyoracle.Oracle(pb)
    lines = ["# %g" % t]
    mass = 0.0
    for i in range(pb.n[0]):
        x = pb.startx[0] + (i + 0.5) * pb.dx[0]
        if pb.geom == P.SPHERICAL:
            x = abs(x)
        g = o.geom(i)
        vol, s00 = g[0], g[11]          # volume, scale[0][0]
        f = ["%16.14e " % x]
        f += ["%16.14e " % (prim[i, v] * (s00 if v == 2 else 1.0)) for v in range(5)]
        f += ["%16.15e " % eos[i, v] for v in range(5)]
        dm = vol * prim[i, 0]
        f.append("%16.15e " % (mass + 0.5 * dm))
        mass += dm
        f.append("%16.15e %16.15e " % (1.0, 1.0))
        lines.append("".join(f))
    return "\n".join(lines) + "\n"


@pytest.mark.parametrize("pb", [P.spherical_1d("sedov", 200, 1.4, p_ratio=1.0e4, r0=0.05),
                                P.sod(256), P.spherical_1d("sod", 96, 4.0 / 3.0).copy(eos=P.POLYTROPIC)],
                         ids=["sph_sedov", "sod", "sph_poly"])
def test_dump_ascii1_matches_reference_format(pb, tmp_path):
    with Solver(pb) as s:
        s.step(30)
        prim, eos = s.update_cpu(0, with_eos=True)
        t = s.time(0)[0]
        path = tmp_path / "dump_00000"
        s.dump_ascii1(path)
    assert path.read_text() == _dump_text(pb, prim, eos, t)


def test_snapshot_overlaps_later_steps():
    """The snapshot holds the state at the time it was taken, while the solver keeps
    stepping; reading it waits for its host copy only."""
    pb = P.spherical_1d("sod", 4000, 1.4)
    with Solver(pb) as ref:
        ref.step(10)
        want, want_eos = ref.update_cpu(0, with_eos=True)
        t10 = ref.time(0)[0]
    with Solver(pb) as s:
        s.step(10)
        s.snapshot(0)
        s.step(40)                     # queued behind the device-side copies only
        prim, eos, t = s.snapshot_read()
        later = s.update_cpu(0)
    assert t == t10
    assert np.array_equal(prim, want) and np.array_equal(eos, want_eos)
    assert not np.array_equal(later, want)


def test_snapshot_3d_and_errors():
    pb = P.sedov_3d(12, 8, 16, r_dep=0.3)
    with Solver(pb) as s:
        with pytest.raises(MdgError) as e:
            s.snapshot_read()
        assert e.value.code == 8
        s.step(3)
        s.snapshot(0)
        prim, eos, t = s.snapshot_read()
        assert np.array_equal(prim, s.update_cpu(0)) and t == s.time(0)[0]
        with pytest.raises(MdgError) as e:
            s.snapshot_write_ascii1("/dev/null")
        assert e.value.code == 5


def _restart_against_oracle(pb, n_before, n_after, tmp_path):
    """Run n_before steps, write a restart file, resume it in a new solver for n_after
    steps; the oracle does the same through its restart (a new reference process reading
    the file: the state's EOS, dtold = 1e100, estimate_dt's first-call reset)."""
    path = str(tmp_path / "restart.bin")
    with Solver(pb) as s:
        s.step(n_before)
        s.synchronize()
        saved = s.update_cpu(0)
        t0, _, ist0 = s.time(0)
        s.restart_write(path, 0)
    raw = np.fromfile(path, dtype=np.uint8)
    assert raw[:8].tobytes() == b"MDGRST1\x00"
    hdr = np.frombuffer(raw[:48].tobytes(), dtype=np.dtype([("m", "S8"), ("ndim", "<i4"), ("n1", "<i4"),
                                                          ("n2", "<i4"), ("n3", "<i4"), ("istep", "<i4"),
                                                          ("res", "<i4"), ("ncell", "<i8"), ("t", "<f8")]))[0]
    assert hdr["istep"] == ist0 and hdr["t"] == t0 and hdr["ncell"] == saved.shape[0]
    assert np.array_equal(np.frombuffer(raw[48:].tobytes(), dtype="<f8").reshape(-1, 5), saved)
    with Solver(pb) as s:
        s.restart_read(path, 0)
        t1, _, ist1 = s.time(0)
        assert t1 == t0 and ist1 == ist0
        s.step(n_after)
        s.synchronize()
        got = s.update_cpu(0)
        tg, _, istg = s.time(0)
    return saved, t0, got, tg, istg


@pytest.mark.parametrize("pb", [P.spherical_1d("sedov", 200, 1.4, p_ratio=1.0e4, r0=0.05),
                                P.kelvin_helmholtz(48, 40, seed=2)], ids=["sph_sedov", "kh"])
def test_restart_resumes_as_the_reference_does(pb, tmp_path):
    from tests._cases import pointwise_rel_err
    saved, t0, got, tg, istg = _restart_against_oracle(pb, 30, 20, tmp_path)
    o = pyoracle.Oracle(pb)
    o.advance(30)
    ostate, _ = o.state()
    assert pointwise_rel_err(saved, ostate, pb) <= 1.0e-9
    o2 = pyoracle.Oracle(pb)
    o2.restart(saved, t0, 30)
    o2.advance(20)
    ref, _ = o2.state()
    assert istg == 50
    assert abs(tg - o2.t) <= 1.0e-12 * o2.t
    assert pointwise_rel_err(got, ref, pb) <= 1.0e-9


def test_restart_of_a_dendritic_grid_and_wrong_file(tmp_path):
    """3-D dendritic: resuming from the file equals uploading the saved state and setting
    the time record by hand, bit for bit; a file of another grid is refused."""
    pb = P.sedov_3d(16, 8, 16, r_dep=0.25, noise=0.05)
    saved, t0, got, tg, istg = _restart_against_oracle(pb, 10, 6, tmp_path)
    with Solver(pb) as s:
        s.upload(0, saved)
        s.set_time(0, t0, 10)
        s.step(6)
        s.synchronize()
        by_hand = s.update_cpu(0)
        assert s.time(0)[0] == tg
    assert np.array_equal(got, by_hand)
    with Solver(P.sedov_3d(16, 8, 32, r_dep=0.25)) as s:
        with pytest.raises(MdgError) as e:
            s.restart_read(str(tmp_path / "restart.bin"), 0)
        assert e.value.code == 1


def test_write_timers_in_the_reference_timing_csv_columns(tmp_path):
    """timing.csv as output_timers (io.c:51-108) lays it out: a header row when the file is
    new, then per timer its name, t, step, cycle count and max/min/avg seconds; a second
    call appends."""
    import csv
    path = str(tmp_path / "timing.csv")
    with Solver(P.spherical_1d("sedov", 300, 1.4, p_ratio=1.0e4, r0=0.05)) as s:
        s.set_timing(True)
        s.step(5)
        s.write_timers(path)
        s.step(3)
        s.write_timers(path)
        t, _, ist = s.time(0)
    rows = list(csv.reader(open(path)))
    assert rows[0] == ["timer", "time", "step", "ncycle", "max", "min", "avg"]
    assert len(rows) == 1 + 2 * 4
    names = [r[0] for r in rows[1:5]]
    assert names == ["estimate_dt", "stage0", "stage1", "finish"]
    assert all(int(r[3]) == 5 for r in rows[1:5]) and all(int(r[3]) == 8 for r in rows[5:])
    assert all(int(r[2]) == 5 for r in rows[1:5]) and all(int(r[2]) == ist for r in rows[5:])
    assert abs(float(rows[5][1]) - t) <= 1.0e-6 * max(t, 1e-30) + 1e-6
    assert all(float(r[4]) > 0.0 and r[4] == r[5] == r[6] for r in rows[1:])
