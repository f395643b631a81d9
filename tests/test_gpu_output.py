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
