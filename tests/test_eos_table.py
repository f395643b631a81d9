"""Tabulated EOS without a GPU: the oracle's restatement of eos_given_rex_per_zone
(oracle/eos_table_oracle.c) against the reference's own function (eos/burrows/
eos_stuff.c:768-902, built unmodified as oracle/_ref/refeos) -- bit for bit on the
committed fixture (tests/golden/make_eos_fixture.py) and live on fresh zones -- and the
C ABI's validation before any device work."""
import ctypes
import os
import subprocess
import tempfile

import numpy as np
import pytest

from medusa_b200 import eos_table as ET
from medusa_b200 import solver as S
from oracle import pyoracle

HERE = os.path.dirname(os.path.abspath(__file__))
REFEOS = os.path.join(pyoracle.REF_DIR, "refeos")


def _grid(g):
    return pyoracle.EosGrid(g.nrec, g.ny, g.nr, g.nt, g.r1, g.r2, g.t1, g.t2, g.y1, g.y2, g.const_hack)


@pytest.fixture(scope="module")
def ref_table():
    return ET.synthetic_table(ET.REFERENCE_GRID)


def test_oracle_matches_reference_fixture(ref_table):
    f = np.load(os.path.join(HERE, "golden", "eos_table_ref.npz"))
    out = pyoracle.eos_given_rex(ref_table, _grid(ET.REFERENCE_GRID), f["rho"], f["u"], f["ye"], f["temp_guess"])
    assert out.shape == f["out"].shape == (f["rho"].size, 5)
    assert np.array_equal(out, f["out"])
    assert np.all(np.isfinite(out)) and np.all(out[:, 0] > 0) and np.all(out[:, 2] > 0)


def test_oracle_matches_reference_build_live(ref_table):
    if not os.path.exists(REFEOS):
        pytest.skip("oracle/_ref/refeos absent (python oracle/build_ref.py)")
    g = ET.REFERENCE_GRID
    rho, u, ye, tg = ET.synthetic_zones(g, 512, seed=21, table=ref_table)
    with tempfile.TemporaryDirectory() as td:
        ft, fz, fo = (os.path.join(td, x) for x in ("table.bin", "zones.bin", "out.bin"))
        ref_table.tofile(ft)
        with open(fz, "wb") as fh:
            fh.write(np.int64(rho.size).tobytes())
            fh.write(np.ascontiguousarray(np.stack([rho, u, ye, tg], axis=1)).tobytes())
        subprocess.run([REFEOS, ft, fz, fo], check=True, stdout=subprocess.DEVNULL)
        ref = np.fromfile(fo, dtype=np.float64).reshape(-1, 5)
    assert np.array_equal(pyoracle.eos_given_rex(ref_table, _grid(g), rho, u, ye, tg), ref)


def test_synthetic_zones_recover_their_temperature(ref_table):
    """The zones' energies come from a target temperature; the update finds it again to
    the accuracy of the table's linear-in-T model between rows."""
    g = ET.REFERENCE_GRID
    rho, u, ye, tg = ET.synthetic_zones(g, 256, seed=5, table=ref_table)
    w = np.array(ET.uniform01(5, 4 * 256)).reshape(256, 4)
    tl = g.t1 + (g.t2 - g.t1) * (0.002 + 0.996 * w[:, 2])
    out = pyoracle.eos_given_rex(ref_table, _grid(g), rho, u, ye, tg)
    assert np.max(np.abs(np.log10(out[:, 2]) - tl)) < 1e-9


def test_abi_checks_before_device_work():
    L = S.library()
    ET._declare(L)
    h = ctypes.c_void_p()
    assert L.mdg_eos_table_create(None, None, 0, ctypes.byref(h)) == 1
    table = np.zeros(4)
    for bad in (ET.EosGrid(nrec=4), ET.EosGrid(nt=1), ET.EosGrid(r2=0.5), ET.EosGrid(y1=0.7)):
        gc = ET.EosGridC.of(bad)
        assert L.mdg_eos_table_create(ctypes.byref(gc), table.ctypes.data, 0, ctypes.byref(h)) == 1
    assert L.mdg_eos_given_rex(None, 1, *([None] * 9)) == 1
    assert L.mdg_eos_given_rex_host(None, 1, *([None] * 8)) == 1
    assert L.mdg_eos_table_destroy(None) == 0


def test_top_row_guess_is_the_reference_result(ref_table):
    """A temperature guess on the table's last row makes the reference start its scan at
    jt = nt; the restatement (and the device kernel) start one row lower.  Where the zone's
    energy lies inside the table the scan goes down in both and brackets the same rows:
    the results are the same bits."""
    if not os.path.exists(REFEOS):
        pytest.skip("oracle/_ref/refeos absent (python oracle/build_ref.py)")
    g = ET.REFERENCE_GRID
    rho, u, ye, _ = ET.synthetic_zones(g, 64, seed=41, table=ref_table)
    tg = np.full(rho.size, 10.0 ** g.t2)
    with tempfile.TemporaryDirectory() as td:
        ft, fz, fo = (os.path.join(td, x) for x in ("table.bin", "zones.bin", "out.bin"))
        ref_table.tofile(ft)
        with open(fz, "wb") as fh:
            fh.write(np.int64(rho.size).tobytes())
            fh.write(np.ascontiguousarray(np.stack([rho, u, ye, tg], axis=1)).tobytes())
        subprocess.run([REFEOS, ft, fz, fo], check=True, stdout=subprocess.DEVNULL)
        ref = np.fromfile(fo, dtype=np.float64).reshape(-1, 5)
    assert np.array_equal(pyoracle.eos_given_rex(ref_table, _grid(g), rho, u, ye, tg), ref)

