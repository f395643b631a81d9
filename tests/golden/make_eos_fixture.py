"""Regenerate tests/golden/eos_table_ref.npz: the reference's own tabulated-EOS zone
update (eos/burrows/eos_stuff.c:768-902, built unmodified as oracle/_ref/refeos by
oracle/build_ref.py) on the seeded synthetic table of medusa_b200.eos_table at the
reference's table sizes, for seeded zones inside the table plus edge cases (a temperature
guess below 1e-10, guesses on the first and last temperature rows, densities and Ye on
grid lines).  The table itself is not stored: synthetic_table() regenerates it.

    python oracle/build_ref.py && python tests/golden/make_eos_fixture.py
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from medusa_b200 import eos_table as ET  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "eos_table_ref.npz")


def zones(g, tab):
    rho, u, ye, tg = ET.synthetic_zones(g, 2048, seed=11, table=tab)
    rl, tl, yg = g.axes()
    # temperature guesses below 1e-10 (the update starts from 1 MeV), on the first and the
    # last temperature row, and mid-table
    r2, u2, y2, _ = ET.synthetic_zones(g, 4, seed=12, table=tab)
    guesses = np.array([1.0e-12, 10.0 ** g.t1, 10.0 ** g.t2, 10.0 ** tl[150]])
    # density and Ye on grid lines, with the energy halfway between two temperature rows
    gr = []
    for jr, jy in ((10, 3), (200, 40), (0, 0)):
        rho_g = 10.0 ** rl[jr]
        e = 0.5 * (tab[0, jy, jr, 120] + tab[0, jy, jr, 121])
        gr.append((rho_g, rho_g * (e + g.const_hack) * ET.ERG_PER_UNIT, yg[jy], 10.0 ** tl[60]))
    gr = np.array(gr)
    return (np.concatenate([rho, r2, gr[:, 0]]), np.concatenate([u, u2, gr[:, 1]]),
            np.concatenate([ye, y2, gr[:, 2]]), np.concatenate([tg, guesses, gr[:, 3]]))


def run_reference(tab, rho, u, ye, tg):
    exe = os.path.join(ROOT, "oracle", "_ref", "refeos")
    with tempfile.TemporaryDirectory() as td:
        ft, fz, fo = (os.path.join(td, x) for x in ("table.bin", "zones.bin", "out.bin"))
        np.ascontiguousarray(tab, dtype=np.float64).tofile(ft)
        with open(fz, "wb") as f:
            f.write(np.int64(rho.size).tobytes())
            f.write(np.ascontiguousarray(np.stack([rho, u, ye, tg], axis=1)).tobytes())
        subprocess.run([exe, ft, fz, fo], check=True, stdout=subprocess.DEVNULL)
        return np.fromfile(fo, dtype=np.float64).reshape(-1, 5)


def main():
    g = ET.REFERENCE_GRID
    tab = ET.synthetic_table(g)
    rho, u, ye, tg = zones(g, tab)
    out = run_reference(tab, rho, u, ye, tg)
    np.savez_compressed(OUT, rho=rho, u=u, ye=ye, temp_guess=tg, out=out)
    print("wrote %s (%d zones)" % (OUT, rho.size))


if __name__ == "__main__":
    main()
