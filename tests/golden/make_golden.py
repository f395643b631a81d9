"""Regenerate the golden fixtures from the reference itself.

Runs the UNMODIFIED reference hydro (built by oracle/build_ref.py from the reference
tree into oracle/_ref/) on small seeded cases and stores the initial and final
primitive states, the time and the last dt as compressed .npz files next to this script.
The fixtures pin the CPU oracle (tests/test_golden.py) and the GPU sweep
(tests/test_gpu_parity.py) without needing the reference tree at test time.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from medusa_b200 import problems as P  # noqa: E402
from oracle import build_ref, pyoracle  # noqa: E402


def cases():
    """name -> (problem, nsteps).  Kept small: every fixture is a few tens of KB."""
    return {
        "sod1d_1024": (P.sod(1024), 60),
        "sph1d_sod_128": (P.spherical_1d("sod", 128, 1.4, rho_ratio=8.0, p_ratio=50.0), 80),
        "sph1d_noh_200": (P.spherical_1d("noh", 200, 5.0 / 3.0), 100),
        "sph1d_noh_nofloor_160": (P.spherical_1d("noh", 160, 1.4, floors=False), 90),
        "double_rare1d_v6_floors_200": (P.double_rarefaction(200, v=6.0, rho_floor=1.0e-2, e_floor=5.0e-3), 80),
        "sph1d_sedov_256": (P.spherical_1d("sedov", 256, 1.4, p_ratio=1.0e4, r0=0.05), 100),
        "sph1d_sod_poly_lin_96": (P.spherical_1d("sod", 96, 4.0 / 3.0, rho_ratio=20.0)
                                  .copy(eos=P.POLYTROPIC, Kpoly=1.0, hydro_interp_order=2), 60),
        "sod1d_pcm_256": (P.sod(256).copy(hydro_interp_order=1), 40),
        "kh2d_48x40": (P.kelvin_helmholtz(48, 40, seed=11), 25),
        "blast2d_40x48_reflect": (P.blast_2d(40, 48, bc=P.REFLECT), 40),
        "blast2d_44x36_outflow": (P.blast_2d(44, 36, bc=P.OUTFLOW), 40),
        "rt2d_32x64_grav": (P.rayleigh_taylor_2d(32, 64, g=-0.5, noise=0.05), 40),
    }


def main():
    build_ref.build()
    for name, (pb, n) in cases().items():
        snaps = pyoracle.run_reference(pb, n, every=n)
        first, last = snaps[0], snaps[-1]
        out = os.path.join(HERE, name + ".npz")
        np.savez_compressed(out, ic=first[4], prim=last[4], t=last[1], dt=last[2], nsteps=n,
                            istep=last[0])
        print(name, "steps", last[0], "t", last[1], "->", os.path.relpath(out, ROOT))


if __name__ == "__main__":
    main()
