"""Regenerate the golden fixtures from the reference itself.

Runs the UNMODIFIED reference hydro (built by oracle/build_ref.py from the reference
tree into oracle/_ref/) on small seeded cases and stores the initial and final
primitive states, the time and the last dt as compressed .npz files next to this script.
The fixtures pin the CPU oracle (tests/test_golden.py) and the GPU sweep
(tests/test_gpu_parity.py) without needing the reference tree at test time.

    python tests/golden/make_golden.py [fixture names]
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
        # the SINH radial map (zones 2e-3 wide at the centre, widening outwards)
        "sph1d_sinh_sedov_192": (P.spherical_1d("sedov", 192, 1.4, p_ratio=1.0e4, r0=0.05, dr_min=2.0e-3), 100),
        # the log-spaced radius on [1e-3, 1] with a reflecting inner sphere (RCOORD=LOG)
        "sph1d_log_sedov_160": (P.spherical_1d("sedov", 160, 1.4, p_ratio=1.0e4, r0=0.02, coords="log",
                                               r_in=1.0e-3), 100),
    }


def cases3d():
    """Dendritic spherical cases (Sedov blast, 3-D and 2-D): name -> (problem, nsteps).
    Their fixtures also hold one step started afresh from the final state (prim1)."""
    return {
        "sedov3d_20x16x32": (P.sedov_3d(20, 16, 32, r_dep=0.2), 30),
        "sedov3d_noisy_18x8x16": (P.sedov_3d(18, 8, 16, r_dep=0.25, noise=0.1), 30),
        "sedov3d_noisy_origin_16x8x16": (P.sedov_3d(16, 8, 16, r_dep=0.25, noise=0.05, bc_inner=P.SPHERICAL_ORIGIN,
                                                    bc_pole=P.SPHERICAL_ORIGIN), 30),
        # 2-D (r, theta) grids: the same machinery without phi faces
        "sedov2dsph_24x16": (P.sedov_2d_spherical(24, 16, r_dep=0.2), 40),
        "sedov2dsph_noisy_40x32": (P.sedov_2d_spherical(40, 32, r_dep=0.2, noise=0.1), 40),
        "sedov2dsph_noisy_origin_32x16": (P.sedov_2d_spherical(32, 16, r_dep=0.25, noise=0.05,
                                                               bc_inner=P.SPHERICAL_ORIGIN,
                                                               bc_pole=P.SPHERICAL_ORIGIN), 40),
        # the SINH radial map on both dendritic grids
        "sedov3d_sinh_24x16x32": (P.sedov_3d(24, 16, 32, r_dep=0.2, dr_min=0.02), 30),
        "sedov2dsph_sinh_noisy_40x32": (P.sedov_2d_spherical(40, 32, r_dep=0.15, noise=0.05, dr_min=0.01), 40),
        # the reference's default build maps (SINH_MODIFIED radius, POLYTH theta); the 1-D
        # case carries the one-step-afresh state (prim1) of this group as well
        "sedov3d_default_24x16x32": (P.sedov_3d(24, 16, 32, r_dep=0.2, dr_min=0.02, coords="default"), 30),
        "sedov2dsph_default_noisy_40x32": (P.sedov_2d_spherical(40, 32, r_dep=0.15, noise=0.05, dr_min=0.01,
                                                                coords="default"), 40),
        "sph1d_default_sedov_192": (P.spherical_1d("sedov", 192, 1.4, p_ratio=1.0e4, r0=0.05, dr_min=2.0e-3,
                                                   coords="default"), 60),
        # the log-spaced radius (RCOORD=LOG) on the 2-D grid, which the reference accepts (on
        # the 3-D grid its init_dendritic rejects it), and the 3-D workload's map: SINH with the
        # transition radius small, zones log-spaced outside it
        "sedov2dsph_log_noisy_40x32": (P.sedov_2d_spherical(40, 32, r_dep=0.15, noise=0.02, coords="log",
                                                            r_in=1.0e-2), 40),
        "sedov3d_sinhrt_noisy_24x16x32": (P.sedov_3d(24, 16, 32, r_dep=0.1, noise=0.02, coords="sinh_rt",
                                                     r_in=1.0e-2), 30),
    }


def cases_gravity():
    """Self-gravity in the monopole approximation (the reference's
    GRAV=SPHERICAL_MONOPOLE_GRAV builds; the C restatement does not cover it): the
    dust-collapse setup of problems/init_dustcollapse.c in 1-D (SINH radius, floors,
    the outer v^r hook; uniform radius without floors) and on the 2-D and 3-D dendritic
    grids; and fixed gravity (GRAV=FIXED_GRAV builds) on the dendritic grids.  Fixtures
    as for cases3d (the state after n steps and one step from it)."""
    return {
        "dust1d_sinh_200": (P.dust_collapse(200), 60),
        "dust1d_uniform_nofloor_128": (P.dust_collapse(128, radius="uniform", floors=False), 60),
        "dust2d_uniform_24x16": (P.dust_collapse(24, 16, ndim=2, radius="uniform", floors=False), 40),
        "dust3d_uniform_16x8x16": (P.dust_collapse(16, 8, 16, ndim=3, radius="uniform", floors=False), 30),
        # the constant acceleration of GRAV=FIXED_GRAV (a contravariant vector, gravity.c:38-64)
        # on the dendritic grids: inward radial, and with theta and phi components as well
        "sedov3d_grav_noisy_16x8x16": (P.sedov_3d(16, 8, 16, r_dep=0.25, noise=0.05).copy(
            grav=(-0.5, 0.0, 0.0), name="sedov3d_grav_noisy_16x8x16"), 30),
        "sedov3d_sinh_grav3_18x8x16": (P.sedov_3d(18, 8, 16, r_dep=0.2, noise=0.05, dr_min=0.02).copy(
            grav=(-0.4, 0.3, 0.2), name="sedov3d_sinh_grav3_18x8x16"), 30),
        "sedov2dsph_grav_noisy_24x16": (P.sedov_2d_spherical(24, 16, r_dep=0.2, noise=0.05).copy(
            grav=(-0.6, 0.25, 0.1), name="sedov2dsph_grav_noisy_24x16"), 40),
    }


def main(only=()):
    """Regenerate every fixture, or only those named in `only`."""
    build_ref.build()
    for name, (pb, n) in list(cases3d().items()) + list(cases_gravity().items()):
        if only and name not in only:
            continue
        snaps = pyoracle.run_reference(pb, n, every=n)
        last = snaps[-1]
        one = pyoracle.run_reference(pb.copy(ic=last[4]), 1, every=1)[-1]
        out = os.path.join(HERE, name + ".npz")
        np.savez_compressed(out, prim=last[4], t=last[1], dt=last[2], nsteps=n, istep=last[0],
                            prim1=one[4], t1=one[1], dt1=one[2])
        print(name, "steps", last[0], "t", last[1], "->", os.path.relpath(out, ROOT))
    for name, (pb, n) in cases().items():
        if only and name not in only:
            continue
        snaps = pyoracle.run_reference(pb, n, every=n)
        first, last = snaps[0], snaps[-1]
        out = os.path.join(HERE, name + ".npz")
        np.savez_compressed(out, ic=first[4], prim=last[4], t=last[1], dt=last[2], nsteps=n,
                            istep=last[0])
        print(name, "steps", last[0], "t", last[1], "->", os.path.relpath(out, ROOT))


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
