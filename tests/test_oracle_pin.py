"""Pin the oracle against the reference run live (needs oracle/_ref, built by
oracle/build_ref.py from the reference tree; skipped where that build is absent)."""
import numpy as np
import pytest

from medusa_b200 import problems as P
from oracle import pyoracle


def _cases():
    out = []
    for seed, kind in enumerate(("sod", "noh", "sedov")):
        for gam in (4.0 / 3.0, 1.4, 5.0 / 3.0):
            out.append(P.spherical_1d(kind, 64 + 37 * seed, gam, rho_ratio=3.0 + seed, p_ratio=30.0 ** (1 + seed),
                                      r0=0.3 if kind == "sod" else 0.08))
    out.append(P.sod(300).copy(bc_lo=(P.REFLECT, 0, 0), bc_hi=(P.EXTRAP, 0, 0)))
    out.append(P.sod(200).copy(bc_lo=(P.PERIODIC, 0, 0), bc_hi=(P.PERIODIC, 0, 0)))
    out.append(P.blast_2d(24, 30, bc=P.PERIODIC))
    out.append(P.blast_2d(30, 24, bc=P.OUTFLOW).copy(bc_lo=(P.EXTRAP, P.OUTFLOW, 0), bc_hi=(P.EXTRAP, P.REFLECT, 0)))
    out.append(P.kelvin_helmholtz(32, 24, seed=3))
    out.append(P.double_rarefaction(150, v=6.0, rho_floor=1.0e-2, e_floor=5.0e-3))
    out.append(P.rayleigh_taylor_2d(24, 40, g=-0.3, noise=0.05))
    out.append(P.sod(160).copy(grav=(-0.9, 0.0, 0.0), name="sod_grav"))
    out.append(P.spherical_1d("sod", 120, 1.4).copy(grav=(-0.4, 0.0, 0.0), name="sph_sod_grav"))
    # the log-spaced radius on [r_in, 1] with a reflecting inner sphere (RCOORD=LOG)
    out.append(P.spherical_1d("sedov", 160, 1.4, p_ratio=1.0e4, r0=0.02, coords="log", r_in=1.0e-3))
    out.append(P.spherical_1d("sod", 96, 5.0 / 3.0, rho_ratio=5.0, p_ratio=50.0, r0=0.1, coords="log", r_in=1.0e-2))
    # the reference's default build maps (SINH_MODIFIED radius, POLYTH theta)
    out.append(P.spherical_1d("sod", 256, 1.4, rho_ratio=10.0, p_ratio=100.0, dr_min=1.0e-3, coords="default"))
    out.append(P.spherical_1d("sedov", 200, 5.0 / 3.0, p_ratio=3.0e3, r0=0.08, dr_min=3.0e-3, coords="default"))
    return out


@pytest.mark.parametrize("pb", _cases(), ids=lambda p: p.name + "_" + "".join(map(str, p.bc_lo + p.bc_hi)))
def test_oracle_equals_live_reference(pb):
    if not pyoracle.ref_available(pb):
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    n = 40
    snaps = pyoracle.run_reference(pb, n, every=10)
    o = pyoracle.Oracle(pb)
    k = 0
    for s in snaps[1:]:
        while k < s[0]:
            o.advance(1)
            k += 1
        prim, _ = o.state()
        assert np.array_equal(prim, s[4]), "diverged at step %d" % s[0]
        assert o.t == s[1]
