"""The dendritic spherical grid (3-D, and 2-D in r and theta) on the host: zone counts (compute_dj/compute_dk,
utils.c:181-354) and per-row zone geometry (init_geometry, metric_spherical_general.c)
of the library against the Python restatement and against the reference build itself;
the 3-D fixtures against the problem generator and the live reference."""
import subprocess

import numpy as np
import pytest

from medusa_b200 import problems as P
from medusa_b200 import solver as S
from medusa_b200.solver import MdgError
from oracle import pyoracle
from tests._cases import golden_cases3d, load_golden

CASES3 = golden_cases3d()
# the reference record of ref_get_geom: vol, area[3], gcov[4][3], gcon[3], scale[4][3],
# conn[27]; the library keeps the 11 coefficients the spherical metric sets
CONN_SET = [0, 4, 8, 10, 12, 13, 17, 20, 24, 23, 25]


@pytest.mark.parametrize("dims", [(20, 16, 32), (64, 64, 128), (384, 128, 256), (7, 2, 4)])
def test_zone_counts_match_restatement(dims):
    pb = P.sedov_3d(*dims, r_dep=0.3)
    nj, nk, n = S.grid3d_counts(pb)
    pj, pk = P.dendritic_grid(*dims, pb.startx, pb.dx)
    assert list(nj) == pj
    assert list(nk) == [x for row in pk for x in row]
    assert n == pb.ncell == sum(sum(r) for r in pk)


@pytest.mark.parametrize("dims,dr_min", [((24, 16, 32), 0.02), ((384, 128, 256), 1.0e-3)])
def test_sinh_zone_counts_match_restatement_and_reference(dims, dr_min):
    pb = P.sedov_3d(*dims, r_dep=0.2, dr_min=dr_min)
    nj, nk, n = S.grid3d_counts(pb)
    pj, pk = P.dendritic_grid(*dims, pb.startx, pb.dx, rtrans=pb.rtrans)
    assert list(nj) == pj and list(nk) == [x for row in pk for x in row] and n == pb.ncell
    if dims[0] <= 64 and pyoracle.ref_available(pb):
        rnj, rnk = pyoracle.reference_grid(pb)
        assert list(nj) == rnj[2:-2]
    edges = P.radial_edges(pb)
    assert abs(edges[-1] - 1.0) <= 1.0e-9 and abs(edges[1] - dr_min) <= 1.0e-2 * dr_min


@pytest.mark.parametrize("dims,r_in", [((24, 16, 32), 1.0e-2), ((48, 32, 64), 1.0e-3), ((384, 128, 256), 1.0e-3)])
def test_log_radius_3d_grid_refused_as_by_the_reference(dims, r_in):
    """The log-spaced radius (RCOORD=LOG, zone edges r_in (1/r_in)^(i/n1)) on the 3-D
    dendritic grid: theta zones double at every radial row from nj = 2 and the phi zones
    then refine 4-to-1 between neighbouring rows, which the reference's init_dendritic
    rejects (it prints the cells and exits, utils.c:548-586).  The library refuses the
    same grids with MDG_ERR_INVALID; the restatement finds 4-to-1 cells too."""
    pb = P.sedov_3d(*dims, r_dep=0.2, coords="log", r_in=r_in)
    with pytest.raises(MdgError) as e:
        S.grid3d_counts(pb)
    assert e.value.code == 1 and "4-to-1" in str(e.value)
    nj, nk = P.dendritic_grid(*dims, pb.startx, pb.dx, maps=P.CoordMaps.of(pb))
    assert P.dendritic_refine_errors(dims[1], dims[2], nj, nk) > 0
    if dims[0] <= 64 and pyoracle.ref_available(pb):
        with pytest.raises(subprocess.CalledProcessError):
            pyoracle.reference_grid(pb)


@pytest.mark.parametrize("dims,r_in", [((24, 16), 1.0e-2), ((48, 32), 1.0e-3), ((384, 128), 1.0e-3)])
def test_log_radius_2d_zone_counts_match_restatement_and_reference(dims, r_in):
    """On the 2-D (r, theta) grid the log-spaced radius is accepted (no phi refinement)."""
    pb = P.sedov_2d_spherical(*dims, r_dep=0.2, coords="log", r_in=r_in)
    nj, nk, n = S.grid3d_counts(pb)
    pj, _ = P.dendritic_grid(dims[0], dims[1], 1, pb.startx, pb.dx, ndim=2, maps=P.CoordMaps.of(pb))
    assert list(nj) == pj and n == pb.ncell == sum(pj)
    if dims[0] <= 64 and pyoracle.ref_available(pb):
        rnj, _ = pyoracle.reference_grid(pb)
        assert list(nj) == rnj[2:-2]
    edges = P.radial_edges(pb)
    want = r_in * (1.0 / r_in) ** (np.arange(dims[0] + 1) / dims[0])
    assert np.allclose(edges, want, rtol=1.0e-12, atol=0.0)


def test_c3_grid_size():
    """The measured 3-D workload: 384 x 128 x 256 before coarsening."""
    pb = P.sedov_3d(384, 128, 256)
    nj, nk, n = S.grid3d_counts(pb)
    assert nj[0] == 2 and nj[-1] == 128 and nk.min() == 4 and nk.max() == 256
    assert n == pb.ncell < 384 * 128 * 256


@pytest.mark.parametrize("dims,dr_min,coords", [((24, 16, 32), None, "sinh"), ((40, 32, 64), None, "sinh"),
                                                ((48, 64, 128), None, "sinh"), ((24, 16, 32), 0.02, "sinh"),
                                                ((48, 32, 64), 0.01, "sinh"), ((24, 16, 32), 0.02, "default"),
                                                ((48, 32, 64), 0.01, "default"), ((384, 128, 256), 1.98e-5, "sinh")])
def test_geometry_bit_identical_to_reference(dims, dr_min, coords):
    """Uniform radius, the SINH radial map (against the reference's RCOORD=SINH build; the
    last case is the measured 3-D workload's grid, rtrans about 1e-3: zones log-spaced
    from r = 1e-3 to 1, 2e-5 wide inside) and the default build maps SINH_MODIFIED +
    POLYTH."""
    pb = P.sedov_3d(*dims, r_dep=0.2, dr_min=dr_min, coords=coords)
    if not pyoracle.ref_available(pb):
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    rnj, _ = pyoracle.reference_grid(pb)
    geo = S.grid3d_geometry(pb)
    ref = pyoracle.reference_geometry(pb)
    theirs = np.concatenate([ref[:, 0:31], ref[:, 31:58][:, CONN_SET]], axis=1)
    assert geo.shape == theirs.shape
    n1 = dims[0]
    r = 0
    for i in range(-2, n1 + 2):
        for j in range(-2, rnj[i + 2] + 2):
            # volume, gcov, gcon, scale on every row; areas on the face rows; conn inside
            fields = [0] + list(range(4, 31))
            if 0 <= i <= n1 and 0 <= j <= rnj[i + 2]:
                fields += [1, 2, 3]
            if 0 <= i < n1 and 0 <= j < rnj[i + 2]:
                fields += list(range(31, 42))
            assert np.array_equal(geo[r, fields], theirs[r, fields]), (i, j)
            r += 1


@pytest.mark.parametrize("dims", [(24, 16), (256, 128), (5, 2)])
def test_2d_zone_counts_match_restatement(dims):
    pb = P.sedov_2d_spherical(*dims, r_dep=0.3)
    nj, nk, n = S.grid3d_counts(pb)
    pj, _ = P.dendritic_grid(dims[0], dims[1], 1, pb.startx, pb.dx, ndim=2)
    assert list(nj) == pj
    assert np.all(nk == 1)
    assert n == pb.ncell == sum(pj)


# the NDIM=2 record of ref_get_geom: vol, area[2], gcov[3][3], gcon[3], scale[3][3], conn[27]
@pytest.mark.parametrize("dims,dr_min,coords", [((24, 16), None, "sinh"), ((48, 32), None, "sinh"),
                                                ((40, 64), None, "sinh"), ((40, 32), 0.01, "sinh"),
                                                ((40, 32), 0.01, "default"), ((40, 32), 1.0e-2, "log"),
                                                ((64, 32), 1.0e-3, "log")])
def test_2d_geometry_bit_identical_to_reference(dims, dr_min, coords):
    """As the 3-D test; for coords "log" (the RCOORD=LOG build) dr_min is the inner radius."""
    if coords == "log":
        pb = P.sedov_2d_spherical(*dims, r_dep=0.2, coords="log", r_in=dr_min)
    else:
        pb = P.sedov_2d_spherical(*dims, r_dep=0.2, dr_min=dr_min, coords=coords)
    if not pyoracle.ref_available(pb):
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    rnj, _ = pyoracle.reference_grid(pb)
    geo = S.grid3d_geometry(pb)
    ref = pyoracle.reference_geometry(pb)
    assert geo.shape[0] == ref.shape[0]
    assert not np.any(ref[:, 24:51][:, [c for c in range(27) if c not in CONN_SET]])
    n1 = dims[0]
    r = 0
    for i in range(-2, n1 + 2):
        for j in range(-2, rnj[i + 2] + 2):
            pairs = [(geo[r, 0:1], ref[r, 0:1]), (geo[r, 4:13], ref[r, 3:12]), (geo[r, 16:19], ref[r, 12:15]),
                     (geo[r, 19:28], ref[r, 15:24])]
            if 0 <= i <= n1 and 0 <= j <= rnj[i + 2]:
                pairs.append((geo[r, 1:3], ref[r, 1:3]))
            if 0 <= i < n1 and 0 <= j < rnj[i + 2]:
                pairs.append((geo[r, 31:42], ref[r, 24:51][CONN_SET]))
            for a, b in pairs:
                assert np.array_equal(a, b), (i, j)
            r += 1


def test_2d_zone_volumes_fill_the_sphere():
    pb = P.sedov_2d_spherical(32, 16, r_dep=0.2)
    vol = S.grid3d_zone_volumes(pb)
    assert vol.shape == (pb.ncell,) and np.all(vol > 0)
    assert abs(vol.sum() - 4.0 / 3.0 * np.pi) <= 1.0e-12


def test_grid_calls_validate():
    pb = P.sedov_3d(16, 8, 16)
    with pytest.raises(MdgError) as e:
        S.grid3d_counts(pb.copy(n=(16, 12, 16)))
    assert e.value.code == 1
    with pytest.raises(MdgError) as e:
        S.grid3d_counts(pb.copy(geom=P.CARTESIAN))
    assert e.value.code == 5
    with pytest.raises(MdgError) as e:
        S.grid3d_counts(P.kelvin_helmholtz(16, 16, nsteps=1))
    assert e.value.code == 5


@pytest.mark.parametrize("name", sorted(CASES3))
def test_fixture_matches_generator(name):
    pb, n = CASES3[name]
    g = load_golden(name)
    assert g["prim"].shape == (pb.ncell, 5) and g["prim1"].shape == (pb.ncell, 5)
    assert int(g["istep"]) == n
    assert np.all(np.isfinite(g["prim"]))


@pytest.mark.parametrize("name", sorted(CASES3))
def test_fixture_reproduced_by_live_reference(name):
    pb, n = CASES3[name]
    if not pyoracle.ref_available(pb):
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    g = load_golden(name)
    snaps = pyoracle.run_reference(pb, n, every=n)
    assert np.array_equal(snaps[-1][4], g["prim"])
    assert snaps[-1][1] == float(g["t"])


def test_zone_volumes_fill_the_sphere():
    pb = P.sedov_3d(24, 16, 32, r_dep=0.2)
    vol = S.grid3d_zone_volumes(pb)
    assert vol.shape == (pb.ncell,) and np.all(vol > 0)
    assert abs(vol.sum() - 4.0 / 3.0 * np.pi) <= 1.0e-12
    prof = S.grid3d_radial_mean(pb, np.ones(pb.ncell))
    assert np.allclose(prof, 1.0, rtol=0, atol=1e-14)
