// 3-D spherical grid with dendritic coarsening (utils.c:181-525): radial row i has
// nj[i] theta zones and row (i, j) has nk[i][j] phi zones; the interior zones are stored
// in the reference's zone order (i, then j, then k: ZLOOP, decs.h:614), structure of
// arrays, no ghost zones.  Everything that depends only on (i, j) -- the zone geometry,
// the refinement factors -- lives in "row tables" indexed by
//     ij = rowbase[i + NG] + j + NG,   i in [-NG, n1+NG), j in [-NG, nj[i]+NG)
// (ghost rows included: the boundary maps, the restriction volumes and the pole
// faces read them).  The reconstruction moments of directions 1 and 2 depend on the
// refinement level only (init_interp_vol, metric_spherical_general.c:592-668) and are
// tabulated per level.
#pragma once
#include <stdint.h>
#include <vector>
#include "mdg_internal.h"

namespace mdg {

constexpr int G3_MAXLEV = 16;

// Per-row geometry fields of zone (i, j, k) (every k of a row has the same record).
enum Geo3Field {
  G3_VOL,                     // volume
  G3_A0, G3_A1, G3_A2,        // area[0..2] of the lower faces
  G3_GCOV,                    // gcov[loc][m] at G3_GCOV + 3*loc + m, loc 0 (zone), 1..3 (faces)
  G3_GCON = G3_GCOV + 12,     // gcon[m]
  G3_SCALE = G3_GCON + 3,     // scale[loc][m] at G3_SCALE + 3*loc + m
  G3_C000 = G3_SCALE + 12,    // the connection coefficients the spherical metric sets
  G3_C011, G3_C022, G3_C101, G3_C110, G3_C111, G3_C122, G3_C202, G3_C220, G3_C212, G3_C221,
  G3_NFIELDS
};
static_assert(G3_NFIELDS == MDG_GEO3_FIELDS, "row geometry record of mdg_grid3d_geometry");

// Device view of the grid and its tables (pointers into one device allocation).
// Flux addresses push() reads for the zones of one interior row (i, j), precomputed on the
// host from the dendritic structure (the device then issues every flux load of a zone at
// once instead of walking the row tables): the direction-0 faces of the one or two rows
// of radial row i+1 over it (zone k collects nkp consecutive faces of each, from face
// k*nkp), its own lower direction-0 faces, the direction-1 faces of rows (i, j+1) and
// (i, j) with their fan-in, and its direction-2 faces.
struct PushRow3 {
  int64_t f0o[2];   // first direction-0 face of the outer rows (i+1, jp), (i+1, jp+1)
  int64_t f0i;      // first direction-0 face of row (i, j)
  int64_t f1o, f1i; // first direction-1 face of rows (i, j+1) and (i, j)
  int64_t f2;       // first direction-2 face of row (i, j) (3-D grids)
  int64_t cell;     // first zone of row (i, j)
  int nf0o;         // outer rows: 1 or 2
  int nkp[2];       // outer faces per zone of each outer row
  int mo;           // outer theta faces: 0 one per zone, 1 half of a coarser row's face, 2 two faces
  int mi;           // inner theta faces: 0 one per zone, 1 halves of two faces
};

struct Grid3 {
  int ndim;                   // 3, or 2 for the axisymmetric (r, theta) grid (n3 = 1, no phi faces)
  int n1, n2, n3;
  int bc_lo0, bc_hi0, bc_lo1, bc_hi1, bc_lo2, bc_hi2;
  double dx0, dx1, dx2;
  int64_t nij;                // row-table length
  int64_t ncell;              // interior zones
  int64_t nf0, nf1, nf2;      // faces per direction
  const int *nj;              // [n1+2NG] theta zones of row i (i+NG)
  const int *rowbase;         // [n1+2NG] row-table index of (i, -NG)
  const int *nk;              // [nij] phi zones of row (i, j)
  const int64_t *cell;        // [nij] first zone of an interior row, -1 otherwise
  const int64_t *f0;          // [nij] first direction-0 face of row (i, j), i in [0, n1], j in [0, nj)
  const int64_t *f1;          // [nij] first direction-1 face, i in [0, n1), j in [0, nj]
  const int64_t *f2;          // [nij] first direction-2 face, i in [0, n1), j in [0, nj)
  const double *geo;          // [G3_NFIELDS][nij]
  const double *rc0;          // [RC_NFIELDS][n1+2NG] direction-0 reconstruction table
  const double *rc1;          // [RC_NFIELDS][cols1] per (level, j): column rc1_base[lev] + j + NG
  const double *rc2;          // [RC_NFIELDS][cols2] per (level, k)
  int64_t cols1, cols2;
  int rc1_base[G3_MAXLEV], rc2_base[G3_MAXLEV];
  const double *xc1, *xc2;    // beta/Gamma (volume centroid coordinate) in the rc1/rc2 columns
  const double *sth, *cth;    // sin/cos(theta(beta1s/Gamma1s)) in the rc1 columns (polar fix)
  const double *sphc, *cphc;  // sin/cos(phi) at the zone centre, rc2 columns
  const double *sphl, *cphl;  // sin/cos(phi) at the lower phi face, rc2 columns
  const float *mx0, *mx1, *mx2;   // FP32 reconstruction weights (MixField) of the rc0/rc1/rc2 columns
  const double *medge;        // [2][n1+1] SQR(redge[i]), dr_dx at radial edge i (monopole gravity)
  double *gmono;              // [n1] monopole gravity at the radial zone centroids (shell masses first)
  double x0;                  // startx[0]
  int mono;                   // GRAV=SPHERICAL_MONOPOLE_GRAV
  const PushRow3 *prow;       // [nij] push() flux addresses of interior rows
};

MDG_HD inline int ilog2(int s)
{
  int l = 0;
  while (s >>= 1) l++;
  return l;
}

// Host-side tables of the grid (built by build_grid3 in mdg_geometry.cpp).
struct Grid3Host {
  int ndim = 3, n1 = 0, n2 = 0, n3 = 0;
  std::vector<int> nj, rowbase, nk;
  std::vector<int64_t> cell, f0, f1, f2;
  std::vector<double> geo, rc0, rc1, rc2, xc1, xc2, sth, cth, sphc, cphc, sphl, cphl, medge;
  std::vector<float> mx0, mx1, mx2;
  int64_t nij = 0, ncell = 0, nf0 = 0, nf1 = 0, nf2 = 0, cols1 = 0, cols2 = 0;
  int nlev1 = 0, nlev2 = 0;
  int rc1_base[G3_MAXLEV] = {}, rc2_base[G3_MAXLEV] = {};
  int row(int i, int j) const { return rowbase[i + NG] + j + NG; }
  int njr(int i) const { return nj[i + NG]; }
  int dj(int i) const { return n2 / nj[i + NG]; }
  int dk(int i, int j) const { return n3 / nk[row(i, j)]; }
};

}  // namespace mdg
