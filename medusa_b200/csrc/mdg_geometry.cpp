// Host-side geometry tables of the sweep, rebuilt from the problem description exactly
// as the reference's init_geometry() builds them (geometry.c:4-63), and reduced to the
// per-index tables the kernels read.
//
//   Cartesian: metrics/metric_cartesian.c:47-55 (volume moments), 127-295 (volume,
//              area, gcov, gcon, scale; conn = 0)
//   Spherical, 1-D, radius UNIFORM or SINH (the RCOORD switch), THCOORD=UNIFORM:
//              metrics/metric_spherical_general.c:149-243 (maps), 558-568 (moments),
//              708-740 (volume), 745-779 (area), 820-930 (conn), 941-1051 (gcov, gcon,
//              scale); Romberg integration as utils.c:16-62.
//
// Compiled with -ffp-contract=off so that every product and sum rounds as in the
// reference's CPU build.
#include <cmath>
#include <cstring>
#include <vector>
#include "mdg_internal.h"
#include "mdg_tables.cuh"
#include "mdg_grid3d.cuh"
#include <algorithm>
#include "../../include/medusa_b200.h"

namespace mdg {

// ----------------------------------------------------------------- Romberg (utils.c:16-62)
static double rtrap(double x0, double x1, int rstage, double (*f)(double))
{
  unsigned long long nseg = 1ULL << rstage, i;
  double dx = (x1 - x0) / nseg, sum = 0.0;
  if (rstage == 0) return 0.5 * dx * ((*f)(x0) + (*f)(x1));
  for (i = 0; i < (1ULL << (rstage - 1)); i++) sum += (*f)(x0 + (2 * i + 1) * dx);
  return dx * sum;
}

static double romb(double x0, double x1, double (*f)(double))
{
  double rvec[16], R0, R1;
  unsigned long long fm;
  rvec[0] = rtrap(x0, x1, 0, f);
  for (int rstage = 1; rstage <= 15; rstage++) {
    R0 = rvec[0];
    rvec[0] = 0.5 * R0 + rtrap(x0, x1, rstage, f);
    for (int m = 1; m <= rstage; m++) {
      fm = 1ULL << (2 * m);
      R1 = rvec[m];
      rvec[m] = 1.0 / (fm - 1) * (fm * rvec[m - 1] - R0);
      R0 = R1;
    }
    if (std::fabs((rvec[rstage] - rvec[rstage - 1]) / rvec[rstage]) < 1.e-15 ||
        (rstage > 2 && std::fabs(rvec[rstage]) < 1.e-15))
      return rvec[rstage];
  }
  return rvec[15];
}

// The coordinate maps of the problem being built (RCOORD and THCOORD,
// metric_spherical_general.c:149-290): r(x) UNIFORM |x|, SINH rtrans sinh(|x|/rtrans),
// SINH_MODIFIED (the SINH map minus a sigmoid step of height facta) or LOG
// rtrans exp(|x|/rtrans) (zones log-spaced outwards from r = rtrans at x = 0; the
// reference has no such map: it is written in the form of its SINH branch, and the
// oracle's reference builds with RCOORD=LOG carry the same three expressions), th(x)
// UNIFORM or POLYTH.  The integrands below are plain functions handed to romb(), so the maps are
// per-thread state that CoordMap sets for the duration of one public build call (the
// solve server builds tables in the submitting threads).
namespace {
struct MapState {
  int rcoord = MDG_RCOORD_UNIFORM;
  double rtrans = 1.0, facta = 0.0, factb = 0.0, factc = 1.0;
  int thcoord = MDG_THCOORD_UNIFORM;
  double poly_norm = 0.0, poly_xt = 1.0, poly_alpha = 0.0;
};
thread_local MapState t_map;
struct CoordMap {
  MapState saved;
  explicit CoordMap(const mdg_problem_desc &d) : saved(t_map)
  {
    t_map.rcoord = d.rcoord;
    t_map.rtrans = d.rtrans;
    t_map.facta = d.rfact[0];
    t_map.factb = d.rfact[1];
    t_map.factc = d.rfact[2];
    t_map.thcoord = d.thcoord;
    t_map.poly_xt = d.poly_xt;
    t_map.poly_alpha = d.poly_alpha;
    // init_coords (metric_spherical_general.c:565-567)
    if (d.thcoord == MDG_THCOORD_POLYTH)
      t_map.poly_norm = 0.5 * M_PI * 1.0 / (1.0 + 1.0 / (d.poly_alpha + 1.0) * 1.0 / std::pow(d.poly_xt, d.poly_alpha));
  }
  ~CoordMap() { t_map = saved; }
};
}  // namespace
using RadialMap = CoordMap;
static double sigmoid(double x) { return 1.0 / (1.0 + std::exp(-x)); }
static double r_of_x(double x)
{
  const MapState &m = t_map;
  if (m.rcoord == MDG_RCOORD_SINH) return m.rtrans * std::sinh(std::fabs(x) / m.rtrans);
  if (m.rcoord == MDG_RCOORD_LOG) return m.rtrans * std::exp(std::fabs(x) / m.rtrans);
  if (m.rcoord == MDG_RCOORD_SINH_MODIFIED)
    return m.rtrans * std::sinh(std::fabs(x) / m.rtrans) - m.facta * sigmoid((std::fabs(x) - m.factb) / m.factc) +
           m.facta * sigmoid(-m.factb / m.factc);
  return std::fabs(x);
}
static double dr_dx(double x)
{
  const MapState &m = t_map;
  if (m.rcoord == MDG_RCOORD_SINH) return std::cosh(std::fabs(x) / m.rtrans);
  if (m.rcoord == MDG_RCOORD_LOG) return std::exp(std::fabs(x) / m.rtrans);
  if (m.rcoord == MDG_RCOORD_SINH_MODIFIED) {
    const double expval = std::exp(-(std::fabs(x) - m.factb) / m.factc);
    return std::cosh(std::fabs(x) / m.rtrans) - m.facta * expval / m.factc / (1 + expval) / (1 + expval);
  }
  return 1.0;
}
static double d2r_dx2(double x)
{
  const MapState &m = t_map;
  if (m.rcoord == MDG_RCOORD_SINH) return std::sinh(std::fabs(x) / m.rtrans) / m.rtrans;
  if (m.rcoord == MDG_RCOORD_LOG) return std::exp(std::fabs(x) / m.rtrans) / m.rtrans;
  if (m.rcoord == MDG_RCOORD_SINH_MODIFIED) {
    const double expval = std::exp(-(std::fabs(x) - m.factb) / m.factc);
    return std::sinh(std::fabs(x) / m.rtrans) / m.rtrans -
           m.facta / m.factc / m.factc *
               (2 * expval * expval / (1 + expval) / (1 + expval) / (1 + expval) - expval / (1 + expval) / (1 + expval));
  }
  return 0.0;
}
// v^1 of the two outer ghost zones under the dust-collapse boundary hook
// (problems/init_dustcollapse.c:104-113): r at the zone centroid beta0/Gamma0,
// v^r = -1/sqrt(r), divided by the zone's scale[0][0].
void build_moments(const mdg_problem_desc &d, int dir, std::vector<double> &al, std::vector<double> &be,
                   std::vector<double> &ga);
void build_geo_1d(const mdg_problem_desc &d, double *tab, int64_t stride, int64_t off);
void dust_ghost_u1(const mdg_problem_desc &d, double *u1)
{
  RadialMap rmap(d);
  std::vector<double> al, be, ga;
  build_moments(d, 0, al, be, ga);
  const int64_t w = d.n1 + 2 * NG;
  std::vector<double> geo((size_t)GF_NFIELDS * w, 0.0);
  build_geo_1d(d, geo.data(), w, 0);
  for (int q = 0; q < 2; q++) {
    const int i = d.n1 + q;
    const double r = r_of_x(be[i + NG] / ga[i + NG]);
    const double vr = -1.0 / std::sqrt(r);
    u1[q] = vr / geo[(size_t)GF_S00 * w + i + NG];
  }
}

// r(x) of a problem's radial map (ijk_to_x + r_of_x as the dumps use them, io.c:171-174)
double radial_coordinate(const mdg_problem_desc &d, double x)
{
  RadialMap rmap(d);
  return r_of_x(x);
}
// theta map with the reflection about the polar axis (metric_spherical_general.c:222-290)
static double th_of_x(double x)
{
  if (x < -1.0) x = -2.0 - x;
  if (x > 1.0) x = 2.0 - x;
  const MapState &m = t_map;
  if (m.thcoord == MDG_THCOORD_POLYTH)
    return m.poly_norm * x * (1.0 + std::pow(x / m.poly_xt, m.poly_alpha) / (m.poly_alpha + 1.0)) + 0.5 * M_PI;
  return 0.5 * M_PI * (x + 1.0);
}
static double dth_dx(double x)
{
  if (x < -1.0) x = -2.0 - x;
  if (x > 1.0) x = 2.0 - x;
  const MapState &m = t_map;
  if (m.thcoord == MDG_THCOORD_POLYTH) return m.poly_norm * (1.0 + std::pow(x / m.poly_xt, m.poly_alpha));
  return 0.5 * M_PI;
}
static double d2th_dx2(double x)
{
  if (x < -1.0) x = -2.0 - x;
  if (x > 1.0) x = 2.0 - x;
  const MapState &m = t_map;
  if (m.thcoord == MDG_THCOORD_POLYTH)
    return m.poly_norm * m.poly_alpha * std::pow(x / m.poly_xt, m.poly_alpha - 1.0) / m.poly_xt;
  return 0.0;
}
static double f_r2dr_dx(double x) { return std::pow(r_of_x(x), 2) * dr_dx(x); }
static double f_xr1g(double x) { return x * std::pow(r_of_x(x), 2) * dr_dx(x); }
static double f_xr2g(double x) { return x * x * std::pow(r_of_x(x), 2) * dr_dx(x); }
static double f_r2d2r_dx2(double x) { return std::pow(r_of_x(x), 2) * d2r_dx2(x); }
static double f_r3(double x) { return std::pow(r_of_x(x), 3); }
static double f_r2dr_dx3(double x) { return std::pow(r_of_x(x), 2) * std::pow(dr_dx(x), 3); }
static double f_rdr_dx2(double x) { return r_of_x(x) * std::pow(dr_dx(x), 2); }
static double f_sthdth_dx(double x) { return std::sin(th_of_x(x)) * dth_dx(x); }
static double f_sthdth_dx3(double x) { return std::sin(th_of_x(x)) * std::pow(dth_dx(x), 3); }
static double f_sth3dth_dx(double x) { return std::pow(std::sin(th_of_x(x)), 3) * dth_dx(x); }
static double f_sthd2th_dx2(double x) { return std::sin(th_of_x(x)) * d2th_dx2(x); }
static double f_cthdth_dx2(double x) { return std::cos(th_of_x(x)) * std::pow(dth_dx(x), 2); }

// Volume moments alpha/beta/Gamma of direction d over i in [-NG, n+NG), stored at i+NG.
void build_moments(const mdg_problem_desc &d, int dir, std::vector<double> &al,
                   std::vector<double> &be, std::vector<double> &ga)
{
  RadialMap rmap(d);
  const int n = (dir == 0) ? d.n1 : (dir == 1 ? d.n2 : d.n3);
  al.assign(n + 2 * NG, 0.0); be.assign(n + 2 * NG, 0.0); ga.assign(n + 2 * NG, 0.0);
  for (int i = -NG; i < n + NG; i++) {
    if (d.geom == MDG_CARTESIAN) {
      double x0 = d.startx[dir] + i * d.dx[dir], x1 = x0 + d.dx[dir];
      al[i + NG] = (x1 * x1 * x1 - x0 * x0 * x0) / 3.0;
      be[i + NG] = (x1 * x1 - x0 * x0) / 2.0;
      ga[i + NG] = d.dx[dir];
    } else {
      double x0 = d.startx[0] + i * d.dx[0], x1 = d.startx[0] + (i + 1) * d.dx[0];
      ga[i + NG] = romb(x0, x1, f_r2dr_dx);
      be[i + NG] = romb(x0, x1, f_xr1g);
      al[i + NG] = romb(x0, x1, f_xr2g);
    }
  }
}

// Reconstruction coefficient table (RC_NFIELDS x stride, starting at column `off`) for the
// zones of direction dir: zone i at column off+i+NG, i in [-NG, n+NG).
void build_recon_table(const mdg_problem_desc &d, int dir, double *tab, int64_t stride, int64_t off)
{
  std::vector<double> al, be, ga;
  build_moments(d, dir, al, be, ga);
  const int n = (dir == 0) ? d.n1 : d.n2;
  for (int i = -NG; i < n + NG; i++) {
    int im = (i - 1 < -NG) ? -NG : i - 1, ip = (i + 1 >= n + NG) ? n + NG - 1 : i + 1;
    double am = al[im + NG], a0 = al[i + NG], ap = al[ip + NG];
    double bm = be[im + NG], b0 = be[i + NG], bp = be[ip + NG];
    double gm = ga[im + NG], g0 = ga[i + NG], gp = ga[ip + NG];
    // zone edges as prim_to_fluxesN forms them: startx + index*dx (step.c:509,736)
    double xl = d.startx[dir] + i * d.dx[dir];
    double xr = d.startx[dir] + (i + 1) * d.dx[dir];
    double v[RC_NFIELDS];
    rc_fields(am, a0, ap, bm, b0, bp, gm, g0, gp, xl, xr, v);
    for (int f = 0; f < RC_NFIELDS; f++) tab[f * stride + off + i + NG] = v[f];
  }
}

// Face and zone geometry of a 1-D problem (GF_NFIELDS x stride, starting at column off).
void build_geo_1d(const mdg_problem_desc &d, double *tab, int64_t stride, int64_t off)
{
  RadialMap rmap(d);
  const int n1 = d.n1;
  auto put = [&](int f, int i, double v) { tab[f * stride + off + i + NG] = v; };
  for (int i = -NG; i < n1 + NG; i++)
    for (int f = 0; f < GF_NFIELDS; f++) put(f, i, 0.0);
  if (d.geom == MDG_CARTESIAN) {
    for (int i = -NG; i < n1 + NG; i++) {
      double vol = 1.0;
      vol *= d.dx[0];
      double area = 1.0;
      area *= d.dx[0];
      area /= d.dx[0];
      put(GF_VOL, i, vol);
      put(GF_AREA, i, (i >= 0 && i <= n1) ? area : 0.0);
      put(GF_FSCALE, i, 1.0);
      put(GF_FG0, i, 1.0); put(GF_FG1, i, 1.0); put(GF_FG2, i, 1.0);
      put(GF_G0, i, 1.0); put(GF_G1, i, 1.0); put(GF_G2, i, 1.0);
      put(GF_GC0, i, 1.0); put(GF_GC1, i, 1.0); put(GF_GC2, i, 1.0);
      put(GF_S00, i, 1.0);
    }
    return;
  }
  // spherical 1-D: x1 in [-1,1], dx[1] = 2, dx[2] = 2 pi (init_coords)
  const double x1lo = -1.0, x1hi = 1.0, dph = 2.0 * M_PI;
  double vthf = romb(x1lo, x1hi, f_sthdth_dx);
  double th_sthdth_dx3 = romb(x1lo, x1hi, f_sthdth_dx3);
  double th_sth3dth_dx = romb(x1lo, x1hi, f_sth3dth_dx);
  double th_sthd2th_dx2 = romb(x1lo, x1hi, f_sthd2th_dx2);
  double th_cthdth_dx2 = romb(x1lo, x1hi, f_cthdth_dx2);
  for (int i = -NG; i < n1 + NG; i++) {
    double x0lo = d.startx[0] + i * d.dx[0], x0hi = d.startx[0] + (i + 1) * d.dx[0];
    double r2dr_int = romb(x0lo, x0hi, f_r2dr_dx);
    double vrf = r2dr_int;
    double rint_r2dr_dx3 = romb(x0lo, x0hi, f_r2dr_dx3);
    put(GF_VOL, i, r2dr_int * vthf * 1 * dph);
    put(GF_AREA, i, (i >= 0 && i <= n1) ? f_r2dr_dx(x0lo) * vthf * (1 * dph) : 0.0);
    double g00 = rint_r2dr_dx3 / vrf;
    double g01 = std::fabs(0.2 * (std::pow(r_of_x(x0hi), 5) - std::pow(r_of_x(x0lo), 5)) / vrf * th_sthdth_dx3 / vthf);
    double g02 = std::fabs(0.2 * (std::pow(r_of_x(x0hi), 5) - std::pow(r_of_x(x0lo), 5)) / vrf * th_sth3dth_dx / vthf);
    double g10 = std::pow(dr_dx(x0lo), 2);
    double g11 = std::pow(r_of_x(x0lo), 2) * th_sthdth_dx3 / vthf;
    double g12 = std::pow(r_of_x(x0lo), 2) * th_sth3dth_dx / vthf;
    put(GF_G0, i, g00); put(GF_G1, i, g01); put(GF_G2, i, g02);
    put(GF_FG0, i, g10); put(GF_FG1, i, g11); put(GF_FG2, i, g12);
    put(GF_GC0, i, (std::fabs(g00) > 1.0e-50) ? 1.0 / g00 : 0.0);
    put(GF_GC1, i, (std::fabs(g01) > 1.0e-50) ? 1.0 / g01 : 0.0);
    put(GF_GC2, i, (std::fabs(g02) > 1.0e-50) ? 1.0 / g02 : 0.0);
    put(GF_S00, i, std::sqrt(g00));
    put(GF_FSCALE, i, std::sqrt(g10));
    // radial edge i as init_coords (metric_spherical_general.c:577-583) and
    // monopole_gravity_finish (gravity.c:300-303) use it
    const double re = r_of_x(std::fabs(i * d.dx[0] + d.startx[0]));
    put(GF_RE2, i, re * re);
    put(GF_DRDX, i, dr_dx(d.startx[0] + i * d.dx[0]));
    if (i >= 0 && i < n1) {
      double c[3][3][3];
      std::memset(c, 0, sizeof c);
      double rint_r2d2r_dx2 = romb(x0lo, x0hi, f_r2d2r_dx2);
      double rint_r3 = romb(x0lo, x0hi, f_r3);
      double rint_rdr_dx2 = romb(x0lo, x0hi, f_rdr_dx2);
      double vr = romb(x0lo, x0lo + d.dx[0], f_r2dr_dx);
      c[0][0][0] = rint_r2d2r_dx2 / vr;
      c[0][1][1] = -(rint_r3 / vr) * (th_sthdth_dx3 / vthf);
      c[1][0][1] = rint_rdr_dx2 / vr;
      c[1][1][0] = c[1][0][1];
      c[2][0][2] = c[1][0][1];
      c[2][2][0] = c[2][0][2];
      c[2][1][2] = th_cthdth_dx2 / vthf;
      c[2][2][1] = c[2][1][2];
      c[0][2][2] = -c[2][2][0] * g02 / g00;
      c[1][2][2] = -c[2][2][1] * g02 / g01;
      c[1][1][1] = th_sthd2th_dx2 / vthf;
      for (int l = 0; l < 3; l++)
        for (int m = 0; m < 3; m++)
          for (int nn = 0; nn < 3; nn++) put(GF_CONN + (l * 9 + m * 3 + nn), i, c[l][m][nn]);
    }
  }
}

// Cartesian 2-D constants: volume = dx0*dx1, area[loc] = (dx0*dx1)/dx[loc]
// (metric_cartesian.c:127-189, loop order of init_volume/init_area).
void cartesian_2d_constants(const mdg_problem_desc &d, double &vol, double &area0, double &area1)
{
  vol = 1.0; vol *= d.dx[0]; vol *= d.dx[1];
  area0 = 1.0; area0 *= d.dx[0]; area0 *= d.dx[1]; area0 /= d.dx[0];
  area1 = 1.0; area1 *= d.dx[0]; area1 *= d.dx[1]; area1 /= d.dx[1];
}

}  // namespace mdg

namespace mdg {

// Non-allocating variants for callers that provide every buffer: the same moments and
// reconstruction table as build_moments/build_recon_table above, written into caller
// memory (al/be/ga hold n+2*NG entries each).
void build_moments_into(const mdg_problem_desc &d, int dir, double *al, double *be, double *ga)
{
  RadialMap rmap(d);
  const int n = (dir == 0) ? d.n1 : (dir == 1 ? d.n2 : d.n3);
  for (int i = -NG; i < n + NG; i++) {
    if (d.geom == MDG_CARTESIAN) {
      double x0 = d.startx[dir] + i * d.dx[dir], x1 = x0 + d.dx[dir];
      al[i + NG] = (x1 * x1 * x1 - x0 * x0 * x0) / 3.0;
      be[i + NG] = (x1 * x1 - x0 * x0) / 2.0;
      ga[i + NG] = d.dx[dir];
    } else {
      double x0 = d.startx[0] + i * d.dx[0], x1 = d.startx[0] + (i + 1) * d.dx[0];
      ga[i + NG] = romb(x0, x1, f_r2dr_dx);
      be[i + NG] = romb(x0, x1, f_xr1g);
      al[i + NG] = romb(x0, x1, f_xr2g);
    }
  }
}

void build_recon_table_into(const mdg_problem_desc &d, int dir, double *tab, int64_t stride, int64_t off,
                            double *al, double *be, double *ga)
{
  build_moments_into(d, dir, al, be, ga);
  const int n = (dir == 0) ? d.n1 : d.n2;
  for (int i = -NG; i < n + NG; i++) {
    int im = (i - 1 < -NG) ? -NG : i - 1, ip = (i + 1 >= n + NG) ? n + NG - 1 : i + 1;
    double am = al[im + NG], a0 = al[i + NG], ap = al[ip + NG];
    double bm = be[im + NG], b0 = be[i + NG], bp = be[ip + NG];
    double gm = ga[im + NG], g0 = ga[i + NG], gp = ga[ip + NG];
    double xl = d.startx[dir] + i * d.dx[dir];
    double xr = d.startx[dir] + (i + 1) * d.dx[dir];
    double v[RC_NFIELDS];
    rc_fields(am, a0, ap, bm, b0, bp, gm, g0, gp, xl, xr, v);
    for (int f = 0; f < RC_NFIELDS; f++) tab[f * stride + off + i + NG] = v[f];
  }
}

}  // namespace mdg

namespace mdg {

// FP32 reconstruction weights (MX_* fields, see mdg_internal.h) of direction dir, zone i
// at column off+i+NG, computed in FP64 from the volume moments.
void build_mixed_table(const mdg_problem_desc &d, int dir, float *tab, int64_t stride, int64_t off)
{
  std::vector<double> al, be, ga;
  build_moments(d, dir, al, be, ga);
  const int n = (dir == 0) ? d.n1 : d.n2;
  for (int i = -NG; i < n + NG; i++) {
    int im = (i - 1 < -NG) ? -NG : i - 1, ip = (i + 1 >= n + NG) ? n + NG - 1 : i + 1;
    double am = al[im + NG], a0 = al[i + NG], ap = al[ip + NG];
    double bm = be[im + NG], b0 = be[i + NG], bp = be[ip + NG];
    double gm = ga[im + NG], g0 = ga[i + NG], gp = ga[ip + NG];
    double xl = d.startx[dir] + i * d.dx[dir];
    double xr = d.startx[dir] + (i + 1) * d.dx[dir];
    float v[MX_NFIELDS];
    mx_fields(am, a0, ap, bm, b0, bp, gm, g0, gp, xl, xr, v);
    for (int f = 0; f < MX_NFIELDS; f++) tab[f * stride + off + i + NG] = v[f];
  }
}

}  // namespace mdg

namespace mdg {

// 1 when every connection coefficient outside SPARSE_CONN is exactly zero in the nrec
// records of a 1-D geometry table starting at column off.
int conn_is_sparse(const double *tab, int64_t stride, int64_t off, int nrec)
{
  bool keep[27] = {};
  for (int k = 0; k < NSPARSE_CONN; k++) keep[SPARSE_CONN[k]] = true;
  for (int k = 0; k < 27; k++) {
    if (keep[k]) continue;
    for (int i = 0; i < nrec; i++)
      if (tab[(GF_CONN + k) * stride + off + i] != 0.0) return 0;
  }
  return 1;
}

}  // namespace mdg

namespace mdg {

// Angular constants of the 1-D spherical metric (theta integrated over [0, pi], phi over
// 2 pi; metric_spherical_general.c:708-930): area/volume factor vthf*dph, and the
// theta averages th_sthdth_dx3/vthf, th_sth3dth_dx/vthf, th_cthdth_dx2/vthf that scale
// gcov[.][1], gcov[.][2] and conn[2][1][2].  With them every per-zone quantity of the
// uniform-radius grid is a polynomial in the zone's edge radii (see the mixed sweep).
void spherical_1d_constants(double &area_k, double &th1, double &th2, double &tc)
{
  const double x1lo = -1.0, x1hi = 1.0, dph = 2.0 * M_PI;
  const double vthf = romb(x1lo, x1hi, f_sthdth_dx);
  area_k = vthf * 1 * dph;
  th1 = romb(x1lo, x1hi, f_sthdth_dx3) / vthf;
  th2 = romb(x1lo, x1hi, f_sth3dth_dx) / vthf;
  tc = romb(x1lo, x1hi, f_cthdth_dx2) / vthf;
}

}  // namespace mdg

namespace mdg {

static double f_xth1g(double x) { return x * std::sin(th_of_x(x)) * dth_dx(x); }
static double f_xth2g(double x) { return x * x * std::sin(th_of_x(x)) * dth_dx(x); }

// Grid, geometry and reconstruction tables of a 3-D spherical problem on the dendritic
// grid, uniform radius and theta:
//   zone counts      compute_dj / compute_dk (utils.c:181-354; MAX_LOG2_ASPECT utils.c:12)
//   moments          init_interp_vol (metric_spherical_general.c:592-668)
//   volume, area     init_volume / init_area (708-816), axis areas hard-zero
//   gcov, gcon, scale, conn   (941-1051, 837-939), conn[1][1][1] from the dendritic
//                    neighbour areas (897-916)
// with the reference's operation order (every product and sum as written there).
// Zone counts of the dendritic grid, compute_dj / compute_dk (utils.c:181-366): nj per
// radial row and nk per (i, j) row, ghost rows and columns included, and the row tables.
void dendritic_zone_counts(const mdg_problem_desc &d, Grid3Host &h)
{
  RadialMap rmap(d);
  const bool three = d.ndim == 3;
  const int n1 = d.n1, n2 = d.n2, n3 = three ? d.n3 : 1;
  h.ndim = three ? 3 : 2;
  h.n1 = n1; h.n2 = n2; h.n3 = n3;
  const double sx0 = d.startx[0], sx1 = d.startx[1];
  const double dx0 = d.dx[0], dx1 = d.dx[1], dx2 = d.dx[2];
  const double max_log2_aspect = 0.5;
  // theta zones per radial row
  h.nj.assign(n1 + 2 * NG, 0);
  auto NJ = [&](int i) -> int & { return h.nj[i + NG]; };
  NJ(0) = 2;
  {
    const double dth = th_of_x(sx1 + n2 * dx1) - th_of_x(sx1);
    for (int i = 1; i < n1; i++) {
      double r0 = r_of_x(sx0 + (i + 0.0) * dx0);
      double rc = r_of_x(sx0 + (i + 0.5) * dx0);
      double r1 = r_of_x(sx0 + (i + 1.0) * dx0);
      double dr = r1 - r0;
      double nj_ideal = rc * dth / dr;
      NJ(i) = NJ(i - 1);
      if (std::log2(nj_ideal / NJ(i)) > max_log2_aspect) NJ(i) *= 2;
      NJ(i) = std::min(std::max(NJ(i), NJ(i - 1)), n2);
    }
  }
  for (int i = -NG; i < 0; i++) NJ(i) = NJ(-i - 1);
  for (int i = n1; i < n1 + NG; i++) NJ(i) = NJ(n1 - 1);
  auto DJ = [&](int i) { return n2 / NJ(i); };

  // row tables
  h.rowbase.assign(n1 + 2 * NG, 0);
  int64_t nij = 0;
  for (int i = -NG; i < n1 + NG; i++) {
    h.rowbase[i + NG] = (int)nij;
    nij += NJ(i) + 2 * NG;
  }
  h.nij = nij;
  h.nk.assign(nij, 0);
  auto NK = [&](int i, int j) -> int & { return h.nk[h.rowbase[i + NG] + j + NG]; };

  // phi zones per (i, j); a 2-D grid has one (compute_dk's branch for other grids)
  if (!three) {
    for (auto &v : h.nk) v = n3;
  } else {
    const int nk_min = 4;
    const double dph = n3 * dx2;
    NK(0, 0) = nk_min;
    for (int j = 1; j < NJ(0); j++) {
      double r0 = r_of_x(sx0 + (0.0) * dx0);
      double rc = r_of_x(sx0 + (0.5) * dx0);
      double r1 = r_of_x(sx0 + (1.0) * dx0);
      double dr = r1 - r0;
      double thc = th_of_x(sx1 + (j + 0.5) * DJ(0) * dx1);
      double nk_ideal = rc * std::sin(thc) * dph / dr;
      if (j < NJ(0) / 2) {
        NK(0, j) = NK(0, j - 1);
        if (std::log2(nk_ideal / NK(0, j)) > max_log2_aspect) NK(0, j) *= 2;
        NK(0, j) = std::min(NK(0, j), n3);
      } else {
        NK(0, j) = NK(0, NJ(0) - 1 - j);
      }
    }
    for (int i = 1; i < n1; i++) {
      double r0 = r_of_x(sx0 + (i + 0.0) * dx0);
      double rc = r_of_x(sx0 + (i + 0.5) * dx0);
      double r1 = r_of_x(sx0 + (i + 1.0) * dx0);
      double dr = r1 - r0;
      NK(i, 0) = nk_min;
      for (int j = 1; j < NJ(i); j++) {
        double thc = th_of_x(sx1 + (j + 0.5) * DJ(i) * dx1);
        double nk_ideal = rc * std::sin(thc) * dph / dr;
        if (j < NJ(i) / 2) {
          NK(i, j) = NK(i, j - 1);
          if (std::log2(nk_ideal / NK(i, j)) > max_log2_aspect) NK(i, j) *= 2;
          if (NJ(i - 1) == NJ(i)) NK(i, j) = std::min(std::max(NK(i, j), NK(i - 1, j)), n3);
          else NK(i, j) = std::min(std::max(NK(i, j), NK(i - 1, j / 2)), n3);
        } else {
          NK(i, j) = NK(i, NJ(i) - 1 - j);
        }
      }
    }
    for (int i = -NG; i < 0; i++)
      for (int j = 0; j < NJ(i); j++) NK(i, j) = NK(-i - 1, j);
    for (int i = n1; i < n1 + NG; i++)
      for (int j = 0; j < NJ(i); j++) NK(i, j) = NK(n1 - 1, j);
    for (int i = -NG; i < n1 + NG; i++) {
      for (int j = -NG; j < 0; j++) NK(i, j) = NK(i, -j - 1);
      for (int j = NJ(i); j < NJ(i) + NG; j++) NK(i, j) = NK(i, 2 * NJ(i) - 1 - j);
    }
  }
}

// The refinement test of init_dendritic (utils.c:548-586): where theta refines 2:1 from
// radial row i to i+1, phi must not refine 4:1 between the cell (i, j) and either of
// the two cells (i+1, j') beside it; the reference prints each such cell (once per phi
// zone of the row) and exits.  Returns the number of such (i, j, k) cells.  The
// reference's other branch there (an inner row coarser in phi than the outer one,
// which it coarsens to match) cannot occur: compute_dk takes every row's phi count at
// least as large as its inner neighbour's.
int64_t dendritic_refine_errors(const Grid3Host &h)
{
  if (h.ndim != 3) return 0;
  int64_t bad = 0;
  for (int i0 = 0; i0 < h.n1; i0++) {
    const int i1 = i0 + 1;
    if (h.dj(i0) / h.dj(i1) != 2) continue;
    for (int j00 = 0; j00 < h.njr(i0); j00++) {
      const int j10 = j00 * h.dj(i0) / h.dj(i1), j11 = j10 + 1;
      if (h.dk(i0, j00) / h.dk(i1, j10) == 4 || h.dk(i0, j00) / h.dk(i1, j11) == 4) bad += h.n3 / h.dk(i0, j00);
    }
  }
  return bad;
}

void build_grid3(const mdg_problem_desc &d, Grid3Host &h)
{
  RadialMap rmap(d);
  const bool three = d.ndim == 3;
  const int n1 = d.n1, n2 = d.n2, n3 = three ? d.n3 : 1;
  const double sx0 = d.startx[0], sx1 = d.startx[1], sx2 = d.startx[2];
  const double dx0 = d.dx[0], dx1 = d.dx[1], dx2 = d.dx[2];

  // radial edges for the monopole gravity (init_coords, metric_spherical_general.c:577-583;
  // gravity.c:300-303)
  h.medge.assign((size_t)2 * (n1 + 1), 0.0);
  for (int i = 0; i <= n1; i++) {
    const double re = r_of_x(std::fabs(i * dx0 + sx0));
    h.medge[i] = re * re;
    h.medge[n1 + 1 + i] = dr_dx(sx0 + i * dx0);
  }

  dendritic_zone_counts(d, h);
  auto NJ = [&](int i) -> int & { return h.nj[i + NG]; };
  auto DJ = [&](int i) { return n2 / NJ(i); };
  auto NK = [&](int i, int j) -> int & { return h.nk[h.rowbase[i + NG] + j + NG]; };
  const int64_t nij = h.nij;
  auto DK = [&](int i, int j) { return n3 / NK(i, j); };

  // zone and face offsets
  h.cell.assign(nij, -1); h.f0.assign(nij, -1); h.f1.assign(nij, -1); h.f2.assign(nij, -1);
  int64_t c = 0, f0 = 0, f1 = 0, f2 = 0;
  for (int i = 0; i < n1; i++)
    for (int j = 0; j < NJ(i); j++) { h.cell[h.row(i, j)] = c; c += NK(i, j); }
  for (int i = 0; i <= n1; i++)
    for (int j = 0; j < NJ(i); j++) { h.f0[h.row(i, j)] = f0; f0 += NK(i, j); }
  for (int i = 0; i < n1; i++)
    for (int j = 0; j <= NJ(i); j++) { h.f1[h.row(i, j)] = f1; f1 += n3 / std::min(DK(i, j), DK(i, j - 1)); }
  for (int i = 0; i < n1 && three; i++)
    for (int j = 0; j < NJ(i); j++) { h.f2[h.row(i, j)] = f2; f2 += NK(i, j) + 1; }
  h.ncell = c; h.nf0 = f0; h.nf1 = f1; h.nf2 = f2;

  // direction-0 reconstruction table (the 1-D spherical radial moments)
  h.rc0.assign((size_t)RC_NFIELDS * (n1 + 2 * NG), 0.0);
  build_recon_table(d, 0, h.rc0.data(), n1 + 2 * NG, 0);
  h.mx0.assign((size_t)MX_NFIELDS * (n1 + 2 * NG), 0.0f);
  build_mixed_table(d, 0, h.mx0.data(), n1 + 2 * NG, 0);

  // direction-1 and -2 tables per refinement level
  int lev1 = 0, lev2 = 0;
  for (int i = -NG; i < n1 + NG; i++) {
    lev1 = std::max(lev1, ilog2(DJ(i)));
    for (int j = -NG; j < NJ(i) + NG; j++) lev2 = std::max(lev2, ilog2(DK(i, j)));
  }
  h.nlev1 = lev1 + 1; h.nlev2 = lev2 + 1;
  int64_t cols1 = 0, cols2 = 0;
  for (int l = 0; l < h.nlev1; l++) { h.rc1_base[l] = (int)cols1; cols1 += (n2 >> l) + 2 * NG; }
  for (int l = 0; l < h.nlev2; l++) { h.rc2_base[l] = (int)cols2; cols2 += (n3 >> l) + 2 * NG; }
  h.cols1 = cols1; h.cols2 = cols2;
  h.rc1.assign((size_t)RC_NFIELDS * cols1, 0.0); h.rc2.assign((size_t)RC_NFIELDS * cols2, 0.0);
  h.xc1.assign(cols1, 0.0); h.xc2.assign(cols2, 0.0);
  h.mx1.assign((size_t)MX_NFIELDS * cols1, 0.0f); h.mx2.assign((size_t)MX_NFIELDS * cols2, 0.0f);
  h.sth.assign(cols1, 0.0); h.cth.assign(cols1, 0.0);
  h.sphc.assign(cols2, 0.0); h.cphc.assign(cols2, 0.0); h.sphl.assign(cols2, 0.0); h.cphl.assign(cols2, 0.0);
  for (int l = 0; l < h.nlev1; l++) {
    const int s = 1 << l, n = n2 >> l;
    std::vector<double> al(n + 2 * NG), be(n + 2 * NG), ga(n + 2 * NG);
    for (int j = -NG; j < n + NG; j++) {
      double x0 = sx1 + j * s * dx1, x1 = sx1 + (j + 1) * s * dx1;
      ga[j + NG] = romb(x0, x1, f_sthdth_dx);
      be[j + NG] = romb(x0, x1, f_xth1g);
      al[j + NG] = romb(x0, x1, f_xth2g);
    }
    for (int j = -NG; j < n + NG; j++) {
      const int col = h.rc1_base[l] + j + NG;
      int jm = (j - 1 < -NG) ? -NG : j - 1, jp = (j + 1 >= n + NG) ? n + NG - 1 : j + 1;
      double v[RC_NFIELDS];
      rc_fields(al[jm + NG], al[j + NG], al[jp + NG], be[jm + NG], be[j + NG], be[jp + NG], ga[jm + NG],
                ga[j + NG], ga[jp + NG], sx1 + j * s * dx1, sx1 + (j + 1) * s * dx1, v);
      for (int f = 0; f < RC_NFIELDS; f++) h.rc1[(size_t)f * cols1 + col] = v[f];
      float w[MX_NFIELDS];
      mx_fields(al[jm + NG], al[j + NG], al[jp + NG], be[jm + NG], be[j + NG], be[jp + NG], ga[jm + NG],
                ga[j + NG], ga[jp + NG], sx1 + j * s * dx1, sx1 + (j + 1) * s * dx1, w);
      for (int f = 0; f < MX_NFIELDS; f++) h.mx1[(size_t)f * cols1 + col] = w[f];
      h.xc1[col] = be[j + NG] / ga[j + NG];
      double th = th_of_x(be[j + NG] / ga[j + NG]);
      h.sth[col] = std::sin(th);
      h.cth[col] = std::cos(th);
    }
  }
  for (int l = 0; l < h.nlev2; l++) {
    const int s = 1 << l, n = n3 >> l;
    std::vector<double> al(n + 2 * NG), be(n + 2 * NG), ga(n + 2 * NG);
    for (int k = -NG; k < n + NG; k++) {
      double x0 = sx2 + k * s * dx2, x1 = sx2 + (k + 1) * s * dx2;
      ga[k + NG] = s * dx2;
      be[k + NG] = (x1 * x1 - x0 * x0) / 2.0;
      al[k + NG] = (x1 * x1 * x1 - x0 * x0 * x0) / 3.0;
    }
    for (int k = -NG; k < n + NG; k++) {
      const int col = h.rc2_base[l] + k + NG;
      int km = (k - 1 < -NG) ? -NG : k - 1, kp = (k + 1 >= n + NG) ? n + NG - 1 : k + 1;
      double v[RC_NFIELDS];
      rc_fields(al[km + NG], al[k + NG], al[kp + NG], be[km + NG], be[k + NG], be[kp + NG], ga[km + NG],
                ga[k + NG], ga[kp + NG], sx2 + k * s * dx2, sx2 + (k + 1) * s * dx2, v);
      for (int f = 0; f < RC_NFIELDS; f++) h.rc2[(size_t)f * cols2 + col] = v[f];
      float w[MX_NFIELDS];
      mx_fields(al[km + NG], al[k + NG], al[kp + NG], be[km + NG], be[k + NG], be[kp + NG], ga[km + NG],
                ga[k + NG], ga[kp + NG], sx2 + k * s * dx2, sx2 + (k + 1) * s * dx2, w);
      for (int f = 0; f < MX_NFIELDS; f++) h.mx2[(size_t)f * cols2 + col] = w[f];
      h.xc2[col] = be[k + NG] / ga[k + NG];
      double phc = sx2 + (k + 0.5) * s * dx2, phl = sx2 + k * s * dx2;
      h.sphc[col] = std::sin(phc); h.cphc[col] = std::cos(phc);
      h.sphl[col] = std::sin(phl); h.cphl[col] = std::cos(phl);
    }
  }

  // per-row geometry
  h.geo.assign((size_t)G3_NFIELDS * nij, 0.0);
  auto G = [&](int f, int i, int j) -> double & { return h.geo[(size_t)f * nij + h.row(i, j)]; };
  for (int i = -NG; i < n1 + NG; i++) {
    const double x0lo = sx0 + i * dx0, x0hi = sx0 + (i + 1) * dx0;
    const double r2dr_int = romb(x0lo, x0hi, f_r2dr_dx);
    const double rint_r2dr_dx3 = romb(x0lo, x0hi, f_r2dr_dx3);
    const double r5 = std::pow(r_of_x(x0hi), 5) - std::pow(r_of_x(x0lo), 5);
    for (int j = -NG; j < NJ(i) + NG; j++) {
      const double x1lo = sx1 + j * DJ(i) * dx1, x1hi = sx1 + (j + 1) * DJ(i) * dx1;
      const double sthdth_int = romb(x1lo, x1hi, f_sthdth_dx);
      G(G3_VOL, i, j) = r2dr_int * sthdth_int * DK(i, j) * dx2;
      if (i >= 0 && i <= n1 && j >= 0 && j <= NJ(i)) {
        const double dph_int = DK(i, j) * dx2;
        G(G3_A0, i, j) = f_r2dr_dx(x0lo) * sthdth_int * dph_int;
        G(G3_A1, i, j) = r2dr_int * f_sthdth_dx(x1lo) * dph_int;
        G(G3_A2, i, j) = r2dr_int * sthdth_int;
      }
      const double vrf = r2dr_int, vthf = sthdth_int;
      const double th3 = romb(x1lo, x1hi, f_sthdth_dx3);
      const double ts3 = romb(x1lo, x1hi, f_sth3dth_dx);
      double gc[4][3];
      gc[0][0] = rint_r2dr_dx3 / vrf;
      gc[0][1] = std::fabs(0.2 * r5 / vrf * th3 / vthf);
      gc[0][2] = std::fabs(0.2 * r5 / vrf * ts3 / vthf);
      gc[1][0] = std::pow(dr_dx(x0lo), 2);
      gc[1][1] = std::pow(r_of_x(x0lo), 2) * th3 / vthf;
      gc[1][2] = std::pow(r_of_x(x0lo), 2) * ts3 / vthf;
      gc[2][0] = gc[0][0];
      gc[2][1] = std::fabs(0.2 * r5 / vrf * std::pow(dth_dx(x1lo), 2));
      gc[2][2] = std::fabs(0.2 * r5 / vrf * std::pow(std::sin(th_of_x(x1lo)), 2));
      gc[3][0] = gc[0][0]; gc[3][1] = gc[0][1]; gc[3][2] = gc[0][2];
      for (int l = 0; l < 4; l++)
        for (int m = 0; m < 3; m++) {
          G(G3_GCOV + 3 * l + m, i, j) = gc[l][m];
          G(G3_SCALE + 3 * l + m, i, j) = std::sqrt(gc[l][m]);
        }
      for (int m = 0; m < 3; m++) G(G3_GCON + m, i, j) = (std::fabs(gc[0][m]) > 1.0e-50) ? 1.0 / gc[0][m] : 0.0;
    }
  }
  // the areas of the axis faces are exactly zero
  if (sx1 == -1) {
    for (int i = 0; i <= n1; i++) G(G3_A1, i, 0) = 0.0;
  }
  if (std::fabs(sx1 + n2 * dx1 - 1) < 1.0e-15) {
    for (int i = 0; i <= n1; i++) G(G3_A1, i, NJ(i)) = 0.0;
  }
  // connection coefficients of the interior rows
  for (int i = 0; i < n1; i++) {
    const double x0lo = sx0 + i * dx0, x0hi = sx0 + (i + 1) * dx0;
    const double ri_r2d2r = romb(x0lo, x0hi, f_r2d2r_dx2);
    const double ri_r3 = romb(x0lo, x0hi, f_r3);
    const double ri_rdr2 = romb(x0lo, x0hi, f_rdr_dx2);
    const double vrf = romb(x0lo, x0lo + dx0, f_r2dr_dx);
    for (int j = 0; j < NJ(i); j++) {
      const double x1lo = sx1 + j * DJ(i) * dx1, x1hi = sx1 + (j + 1) * DJ(i) * dx1;
      const double vthf = romb(x1lo, x1hi, f_sthdth_dx);
      const double th3 = romb(x1lo, x1hi, f_sthdth_dx3);
      const double tcth = romb(x1lo, x1hi, f_cthdth_dx2);
      const double c000 = ri_r2d2r / vrf;
      const double c011 = -(ri_r3 / vrf) * (th3 / vthf);
      const double c101 = ri_rdr2 / vrf;
      const double c110 = c101, c202 = c101, c220 = c202;
      const double c212 = tcth / vthf, c221 = c212;
      const double c022 = -c220 * G(G3_GCOV + 2, i, j) / G(G3_GCOV + 0, i, j);
      const double c122 = -c221 * G(G3_GCOV + 2, i, j) / G(G3_GCOV + 1, i, j);
      double dA;
      if (DK(i, j + 1) < DK(i, j)) dA = G(G3_A1, i, j + 1) + G(G3_A1, i, j + 1);
      else if (DK(i, j + 1) > DK(i, j)) dA = 0.5 * G(G3_A1, i, j + 1);
      else dA = G(G3_A1, i, j + 1);
      dA -= G(G3_A1, i, j);
      const double dV = G(G3_VOL, i, j);
      const double c111 = dA / dV - c212;
      G(G3_C000, i, j) = c000; G(G3_C011, i, j) = c011; G(G3_C022, i, j) = c022;
      G(G3_C101, i, j) = c101; G(G3_C110, i, j) = c110; G(G3_C111, i, j) = c111;
      G(G3_C122, i, j) = c122; G(G3_C202, i, j) = c202; G(G3_C220, i, j) = c220;
      G(G3_C212, i, j) = c212; G(G3_C221, i, j) = c221;
    }
  }
}

}  // namespace mdg
