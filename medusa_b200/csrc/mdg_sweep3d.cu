// 3-D spherical sweep on the dendritic grid (plain FP64, the reference's operation order).
//
// prim_to_fluxes3 (step.c:1088-1430) visits every zone once and does, in that order, its
// lower direction-0 face, its lower direction-1 face(s) and its lower direction-2 face;
// push (step.c:327-478) then differences the stored face fluxes with the dendritic
// fan-in.  Here each of the three face families is one kernel (one thread per face, the
// faces of a row (i, j) in 128-face tiles), the fluxes go to HBM, and a fourth kernel
// applies push() per zone.  What the serial order of the reference decides is kept:
//
//  * pencils.  A direction-0 face of zone (i, j, k) reads radial zones i-2 .. i+1 at the
//    face's own (theta, phi) resolution: a finer row is restricted (volume-weighted mean,
//    restrict0 step.c:1012-1051; its Gamma slot takes the zone's phi velocity, as
//    restrict0 reads p[..][GAMMA] = p[..][U3]), a coarser or equal row is prolonged by
//    limited slopes in phi and then theta (prolongate0/kslopes0, step.c:905-955, 782-840).
//    Direction-1 faces restrict/prolong across phi-refinement steps (restrict1,
//    prolongate1/kslopes1, step.c:1053-1085, 957-1010, 842-900).
//  * boundaries.  Ghost zones are not stored: a read of a ghost zone is mapped to the
//    interior zone reset_boundaries_gpu copies into it (bc.c:705-1422, i-boundaries on
//    interior (j, k), j-boundaries on interior (i, k), k-boundaries on interior (i, j));
//    ghost zones that no boundary loop writes (corners) hold zeros, as the zero-filled
//    allocation does (utils.c:164-174).
//  * shock flags.  A direction-1 or -2 face uses HLLE next to a direction-0 shock
//    (transverse_shock, fluid.c:189-210) with the flags the serial loop has set when it
//    reaches the face: ghost flags are always "shock" (never reset), the current stage
//    contributes only the zone's own direction-0 face (marks from rows i+1, i+2 come
//    later in the loop), and in the second stage every first-stage mark counts
//    (set_shock_flag(0) resets once per step).  own[c]: zone c's own face in the current
//    stage; all0[c]: any first-stage mark of zone c (faces i, i+1, i+2 map down to it).
//  * the polar-axis fix (step.c:1301-1401): on the last theta row of every radial row
//    the phi-face states are the zone values with the velocity rotated through
//    Cartesian components (host tables of the sines and cosines).
// The FP64 reconstruction is called out of line here (face kernels would otherwise hold
// 14 inlined copies of para_recon): instruction-fetch stalls were the largest stall of
// the face kernels, and the smaller code ran the 384 x 128 x 256 Sedov grid 20 % faster
// on a B200 (same results).
#define MDG_RECON_OUTLINE 1
#include "mdg_hydro.cuh"
#include "mdg_kernels.cuh"
#include "mdg_grid3d.cuh"
#include "mdg_mixed.cuh"
#include <cstring>
#include <type_traits>
#include <string>
#include <vector>

namespace mdg {

struct Tile3 { int i, j, k0, cnt; };
constexpr int NT3 = 128;
// resident CTAs per SM requested from the compiler (register caps): the face kernels
// wait on dependent gathers, and 8 CTAs of 4 warps (64 registers, a few spills) ran
// 1.2x faster than 4 CTAs (128 registers) on the 384x128x256 Sedov grid
#ifndef MDG_F3MINB
#define MDG_F3MINB 8
#endif
#ifndef MDG_P3MINB
#define MDG_P3MINB 8
#endif

__device__ __forceinline__ int rowi(const Grid3 &g, int i, int j) { return __ldg(g.rowbase + i + NG) + j + NG; }
__device__ __forceinline__ int nj_of(const Grid3 &g, int i) { return __ldg(g.nj + i + NG); }
__device__ __forceinline__ int djs(const Grid3 &g, int i) { return g.n2 / nj_of(g, i); }
__device__ __forceinline__ int nk_of(const Grid3 &g, int i, int j) { return __ldg(g.nk + rowi(g, i, j)); }
__device__ __forceinline__ int dks(const Grid3 &g, int i, int j) { return g.n3 / nk_of(g, i, j); }
__device__ __forceinline__ double geo3(const Grid3 &g, int f, int ij) { return __ldg(g.geo + (int64_t)f * g.nij + ij); }
__device__ __forceinline__ double minmod(double a, double b)
{
  // MINMOD, decs.h:629-630
  return 0.5 * ((a < 0.0 ? -1.0 : 1.0) + (b < 0.0 ? -1.0 : 1.0)) * (fabs(a) < fabs(b) ? fabs(a) : fabs(b));
}

// Interior zone that reset_boundaries_gpu copies into zone (i, j, k), with the velocity
// components it negates (bit v set: component v flips sign); -1: a zone no boundary
// loop writes (zero).
__device__ int64_t locate3(const Grid3 &g, int i, int j, int k, int &flip)
{
  flip = 0;
  const int n1 = g.n1;
  const bool ig = (i < 0 || i >= n1);
  const int nji = nj_of(g, i);
  const bool jg = (j < 0 || j >= nji);
  const int nkr = nk_of(g, i, j);
  const bool kg = (k < 0 || k >= nkr);
  int ip = i, jp = j, kp = k;
  if (!ig && !jg && !kg) return __ldg(g.cell + rowi(g, i, j)) + k;
  if (ig && !jg && !kg) {
    if (i < 0) {
      ip = -1 - i;
      if (g.bc_lo0 == BC_SPHERICAL_ORIGIN) {
        const int njp = g.n2 / djs(g, ip);
        jp = njp - 1 - j;
        const int nkp = g.n3 / dks(g, ip, jp);
        kp = (k + nkp / 2) % nkp;
        flip = (1 << U1) | (1 << U3);
      } else {   // REFLECT
        jp = j * djs(g, i) / djs(g, ip);
        kp = k * dks(g, i, j) / dks(g, ip, jp);
        flip = 1 << U1;
      }
    } else {
      if (g.bc_hi0 == BC_REFLECT) {
        ip = 2 * n1 - i - 1;
        flip = 1 << U1;
      } else {   // OUTFLOW
        ip = n1 - 1;
      }
    }
  } else if (!ig && jg && !kg) {
    const int bc = (j < 0) ? g.bc_lo1 : g.bc_hi1;
    if (bc == BC_OUTFLOW) {
      jp = (j < 0) ? 0 : nji - 1;
    } else {
      jp = (j < 0) ? -1 - j : 2 * nji - 1 - j;
      if (bc == BC_SPHERICAL_ORIGIN) {
        const int nkp = g.n3 / dks(g, i, jp);
        kp = (k + nkp / 2) % nkp;
        flip = (1 << U2) | (1 << U3);
      } else {   // REFLECT
        kp = k * dks(g, i, j) / dks(g, i, jp);
        flip = 1 << U2;
      }
    }
  } else if (!ig && !jg && kg) {
    const int bc = (k < 0) ? g.bc_lo2 : g.bc_hi2;
    if (bc == BC_PERIODIC) {
      kp = (k < 0) ? k + nkr : k - nkr;
    } else {
      kp = (k < 0) ? 0 : nkr - 1;
      if (bc == BC_REFLECT) flip = 1 << U3;
    }
  } else {
    return -1;
  }
  // a source outside the interior (boundary kinds that assume no refinement next to the
  // boundary, used on a grid that has some there) reads as an unwritten zone
  if (ip < 0 || ip >= n1 || jp < 0 || jp >= nj_of(g, ip) || kp < 0 || kp >= nk_of(g, ip, jp)) return -1;
  return __ldg(g.cell + rowi(g, ip, jp)) + kp;
}

// Zone (i, j, k) as the pencils see it: primitives, PRESS and GAMMA of its EOS record
// (update_eos / update_eos_ghost fill every zone, eos.c:4-34).
__device__ __forceinline__ void load7(const Grid3 &g, const ProbDev &P, const StateSoA &s, int i, int j, int k,
                                      double *w)
{
  int flip;
  const int64_t c = locate3(g, i, j, k, flip);
#pragma unroll
  for (int v = 0; v < NPRIM; v++) {
    double x = (c >= 0) ? s.v[v][c] : 0.0;
    w[v] = ((flip >> v) & 1) ? -x : x;
  }
  w[5] = eos_press(P.eos, P.gam, P.Kpoly, w[RHO], w[UU]);
  w[6] = P.gam;
}

// kslopes0 / kslopes1: limited phi slope of row (ii, jj) evaluated at the centroid x2p.
__device__ void kslope_point(const Grid3 &g, const ProbDev &P, const StateSoA &s, int ii, int jj, int kk,
                             double x2p, double *pp)
{
  const int lev = ilog2(dks(g, ii, jj));
  const int base = g.rc2_base[lev] + NG;
  const double x20 = __ldg(g.xc2 + base + kk - 1), x21 = __ldg(g.xc2 + base + kk), x22 = __ldg(g.xc2 + base + kk + 1);
  const double idx2m = 1.0 / (x21 - x20), idx2p = 1.0 / (x22 - x21), idx2c = 1.0 / (x22 - x20);
  double a[7], b[7], c[7];
  load7(g, P, s, ii, jj, kk - 1, a);
  load7(g, P, s, ii, jj, kk, b);
  load7(g, P, s, ii, jj, kk + 1, c);
#pragma unroll
  for (int v = 0; v < 7; v++) {
    const double sm = (b[v] - a[v]) * idx2m;
    const double sp = (c[v] - b[v]) * idx2p;
    const double sc = (c[v] - a[v]) * idx2c;
    const double sg = minmod(2.0 * minmod(sm, sp), sc);
    pp[v] = b[v] + sg * (x2p - x21);
  }
}

// Pencil entry of radial row ii for the direction-0 face of zone (i, j, k).
__device__ void pencil0(const Grid3 &g, const ProbDev &P, const StateSoA &s, int i, int j, int k, int ii, double *pp)
{
  const int dji = djs(g, i), djii = djs(g, ii);
  if (djii < dji) {
    // restrict0 (step.c:1012-1051)
    const int njp = dji / djii, jp = j * njp;
    const int dkij = dks(g, i, j);
    double vol_sum = 0.0;
    for (int jj = jp; jj < jp + njp; jj++) {
      const int nkp = dkij / dks(g, ii, jj);
      const double vol = geo3(g, G3_VOL, rowi(g, ii, jj));
      for (int kk = k * nkp; kk < k * nkp + nkp; kk++) vol_sum += vol;
    }
    vol_sum = 1.0 / vol_sum;
#pragma unroll
    for (int v = 0; v < 7; v++) pp[v] = 0.0;
    for (int jj = jp; jj < jp + njp; jj++) {
      const int nkp = dkij / dks(g, ii, jj);
      const double vol = geo3(g, G3_VOL, rowi(g, ii, jj));
      for (int kk = k * nkp; kk < k * nkp + nkp; kk++) {
        const double vol_frac = vol * vol_sum;
        double w[7];
        load7(g, P, s, ii, jj, kk, w);
#pragma unroll
        for (int v = 0; v < NPRIM; v++) pp[v] += w[v] * vol_frac;
        pp[5] += w[5] * vol_frac;
        pp[6] += w[U3] * vol_frac;   // p[..][GAMMA], GAMMA = 4 (decs.h:661)
      }
    }
    return;
  }
  // prolongate0 (step.c:905-955)
  if (djii == dji && dks(g, ii, j) == dks(g, i, j)) {
    // same theta and phi level: both slope corrections are multiplied by an exact +0
    // (the prolongation point is the zone's own centroid), so the result is the zone
    // value itself unless that value is -0 (then the sign of the slope decides the sign
    // of the zero sum, and the full computation below runs)
    load7(g, P, s, ii, j, k, pp);
    bool neg0 = false;
#pragma unroll
    for (int v = 0; v < 7; v++) neg0 = neg0 || (pp[v] == 0.0 && signbit(pp[v]));
    if (!neg0) return;
  }
  const int jj = j * dji / djii;
  const double x1p = __ldg(g.xc1 + g.rc1_base[ilog2(dji)] + NG + j);
  const double x2p = __ldg(g.xc2 + g.rc2_base[ilog2(dks(g, i, j))] + NG + k);
  const int dkij = dks(g, i, j);
  double p0[7], p1[7], p2[7];
  if (g.ndim == 2) {
    // the 2-D prolongate0 (step.c:579-628) has no phi slopes
    load7(g, P, s, ii, jj - 1, 0, p0);
    load7(g, P, s, ii, jj, 0, p1);
    load7(g, P, s, ii, jj + 1, 0, p2);
  } else {
    kslope_point(g, P, s, ii, jj - 1, k * dkij / dks(g, ii, jj - 1), x2p, p0);
    kslope_point(g, P, s, ii, jj, k * dkij / dks(g, ii, jj), x2p, p1);
    kslope_point(g, P, s, ii, jj + 1, k * dkij / dks(g, ii, jj + 1), x2p, p2);
  }
  const int base = g.rc1_base[ilog2(djii)] + NG;
  const double x10 = __ldg(g.xc1 + base + jj - 1), x11 = __ldg(g.xc1 + base + jj), x12 = __ldg(g.xc1 + base + jj + 1);
  const double idx1m = 1.0 / (x11 - x10), idx1p = 1.0 / (x12 - x11), idx1c = 1.0 / (x12 - x10);
#pragma unroll
  for (int v = 0; v < 7; v++) {
    const double sm = (p1[v] - p0[v]) * idx1m;
    const double sp = (p2[v] - p1[v]) * idx1p;
    const double sc = (p2[v] - p0[v]) * idx1c;
    const double sg = minmod(2.0 * minmod(sm, sp), sc);
    pp[v] = p1[v] + sg * (x1p - x11);
  }
}

// Pencil entry of theta row jj for the direction-1 sub-face kk of face row (i, j).
__device__ void pencil1(const Grid3 &g, const ProbDev &P, const StateSoA &s, int i, int j, int kk, int jj,
                        double *pp)
{
  const int dkj = dks(g, i, j), dkjm = dks(g, i, j - 1);
  const int mn = dkj < dkjm ? dkj : dkjm;
  const int dkjj = dks(g, i, jj);
  if (dkjj < mn) {
    // restrict1 (step.c:1053-1085)
    const int nkp = mn / dkjj, kp = kk * nkp;
    const double vol = geo3(g, G3_VOL, rowi(g, i, jj));
    double vol_sum = 0.0;
    for (int k = kp; k < kp + nkp; k++) vol_sum += vol;
    vol_sum = 1.0 / vol_sum;
#pragma unroll
    for (int v = 0; v < 7; v++) pp[v] = 0.0;
    for (int k = kp; k < kp + nkp; k++) {
      const double vol_frac = vol * vol_sum;
      double w[7];
      load7(g, P, s, i, jj, k, w);
#pragma unroll
      for (int v = 0; v < 7; v++) pp[v] += w[v] * vol_frac;
    }
    return;
  }
  // prolongate1 (step.c:957-1010)
  const int k2 = kk * mn / dkjj;
  if (mn == dkjj) {
    load7(g, P, s, i, jj, k2, pp);
    return;
  }
  const double x2p = __ldg(g.xc2 + g.rc2_base[ilog2(mn)] + NG + kk);
  kslope_point(g, P, s, i, jj, k2, x2p, pp);
}

// Wave-speed estimate with per-side Gamma (riemann.c:368-429 / 210-303): the pencils of
// the dendritic grid can carry a reconstructed Gamma slot that differs between sides.
__device__ __forceinline__ void wave_speeds_g(const double *pl, const double *pr, double u_l, double u_r, bool hlle,
                                              double &sl, double &sr, double &ss, double &p_s, int &isshock)
{
  const double p_l = pl[5], p_r = pr[5], G_l = pl[6], G_r = pr[6];
  const double cs_l = sqrt(G_l * p_l / pl[RHO]);
  const double cs_r = sqrt(G_r * p_r / pr[RHO]);
  double p_max, p_min;
  if (p_l > p_r) { p_max = p_l; p_min = p_r; } else { p_max = p_r; p_min = p_l; }
  const double pratio = p_max / p_min;
  isshock = ((p_max - p_min) / p_min > 0.5) ? 1 : 0;
  p_s = 0.5 * (p_l + p_r) - 0.125 * (u_r - u_l) * (pl[RHO] + pr[RHO]) * (cs_l + cs_r);
  if (hlle) p_s = (p_s > 0.0) ? p_s : 0.0;
  else p_s = (0.0 > p_s) ? 0.0 : p_s;
  if (pratio < 2.0 && p_s >= p_min && p_s <= p_max) {
  } else if (p_s < p_min) {
    const double G_avg = 0.5 * (G_l + G_r);
    const double plr = pow(p_l / p_r, (G_avg - 1.0) / (2.0 * G_avg));
    const double s0 = (plr * u_l / cs_l + u_r / cs_r + 2.0 * (plr - 1.0) / (G_avg - 1.0)) / (plr / cs_l + 1.0 / cs_r);
    p_s = 0.5 * (p_l * pow(1.0 + (G_l - 1.0) / (2.0 * cs_l) * (u_l - s0), 2.0 * G_l / (G_l - 1.0))
               + p_r * pow(1.0 + (G_r - 1.0) / (2.0 * cs_r) * (s0 - u_r), 2.0 * G_r / (G_r - 1.0)));
    p_s = (p_s > 0.0) ? p_s : 0.0;
  } else {
    const double a_l = 2.0 / ((G_l + 1.0) * pl[RHO]);
    const double a_r = 2.0 / ((G_r + 1.0) * pr[RHO]);
    const double b_l = (G_l - 1.0) / (G_l + 1.0) * p_l;
    const double b_r = (G_r - 1.0) / (G_r + 1.0) * p_r;
    const double g_l = sqrt(a_l / (p_s + b_l));
    const double g_r = sqrt(a_r / (p_s + b_r));
    p_s = (g_l * p_l + g_r * p_r - (u_r - u_l)) / (g_l + g_r);
    p_s = (p_s > 0.0) ? p_s : 0.0;
  }
  const double q_l = (p_s <= p_l) ? 1.0 : sqrt(1.0 + (G_l + 1.0) / (2.0 * G_l) * (p_s / p_l - 1.0));
  const double q_r = (p_s <= p_r) ? 1.0 : sqrt(1.0 + (G_r + 1.0) / (2.0 * G_r) * (p_s / p_r - 1.0));
  sl = u_l - cs_l * q_l;
  sr = u_r + cs_r * q_r;
  ss = (p_r - p_l + pl[RHO] * u_l * (sl - u_l) - pr[RHO] * u_r * (sr - u_r))
     / (pl[RHO] * (sl - u_l) - pr[RHO] * (sr - u_r));
}

// riemann_flux_HLLC (riemann.c:328-499) with per-side Gamma; returns isshock.
template <int DIR>
__device__ int hllc3(const double *pl, const double *pr, const FaceGeom<double> &g, double *flux, double &sig)
{
  int isshock = 0;
  if (g.area < 1.0e-16) {
    sig = 1.0e-200;
#pragma unroll
    for (int v = 0; v < NPRIM; v++) flux[v] = 0.0;
    return isshock;
  }
  const double sc = g.scale;
  const double u_l = pl[U1 + DIR] * sc, u_r = pr[U1 + DIR] * sc;
  double sl, sr, ss, p_s;
  wave_speeds_g(pl, pr, u_l, u_r, false, sl, sr, ss, p_s, isshock);
  if (ss > sr) sr = 1.001 * ss;
  if (ss < sl) sl = 1.001 * ss;
  sig = tmax(fabs(sl), fabs(sr)) / sc;
  if (sl > 0.0) { pflux<DIR, false, double>(pl, pl[5], g, flux); return isshock; }
  if (sr < 0.0) { pflux<DIR, false, double>(pr, pr[5], g, flux); return isshock; }
  double u[NPRIM], fx[NPRIM], Us[NPRIM], pk[6];
  const bool left = ss > 0.0;
#pragma unroll
  for (int v = 0; v < 6; v++) pk[v] = left ? pl[v] : pr[v];
  const double sk = left ? sl : sr;
  const double uk = left ? u_l : u_r;
  p_uflux<DIR, false, double>(pk, g, pk[5], u, fx);
  Us[0] = pk[RHO] * (sk - uk) / (sk - ss);
  Us[UU] = (u[UU] * (sk - uk) - pk[5] * uk + p_s * ss) / (sk - ss);
  Us[U1] = pk[U1]; Us[U2] = pk[U2]; Us[U3] = pk[U3];
  Us[U1 + DIR] = ss / sc;
  const double slr = sk / sc;
  const double vc0 = g.g0 * Us[U1], vc1 = g.g1 * Us[U2], vc2 = g.g2 * Us[U3];
  Us[U1] = vc0 * Us[0]; Us[U2] = vc1 * Us[0]; Us[U3] = vc2 * Us[0];
#pragma unroll
  for (int v = 0; v < NPRIM; v++) flux[v] = g.area * (fx[v] + slr * (Us[v] - u[v]));
  return isshock;
}

// riemann_flux_HLLE (riemann.c:178-325) with per-side Gamma.
template <int DIR>
__device__ void hlle3(const double *pl, const double *pr, const FaceGeom<double> &g, double *flux, double &sig)
{
  if (g.area < 1.0e-16) {
    sig = 1.0e-200;
#pragma unroll
    for (int v = 0; v < NPRIM; v++) flux[v] = 0.0;
    return;
  }
  const double sc = g.scale;
  const double u_l = pl[U1 + DIR] * sc, u_r = pr[U1 + DIR] * sc;
  double sl, sr, ss, p_s;
  int isshock;
  wave_speeds_g(pl, pr, u_l, u_r, true, sl, sr, ss, p_s, isshock);
  double ul[NPRIM], ur[NPRIM], fl[NPRIM], fr[NPRIM];
  p_uflux<DIR, false, double>(pl, g, pl[5], ul, fl);
  p_uflux<DIR, false, double>(pr, g, pr[5], ur, fr);
  const double cmax = tmax(sr / sc, 0.0);
  const double cmin = fabs(tmin(sl / sc, 0.0));
  sig = tmax(cmax, cmin);
#pragma unroll
  for (int v = 0; v < NPRIM; v++)
    flux[v] = g.area * (cmin * fr[v] + cmax * fl[v] - cmax * cmin * (ur[v] - ul[v])) / (cmax + cmin);
}

// Face geometry of direction d on row (i, j): area[d], scale[1+d][d], gcov[1+d][0..2].
template <int DIR>
__device__ __forceinline__ FaceGeom<double> face_geom3(const Grid3 &g, int ij)
{
  FaceGeom<double> f;
  f.area = geo3(g, G3_A0 + DIR, ij);
  f.scale = geo3(g, G3_SCALE + 3 * (1 + DIR) + DIR, ij);
  f.g0 = geo3(g, G3_GCOV + 3 * (1 + DIR) + 0, ij);
  f.g1 = geo3(g, G3_GCOV + 3 * (1 + DIR) + 1, ij);
  f.g2 = geo3(g, G3_GCOV + 3 * (1 + DIR) + 2, ij);
  return f;
}

// Right face value of pencil zone 1 and left face value of pencil zone 2 (interp() on a
// 4-zone pencil, reconstruct.c:225-279), reconstruction columns c1, c2 of table rc.
__device__ __forceinline__ void recon_face(int order, const double pen[4][7], const double *rc, int64_t stride,
                                           int64_t c1, int64_t c2, double *pl, double *pr)
{
  const RcView<double, true> g1{rc + c1, stride}, g2{rc + c2, stride};
#pragma unroll kReconUnroll
  for (int v = 0; v < 7; v++) {
    double al, ar;
    recon_zone<double>(order, pen[0][v], pen[1][v], pen[2][v], g1, al, ar);
    pl[v] = ar;
    recon_zone<double>(order, pen[1][v], pen[2][v], pen[3][v], g2, al, ar);
    pr[v] = al;
  }
}

// Mixed precision (MIX): the same pencils, para_recon in FP32 difference form with the
// FP32 weights of the zone (face values a + da formed in FP64), HLLC with FP32 wave speeds
// and star-state increments and an FP64 upwind flux.  Faces the FP32 solver declines
// (ill-conditioned, MIX_COND_MAX) or whose Gamma slot is not the constant Gamma (the
// restricted radial entries) are re-solved in FP64 from the pencil; HLLE faces (next to
// a shock) take the FP64 solver on the mixed face states.
__device__ __forceinline__ void recon_face_mixed(const double pen[4][7], const float *mx, int64_t stride,
                                                 int64_t c1, int64_t c2, double *pl, double *pr)
{
  const MixW w1 = load_mixw(mx + c1, stride), w2 = load_mixw(mx + c2, stride);
#pragma unroll
  for (int v = 0; v < 7; v++) {
    float dl, dr;
    mixed_recon((float)(pen[1][v] - pen[0][v]), (float)(pen[2][v] - pen[1][v]), w1, dl, dr);
    pl[v] = pen[1][v] + (double)dr;
    mixed_recon((float)(pen[2][v] - pen[1][v]), (float)(pen[3][v] - pen[2][v]), w2, dl, dr);
    pr[v] = pen[2][v] + (double)dl;
  }
}

template <int DIR>
__device__ __noinline__ int face_fp64_3d(int order, const double *pen, const double *rc, int64_t stride, int64_t c1,
                                         int64_t c2, FaceGeom<double> fg, double *fl, double *ss)
{
  double p[4][7], pl[7], pr[7];
  for (int q = 0; q < 28; q++) p[q / 7][q % 7] = pen[q];
  recon_face(order, p, rc, stride, c1, c2, pl, pr);
  return hllc3<DIR>(pl, pr, fg, fl, *ss);
}

// Reconstruction and solve of one face of the pencil; returns isshock.
template <int DIR, bool MIX>
__device__ __forceinline__ int solve_face(const ProbDev &P, const double pen[4][7], const double *rc, const float *mx,
                                          int64_t stride, int64_t c1, int64_t c2, const FaceGeom<double> &fg,
                                          bool hlle, double *fl, double &ss)
{
  double pl[7], pr[7];
  if (!MIX) {
    recon_face(P.interp_order, pen, rc, stride, c1, c2, pl, pr);
    if (hlle) { hlle3<DIR>(pl, pr, fg, fl, ss); return 0; }
    return hllc3<DIR>(pl, pr, fg, fl, ss);
  }
  recon_face_mixed(pen, mx, stride, c1, c2, pl, pr);
  if (hlle) { hlle3<DIR>(pl, pr, fg, fl, ss); return 0; }
  if (pl[6] == P.gam && pr[6] == P.gam) {
    float sig;
    int isshock;
    if (riemann_hllc_mixed<DIR>(pl, pr, fg, gam_const<float>((float)P.gam), fl, sig, isshock)) {
      ss = (double)sig;
      return isshock;
    }
  }
  return face_fp64_3d<DIR>(P.interp_order, &pen[0][0], rc, stride, c1, c2, fg, fl, &ss);
}

// Flag of zone (i, jj, kc) as transverse_shock reads it at this point of the serial loop.
template <int STAGE>
__device__ __forceinline__ bool flag_shock(const Grid3 &g, int i, int jj, int kc, const unsigned char *own,
                                           const unsigned char *all0)
{
  if (jj < 0 || jj >= nj_of(g, i)) return true;
  if (kc < 0 || kc >= nk_of(g, i, jj)) return true;
  const int64_t c = __ldg(g.cell + rowi(g, i, jj)) + kc;
  return own[c] != 0 || (STAGE == 1 && all0[c] != 0);
}

// Direction-0 faces: face (i, j, k) is the lower radial face of zone (i, j, k), i in [0, n1].
// A work item is a run of up to RUN0 consecutive radial faces i0 .. i0+ni-1 of one (j, k)
// column whose face rows share their theta and phi resolution (djs(i), dks(i, j)), so
// every pencil entry (radial row ii at that resolution) is the same for all faces of the
// run: each thread walks outwards through its column with a ring of pencil entries in
// shared memory, loads one new entry and reconstructs one zone per face (zone i's left
// face value for face i, its right face value kept for face i+1), where the reference's
// interp() builds a 4-zone pencil and reconstructs two zones per face.  The values are
// the same; only their reuse differs.
// A run of faces along one direction: faces r0 .. r0+nr-1 of the fixed row `row` (the
// theta row j for direction 0, the radial row i for direction 1), columns k0 .. k0+cnt-1.
struct Tile3R { int r0, nr, row, k0, cnt; };
constexpr int RUN0 = 16;          // default faces per work item (mdg_launch_config::run_length)

// The RK stage is a run-time argument here (not a template argument as in the other
// face kernels): both stages then run the same code, which measured faster for stage 1
// than its own specialisation.
template <bool MIX>
__global__ void __launch_bounds__(NT3, MDG_F3MINB) face0_kernel(const ProbDev *__restrict__ probs, ProbTime *__restrict__ times,
                                                     Grid3 g, const Tile3R *__restrict__ tiles, StateSoA s,
                                                     double *__restrict__ flux, unsigned char *__restrict__ own,
                                                     unsigned char *__restrict__ all0, int stage)
{
  // ring of pencil entries (radial rows i-1 .. i+1; i-2 as well for the FP64 re-solve of
  // the mixed sweep) and the right face values of the previous zone, [slot][var][thread]
  constexpr int NS = MIX ? 4 : 3;
  __shared__ double win[NS][7][NT3];
  __shared__ double arb[7][NT3];
  __shared__ double sred[32];
  if (times[0].done) return;
  const ProbDev &P = probs[0];
  const Tile3R t = tiles[blockIdx.x];
  const int tid = (int)threadIdx.x;
  const int i0 = t.r0, j = t.row, k = t.k0 + tid;
  double lmin = 1.0e300;
  if (tid < t.cnt) {
    const int64_t rcs = g.n1 + 2 * NG;
    auto slot = [&](int ii) { return (ii - i0 + 2) % NS; };
#pragma unroll 1
    for (int ii = i0 - 2; ii <= i0; ii++) {
      double w[7];
      pencil0(g, P, s, i0, j, k, ii, w);
#pragma unroll
      for (int v = 0; v < 7; v++) win[slot(ii)][v][tid] = w[v];
    }
    {
      // right face values of zone i0-1
      const int sm = slot(i0 - 2), s0 = slot(i0 - 1), sp = slot(i0);
      if (MIX) {
        const MixW w = load_mixw(g.mx0 + i0 - 1 + NG, rcs);
#pragma unroll
        for (int v = 0; v < 7; v++) {
          const double a = win[s0][v][tid];
          float dl, dr;
          mixed_recon((float)(a - win[sm][v][tid]), (float)(win[sp][v][tid] - a), w, dl, dr);
          arb[v][tid] = a + (double)dr;
        }
      } else {
        const RcView<double, true> gz{g.rc0 + i0 - 1 + NG, rcs};
#pragma unroll kReconUnroll
        for (int v = 0; v < 7; v++) {
          double al, ar;
          recon_zone<double>(P.interp_order, win[sm][v][tid], win[s0][v][tid], win[sp][v][tid], gz, al, ar);
          arb[v][tid] = ar;
        }
      }
    }
#pragma unroll 1
    for (int i = i0; i < i0 + t.nr; i++) {
      {
        double w[7];
        pencil0(g, P, s, i0, j, k, i + 1, w);
#pragma unroll
        for (int v = 0; v < 7; v++) win[slot(i + 1)][v][tid] = w[v];
      }
      double pl[7], pr[7];
      const int sm = slot(i - 1), s0 = slot(i), sp = slot(i + 1);
      if (MIX) {
        const MixW w = load_mixw(g.mx0 + i + NG, rcs);
#pragma unroll
        for (int v = 0; v < 7; v++) {
          pl[v] = arb[v][tid];
          const double a = win[s0][v][tid];
          float dl, dr;
          mixed_recon((float)(a - win[sm][v][tid]), (float)(win[sp][v][tid] - a), w, dl, dr);
          pr[v] = a + (double)dl;
          arb[v][tid] = a + (double)dr;
        }
      } else {
        const RcView<double, true> gz{g.rc0 + i + NG, rcs};
#pragma unroll kReconUnroll
        for (int v = 0; v < 7; v++) {
          pl[v] = arb[v][tid];
          double al, ar;
          recon_zone<double>(P.interp_order, win[sm][v][tid], win[s0][v][tid], win[sp][v][tid], gz, al, ar);
          pr[v] = al;
          arb[v][tid] = ar;
        }
      }
      const int ij = rowi(g, i, j);
      const FaceGeom<double> fg = face_geom3<0>(g, ij);
      double fl[NPRIM], ss;
      int isshock = -1;
      if (!MIX) {
        isshock = hllc3<0>(pl, pr, fg, fl, ss);
      } else {
        if (pl[6] == P.gam && pr[6] == P.gam) {
          float sig;
          int sh;
          if (riemann_hllc_mixed<0>(pl, pr, fg, gam_const<float>((float)P.gam), fl, sig, sh)) {
            ss = (double)sig;
            isshock = sh;
          }
        }
        if (isshock < 0) {
          double pen[28];
#pragma unroll
          for (int q = 0; q < 28; q++) pen[q] = win[slot(i - 2 + q / 7)][q % 7][tid];
          isshock = face_fp64_3d<0>(P.interp_order, pen, g.rc0, rcs, i - 1 + NG, i + NG, fg, fl, &ss);
        }
      }
      const int64_t f = __ldg(g.f0 + ij) + k;
#pragma unroll
      for (int v = 0; v < NPRIM; v++) flux[v * g.nf0 + f] = fl[v];
      if (i < g.n1) own[__ldg(g.cell + ij) + k] = (unsigned char)isshock;
      if (stage == 0 && isshock) {
        // shock marks of the zone and of the two zones inside it (step.c:1196-1204)
        if (i < g.n1) all0[__ldg(g.cell + ij) + k] = 1;
        for (int d = 1; d <= 2; d++) {
          const int im = i - d;
          if (im < 0) break;
          const int jm = j * djs(g, i) / djs(g, im);
          const int km = k * dks(g, i, j) / dks(g, im, jm);
          all0[__ldg(g.cell + rowi(g, im, jm)) + km] = 1;
        }
      }
      lmin = tmin(lmin, g.dx0 / fabs(ss));
    }
  }
  block_min_to(lmin, &times[0].minacc, sred);
}

// Direction-1 faces: sub-face kk of face row (i, j), j in [0, nj(i)] (step.c:1212-1265).
// As for direction 0, a work item is a run of up to RUN0 consecutive faces j0 .. j0+nj-1
// of radial row i and sub-face column kk whose face rows share their phi resolution
// mn = min(dks(i, j), dks(i, j-1)) (every pencil entry, theta row jj at that resolution,
// is then the same for all faces of the run); a thread walks northwards through its
// column, one new entry and one zone reconstruction per face.  Tile3R fields here:
// r0 = j0, nr = faces, row = i.
template <bool MIX>
__global__ void __launch_bounds__(NT3, MDG_F3MINB) face1_kernel(const ProbDev *__restrict__ probs, ProbTime *__restrict__ times,
                                                     Grid3 g, const Tile3R *__restrict__ tiles, StateSoA s,
                                                     double *__restrict__ flux, const unsigned char *__restrict__ own,
                                                     const unsigned char *__restrict__ all0, int stage)
{
  constexpr int NS = MIX ? 4 : 3;
  __shared__ double win[NS][7][NT3];
  __shared__ double arb[7][NT3];
  __shared__ double sred[32];
  if (times[0].done) return;
  const ProbDev &P = probs[0];
  const Tile3R t = tiles[blockIdx.x];
  const int tid = (int)threadIdx.x;
  const int j0 = t.r0, i = t.row, kk = t.k0 + tid;
  double lmin = 1.0e300;
  if (tid < t.cnt) {
    const int64_t cs = g.cols1;
    const int64_t base = g.rc1_base[ilog2(djs(g, i))] + NG;
    auto slot = [&](int jj) { return (jj - j0 + 2) % NS; };
#pragma unroll 1
    for (int jj = j0 - 2; jj <= j0; jj++) {
      double w[7];
      pencil1(g, P, s, i, j0, kk, jj, w);
#pragma unroll
      for (int v = 0; v < 7; v++) win[slot(jj)][v][tid] = w[v];
    }
    {
      // right face values of zone j0-1
      const int sm = slot(j0 - 2), s0 = slot(j0 - 1), sp = slot(j0);
      if (MIX) {
        const MixW w = load_mixw(g.mx1 + base + j0 - 1, cs);
#pragma unroll
        for (int v = 0; v < 7; v++) {
          const double a = win[s0][v][tid];
          float dl, dr;
          mixed_recon((float)(a - win[sm][v][tid]), (float)(win[sp][v][tid] - a), w, dl, dr);
          arb[v][tid] = a + (double)dr;
        }
      } else {
        const RcView<double, true> gz{g.rc1 + base + j0 - 1, cs};
#pragma unroll kReconUnroll
        for (int v = 0; v < 7; v++) {
          double al, ar;
          recon_zone<double>(P.interp_order, win[sm][v][tid], win[s0][v][tid], win[sp][v][tid], gz, al, ar);
          arb[v][tid] = ar;
        }
      }
    }
#pragma unroll 1
    for (int j = j0; j < j0 + t.nr; j++) {
      {
        double w[7];
        pencil1(g, P, s, i, j0, kk, j + 1, w);
#pragma unroll
        for (int v = 0; v < 7; v++) win[slot(j + 1)][v][tid] = w[v];
      }
      double pl[7], pr[7];
      const int sm = slot(j - 1), s0 = slot(j), sp = slot(j + 1);
      if (MIX) {
        const MixW w = load_mixw(g.mx1 + base + j, cs);
#pragma unroll
        for (int v = 0; v < 7; v++) {
          pl[v] = arb[v][tid];
          const double a = win[s0][v][tid];
          float dl, dr;
          mixed_recon((float)(a - win[sm][v][tid]), (float)(win[sp][v][tid] - a), w, dl, dr);
          pr[v] = a + (double)dl;
          arb[v][tid] = a + (double)dr;
        }
      } else {
        const RcView<double, true> gz{g.rc1 + base + j, cs};
#pragma unroll kReconUnroll
        for (int v = 0; v < 7; v++) {
          pl[v] = arb[v][tid];
          double al, ar;
          recon_zone<double>(P.interp_order, win[sm][v][tid], win[s0][v][tid], win[sp][v][tid], gz, al, ar);
          pr[v] = al;
          arb[v][tid] = ar;
        }
      }
      // zone k of row j that owns the sub-face, and the transverse_shock test of zone k
      const int dkj = dks(g, i, j), dkjm = dks(g, i, j - 1);
      const int mn = dkj < dkjm ? dkj : dkjm;
      const int k = kk / (dkj / mn);
      const int nkm = dkj / dkjm;
      bool hlle = (stage == 0) ? flag_shock<0>(g, i, j, k, own, all0) : flag_shock<1>(g, i, j, k, own, all0);
      for (int q = k * nkm; q < k * nkm + nkm; q++)
        hlle = hlle || ((stage == 0) ? flag_shock<0>(g, i, j - 1, q, own, all0) : flag_shock<1>(g, i, j - 1, q, own, all0));
      const int ij = rowi(g, i, j);
      const FaceGeom<double> fg = face_geom3<1>(g, ij);
      double fl[NPRIM], ss;
      if (hlle) {
        hlle3<1>(pl, pr, fg, fl, ss);
      } else if (!MIX) {
        hllc3<1>(pl, pr, fg, fl, ss);
      } else {
        bool done = false;
        if (pl[6] == P.gam && pr[6] == P.gam) {
          float sig;
          int sh;
          if (riemann_hllc_mixed<1>(pl, pr, fg, gam_const<float>((float)P.gam), fl, sig, sh)) {
            ss = (double)sig;
            done = true;
          }
        }
        if (!done) {
          double pen[28];
#pragma unroll
          for (int q = 0; q < 28; q++) pen[q] = win[slot(j - 2 + q / 7)][q % 7][tid];
          face_fp64_3d<1>(P.interp_order, pen, g.rc1, cs, base + j - 1, base + j, fg, fl, &ss);
        }
      }
      const int64_t f = __ldg(g.f1 + ij) + kk;
#pragma unroll
      for (int v = 0; v < NPRIM; v++) flux[v * g.nf1 + f] = fl[v];
      lmin = tmin(lmin, djs(g, i) * g.dx1 / fabs(ss));
    }
  }
  block_min_to(lmin, &times[0].minacc, sred);
}

// Direction-2 faces: face k in [0, nk] of row (i, j) (step.c:1267-1425), with the
// polar-axis fix on the last theta row.  A CTA takes NT3-2 consecutive faces of one row:
// it stages the zones they read in shared memory (each zone loaded once) and
// reconstructs every zone once (the reference reconstructs each zone for both of its
// faces), then each thread solves one face.
constexpr int T2 = NT3 - 2;
template <int STAGE, bool MIX>
__global__ void __launch_bounds__(NT3, MDG_F3MINB) face2_kernel(const ProbDev *__restrict__ probs, ProbTime *__restrict__ times,
                                                     Grid3 g, const Tile3 *__restrict__ tiles, StateSoA s,
                                                     double *__restrict__ flux, const unsigned char *__restrict__ own,
                                                     const unsigned char *__restrict__ all0)
{
  __shared__ double sv[7][T2 + 4];    // zones k0-2 .. k0+cnt+1
  __shared__ double sal[7][T2 + 2];   // left / right face values of zones k0-1 .. k0+cnt
  __shared__ double sar[7][T2 + 2];
  __shared__ double sred[32];
  if (times[0].done) return;
  const ProbDev &P = probs[0];
  const Tile3 tl = tiles[blockIdx.x];
  const int i = tl.i, j = tl.j, k0 = tl.k0, cnt = tl.cnt;
  const int t = (int)threadIdx.x;
  const int ij = rowi(g, i, j);
  const int dk = dks(g, i, j);
  const int64_t base = g.rc2_base[ilog2(dk)] + NG;
  const bool pole = (j == nj_of(g, i) - 1);
  for (int q = t; q < cnt + 4; q += NT3) {
    double w[7];
    load7(g, P, s, i, j, k0 - 2 + q, w);
#pragma unroll
    for (int v = 0; v < 7; v++) sv[v][q] = w[v];
  }
  __syncthreads();
  if (!pole && t < cnt + 2) {
    // zone k0-1+t from the staged neighbours (interp() on its 3-zone stencil)
    if (MIX) {
      const MixW w = load_mixw(g.mx2 + base + k0 - 1 + t, g.cols2);
#pragma unroll
      for (int v = 0; v < 7; v++) {
        float dl, dr;
        const double a = sv[v][t + 1];
        mixed_recon((float)(a - sv[v][t]), (float)(sv[v][t + 2] - a), w, dl, dr);
        sal[v][t] = a + (double)dl;
        sar[v][t] = a + (double)dr;
      }
    } else {
      const RcView<double, true> gz{g.rc2 + base + k0 - 1 + t, g.cols2};
#pragma unroll kReconUnroll
      for (int v = 0; v < 7; v++) {
        double al, ar;
        recon_zone<double>(P.interp_order, sv[v][t], sv[v][t + 1], sv[v][t + 2], gz, al, ar);
        sal[v][t] = al;
        sar[v][t] = ar;
      }
    }
  }
  __syncthreads();
  double lmin = 1.0e300;
  if (t < cnt) {
    const int k = k0 + t;
    double pl[7], pr[7];
    if (pole) {
      // polar-axis fix: zone values, velocity rotated at the shared phi face
      const int64_t b1 = g.rc1_base[ilog2(djs(g, i))] + NG + j;
      const double sth = __ldg(g.sth + b1), cth = __ldg(g.cth + b1);
      double s0[3], s3[3];
#pragma unroll
      for (int m = 0; m < 3; m++) {
        s0[m] = geo3(g, G3_SCALE + m, ij);
        s3[m] = geo3(g, G3_SCALE + 9 + m, ij);
      }
      const double sphf = __ldg(g.sphl + base + k), cphf = __ldg(g.cphl + base + k);
      for (int side = 0; side < 2; side++) {
        const int kt = k - 1 + side;
        double w[7];
#pragma unroll
        for (int v = 0; v < 7; v++) w[v] = sv[v][t + 1 + side];
        const double sph = __ldg(g.sphc + base + kt), cph = __ldg(g.cphc + base + kt);
        double lam[3][3] = {{sth * cph, cth * cph, -sph}, {sth * sph, cth * sph, cph}, {cth, -sth, 0.0}};
        double v[3];
        for (int l = 0; l < 3; l++) {
          v[l] = 0.0;
          for (int m = 0; m < 3; m++) v[l] += lam[l][m] * w[U1 + m] * s0[m];
        }
        double lf[3][3] = {{sth * cphf, cth * cphf, -sphf}, {sth * sphf, cth * sphf, cphf}, {cth, -sth, 0.0}};
        double *o = side ? pr : pl;
#pragma unroll
        for (int q = 0; q < 7; q++) o[q] = w[q];
        for (int l = 0; l < 3; l++) {
          o[U1 + l] = 0.0;
          for (int m = 0; m < 3; m++) o[U1 + l] += lf[m][l] * v[m] / s3[l];
        }
      }
    } else {
#pragma unroll
      for (int v = 0; v < 7; v++) {
        pl[v] = sar[v][t];
        pr[v] = sal[v][t + 1];
      }
    }
    const bool hlle = flag_shock<STAGE>(g, i, j, k, own, all0) || flag_shock<STAGE>(g, i, j, k - 1, own, all0);
    const FaceGeom<double> fg = face_geom3<2>(g, ij);
    double fl[NPRIM], ss;
    if (hlle) {
      hlle3<2>(pl, pr, fg, fl, ss);
    } else if (!MIX) {
      hllc3<2>(pl, pr, fg, fl, ss);
    } else {
      float sig;
      int isshock;
      if (pl[6] == P.gam && pr[6] == P.gam &&
          riemann_hllc_mixed<2>(pl, pr, fg, gam_const<float>((float)P.gam), fl, sig, isshock)) {
        ss = (double)sig;
      } else if (pole) {
        hllc3<2>(pl, pr, fg, fl, ss);
      } else {
        double pen[4][7];
#pragma unroll
        for (int q = 0; q < 28; q++) pen[q / 7][q % 7] = sv[q % 7][t + q / 7];
        face_fp64_3d<2>(P.interp_order, &pen[0][0], g.rc2, g.cols2, base + k - 1, base + k, fg, fl, &ss);
      }
    }
    const int64_t f = __ldg(g.f2 + ij) + k;
#pragma unroll
    for (int v = 0; v < NPRIM; v++) flux[v * g.nf2 + f] = fl[v];
    lmin = dk * g.dx2 / fabs(ss);
  }
  block_min_to(lmin, &times[0].minacc, sred);
}

// monopole_gravity_start (gravity.c:238-246): mass vol*rho of radial shell i, summed over
// its zones in zone order (one thread per shell, the reference's serial order).
__global__ void shell_mass3_kernel(const ProbTime *__restrict__ times, Grid3 g, StateSoA s)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.n1 || times[0].done) return;
  double ms = 0.0;
  for (int j = 0; j < nj_of(g, i); j++) {
    const int ij = rowi(g, i, j);
    const double vol = geo3(g, G3_VOL, ij);
    const int64_t c0 = __ldg(g.cell + ij);
    const int nk = __ldg(g.nk + ij);
#pragma unroll 8
    for (int k = 0; k < nk; k++) ms += vol * s.v[RHO][c0 + k];
  }
  g.gmono[i] = ms;
}

// monopole_gravity_finish (gravity.c:300-319, GR_MONOPOLE=FALSE): enclosed mass at the
// radial edges, g = -G mr / r^2 dr/dx there, interpolated to the zone centroids (in place
// over the shell masses).
__global__ void monopole_profile3_kernel(const ProbTime *__restrict__ times, Grid3 g)
{
  if (threadIdx.x != 0 || times[0].done) return;
  const int64_t rcs = g.n1 + 2 * NG;
  double mr = 0.0, gl = 0.0;
  for (int ii = 0; ii < g.n1; ii++) {
    mr = mr + g.gmono[ii];
    const double gr = -GNEWT * mr / __ldg(g.medge + ii + 1) * __ldg(g.medge + g.n1 + 1 + ii + 1);
    g.gmono[ii] = monopole_centroid(gl, gr, g.x0 + ii * g.dx0, g.dx0, __ldg(g.rc0 + RC_B0 * rcs + ii + NG),
                                    __ldg(g.rc0 + RC_G0 * rcs + ii + NG));
    gl = gr;
  }
}

// push() for zone (i, j, k) (step.c:327-478) with the dendritic flux fan-in, the
// geometric sources of the stage state (rad_fluid.c:164-192, fluid.c:56-73), fixed or
// monopole gravity and, in the
// second stage, the zone terms of the next estimate_dt (step.c:177-187).
template <int STAGE>
__global__ void __launch_bounds__(NT3, MDG_P3MINB) push3_kernel(const ProbDev *__restrict__ probs, ProbTime *__restrict__ times,
                                                     Grid3 g, const Tile3 *__restrict__ tiles, StateSoA sst,
                                                     StateSoA sn, StateSoA out, const double *__restrict__ F0,
                                                     const double *__restrict__ F1, const double *__restrict__ F2)
{
  __shared__ double sred[32];
  if (times[0].done) return;
  const ProbDev &P = probs[0];
  const double dt = times[0].dt;
  const Tile3 t = tiles[blockIdx.x];
  const int i = t.i, j = t.j, k = t.k0 + (int)threadIdx.x;
  double lmin = 1.0e300, lmax = 0.0;
  if ((int)threadIdx.x < t.cnt) {
    const int ij = rowi(g, i, j);
    const PushRow3 &pr = g.prow[ij];
    const int64_t c = pr.cell + k;
    double ph[NPRIM], pn[NPRIM], u[NPRIM], uh[NPRIM], src[NPRIM], divF[NPRIM], pf[NPRIM];
#pragma unroll
    for (int v = 0; v < NPRIM; v++) ph[v] = sst.v[v][c];
    if (STAGE == 0) {
#pragma unroll
      for (int v = 0; v < NPRIM; v++) pn[v] = ph[v];
    } else {
#pragma unroll
      for (int v = 0; v < NPRIM; v++) pn[v] = sn.v[v][c];
    }
    const double g0 = geo3(g, G3_GCOV + 0, ij), g1 = geo3(g, G3_GCOV + 1, ij), g2 = geo3(g, G3_GCOV + 2, ij);
    const double press = eos_press(P.eos, P.gam, P.Kpoly, ph[RHO], ph[UU]);
    {
      // p_to_geom_src: src[U1+m] = sum_l sum_n T[l][n] conn[l][m][n] over the non-zero conn
      const double vcov[3] = {g0 * ph[U1], g1 * ph[U2], g2 * ph[U3]};
      double T[3][3];
#pragma unroll
      for (int l = 0; l < 3; l++) {
#pragma unroll
        for (int m = 0; m < 3; m++) T[l][m] = ph[RHO] * ph[U1 + m] * vcov[l];
        T[l][l] += press;
      }
      double s0 = 0.0, s1 = 0.0, s2 = 0.0;
      s0 += T[0][0] * geo3(g, G3_C000, ij);
      s0 += T[1][1] * geo3(g, G3_C101, ij);
      s0 += T[2][2] * geo3(g, G3_C202, ij);
      s1 += T[0][1] * geo3(g, G3_C011, ij);
      s1 += T[1][0] * geo3(g, G3_C110, ij);
      s1 += T[1][1] * geo3(g, G3_C111, ij);
      s1 += T[2][2] * geo3(g, G3_C212, ij);
      s2 += T[0][2] * geo3(g, G3_C022, ij);
      s2 += T[1][2] * geo3(g, G3_C122, ij);
      s2 += T[2][0] * geo3(g, G3_C220, ij);
      s2 += T[2][1] * geo3(g, G3_C221, ij);
      src[RHO] = 0.0; src[UU] = 0.0; src[U1] = s0; src[U2] = s1; src[U3] = s2;
    }
    // GRAV=FIXED_GRAV (gravity.c:38-64): the constant contravariant acceleration, lowered
    // with the zone's metric, on the momenta of the grid's directions and the energy
    if (P.grav_on) add_fixed_gravity(ph, P.grav, g0, g1, g2, g.ndim, src);
    if (g.mono) {
      // monopole gravity (gravity.c:373-401): mass flux density on the outer faces of the
      // zone (row i+1, the fan-in below) and on its inner face
      const int dji = djs(g, i), djo = djs(g, i + 1);
      const int jp = j * dji / djo, njp = dji / djo, dkij = dks(g, i, j);
      double vr = 0.0, area = 0.0;
      for (int jj = jp; jj < jp + njp; jj++) {
        const int nkp = dkij / dks(g, i + 1, jj);
        const int ijo = rowi(g, i + 1, jj);
        const int64_t fb = __ldg(g.f0 + ijo);
        const double ao = geo3(g, G3_A0, ijo);
        for (int kk = k * nkp; kk < k * nkp + nkp; kk++) {
          vr += F0[RHO * g.nf0 + fb + kk];
          area += ao + 1.0e-16;
        }
      }
      vr /= area;
      const double vl = F0[RHO * g.nf0 + __ldg(g.f0 + ij) + k] / (geo3(g, G3_A0, ij) + 1.0e-16);
      const int64_t rcs = g.n1 + 2 * NG;
      add_monopole_gravity(ph[RHO], g.gmono[i], vl, vr, g.x0 + i * g.dx0, g.dx0, __ldg(g.rc0 + RC_B0 * rcs + i + NG),
                           __ldg(g.rc0 + RC_G0 * rcs + i + NG), src);
    }
    p_to_u(pn, u, g0, g1, g2);
    p_to_u(ph, uh, g0, g1, g2);
    lmin = dt_source_control(pn, u, src);
#pragma unroll
    for (int v = 0; v < NPRIM; v++) divF[v] = 0.0;
    // direction 0: outer face(s) on row i+1, inner face
    {
      const int nf0o = pr.nf0o;
      for (int q = 0; q < nf0o; q++) {
        const int nkp = pr.nkp[q];
        const int64_t fb = pr.f0o[q];
        for (int kk = k * nkp; kk < k * nkp + nkp; kk++) {
#pragma unroll
          for (int v = 0; v < NPRIM; v++) divF[v] += F0[v * g.nf0 + fb + kk];
        }
      }
      const int64_t fi = pr.f0i + k;
#pragma unroll
      for (int v = 0; v < NPRIM; v++) divF[v] -= F0[v * g.nf0 + fi];
    }
    // direction 1
    {
      const int64_t fo = pr.f1o, fin = pr.f1i;
      const int mo = pr.mo, mi = pr.mi;
      if (mo == 1) {
#pragma unroll
        for (int v = 0; v < NPRIM; v++) divF[v] += 0.5 * F1[v * g.nf1 + fo + k];
      } else if (mo == 2) {
#pragma unroll
        for (int v = 0; v < NPRIM; v++) divF[v] += F1[v * g.nf1 + fo + 2 * k] + F1[v * g.nf1 + fo + 2 * k + 1];
      } else {
#pragma unroll
        for (int v = 0; v < NPRIM; v++) divF[v] += F1[v * g.nf1 + fo + k];
      }
      if (mi == 1) {
#pragma unroll
        for (int v = 0; v < NPRIM; v++)
          divF[v] -= 0.5 * F1[v * g.nf1 + fin + 2 * k] + 0.5 * F1[v * g.nf1 + fin + 2 * k + 1];
      } else {
#pragma unroll
        for (int v = 0; v < NPRIM; v++) divF[v] -= F1[v * g.nf1 + fin + k];
      }
    }
    // direction 2
    if (g.ndim == 3) {
      const int64_t f2 = pr.f2 + k;
#pragma unroll
      for (int v = 0; v < NPRIM; v++) divF[v] += F2[v * g.nf2 + f2 + 1] - F2[v * g.nf2 + f2];
    }
    const double vol = geo3(g, G3_VOL, ij);
    const double pfact = STAGE ? 0.5 : 1.0, phfact = STAGE ? 0.5 : 0.0, ffact = STAGE ? 0.5 : 1.0;
#pragma unroll
    for (int v = 0; v < NPRIM; v++) {
      const double ddt = divF[v] / vol - src[v];
      u[v] = pfact * u[v] + phfact * uh[v] - ffact * dt * ddt;
    }
    u_to_p(u, pf, geo3(g, G3_GCON + 0, ij), geo3(g, G3_GCON + 1, ij), geo3(g, G3_GCON + 2, ij), P.floors != 0,
           P.rho_floor, P.e_floor);
#pragma unroll
    for (int v = 0; v < NPRIM; v++) out.v[v][c] = pf[v];
    flag_nonfinite(pf, &times[0]);
    if (STAGE == 1) {
      // next estimate_dt: velocity of the new state, sound speed of the stage state
      const double cs = sqrt(P.gam * press / ph[RHO]);
      double local_dt = 0.0;
      local_dt += (fabs(pf[U1]) + cs / geo3(g, G3_SCALE + 0, ij)) / g.dx0;
      lmin = tmin(lmin, 1.0 / local_dt);
      local_dt += (fabs(pf[U2]) + cs / geo3(g, G3_SCALE + 1, ij)) / (g.dx1 * djs(g, i));
      lmin = tmin(lmin, 1.0 / local_dt);
      if (g.ndim == 3) {
        local_dt += (fabs(pf[U3]) + cs / geo3(g, G3_SCALE + 2, ij)) / (g.dx2 * dks(g, i, j));
        lmin = tmin(lmin, 1.0 / local_dt);
      }
    }
  }
  (void)lmax;
  block_min_to(lmin, &times[0].minacc, sred);
}

// First estimate_dt of the problem (step.c:171-187, the EOS of the state itself).
__global__ void __launch_bounds__(NT3) estimate3_kernel(const ProbDev *__restrict__ probs,
                                                         ProbTime *__restrict__ times, Grid3 g,
                                                         const Tile3 *__restrict__ tiles, StateSoA s)
{
  __shared__ double sred[32];
  const ProbDev &P = probs[0];
  const Tile3 t = tiles[blockIdx.x];
  const int i = t.i, j = t.j, k = t.k0 + (int)threadIdx.x;
  double lmin = 1.0e300;
  if ((int)threadIdx.x < t.cnt) {
    const int ij = rowi(g, i, j);
    const int64_t c = __ldg(g.cell + ij) + k;
    const double rho = s.v[RHO][c], uu = s.v[UU][c];
    const double cs = sqrt(P.gam * eos_press(P.eos, P.gam, P.Kpoly, rho, uu) / rho);
    double local_dt = 0.0;
    local_dt += (fabs(s.v[U1][c]) + cs / geo3(g, G3_SCALE + 0, ij)) / g.dx0;
    lmin = tmin(lmin, 1.0 / local_dt);
    local_dt += (fabs(s.v[U2][c]) + cs / geo3(g, G3_SCALE + 1, ij)) / (g.dx1 * djs(g, i));
    lmin = tmin(lmin, 1.0 / local_dt);
    if (g.ndim == 3) {
      local_dt += (fabs(s.v[U3][c]) + cs / geo3(g, G3_SCALE + 2, ij)) / (g.dx2 * dks(g, i, j));
      lmin = tmin(lmin, 1.0 / local_dt);
    }
  }
  block_min_to(lmin, &times[0].minacc, sred);
}


// Mass and total energy (utils.c:2337-2361, 2581-2612) with compensated sums: one CTA,
// each thread over a fixed subset of the zone tiles, then the threads in order.
__device__ __forceinline__ void neumaier3(double &s, double &c, double x)
{
  const double t = s + x;
  if (fabs(s) >= fabs(x)) c += (s - t) + x;
  else c += (x - t) + s;
  s = t;
}

__global__ void __launch_bounds__(256) totals3_kernel(Grid3 g, const Tile3 *__restrict__ tiles, int ntiles,
                                                       StateSoA s, double *__restrict__ out)
{
  __shared__ double sh[4][256];
  const int t = threadIdx.x;
  double ms = 0.0, mc = 0.0, es = 0.0, ec = 0.0;
  for (int q = t; q < ntiles; q += blockDim.x) {
    const Tile3 tl = tiles[q];
    const int ij = rowi(g, tl.i, tl.j);
    const double vol = geo3(g, G3_VOL, ij);
    const double g0 = geo3(g, G3_GCOV + 0, ij), g1 = geo3(g, G3_GCOV + 1, ij), g2 = geo3(g, G3_GCOV + 2, ij);
    for (int k = tl.k0; k < tl.k0 + tl.cnt; k++) {
      const int64_t c = __ldg(g.cell + ij) + k;
      double p[NPRIM], u[NPRIM];
#pragma unroll
      for (int v = 0; v < NPRIM; v++) p[v] = s.v[v][c];
      p_to_u(p, u, g0, g1, g2);
      neumaier3(ms, mc, p[RHO] * vol);
      neumaier3(es, ec, u[UU] * vol);
    }
  }
  sh[0][t] = ms; sh[1][t] = mc; sh[2][t] = es; sh[3][t] = ec;
  __syncthreads();
  if (t == 0) {
    double S = 0.0, C = 0.0, E = 0.0, D = 0.0;
    for (int k = 0; k < (int)blockDim.x; k++) {
      neumaier3(S, C, sh[0][k]); C += sh[1][k];
      neumaier3(E, D, sh[2][k]); D += sh[3][k];
    }
    out[0] = S + C;
    out[1] = E + D;
  }
}

// ------------------------------------------------------------------------ host driver

void build_grid3(const mdg_problem_desc &d, Grid3Host &h);

struct Sweep3 {
  Grid3 g{};
  char *d_tab = nullptr;           // all grid tables in one allocation
  double *d_flux = nullptr;        // F0 | F1 | F2, 5 arrays each
  unsigned char *d_bits = nullptr; // own0 | own1 | all0, one byte per zone each
  Tile3 *d_tiles = nullptr;        // face2 | zone tiles
  Tile3R *d_runs = nullptr;        // direction-0 face runs | direction-1 face runs
  size_t runs_cap = 0;             // Tile3R entries d_runs holds
  int run_len = RUN0;
  // the row structure the run lists are cut from (a copy of the host grid's)
  int n1 = 0, n2 = 0, n3 = 0;
  std::vector<int> nj, rowbase, nk;
  double *d_gmono = nullptr;       // monopole gravity per radial row
  int nt[4] = {0, 0, 0, 0};
  int64_t ncell = 0;
  int64_t bytes = 0;               // device memory held
};

static void tiles_of_rows(std::vector<Tile3> &out, int i, int j, int count, int chunk = NT3)
{
  for (int k0 = 0; k0 < count; k0 += chunk) out.push_back(Tile3{i, j, k0, (count - k0 < chunk) ? count - k0 : chunk});
}

// Work lists of the radial and theta run kernels for runs of at most run_len faces.
static void build_runs(const Sweep3 &w, int run_len, std::vector<Tile3R> &t0, std::vector<Tile3R> &t1)
{
  auto njr = [&](int i) { return w.nj[i + NG]; };
  auto row = [&](int i, int j) { return w.rowbase[i + NG] + j + NG; };
  auto dj = [&](int i) { return w.n2 / w.nj[i + NG]; };
  auto dk = [&](int i, int j) { return w.n3 / w.nk[row(i, j)]; };
  t0.clear();
  t1.clear();
  // direction-0 runs: faces i in [0, n1] grouped by constant theta resolution, then per
  // theta row j by constant phi resolution, cut into run_len faces and NT3 phi columns
  for (int i = 0; i <= w.n1;) {
    int ie = i + 1;
    while (ie <= w.n1 && dj(ie) == dj(i)) ie++;
    for (int j = 0; j < njr(i); j++) {
      for (int a = i; a < ie;) {
        int b = a + 1;
        while (b < ie && dk(b, j) == dk(a, j)) b++;
        const int nk = w.nk[row(a, j)];
        for (int c = a; c < b; c += run_len)
          for (int k0 = 0; k0 < nk; k0 += NT3)
            t0.push_back(Tile3R{c, std::min(run_len, b - c), j, k0, std::min(NT3, nk - k0)});
        a = b;
      }
    }
    i = ie;
  }
  // direction-1 runs: faces j in [0, nj(i)] of radial row i grouped by constant phi
  // resolution of the face, min(dk(i, j), dk(i, j-1)), cut into run_len faces and NT3 columns
  for (int i = 0; i < w.n1; i++) {
    const int nj = njr(i);
    auto mn = [&](int j) { return std::min(dk(i, j), dk(i, j - 1)); };
    for (int a = 0; a <= nj;) {
      int b = a + 1;
      while (b <= nj && mn(b) == mn(a)) b++;
      const int cnt = w.n3 / mn(a);
      for (int c = a; c < b; c += run_len)
        for (int k0 = 0; k0 < cnt; k0 += NT3)
          t1.push_back(Tile3R{c, std::min(run_len, b - c), i, k0, std::min(NT3, cnt - k0)});
      a = b;
    }
  }
}

int sweep3_set_run_length(Sweep3 *w, int run_length, std::string &why)
{
  if (run_length < 1 || run_length > 64) { why = "run_length out of [1, 64]"; return MDG_ERR_INVALID; }
  if (run_length == w->run_len) return MDG_OK;
  std::vector<Tile3R> t0, t1;
  build_runs(*w, run_length, t0, t1);
  const int n0 = (int)t0.size(), n1 = (int)t1.size();
  t0.insert(t0.end(), t1.begin(), t1.end());
  cudaError_t e = cudaSuccess;
  if (t0.size() > w->runs_cap) {
    Tile3R *d = nullptr;
    e = cudaMalloc(&d, sizeof(Tile3R) * t0.size());
    if (e != cudaSuccess) { why = cudaGetErrorString(e); return MDG_ERR_OUTOFMEM; }
    cudaFree(w->d_runs);
    w->d_runs = d;
    w->runs_cap = t0.size();
  }
  e = cudaMemcpy(w->d_runs, t0.data(), sizeof(Tile3R) * t0.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { why = cudaGetErrorString(e); return MDG_ERR_CUDA; }
  w->nt[0] = n0;
  w->nt[1] = n1;
  w->run_len = run_length;
  return MDG_OK;
}

int sweep3_create(const mdg_problem_desc &d, Sweep3 **out, std::string &why)
{
  *out = nullptr;
  Grid3Host h;
  build_grid3(d, h);
  if (h.nlev1 > G3_MAXLEV || h.nlev2 > G3_MAXLEV) { why = "too many refinement levels"; return MDG_ERR_INVALID; }
  Sweep3 *w = new Sweep3();
  w->ncell = h.ncell;
  // push() flux addresses of every interior row (the fan-in rules of push3_kernel)
  std::vector<PushRow3> prow((size_t)h.nij);
  for (int i = 0; i < h.n1; i++) {
    for (int j = 0; j < h.njr(i); j++) {
      PushRow3 r{};
      const int ij = h.row(i, j);
      const int dji = h.dj(i), djo = h.dj(i + 1), dkij = h.dk(i, j);
      const int jp = j * dji / djo;
      r.nf0o = (djo < dji) ? dji / djo : 1;
      for (int q = 0; q < r.nf0o; q++) {
        r.nkp[q] = dkij / h.dk(i + 1, jp + q);
        r.f0o[q] = h.f0[h.row(i + 1, jp + q)];
      }
      r.f0i = h.f0[ij];
      const int dkp = h.dk(i, j + 1), dkm = h.dk(i, j - 1);
      r.f1o = h.f1[h.row(i, j + 1)];
      r.f1i = h.f1[ij];
      r.mo = (dkp > dkij) ? 1 : (dkp < dkij ? 2 : 0);
      r.mi = (dkm < dkij) ? 1 : 0;
      r.f2 = h.ndim == 3 ? h.f2[ij] : 0;
      r.cell = h.cell[ij];
      prow[ij] = r;
    }
  }
  // one allocation for every table, each part 256-byte aligned
  std::vector<std::pair<const void *, size_t>> parts = {
      {h.nj.data(), h.nj.size() * sizeof(int)},         {h.rowbase.data(), h.rowbase.size() * sizeof(int)},
      {h.nk.data(), h.nk.size() * sizeof(int)},         {h.cell.data(), h.cell.size() * sizeof(int64_t)},
      {h.f0.data(), h.f0.size() * sizeof(int64_t)},     {h.f1.data(), h.f1.size() * sizeof(int64_t)},
      {h.f2.data(), h.f2.size() * sizeof(int64_t)},     {h.geo.data(), h.geo.size() * sizeof(double)},
      {h.rc0.data(), h.rc0.size() * sizeof(double)},    {h.rc1.data(), h.rc1.size() * sizeof(double)},
      {h.rc2.data(), h.rc2.size() * sizeof(double)},    {h.xc1.data(), h.xc1.size() * sizeof(double)},
      {h.xc2.data(), h.xc2.size() * sizeof(double)},    {h.sth.data(), h.sth.size() * sizeof(double)},
      {h.cth.data(), h.cth.size() * sizeof(double)},    {h.sphc.data(), h.sphc.size() * sizeof(double)},
      {h.cphc.data(), h.cphc.size() * sizeof(double)},  {h.sphl.data(), h.sphl.size() * sizeof(double)},
      {h.cphl.data(), h.cphl.size() * sizeof(double)},  {h.mx0.data(), h.mx0.size() * sizeof(float)},
      {h.mx1.data(), h.mx1.size() * sizeof(float)},     {h.mx2.data(), h.mx2.size() * sizeof(float)},
      {h.medge.data(), h.medge.size() * sizeof(double)},    {prow.data(), prow.size() * sizeof(PushRow3)}};
  std::vector<size_t> off(parts.size());
  size_t tot = 0;
  for (size_t q = 0; q < parts.size(); q++) {
    off[q] = tot;
    tot += (parts[q].second + 255) / 256 * 256;
  }
  w->bytes = (int64_t)tot + (int64_t)sizeof(double) * NPRIM * (h.nf0 + h.nf1 + h.nf2) + 3 * h.ncell +
             (int64_t)sizeof(double) * h.n1;
  std::vector<char> host(tot, 0);
  for (size_t q = 0; q < parts.size(); q++) std::memcpy(host.data() + off[q], parts[q].first, parts[q].second);
  auto fail3 = [&](cudaError_t e) {
    why = cudaGetErrorString(e);
    cudaFree(w->d_tab); cudaFree(w->d_flux); cudaFree(w->d_bits); cudaFree(w->d_tiles); cudaFree(w->d_gmono);
    cudaFree(w->d_runs);
    delete w;
    return e == cudaErrorMemoryAllocation ? MDG_ERR_OUTOFMEM : MDG_ERR_CUDA;
  };
  cudaError_t e = cudaMalloc(&w->d_tab, tot);
  if (e != cudaSuccess) return fail3(e);
  e = cudaMemcpy(w->d_tab, host.data(), tot, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail3(e);
  Grid3 &g = w->g;
  g.ndim = h.ndim;
  g.n1 = h.n1; g.n2 = h.n2; g.n3 = h.n3;
  g.bc_lo0 = d.bc_lo[0]; g.bc_hi0 = d.bc_hi[0]; g.bc_lo1 = d.bc_lo[1]; g.bc_hi1 = d.bc_hi[1];
  g.bc_lo2 = d.bc_lo[2]; g.bc_hi2 = d.bc_hi[2];
  g.dx0 = d.dx[0]; g.dx1 = d.dx[1]; g.dx2 = d.dx[2];
  g.nij = h.nij; g.ncell = h.ncell; g.nf0 = h.nf0; g.nf1 = h.nf1; g.nf2 = h.nf2;
  g.cols1 = h.cols1; g.cols2 = h.cols2;
  for (int l = 0; l < G3_MAXLEV; l++) { g.rc1_base[l] = h.rc1_base[l]; g.rc2_base[l] = h.rc2_base[l]; }
  char *b = w->d_tab;
  g.nj = (const int *)(b + off[0]); g.rowbase = (const int *)(b + off[1]); g.nk = (const int *)(b + off[2]);
  g.cell = (const int64_t *)(b + off[3]); g.f0 = (const int64_t *)(b + off[4]);
  g.f1 = (const int64_t *)(b + off[5]); g.f2 = (const int64_t *)(b + off[6]);
  g.geo = (const double *)(b + off[7]); g.rc0 = (const double *)(b + off[8]);
  g.rc1 = (const double *)(b + off[9]); g.rc2 = (const double *)(b + off[10]);
  g.xc1 = (const double *)(b + off[11]); g.xc2 = (const double *)(b + off[12]);
  g.sth = (const double *)(b + off[13]); g.cth = (const double *)(b + off[14]);
  g.sphc = (const double *)(b + off[15]); g.cphc = (const double *)(b + off[16]);
  g.sphl = (const double *)(b + off[17]); g.cphl = (const double *)(b + off[18]);
  g.mx0 = (const float *)(b + off[19]); g.mx1 = (const float *)(b + off[20]); g.mx2 = (const float *)(b + off[21]);
  g.medge = (const double *)(b + off[22]);
  g.prow = (const PushRow3 *)(b + off[23]);
  g.x0 = d.startx[0];
  g.mono = d.monopole;
  e = cudaMalloc(&w->d_gmono, sizeof(double) * (size_t)h.n1);
  if (e != cudaSuccess) return fail3(e);
  g.gmono = w->d_gmono;
  // flux arrays, shock bits
  e = cudaMalloc(&w->d_flux, sizeof(double) * NPRIM * (size_t)(h.nf0 + h.nf1 + h.nf2));
  if (e != cudaSuccess) return fail3(e);
  e = cudaMalloc(&w->d_bits, (size_t)3 * h.ncell);
  if (e != cudaSuccess) return fail3(e);
  e = cudaMemset(w->d_bits, 0, (size_t)3 * h.ncell);
  if (e != cudaSuccess) return fail3(e);
  // tiles of each kernel
  std::vector<Tile3> t2, tc;
  std::vector<Tile3R> t0, t1;
  w->n1 = h.n1; w->n2 = h.n2; w->n3 = h.n3;
  w->nj = h.nj; w->rowbase = h.rowbase; w->nk = h.nk;
  build_runs(*w, RUN0, t0, t1);
  for (int i = 0; i < h.n1 && h.ndim == 3; i++)
    for (int j = 0; j < h.njr(i); j++) tiles_of_rows(t2, i, j, h.nk[h.row(i, j)] + 1, T2);
  for (int i = 0; i < h.n1; i++)
    for (int j = 0; j < h.njr(i); j++) tiles_of_rows(tc, i, j, h.nk[h.row(i, j)]);
  w->nt[0] = (int)t0.size(); w->nt[1] = (int)t1.size(); w->nt[2] = (int)t2.size(); w->nt[3] = (int)tc.size();
  std::vector<Tile3> all;
  all.insert(all.end(), t2.begin(), t2.end());
  all.insert(all.end(), tc.begin(), tc.end());
  e = cudaMalloc(&w->d_tiles, sizeof(Tile3) * all.size());
  if (e != cudaSuccess) return fail3(e);
  e = cudaMemcpy(w->d_tiles, all.data(), sizeof(Tile3) * all.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail3(e);
  t0.insert(t0.end(), t1.begin(), t1.end());
  e = cudaMalloc(&w->d_runs, sizeof(Tile3R) * t0.size());
  if (e != cudaSuccess) return fail3(e);
  w->runs_cap = t0.size();
  e = cudaMemcpy(w->d_runs, t0.data(), sizeof(Tile3R) * t0.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail3(e);
  *out = w;
  return MDG_OK;
}

void sweep3_destroy(Sweep3 *w)
{
  if (!w) return;
  cudaFree(w->d_tab); cudaFree(w->d_flux); cudaFree(w->d_bits); cudaFree(w->d_tiles); cudaFree(w->d_gmono);
  cudaFree(w->d_runs);
  delete w;
}

int64_t sweep3_ncell(const Sweep3 *w) { return w->ncell; }
int64_t sweep3_bytes(const Sweep3 *w) { return w->bytes; }

// Kernel launches of one RK stage of the single 3-D problem (slot 0).
void launch_stage3d(int stage, bool mixed, Sweep3 *w, const ProbDev *probs, ProbTime *times, StateSoA sst,
                    StateSoA sn, StateSoA out, cudaStream_t st)
{
  const Grid3 &g = w->g;
  double *F0 = w->d_flux, *F1 = F0 + NPRIM * g.nf0, *F2 = F1 + NPRIM * g.nf1;
  unsigned char *own = w->d_bits + (size_t)stage * g.ncell, *all0 = w->d_bits + (size_t)2 * g.ncell;
  const Tile3R *t0 = w->d_runs, *t1 = t0 + w->nt[0];
  const Tile3 *t2 = w->d_tiles, *tc = t2 + w->nt[2];
  if (stage == 0) cudaMemsetAsync(all0, 0, (size_t)g.ncell, st);
  if (g.mono) {
    shell_mass3_kernel<<<(g.n1 + 127) / 128, 128, 0, st>>>(times, g, sst);
    monopole_profile3_kernel<<<1, 32, 0, st>>>(times, g);
  }
  auto faces = [&](auto s0, auto mix) {
    constexpr int S = decltype(s0)::value;
    constexpr bool M = decltype(mix)::value;
    face0_kernel<M><<<w->nt[0], NT3, 0, st>>>(probs, times, g, t0, sst, F0, own, all0, S);
    face1_kernel<M><<<w->nt[1], NT3, 0, st>>>(probs, times, g, t1, sst, F1, own, all0, S);
    if (w->nt[2] > 0) face2_kernel<S, M><<<w->nt[2], NT3, 0, st>>>(probs, times, g, t2, sst, F2, own, all0);
  };
  using I0 = std::integral_constant<int, 0>;
  using I1 = std::integral_constant<int, 1>;
  using BF = std::integral_constant<bool, false>;
  using BT = std::integral_constant<bool, true>;
  if (stage == 0) {
    if (mixed) faces(I0{}, BT{}); else faces(I0{}, BF{});
    push3_kernel<0><<<w->nt[3], NT3, 0, st>>>(probs, times, g, tc, sst, sn, out, F0, F1, F2);
  } else {
    if (mixed) faces(I1{}, BT{}); else faces(I1{}, BF{});
    push3_kernel<1><<<w->nt[3], NT3, 0, st>>>(probs, times, g, tc, sst, sn, out, F0, F1, F2);
  }
}

void launch_totals3(Sweep3 *w, StateSoA s, double *out, cudaStream_t st)
{
  const Tile3 *tc = w->d_tiles + w->nt[2];
  totals3_kernel<<<1, 256, 0, st>>>(w->g, tc, w->nt[3], s, out);
}

void launch_initial_estimate3(Sweep3 *w, const ProbDev *probs, ProbTime *times, StateSoA s, cudaStream_t st)
{
  const Tile3 *tc = w->d_tiles + w->nt[2];
  estimate3_kernel<<<w->nt[3], NT3, 0, st>>>(probs, times, w->g, tc, s);
}

}  // namespace mdg
