// Per-zone table entries of the 1-D sweeps as host/device functions of the volume
// moments, shared by the host table builders (mdg_geometry.cpp, from the reference's
// Romberg moments: bit-identical to the reference) and the device builder of the
// mixed-precision tables (mdg_tables.cu, from closed-form moments).
#pragma once
#include "mdg_internal.h"

namespace mdg {

// Reconstruction coefficients of one zone (ReconField) from the moments alpha/beta/Gamma
// of the zone (a0, b0, g0) and its neighbours (m: i-1, p: i+1) and its edges xl, xr:
// the geometry-only sub-expressions of para_recon (reconstruct.c:151-157,174-175) and
// lin_recon (reconstruct.c:100-104) in the reference's operation order.
MDG_HD inline void rc_fields(double am, double a0, double ap, double bm, double b0, double bp, double gm,
                             double g0, double gp, double xl, double xr, double *v)
{
  double a0b1g2 = am * b0 * gp, a0b2g1 = am * bp * g0, a1b0g2 = a0 * bm * gp;
  double a1b2g0 = a0 * bp * gm, a2b0g1 = ap * bm * g0, a2b1g0 = ap * b0 * gm;
  double den1 = 1.0 / (a0b1g2 + a1b2g0 + a2b0g1 - a0b2g1 - a1b0g2 - a2b1g0);
  double den2 = (xl - xr) * (a0 + g0 * xl * xr - b0 * (xl + xr));
  den2 = 1.0 / den2;
  double xm = bm / gm, xp = bp / gp, xc = b0 / g0;
  v[RC_AM] = am; v[RC_A0] = a0; v[RC_AP] = ap;
  v[RC_BM] = bm; v[RC_B0] = b0; v[RC_BP] = bp;
  v[RC_GM] = gm; v[RC_G0] = g0; v[RC_GP] = gp;
  v[RC_XL] = xl; v[RC_XR] = xr;
  v[RC_DEN1] = den1; v[RC_DEN2] = den2;
  v[RC_XLR] = xl - xr;
  v[RC_XL2] = xl * xl; v[RC_XR2] = xr * xr;
  v[RC_XMID] = 0.5 * (xl + xr);
  v[RC_DMR] = a0 + xr * (g0 * xr - 2.0 * b0);
  v[RC_DML] = a0 + xl * (g0 * xl - 2.0 * b0);
  v[RC_LSM] = xc - 0.5 * (xl + xm);
  v[RC_LSP] = 0.5 * (xr + xp) - xc;
  v[RC_LSC] = xp - xm;
}

// FP32 reconstruction weights of one zone (MixField; the parabola of para_recon on the
// differences dqm, dqp, with the geometry folded in), computed in FP64.
MDG_HD inline void mx_fields(double am, double a0, double ap, double bm, double b0, double bp, double gm,
                             double g0, double gp, double xl, double xr, float *out)
{
  double den1 = 1.0 / (am * b0 * gp + a0 * bp * gm + ap * bm * g0 - am * bp * g0 - a0 * bm * gp - ap * b0 * gm);
  double kAm = (bp * gm * g0 - gp * b0 * gm) * den1, kAp = (gp * bm * g0 - gp * b0 * gm) * den1;
  double kBm = -(ap * gm * g0 - gp * a0 * gm) * den1, kBp = -(gp * am * g0 - gp * a0 * gm) * den1;
  double cl2 = xl * xl - a0 / g0, cl1 = xl - b0 / g0, cr2 = xr * xr - a0 / g0, cr1 = xr - b0 / g0;
  double den2 = 1.0 / ((xl - xr) * (a0 + g0 * xl * xr - b0 * (xl + xr)));
  double eAl = (g0 * xr - b0) * den2, eAr = (b0 - g0 * xl) * den2;
  double eBl = (a0 - g0 * xr * xr) * den2, eBr = (g0 * xl * xl - a0) * den2;
  double dmr = a0 + xr * (g0 * xr - 2.0 * b0), dml = a0 + xl * (g0 * xl - 2.0 * b0);
  double v[MX_NFIELDS];
  v[MX_WLM] = kAm * cl2 + kBm * cl1;
  v[MX_WLP] = kAp * cl2 + kBp * cl1;
  v[MX_WRM] = kAm * cr2 + kBm * cr1;
  v[MX_WRP] = kAp * cr2 + kBp * cr1;
  v[MX_EAL] = eAl;
  v[MX_EAR] = eAr;
  v[MX_EBL] = eBl + 2.0 * xl * eAl;
  v[MX_EBR] = eBr + 2.0 * xl * eAr;
  v[MX_DXZ] = xr - xl;
  v[MX_MR] = (-g0 / dmr) * (cl2 - 2.0 * xr * cl1);
  v[MX_ML] = (-g0 / dml) * (cr2 - 2.0 * xl * cr1);
  for (int f = 0; f < MX_NFIELDS; f++) out[f] = (float)v[f];
}

// Volume moments of zone i of a uniform 1-D grid in closed form: for the spherical metric
// with r = |x|, dr/dx = 1 (metric_spherical_general.c:558-568) Gamma = int x^2 dx,
// beta = int x^3 dx, alpha = int x^4 dx over the zone (what the reference integrates by
// Romberg quadrature, exact for these polynomials up to rounding); Cartesian as
// metric_cartesian.c:47-55.
MDG_HD inline void moments_closed(int spherical, double x0, double dx, int i, double &al, double &be, double &ga)
{
  const double a = x0 + i * dx, b = x0 + (i + 1) * dx;
  if (spherical) {
    const double h = b - a, a2 = a * a, b2 = b * b;
    ga = h * (b2 + a * b + a2) * (1.0 / 3.0);
    be = h * (a + b) * (a2 + b2) * 0.25;
    al = h * (b2 * b2 + b2 * b * a + b2 * a2 + b * a2 * a + a2 * a2) * 0.2;
  } else {
    al = (b * b * b - a * a * a) / 3.0;
    be = (b * b - a * a) / 2.0;
    ga = dx;
  }
}

}  // namespace mdg
