// Tables of the mixed-precision 1-D sweep built on the device.
//
// The plain FP64 sweep needs the reference's own table values, so its tables are built on
// the host from Romberg moments exactly as the reference computes them (mdg_geometry.cpp).
// The mixed-precision sweep only needs them to FP64 accuracy: here one thread per table
// column evaluates the closed-form moments of its zone and its neighbours
// (moments_closed) and derives the reconstruction coefficients, the FP32 weights and the
// face/zone geometry from them.  This takes the per-problem set-up cost off the host --
// for a 2048-problem ensemble, seconds of Romberg quadrature -- which is what a solve
// server admitting thousands of requests per second needs.
#include <cuda_runtime.h>
#include <math.h>
#include "mdg_kernels.cuh"
#include "mdg_tables.cuh"

namespace mdg {

__global__ void build_tables_1d_kernel(const ProbDev *__restrict__ probs, int m, double *__restrict__ rc,
                                       double *__restrict__ geo, float *__restrict__ mx, int64_t stride)
{
  const ProbDev &P = probs[m];
  const int n = P.n1;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;   // column c holds zone i = c - NG
  if (c >= n + 2 * NG) return;
  const int i = c - NG;
  const int im = (i - 1 < -NG) ? -NG : i - 1, ip = (i + 1 >= n + NG) ? n + NG - 1 : i + 1;
  const int sph = P.has_src;
  double am, bm, gm, a0, b0, g0, ap, bp, gp;
  moments_closed(sph, P.x0, P.dx0, im, am, bm, gm);
  moments_closed(sph, P.x0, P.dx0, i, a0, b0, g0);
  moments_closed(sph, P.x0, P.dx0, ip, ap, bp, gp);
  const double xl = P.x0 + i * P.dx0, xr = P.x0 + (i + 1) * P.dx0;
  const int64_t col = P.geo_off + c;
  double v[RC_NFIELDS];
  rc_fields(am, a0, ap, bm, b0, bp, gm, g0, gp, xl, xr, v);
  for (int f = 0; f < RC_NFIELDS; f++) rc[f * stride + col] = v[f];
  float w[MX_NFIELDS];
  mx_fields(am, a0, ap, bm, b0, bp, gm, g0, gp, xl, xr, w);
  for (int f = 0; f < MX_NFIELDS; f++) mx[f * stride + col] = w[f];

  // face i and zone i geometry (the closed forms of the mixed sweep; ghost zones of the
  // spherical grid may have x < 0, where r = |x|)
  double g[GF_NFIELDS];
  for (int f = 0; f < GF_NFIELDS; f++) g[f] = 0.0;
  g[GF_FSCALE] = 1.0; g[GF_FG0] = 1.0; g[GF_G0] = 1.0; g[GF_GC0] = 1.0; g[GF_S00] = 1.0;
  const bool face = (i >= 0 && i <= n);
  if (sph) {
    const double xl2 = xl * xl;
    g[GF_AREA] = face ? xl2 * P.gk_area : 0.0;
    g[GF_FG1] = xl2 * P.gk_th1;
    g[GF_FG2] = xl2 * P.gk_th2;
    const double vr = g0;   // int x^2 dx over the zone
    const double ra = fabs(xl), rb = fabs(xr);
    const double F = fabs(0.2 * (rb * rb * rb * rb * rb - ra * ra * ra * ra * ra) / vr);
    g[GF_VOL] = vr * P.gk_area;
    g[GF_G1] = F * P.gk_th1;
    g[GF_G2] = F * P.gk_th2;
    g[GF_GC1] = (g[GF_G1] > 1.0e-50) ? 1.0 / g[GF_G1] : 0.0;
    g[GF_GC2] = (g[GF_G2] > 1.0e-50) ? 1.0 / g[GF_G2] : 0.0;
    if (i >= 0 && i < n) {
      const double h = xr - xl;
      const double c101 = 0.5 * h * (xl + xr) / vr;
      g[GF_CONN + 10] = c101;                                   // conn[1][0][1]
      g[GF_CONN + 12] = c101;                                   // conn[1][1][0]
      g[GF_CONN + 20] = c101;                                   // conn[2][0][2]
      g[GF_CONN + 24] = c101;                                   // conn[2][2][0]
      g[GF_CONN + 4] = -(0.25 * h * (xl + xr) * (xl * xl + xr * xr) / vr) * P.gk_th1;   // conn[0][1][1]
      g[GF_CONN + 23] = P.gk_tc;                                // conn[2][1][2]
      g[GF_CONN + 25] = P.gk_tc;                                // conn[2][2][1]
      g[GF_CONN + 8] = -c101 * g[GF_G2];                        // conn[0][2][2]
      g[GF_CONN + 17] = -P.gk_tc * g[GF_G2] / g[GF_G1];         // conn[1][2][2]
    }
  } else {
    g[GF_AREA] = face ? 1.0 : 0.0;
    g[GF_FG1] = 1.0; g[GF_FG2] = 1.0;
    g[GF_VOL] = P.dx0;
    g[GF_G1] = 1.0; g[GF_G2] = 1.0; g[GF_GC1] = 1.0; g[GF_GC2] = 1.0;
  }
  for (int f = 0; f < GF_NFIELDS; f++) geo[f * stride + col] = g[f];
}

void launch_build_tables_1d(const ProbDev *probs, int m, int n1, double *rc, double *geo, float *mx,
                            int64_t stride, cudaStream_t st)
{
  const int ncol = n1 + 2 * NG;
  build_tables_1d_kernel<<<(ncol + 127) / 128, 128, 0, st>>>(probs, m, rc, geo, mx, stride);
}

}  // namespace mdg
