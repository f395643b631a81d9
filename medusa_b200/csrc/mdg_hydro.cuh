// Device restatement of the reference's per-zone and per-face hydro arithmetic.
//
// Every function keeps the reference's floating-point expression trees (operation order
// and grouping) so that, compiled with -fmad=false, the FP64 instantiation reproduces the
// reference CPU build bit for bit; the only libm dependence is pow() in the
// two-rarefaction branch of the wave-speed estimate (CUDA's pow and the host's may differ
// in the last place) and sqrt/division, which are correctly rounded on both.
//
// Templated on the arithmetic type T so that the mixed-precision sweep can instantiate
// the reconstruction and Riemann solver in FP32.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include "mdg_internal.h"

namespace mdg {

template <typename T> __device__ __forceinline__ T tmin(T a, T b) { return (a < b) ? a : b; }
template <typename T> __device__ __forceinline__ T tmax(T a, T b) { return (a > b) ? a : b; }
template <typename T> __device__ __forceinline__ T tsign(T a) { return (a < T(0)) ? T(-1) : T(1); }

// Reconstruction coefficients of one zone (the geometry of para_recon/lin_recon).
template <typename T>
struct Rc {
  T am, a0, ap, bm, b0, bp, gm, g0, gp;
  T xl, xr, den1, den2, xlr, xl2, xr2, xmid, dmr, dml, lsm, lsp, lsc;
};

template <typename T>
__device__ __forceinline__ void load_rc(Rc<T> &r, const double *__restrict__ tab, int64_t stride, int64_t idx)
{
  r.am = T(__ldg(tab + RC_AM * stride + idx)); r.a0 = T(__ldg(tab + RC_A0 * stride + idx));
  r.ap = T(__ldg(tab + RC_AP * stride + idx));
  r.bm = T(__ldg(tab + RC_BM * stride + idx)); r.b0 = T(__ldg(tab + RC_B0 * stride + idx));
  r.bp = T(__ldg(tab + RC_BP * stride + idx));
  r.gm = T(__ldg(tab + RC_GM * stride + idx)); r.g0 = T(__ldg(tab + RC_G0 * stride + idx));
  r.gp = T(__ldg(tab + RC_GP * stride + idx));
  r.xl = T(__ldg(tab + RC_XL * stride + idx)); r.xr = T(__ldg(tab + RC_XR * stride + idx));
  r.den1 = T(__ldg(tab + RC_DEN1 * stride + idx)); r.den2 = T(__ldg(tab + RC_DEN2 * stride + idx));
  r.xlr = T(__ldg(tab + RC_XLR * stride + idx));
  r.xl2 = T(__ldg(tab + RC_XL2 * stride + idx)); r.xr2 = T(__ldg(tab + RC_XR2 * stride + idx));
  r.xmid = T(__ldg(tab + RC_XMID * stride + idx));
  r.dmr = T(__ldg(tab + RC_DMR * stride + idx)); r.dml = T(__ldg(tab + RC_DML * stride + idx));
  r.lsm = T(__ldg(tab + RC_LSM * stride + idx)); r.lsp = T(__ldg(tab + RC_LSP * stride + idx));
  r.lsc = T(__ldg(tab + RC_LSC * stride + idx));
}

// para_recon for one zone (reconstruct.c:142-201): am/a0/ap are the zone averages at
// i-1, i, i+1; returns the left (al) and right (ar) face values of zone i.
template <typename T>
__device__ __forceinline__ void para_recon_zone(T am_v, T a, T ap_v, const Rc<T> &g, T &al, T &ar)
{
  T dqm = a - am_v;
  T dqp = ap_v - a;
  if (dqm * dqp <= T(0)) { al = a; ar = a; return; }
  T dqc = ap_v - am_v;
  T A = (dqm * g.bp * g.gm * g.g0 + g.gp * (dqp * g.bm * g.g0 - dqc * g.b0 * g.gm)) * g.den1;
  T B = -(dqm * g.ap * g.gm * g.g0 + g.gp * (dqp * g.am * g.g0 - dqc * g.a0 * g.gm)) * g.den1;
  T C = a - (g.a0 * A + g.b0 * B) / g.g0;
  T l = g.xl * (A * g.xl + B) + C;
  T r = g.xr * (A * g.xr + B) + C;
  T mean = T(0.75) * am_v + T(0.25) * a;
  T mask = (a - l) * (l - mean);
  l = (mask < T(0)) ? mean : l;
  mean = T(0.75) * ap_v + T(0.25) * a;
  mask = (mean - r) * (r - a);
  r = (mask < T(0)) ? mean : r;
  A = (g.b0 * (r - l) + g.g0 * (a * g.xlr - r * g.xl + l * g.xr)) * g.den2;
  B = (g.a0 * (l - r) + g.g0 * (r - a) * g.xl2 + g.g0 * (a - l) * g.xr2) * g.den2;
  T xzero = -B / (T(2) * A + T(1.0e-16));
  if (isinf(xzero) || isnan(xzero)) xzero = T(-1.0e-200);
  if (xzero > g.xl && xzero < g.xr) {
    if (xzero > g.xmid) {
      A = g.g0 * (a - r) / g.dmr;
      B = T(-2.0) * A * g.xr;
      C = a - (g.a0 * A + g.b0 * B) / g.g0;
      l = g.xl * (A * g.xl + B) + C;
    } else {
      A = g.g0 * (a - l) / g.dml;
      B = T(-2.0) * A * g.xl;
      C = a - (g.a0 * A + g.b0 * B) / g.g0;
      r = g.xr * (A * g.xr + B) + C;
    }
  }
  al = l;
  ar = r;
}

// lin_recon for one zone (reconstruct.c:99-121)
template <typename T>
__device__ __forceinline__ void lin_recon_zone(T am_v, T a, T ap_v, const Rc<T> &g, T &al, T &ar)
{
  T sm = (a - am_v) / g.lsm;
  T sp = (ap_v - a) / g.lsp;
  if (sm * sp <= T(0)) { al = a; ar = a; return; }
  T sc = (ap_v - am_v) / g.lsc;
  T A = tsign(sc) * tmin(tmin(fabs(sm), fabs(sp)), fabs(sc));
  T B = a - A * g.b0 / g.g0;
  al = A * g.xl + B;
  ar = A * g.xr + B;
}

template <typename T>
__device__ __forceinline__ void recon_zone(int order, T am_v, T a, T ap_v, const Rc<T> &g, T &al, T &ar)
{
  if (order == 3) para_recon_zone(am_v, a, ap_v, g, al, ar);
  else if (order == 2) lin_recon_zone(am_v, a, ap_v, g, al, ar);
  else { al = a; ar = a; }
}

// Geometry of one face as the Riemann solver sees it (zone_geom at the face's cell).
template <typename T>
struct FaceGeom { T area, scale; T g0, g1, g2; };

// Wave-speed estimate shared by HLLC and HLLE (riemann.c:368-429 / 210-303).
// w[0..4] primitives, w[5] pressure, w[6] Gamma.
template <typename T>
__device__ __forceinline__ void wave_speeds(const T *pl, const T *pr, T u_l, T u_r, bool hlle,
                                            T &sl, T &sr, T &ss, T &p_s, int &isshock)
{
  const T p_l = pl[5], p_r = pr[5], G_l = pl[6], G_r = pr[6];
  T cs_l = sqrt(G_l * p_l / pl[RHO]);
  T cs_r = sqrt(G_r * p_r / pr[RHO]);
  T p_max, p_min;
  if (p_l > p_r) { p_max = p_l; p_min = p_r; } else { p_max = p_r; p_min = p_l; }
  T pratio = p_max / p_min;
  isshock = ((p_max - p_min) / p_min > T(0.5)) ? 1 : 0;
  p_s = T(0.5) * (p_l + p_r) - T(0.125) * (u_r - u_l) * (pl[RHO] + pr[RHO]) * (cs_l + cs_r);
  // HLLC clamps with MAX(0,p_s), HLLE with MAX(p_s,0.0): they differ only for NaN
  if (hlle) p_s = (p_s > T(0)) ? p_s : T(0);
  else p_s = (T(0) > p_s) ? T(0) : p_s;
  if (pratio < T(2) && p_s >= p_min && p_s <= p_max) {
    // primitive-variable estimate kept
  } else if (p_s < p_min) {
    // two rarefactions (Toro 9.35-9.36)
    T G_avg = T(0.5) * (G_l + G_r);
    T plr = pow(p_l / p_r, (G_avg - T(1)) / (T(2) * G_avg));
    T s0 = (plr * u_l / cs_l + u_r / cs_r + T(2) * (plr - T(1)) / (G_avg - T(1))) / (plr / cs_l + T(1) / cs_r);
    p_s = T(0.5) * (p_l * pow(T(1) + (G_l - T(1)) / (T(2) * cs_l) * (u_l - s0), T(2) * G_l / (G_l - T(1)))
                  + p_r * pow(T(1) + (G_r - T(1)) / (T(2) * cs_r) * (s0 - u_r), T(2) * G_r / (G_r - T(1))));
    p_s = tmax(p_s, T(0));
  } else {
    // two shocks (Toro 9.42-9.43)
    T a_l = T(2) / ((G_l + T(1)) * pl[RHO]);
    T a_r = T(2) / ((G_r + T(1)) * pr[RHO]);
    T b_l = (G_l - T(1)) / (G_l + T(1)) * p_l;
    T b_r = (G_r - T(1)) / (G_r + T(1)) * p_r;
    T g_l = sqrt(a_l / (p_s + b_l));
    T g_r = sqrt(a_r / (p_s + b_r));
    p_s = (g_l * p_l + g_r * p_r - (u_r - u_l)) / (g_l + g_r);
    p_s = tmax(p_s, T(0));
  }
  T q_l = (p_s <= p_l) ? T(1) : sqrt(T(1) + (G_l + T(1)) / (T(2) * G_l) * (p_s / p_l - T(1)));
  T q_r = (p_s <= p_r) ? T(1) : sqrt(T(1) + (G_r + T(1)) / (T(2) * G_r) * (p_s / p_r - T(1)));
  sl = u_l - cs_l * q_l;
  sr = u_r + cs_r * q_r;
  ss = (p_r - p_l + pl[RHO] * u_l * (sl - u_l) - pr[RHO] * u_r * (sr - u_r))
     / (pl[RHO] * (sl - u_l) - pr[RHO] * (sr - u_r));
}

// p_uflux (riemann.c:4-37) for direction DIR
template <int DIR, typename T>
__device__ __forceinline__ void p_uflux(const T *p, const FaceGeom<T> &g, T press, T *u, T *f)
{
  T vc0 = g.g0 * p[U1], vc1 = g.g1 * p[U2], vc2 = g.g2 * p[U3];
  T v = p[U1 + DIR];
  u[RHO] = p[RHO];
  T vsq = T(0);
  vsq += p[U1] * vc0; vsq += p[U2] * vc1; vsq += p[U3] * vc2;
  T etot = T(0.5) * u[RHO] * vsq + p[UU];
  u[UU] = etot;
  u[U1] = u[RHO] * vc0; u[U2] = u[RHO] * vc1; u[U3] = u[RHO] * vc2;
  f[RHO] = u[RHO] * v;
  f[UU] = v * (etot + press);
  f[U1] = f[RHO] * vc0; f[U2] = f[RHO] * vc1; f[U3] = f[RHO] * vc2;
  f[U1 + DIR] += press;
}

// pflux (riemann.c:39-62)
template <int DIR, typename T>
__device__ __forceinline__ void pflux(const T *p, T press, const FaceGeom<T> &g, T *f)
{
  T vc0 = g.g0 * p[U1], vc1 = g.g1 * p[U2], vc2 = g.g2 * p[U3];
  T v = p[U1 + DIR];
  T area = g.area;
  f[RHO] = area * p[RHO] * v;
  f[U1] = f[RHO] * vc0; f[U2] = f[RHO] * vc1; f[U3] = f[RHO] * vc2;
  f[U1 + DIR] += area * press;
  T vsq = T(0);
  vsq += p[U1] * vc0; vsq += p[U2] * vc1; vsq += p[U3] * vc2;
  T etot = T(0.5) * p[RHO] * vsq + p[UU];
  f[UU] = area * v * (etot + press);
}

// riemann_flux_HLLC (riemann.c:328-499); returns isshock, writes flux[5] and the signal
// speed used by the CFL reduction.
template <int DIR, typename T>
__device__ __forceinline__ int riemann_hllc(const T *pl, const T *pr, const FaceGeom<T> &g, T *flux, T &sig)
{
  int isshock = 0;
  if (g.area < T(1.0e-16)) {
    sig = T(1.0e-200);
#pragma unroll
    for (int v = 0; v < NPRIM; v++) flux[v] = T(0);
    return isshock;
  }
  const T sc = g.scale;
  T u_l = pl[U1 + DIR] * sc;
  T u_r = pr[U1 + DIR] * sc;
  T sl, sr, ss, p_s;
  wave_speeds<T>(pl, pr, u_l, u_r, false, sl, sr, ss, p_s, isshock);
  if (ss > sr) sr = T(1.001) * ss;
  if (ss < sl) sl = T(1.001) * ss;
  sig = tmax(fabs(sl), fabs(sr)) / sc;
  if (sl > T(0)) { pflux<DIR, T>(pl, pl[5], g, flux); return isshock; }
  if (sr < T(0)) { pflux<DIR, T>(pr, pr[5], g, flux); return isshock; }
  T u[NPRIM], fx[NPRIM], Us[NPRIM], slr;
  if (ss > T(0)) {
    p_uflux<DIR, T>(pl, g, pl[5], u, fx);
    Us[0] = pl[RHO] * (sl - u_l) / (sl - ss);
    Us[UU] = (u[UU] * (sl - u_l) - pl[5] * u_l + p_s * ss) / (sl - ss);
    Us[U1] = pl[U1]; Us[U2] = pl[U2]; Us[U3] = pl[U3];
    Us[U1 + DIR] = ss / sc;
    slr = sl / sc;
  } else {
    p_uflux<DIR, T>(pr, g, pr[5], u, fx);
    Us[0] = pr[RHO] * (sr - u_r) / (sr - ss);
    Us[UU] = (u[UU] * (u_r - sr) + pr[5] * u_r - p_s * ss) / (ss - sr);
    Us[U1] = pr[U1]; Us[U2] = pr[U2]; Us[U3] = pr[U3];
    Us[U1 + DIR] = ss / sc;
    slr = sr / sc;
  }
  T vc0 = g.g0 * Us[U1], vc1 = g.g1 * Us[U2], vc2 = g.g2 * Us[U3];
  Us[U1] = vc0 * Us[0]; Us[U2] = vc1 * Us[0]; Us[U3] = vc2 * Us[0];
#pragma unroll
  for (int v = 0; v < NPRIM; v++) flux[v] = g.area * (fx[v] + slr * (Us[v] - u[v]));
  return isshock;
}

// riemann_flux_HLLE (riemann.c:178-325)
template <int DIR, typename T>
__device__ __forceinline__ void riemann_hlle(const T *pl, const T *pr, const FaceGeom<T> &g, T *flux, T &sig)
{
  if (g.area < T(1.0e-16)) {
    sig = T(1.0e-200);
#pragma unroll
    for (int v = 0; v < NPRIM; v++) flux[v] = T(0);
    return;
  }
  const T sc = g.scale;
  T u_l = pl[U1 + DIR] * sc;
  T u_r = pr[U1 + DIR] * sc;
  T sl, sr, ss, p_s;
  int isshock;
  wave_speeds<T>(pl, pr, u_l, u_r, true, sl, sr, ss, p_s, isshock);
  T ul[NPRIM], ur[NPRIM], fl[NPRIM], fr[NPRIM];
  p_uflux<DIR, T>(pl, g, pl[5], ul, fl);
  p_uflux<DIR, T>(pr, g, pr[5], ur, fr);
  T cmax = tmax(sr / sc, T(0));
  T cmin = fabs(tmin(sl / sc, T(0)));
  sig = tmax(cmax, cmin);
#pragma unroll
  for (int v = 0; v < NPRIM; v++)
    flux[v] = g.area * (cmin * fr[v] + cmax * fl[v] - cmax * cmin * (ur[v] - ul[v])) / (cmax + cmin);
}

// hydro_p_to_u (fluid.c:4-24) with the zone-centred gcov
__device__ __forceinline__ void p_to_u(const double *p, double *u, double g0, double g1, double g2)
{
  double vc0 = g0 * p[U1], vc1 = g1 * p[U2], vc2 = g2 * p[U3];
  u[RHO] = p[RHO];
  double vsq = 0.0;
  vsq += p[U1] * vc0; u[U1] = u[RHO] * vc0;
  vsq += p[U2] * vc1; u[U2] = u[RHO] * vc1;
  vsq += p[U3] * vc2; u[U3] = u[RHO] * vc2;
  u[UU] = 0.5 * u[RHO] * vsq + p[UU];
}

// hydro_u_to_p (fluid.c:27-53, ENFORCE_FLOORS off); u is modified as in the reference
__device__ __forceinline__ void u_to_p(double *u, double *p, double gc0, double gc1, double gc2)
{
  p[RHO] = u[RHO];
  u[U1] /= u[RHO]; u[U2] /= u[RHO]; u[U3] /= u[RHO];
  p[U1] = gc0 * u[U1]; p[U2] = gc1 * u[U2]; p[U3] = gc2 * u[U3];
  double vsq = 0.0;
  vsq += u[U1] * p[U1]; vsq += u[U2] * p[U2]; vsq += u[U3] * p[U3];
  p[UU] = u[UU] - 0.5 * p[RHO] * vsq;
}

// dt_source_control (step.c:205-223)
__device__ __forceinline__ double dt_source_control(const double *p, const double *u, const double *s)
{
  const double alpha = 0.02;
  double mdt = 1.0e100, local_dt, momterm = 0.0;
  local_dt = alpha * u[0] / (fabs(s[0]) + 1.0e-16);
  mdt = tmin(mdt, local_dt);
  local_dt = alpha * u[1] / (fabs(s[1]) + 1.0e-16);
  mdt = tmin(mdt, local_dt);
  momterm += p[U1] * s[U1]; momterm += p[U2] * s[U2]; momterm += p[U3] * s[U3];
  local_dt = 100 * alpha * p[UU] / (fabs(fabs(s[1]) - fabs(momterm)) + 1.0e-16);
  mdt = tmin(mdt, local_dt);
  return mdt;
}

// gamma-law / polytrope pressure (eos_gamma.c:7, eos_poly.c:7)
__device__ __forceinline__ double eos_press(int eos, double gam, double Kpoly, double rho, double uu)
{
  return (eos == 0) ? (gam - 1.0) * uu : Kpoly * pow(rho, gam);
}

// Block-wide min of a double, folded into an order-preserving atomic accumulator.
__device__ __forceinline__ void block_min_to(double v, unsigned long long *acc, double *sbuf)
{
  for (int o = 16; o > 0; o >>= 1) v = tmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sbuf[warp] = v;
  __syncthreads();
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    v = (lane < nw) ? sbuf[lane] : 1.0e300;
    for (int o = 16; o > 0; o >>= 1) v = tmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (lane == 0) atomicMin(acc, dbl_to_ord(v));
  }
}

}  // namespace mdg
