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

// Read access to the reconstruction coefficients of one zone (the geometry-only
// sub-expressions of para_recon/lin_recon, field f at p[f*stride]).  Fields are read when
// used, so the 22 coefficients never occupy registers all at once; LDG selects the
// read-only global path (tables in HBM) or plain loads (tables staged in shared memory).
template <typename T, bool LDG>
struct RcView {
  const double *p;
  int64_t stride;
  __device__ __forceinline__ T operator()(int f) const
  {
    return LDG ? T(__ldg(p + f * stride)) : T(p[f * stride]);
  }
};

// para_recon for one zone (reconstruct.c:142-201): am/a0/ap are the zone averages at
// i-1, i, i+1; returns the left (al) and right (ar) face values of zone i.
//
// Control flow is arranged for the SIMT machine without changing any result: the
// extremum test (reconstruct.c:145) only skips the work when every active lane of the
// warp is at an extremum; otherwise all lanes compute and extremum lanes select a[i] at
// the end, so the six variables of a zone run as independent instruction streams.  The
// two "move the zero" cases (reconstruct.c:190-200) share one code path.
template <typename T, typename G>
__device__ __forceinline__ void para_recon_zone(T am_v, T a, T ap_v, const G &g, T &al, T &ar)
{
  T dqm = a - am_v;
  T dqp = ap_v - a;
  const bool flat = (dqm * dqp <= T(0));
  if (__all_sync(__activemask(), flat)) { al = a; ar = a; return; }
  T dqc = ap_v - am_v;
  T A = (dqm * g(RC_BP) * g(RC_GM) * g(RC_G0) + g(RC_GP) * (dqp * g(RC_BM) * g(RC_G0) - dqc * g(RC_B0) * g(RC_GM))) * g(RC_DEN1);
  T B = -(dqm * g(RC_AP) * g(RC_GM) * g(RC_G0) + g(RC_GP) * (dqp * g(RC_AM) * g(RC_G0) - dqc * g(RC_A0) * g(RC_GM))) * g(RC_DEN1);
  T C = a - (g(RC_A0) * A + g(RC_B0) * B) / g(RC_G0);
  const T xl = g(RC_XL), xr = g(RC_XR);
  T l = xl * (A * xl + B) + C;
  T r = xr * (A * xr + B) + C;
  T mean = T(0.75) * am_v + T(0.25) * a;
  T mask = (a - l) * (l - mean);
  l = (mask < T(0)) ? mean : l;
  mean = T(0.75) * ap_v + T(0.25) * a;
  mask = (mean - r) * (r - a);
  r = (mask < T(0)) ? mean : r;
  A = (g(RC_B0) * (r - l) + g(RC_G0) * (a * g(RC_XLR) - r * xl + l * xr)) * g(RC_DEN2);
  B = (g(RC_A0) * (l - r) + g(RC_G0) * (r - a) * g(RC_XL2) + g(RC_G0) * (a - l) * g(RC_XR2)) * g(RC_DEN2);
  T xzero = -B / (T(2) * A + T(1.0e-16));
  if (isinf(xzero) || isnan(xzero)) xzero = T(-1.0e-200);
  const bool inside = !flat && (xzero > xl && xzero < xr);
  if (__any_sync(__activemask(), inside)) {
    // move the zero to the right edge (replace al) or to the left edge (replace ar)
    const bool right = xzero > g(RC_XMID);
    const T e = right ? r : l;
    const T xe = right ? xr : xl;
    const T xo = right ? xl : xr;
    A = g(RC_G0) * (a - e) / (right ? g(RC_DMR) : g(RC_DML));
    B = T(-2.0) * A * xe;
    C = a - (g(RC_A0) * A + g(RC_B0) * B) / g(RC_G0);
    const T val = xo * (A * xo + B) + C;
    if (inside) {
      if (right) l = val;
      else r = val;
    }
  }
  al = flat ? a : l;
  ar = flat ? a : r;
}

// lin_recon for one zone (reconstruct.c:99-121)
template <typename T, typename G>
__device__ __forceinline__ void lin_recon_zone(T am_v, T a, T ap_v, const G &g, T &al, T &ar)
{
  T sm = (a - am_v) / g(RC_LSM);
  T sp = (ap_v - a) / g(RC_LSP);
  if (sm * sp <= T(0)) { al = a; ar = a; return; }
  T sc = (ap_v - am_v) / g(RC_LSC);
  T A = tsign(sc) * tmin(tmin(fabs(sm), fabs(sp)), fabs(sc));
  T B = a - A * g(RC_B0) / g(RC_G0);
  al = A * g(RC_XL) + B;
  ar = A * g(RC_XR) + B;
}

// How the FP64 reconstruction is emitted, chosen per translation unit before this header
// is included (the results are the same either way):
//   MDG_RECON_OUTLINE 1 -- recon_zone calls one out-of-line copy of para_recon/lin_recon
//                          (kernels whose many inlined copies overflow the instruction
//                          cache: the 1-D stage and the 3-D face kernels);
//   MDG_RECON_UNROLL n  -- unroll factor of the loops over the reconstructed variables
//                          (1: one inlined copy per loop, the 2-D split sweep).
#ifndef MDG_RECON_OUTLINE
#define MDG_RECON_OUTLINE 0
#endif
#ifndef MDG_RECON_UNROLL
#define MDG_RECON_UNROLL 8
#endif
constexpr int kReconUnroll = MDG_RECON_UNROLL;
struct FacePair { double al, ar; };
template <typename G>
__device__ __noinline__ FacePair recon_zone_call(int order, double am_v, double a, double ap_v, G g)
{
  FacePair o;
  if (order == 3) para_recon_zone(am_v, a, ap_v, g, o.al, o.ar);
  else if (order == 2) lin_recon_zone(am_v, a, ap_v, g, o.al, o.ar);
  else { o.al = a; o.ar = a; }
  return o;
}

template <typename T, typename G>
__device__ __forceinline__ void recon_zone(int order, T am_v, T a, T ap_v, const G &g, T &al, T &ar)
{
  if (MDG_RECON_OUTLINE && sizeof(T) == 8) {
    const FacePair o = recon_zone_call<G>(order, am_v, a, ap_v, g);
    al = o.al;
    ar = o.ar;
    return;
  }
  if (order == 3) para_recon_zone(am_v, a, ap_v, g, al, ar);
  else if (order == 2) lin_recon_zone(am_v, a, ap_v, g, al, ar);
  else { al = a; ar = a; }
}

// Geometry of one face as the Riemann solver sees it (zone_geom at the face's cell).
template <typename T>
struct FaceGeom { T area, scale; T g0, g1, g2; };

// Metric factors: with UNIT (Cartesian grids: gcov = scale = 1) the multiplications and
// divisions by 1.0 are dropped; x*1.0 == x and x/1.0 == x exactly, so results are unchanged.
template <bool UNIT, typename T> __device__ __forceinline__ T gmul(T g, T x) { return UNIT ? x : g * x; }
template <bool UNIT, typename T> __device__ __forceinline__ T gdiv(T x, T s) { return UNIT ? x : x / s; }

// Adiabatic-index constants of the wave-speed estimate.  Every cell carries Gamma = gam
// (gamma-law and polytrope), so these sub-expressions of riemann.c are constants;
// computed here with the reference's own operation order they are bit-identical.
template <typename T>
struct GamConst {
  T g;      // Gamma
  T cq;     // (Gamma+1)/(2 Gamma)        riemann.c:389-390
  T gp1;    // Gamma+1                    riemann.c:413-414
  T cb;     // (Gamma-1)/(Gamma+1)        riemann.c:415-416
  T ce;     // (Gamma_avg-1)/(2 Gamma_avg), Gamma_avg = 0.5(Gamma+Gamma) = Gamma   riemann.c:400
  T gm1;    // Gamma-1
  T cx;     // 2 Gamma/(Gamma-1)          riemann.c:402
};
template <typename T>
__device__ __forceinline__ GamConst<T> gam_const(T G)
{
  GamConst<T> c;
  T Gavg = T(0.5) * (G + G);
  c.g = G;
  c.cq = (G + T(1)) / (T(2) * G);
  c.gp1 = G + T(1);
  c.cb = (G - T(1)) / (G + T(1));
  c.ce = (Gavg - T(1)) / (T(2) * Gavg);
  c.gm1 = G - T(1);
  c.cx = T(2) * G / (G - T(1));
  return c;
}

// Wave-speed estimate shared by HLLC and HLLE (riemann.c:368-429 / 210-303).
// w[0..4] primitives, w[5] pressure (w[6], Gamma, equals gc.g).
template <typename T>
__device__ __forceinline__ void wave_speeds(const T *pl, const T *pr, T u_l, T u_r, bool hlle,
                                            const GamConst<T> &gc, T &sl, T &sr, T &ss, T &p_s, int &isshock)
{
  const T p_l = pl[5], p_r = pr[5], G = gc.g;
  T cs_l = sqrt(G * p_l / pl[RHO]);
  T cs_r = sqrt(G * p_r / pr[RHO]);
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
    T plr = pow(p_l / p_r, gc.ce);
    T s0 = (plr * u_l / cs_l + u_r / cs_r + T(2) * (plr - T(1)) / gc.gm1) / (plr / cs_l + T(1) / cs_r);
    p_s = T(0.5) * (p_l * pow(T(1) + gc.gm1 / (T(2) * cs_l) * (u_l - s0), gc.cx)
                  + p_r * pow(T(1) + gc.gm1 / (T(2) * cs_r) * (s0 - u_r), gc.cx));
    p_s = tmax(p_s, T(0));
  } else {
    // two shocks (Toro 9.42-9.43)
    T a_l = T(2) / (gc.gp1 * pl[RHO]);
    T a_r = T(2) / (gc.gp1 * pr[RHO]);
    T b_l = gc.cb * p_l;
    T b_r = gc.cb * p_r;
    T g_l = sqrt(a_l / (p_s + b_l));
    T g_r = sqrt(a_r / (p_s + b_r));
    p_s = (g_l * p_l + g_r * p_r - (u_r - u_l)) / (g_l + g_r);
    p_s = tmax(p_s, T(0));
  }
  // q = 1 when p_s <= p, else sqrt(1 + (G+1)/(2G) (p_s/p - 1)); sqrt(1) == 1 exactly, so
  // the square root is taken unconditionally on the selected argument (no branch)
  T q_l = sqrt((p_s <= p_l) ? T(1) : T(1) + gc.cq * (p_s / p_l - T(1)));
  T q_r = sqrt((p_s <= p_r) ? T(1) : T(1) + gc.cq * (p_s / p_r - T(1)));
  sl = u_l - cs_l * q_l;
  sr = u_r + cs_r * q_r;
  ss = (p_r - p_l + pl[RHO] * u_l * (sl - u_l) - pr[RHO] * u_r * (sr - u_r))
     / (pl[RHO] * (sl - u_l) - pr[RHO] * (sr - u_r));
}

// p_uflux (riemann.c:4-37) for direction DIR
template <int DIR, bool UNIT, typename T>
__device__ __forceinline__ void p_uflux(const T *p, const FaceGeom<T> &g, T press, T *u, T *f)
{
  T vc0 = gmul<UNIT>(g.g0, p[U1]), vc1 = gmul<UNIT>(g.g1, p[U2]), vc2 = gmul<UNIT>(g.g2, p[U3]);
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
template <int DIR, bool UNIT, typename T>
__device__ __forceinline__ void pflux(const T *p, T press, const FaceGeom<T> &g, T *f)
{
  T vc0 = gmul<UNIT>(g.g0, p[U1]), vc1 = gmul<UNIT>(g.g1, p[U2]), vc2 = gmul<UNIT>(g.g2, p[U3]);
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
template <int DIR, bool UNIT, typename T>
__device__ __forceinline__ int riemann_hllc(const T *pl, const T *pr, const FaceGeom<T> &g, const GamConst<T> &gc,
                                            T *flux, T &sig)
{
  int isshock = 0;
  if (g.area < T(1.0e-16)) {
    sig = T(1.0e-200);
#pragma unroll
    for (int v = 0; v < NPRIM; v++) flux[v] = T(0);
    return isshock;
  }
  const T sc = g.scale;
  T u_l = gmul<UNIT>(sc, pl[U1 + DIR]);
  T u_r = gmul<UNIT>(sc, pr[U1 + DIR]);
  T sl, sr, ss, p_s;
  wave_speeds<T>(pl, pr, u_l, u_r, false, gc, sl, sr, ss, p_s, isshock);
  if (ss > sr) sr = T(1.001) * ss;
  if (ss < sl) sl = T(1.001) * ss;
  sig = gdiv<UNIT>(tmax(fabs(sl), fabs(sr)), sc);
  if (sl > T(0)) { pflux<DIR, UNIT, T>(pl, pl[5], g, flux); return isshock; }
  if (sr < T(0)) { pflux<DIR, UNIT, T>(pr, pr[5], g, flux); return isshock; }
  // Star state of the upwind side k (k = left if ss > 0, riemann.c:453-491).  The
  // right-side formula of the reference, (E(u_r - s_r) + p_r u_r - p_s ss)/(ss - s_r), is
  // the left-side formula with every sum and difference negated; round-to-nearest is
  // symmetric under negation, so one code path gives bit-identical results for both sides.
  T u[NPRIM], fx[NPRIM], Us[NPRIM], pk[6];
  const bool left = ss > T(0);
#pragma unroll
  for (int v = 0; v < 6; v++) pk[v] = left ? pl[v] : pr[v];
  const T sk = left ? sl : sr;
  const T uk = left ? u_l : u_r;
  p_uflux<DIR, UNIT, T>(pk, g, pk[5], u, fx);
  Us[0] = pk[RHO] * (sk - uk) / (sk - ss);
  Us[UU] = (u[UU] * (sk - uk) - pk[5] * uk + p_s * ss) / (sk - ss);
  Us[U1] = pk[U1]; Us[U2] = pk[U2]; Us[U3] = pk[U3];
  Us[U1 + DIR] = gdiv<UNIT>(ss, sc);
  const T slr = gdiv<UNIT>(sk, sc);
  T vc0 = gmul<UNIT>(g.g0, Us[U1]), vc1 = gmul<UNIT>(g.g1, Us[U2]), vc2 = gmul<UNIT>(g.g2, Us[U3]);
  Us[U1] = vc0 * Us[0]; Us[U2] = vc1 * Us[0]; Us[U3] = vc2 * Us[0];
#pragma unroll
  for (int v = 0; v < NPRIM; v++) flux[v] = g.area * (fx[v] + slr * (Us[v] - u[v]));
  return isshock;
}

// riemann_flux_HLLE (riemann.c:178-325)
template <int DIR, bool UNIT, typename T>
__device__ __forceinline__ void riemann_hlle(const T *pl, const T *pr, const FaceGeom<T> &g, const GamConst<T> &gc,
                                             T *flux, T &sig)
{
  if (g.area < T(1.0e-16)) {
    sig = T(1.0e-200);
#pragma unroll
    for (int v = 0; v < NPRIM; v++) flux[v] = T(0);
    return;
  }
  const T sc = g.scale;
  T u_l = gmul<UNIT>(sc, pl[U1 + DIR]);
  T u_r = gmul<UNIT>(sc, pr[U1 + DIR]);
  T sl, sr, ss, p_s;
  int isshock;
  wave_speeds<T>(pl, pr, u_l, u_r, true, gc, sl, sr, ss, p_s, isshock);
  T ul[NPRIM], ur[NPRIM], fl[NPRIM], fr[NPRIM];
  p_uflux<DIR, UNIT, T>(pl, g, pl[5], ul, fl);
  p_uflux<DIR, UNIT, T>(pr, g, pr[5], ur, fr);
  T cmax = tmax(gdiv<UNIT>(sr, sc), T(0));
  T cmin = fabs(tmin(gdiv<UNIT>(sl, sc), T(0)));
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

// hydro_u_to_p (fluid.c:27-53); u is modified as in the reference.  With floors (the
// ENFORCE_FLOORS build, fluid.c:43-46) density and internal energy are clamped from below
// with the reference's MAX (decs.h:628) after the velocities are formed.
__device__ __forceinline__ void u_to_p(double *u, double *p, double gc0, double gc1, double gc2,
                                       bool floors = false, double rho_floor = 0.0, double e_floor = 0.0)
{
  p[RHO] = u[RHO];
  u[U1] /= u[RHO]; u[U2] /= u[RHO]; u[U3] /= u[RHO];
  p[U1] = gc0 * u[U1]; p[U2] = gc1 * u[U2]; p[U3] = gc2 * u[U3];
  double vsq = 0.0;
  vsq += u[U1] * p[U1]; vsq += u[U2] * p[U2]; vsq += u[U3] * p[U3];
  p[UU] = u[UU] - 0.5 * p[RHO] * vsq;
  if (floors) {
    p[RHO] = (p[RHO] > rho_floor) ? p[RHO] : rho_floor;
    p[UU] = (p[UU] > e_floor) ? p[UU] : e_floor;
  }
}

// A non-finite updated state marks its problem (ProbTime::err, reported by
// mdg_synchronize and the server's results); the values themselves are left as computed.
__device__ __forceinline__ void flag_nonfinite(const double *pf, ProbTime *T)
{
  bool bad = false;
#pragma unroll
  for (int v = 0; v < NPRIM; v++) bad = bad || !isfinite(pf[v]);
  if (bad) T->err = MDG_ERR_NONFINITE;
}

// Gravitational constant of constants.h:3 (cgs).
constexpr double GNEWT = 6.67384e-8;

// The monopole gravity sources of a zone (monopole_gravity_finish, gravity.c:389-407):
// momentum rho g, and energy g times the mass flux density interpolated linearly in x
// from the inner face (vl) to the outer face(s) (vr) to the zone centroid beta0/Gamma0.
__device__ __forceinline__ void add_monopole_gravity(double rho, double g, double vl, double vr, double x0l,
                                                     double dx0, double b0, double g0, double *src)
{
  const double A = (vr - vl) / dx0;
  const double B = vl - A * x0l;
  src[U1] += rho * g;
  src[UU] += (A * b0 / g0 + B) * g;
}

// One step of the edge-to-centroid interpolation of the monopole acceleration
// (gravity.c:302-319): zone ii between edges with accelerations gl, gr.
__device__ __forceinline__ double monopole_centroid(double gl, double gr, double x0l, double dx0, double b0, double g0)
{
  const double A = (gr - gl) / dx0;
  const double B = gl - A * x0l;
  return A * b0 / g0 + B;
}

// fixed_gravity (gravity.c:38-64) added to the sources of a zone: src[ETOT] += rho
// geom_dot(v, g0, gcov) (geometry.c:65-73, over all three components) and
// src[P1+d] += rho g0[d] gcov[d] for the grid's directions d < ndim.
__device__ __forceinline__ void add_fixed_gravity(const double *p, const double *g, double gc0, double gc1,
                                                  double gc2, int ndim, double *src)
{
  double vsq = 0.0;
  vsq += p[U1] * g[0] * gc0;
  vsq += p[U2] * g[1] * gc1;
  vsq += p[U3] * g[2] * gc2;
  src[UU] += p[RHO] * vsq;
  src[U1] += p[RHO] * g[0] * gc0;
  if (ndim > 1) src[U2] += p[RHO] * g[1] * gc1;
  if (ndim > 2) src[U3] += p[RHO] * g[2] * gc2;
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

// The CFL reduction without a division per term.  Correctly rounded division is
// monotone, so for a fixed c > 0:  min_k fl(x_k / c) == fl(min_k x_k / c)  and, for
// y_k >= 0,  min_k fl(c / y_k) == fl(c / max_k y_k).  The face terms dx/|sig| and the zone
// terms 1/local_dt are therefore reduced as maxima of their denominators, and with zero
// source terms (Cartesian grids) dt_source_control's three terms share the denominator
// |0| + 1e-16 and are reduced on their numerators.  The results are bit-identical.
__device__ __forceinline__ double src_dt_numerator_min(const double *p, const double *u)
{
  const double alpha = 0.02;
  double m = alpha * u[0];
  m = tmin(m, alpha * u[1]);
  m = tmin(m, 100 * alpha * p[UU]);
  return m;
}
// dt_source_control's minimum over zones with zero sources, from the numerator minimum
__device__ __forceinline__ double src_dt_from_numerator(double nmin)
{
  return tmin(1.0e100, nmin / (fabs(0.0) + 1.0e-16));
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
