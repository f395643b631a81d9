// Mixed-precision batched 1-D RK stage kernel.
//
// The batched ensemble path: many independent 1-D problems of different sizes advance
// together, one launch per RK stage.  In persistent mode the grid is a fixed number of
// CTAs (chosen by the autotuner) that pull (problem, tile) work items from a device work
// queue (an atomic counter over the tile list, whose length is read from device memory,
// so a captured CUDA graph serves any batch composition); otherwise CTA b takes tile b.
//
// Precision split:
//  * FP32: reconstruction and limiting (para_recon on the differences dqm, dqp with the
//    geometry folded into FP64-computed weights, MixField), the wave speeds and the
//    star-state increments U* - U of the HLLC solver (faces where FP32 cannot resolve
//    the internal energy of the colder side are re-solved in FP64, MIX_COND_MAX);
//  * FP64: the state, the face states a + da, the upwind physical flux, area and volume
//    factors, the geometric source terms, the conserved-variable update and the dt
//    reduction.
// Each FP64 face flux is used once with each sign, so the flux differences conserve mass
// and energy to FP64 round-off.
//
// This translation unit is compiled with fast FP32 math (approximate FP32 division and
// square root); FP64 division and square root stay IEEE.
#include "mdg_hydro.cuh"
#include "mdg_kernels.cuh"
#include "mdg_load1d.cuh"
#include "mdg_mixed.cuh"

namespace mdg {

// FP64 re-solve of an ill-conditioned face (MIX_COND_MAX), out of line so that its
// register demand does not raise the common path's.  c = &sv[0][k] holds the stencil of
// the face (zones z-2 .. z+1 at c[v*cs + 0..3]); both face states are reconstructed in FP64
// (right face of zone z-1, left face of zone z; reconstruct.c:142-201), the FP64 solver
// writes flux[v * fs] and the signal speed is returned.
__device__ __noinline__ float face_fp64(const double *c, int cs, const double *rc_zm, const double *rc_z,
                                        int64_t rcs, double gam, double area, double scale, double g0,
                                        double g1, double g2, double *flux, int fs)
{
  double xs[12];
  const RcView<double, true> gm{rc_zm, rcs};
  const RcView<double, true> gz{rc_z, rcs};
#pragma unroll 1
  for (int v = 0; v < 6; v++) {
    const double *q = c + v * cs;
    double lo, hi;
    para_recon_zone<double>(q[0], q[1], q[2], gm, lo, hi);
    xs[v] = hi;
    para_recon_zone<double>(q[1], q[2], q[3], gz, lo, hi);
    xs[6 + v] = lo;
  }
  FaceGeom<double> fg;
  fg.area = area; fg.scale = scale; fg.g0 = g0; fg.g1 = g1; fg.g2 = g2;
  double f[NPRIM], sig64;
  riemann_hllc<0, false, double>(xs, xs + 6, fg, gam_const<double>(gam), f, sig64);
#pragma unroll
  for (int v = 0; v < NPRIM; v++) flux[v * fs] = f[v];
  return (float)sig64;
}

// 1-D geometry in closed form, in FP64.  On the uniform-radius spherical grid (r = x,
// dr/dx = 1) every quantity of metric_spherical_general.c is a polynomial integral over the
// zone's edge radii a < b times an angular constant (ProbDev::gk_*); written with the
// factor h = b - a taken out, nothing cancels as r -> 0 or at large r.  This replaces the
// 320 bytes of geometry tables per zone that the FP64 sweep reads (it must reproduce the
// reference's Romberg values bit for bit; these agree with them to ~1e-15).
//   face at x: area = x^2 vthf dph, gcov = (1, x^2 th1, x^2 th2), scale = 1   (745-779, 941-1051)
//   zone:      vol = int r^2 dr vthf dph; gcov = (1, F th1, F th2), F = (b^5 - a^5)/(5 int r^2 dr)
//              conn[1][0][1] = conn[1][1][0] = conn[2][0][2] = conn[2][2][0] = int r dr / int r^2 dr,
//              conn[0][1][1] = -(int r^3 dr / int r^2 dr) th1, conn[2][1][2] = conn[2][2][1] = tc,
//              conn[0][2][2] = -conn[2][2][0] gcov[2], conn[1][2][2] = -tc gcov[2]/gcov[1]   (820-930)
// Cartesian: unit metric, area 1, volume dx, no connection.  Problems on a non-uniform
// coordinate map (SINH, SINH_MODIFIED or LOG radius, POLYTH theta; ProbDev::geo_tab) read
// the reference's Romberg geometry tables instead, with the FP64 source routine of the
// plain sweep.
__device__ __forceinline__ FaceGeom<double> face_geom_1d(const ProbDev &P, int zf)
{
  FaceGeom<double> g;
  g.scale = 1.0;
  g.g0 = 1.0;
  if (P.has_src) {
    const double x = P.x0 + zf * P.dx0;
    const double x2 = x * x;
    g.area = x2 * P.gk_area;
    g.g1 = x2 * P.gk_th1;
    g.g2 = x2 * P.gk_th2;
  } else {
    g.area = 1.0;
    g.g1 = 1.0;
    g.g2 = 1.0;
  }
  return g;
}

struct ZoneGeo1 { double vol, g1, g2, gc1, gc2, c101, c011, c022, c122; };

__device__ __forceinline__ ZoneGeo1 zone_geom_1d(const ProbDev &P, int z)
{
  ZoneGeo1 q;
  if (P.has_src) {
    const double a = P.x0 + z * P.dx0, b = P.x0 + (z + 1) * P.dx0, h = b - a;
    const double a2 = a * a, b2 = b * b;
    const double vr = h * (b2 + a * b + a2) * (1.0 / 3.0);
    const double ivr = 1.0 / vr;
    const double F = 0.2 * h * (b2 * b2 + b2 * b * a + b2 * a2 + b * a2 * a + a2 * a2) * ivr;
    q.vol = vr * P.gk_area;
    q.g1 = F * P.gk_th1;
    q.g2 = F * P.gk_th2;
    q.gc1 = (q.g1 > 1.0e-50) ? 1.0 / q.g1 : 0.0;
    q.gc2 = (q.g2 > 1.0e-50) ? 1.0 / q.g2 : 0.0;
    q.c101 = 0.5 * h * (a + b) * ivr;
    q.c011 = -(0.25 * h * (a + b) * (a2 + b2) * ivr) * P.gk_th1;
    q.c022 = -q.c101 * q.g2;
    q.c122 = -P.gk_tc * q.g2 * q.gc1;
  } else {
    q.vol = P.dx0;
    q.g1 = q.g2 = q.gc1 = q.gc2 = 1.0;
    q.c101 = q.c011 = q.c022 = q.c122 = 0.0;
  }
  return q;
}

// Geometric source terms (rad_fluid.c:164-192, fluid.c:56-73) with the connection above:
// src[U1+m] = sum over l, n of T[l][n] conn[l][m][n], T[l][m] = rho v^m v_l + p delta_lm.
__device__ __forceinline__ void geo_sources_closed(const ProbDev &P, const ZoneGeo1 &q, const double *ph,
                                                   double press, double *src)
{
  const double vcov[3] = {ph[U1], q.g1 * ph[U2], q.g2 * ph[U3]};
  double T[3][3];
#pragma unroll
  for (int l = 0; l < 3; l++) {
#pragma unroll
    for (int m = 0; m < 3; m++) T[l][m] = ph[RHO] * ph[U1 + m] * vcov[l];
    T[l][l] += press;
  }
  src[RHO] = 0.0;
  src[UU] = 0.0;
  src[U1] = (T[1][1] + T[2][2]) * q.c101;
  src[U2] = T[0][1] * q.c011 + T[1][0] * q.c101 + T[2][2] * P.gk_tc;
  src[U3] = T[0][2] * q.c022 + T[1][2] * q.c122 + T[2][0] * q.c101 + T[2][1] * P.gk_tc;
}

// dt_source_control (step.c:205-223) with one division: the three ratios a_k/b_k have
// positive denominators, so the smallest is selected by cross-multiplication.
__device__ __forceinline__ double dt_source_control_1div(const double *p, const double *u, const double *s)
{
  const double alpha = 0.02;
  double num = alpha * u[0], den = fabs(s[0]) + 1.0e-16;
  const double n1 = alpha * u[1], d1 = fabs(s[1]) + 1.0e-16;
  if (n1 * den < num * d1) { num = n1; den = d1; }
  const double momterm = p[U1] * s[U1] + p[U2] * s[U2] + p[U3] * s[U3];
  const double n2 = 100 * alpha * p[UU], d2 = fabs(fabs(s[1]) - fabs(momterm)) + 1.0e-16;
  if (n2 * den < num * d2) { num = n2; den = d2; }
  return fmin(1.0e100, num / den);
}

// Face geometry of a problem on a non-uniform coordinate map (the Romberg tables).
__device__ __forceinline__ FaceGeom<double> face_geom_tab(const double *geo, int64_t gs, int64_t gi)
{
  FaceGeom<double> fg;
  fg.area = __ldg(geo + GF_AREA * gs + gi);
  fg.scale = __ldg(geo + GF_FSCALE * gs + gi);
  fg.g0 = __ldg(geo + GF_FG0 * gs + gi);
  fg.g1 = __ldg(geo + GF_FG1 * gs + gi);
  fg.g2 = __ldg(geo + GF_FG2 * gs + gi);
  return fg;
}

// push() of zone z (thread t of the tile) for a problem that reads the Romberg tables (a
// non-uniform coordinate map, or monopole gravity): the zone geometry and connection of
// the tables with the FP64 source routine of the plain sweep, fixed or monopole gravity,
// the update, u -> p and the next-dt zone term.  sv and sfl are the kernel's shared
// pencil ([6][NT+2]) and face fluxes ([NPRIM][NT]).  Returns (source dt limit, zone term).
template <int STAGE, int NT>
__device__ __forceinline__ double2 push_zone_tab(const ProbDev &P, const Tables &tb, int z, int t, double dt,
                                              const double *sv, const double *sfl, StateSoA sn, StateSoA out,
                                              int64_t cell, ProbTime *tm)
{
  const int64_t gs = tb.geo_stride, rcs = tb.rc0_stride;
  const int64_t gi = P.geo_off + z + NG;
  const double *geo = tb.geo;
  double ph[NPRIM], pn[NPRIM], u[NPRIM], uh[NPRIM], src[NPRIM];
#pragma unroll
  for (int v = 0; v < NPRIM; v++) ph[v] = sv[v * (NT + 2) + t + 1];
  const double press = sv[5 * (NT + 2) + t + 1];
#pragma unroll
  for (int v = 0; v < NPRIM; v++) pn[v] = STAGE ? sn.v[v][cell] : ph[v];
  const double vol = __ldg(geo + GF_VOL * gs + gi);
  const double g0 = __ldg(geo + GF_G0 * gs + gi), g1 = __ldg(geo + GF_G1 * gs + gi), g2 = __ldg(geo + GF_G2 * gs + gi);
  const double gc0 = __ldg(geo + GF_GC0 * gs + gi), gc1 = __ldg(geo + GF_GC1 * gs + gi);
  const double gc2 = __ldg(geo + GF_GC2 * gs + gi), s00 = __ldg(geo + GF_S00 * gs + gi);
  if (P.has_src) {
    geo_sources_1d(geo, gs, gi, P.sparse_conn != 0, ph, press, g0, g1, g2, src);
  } else {
#pragma unroll
    for (int v = 0; v < NPRIM; v++) src[v] = 0.0;
  }
  if (P.grav_on) add_fixed_gravity(ph, P.grav, g0, g1, g2, 1, src);
  if (P.mono) {
    // monopole gravity (gravity.c:373-401) with the mass flux densities of the zone's
    // FP64 face fluxes
    const double vr = sfl[RHO * NT + t + 1] / (__ldg(geo + GF_AREA * gs + gi + 1) + 1.0e-16);
    const double vl = sfl[RHO * NT + t] / (__ldg(geo + GF_AREA * gs + gi) + 1.0e-16);
    add_monopole_gravity(ph[RHO], tb.gmono[P.mono_off + z], vl, vr, P.x0 + z * P.dx0, P.dx0,
                         __ldg(tb.rc0 + RC_B0 * rcs + gi), __ldg(tb.rc0 + RC_G0 * rcs + gi), src);
  }
  p_to_u(pn, u, g0, g1, g2);
  p_to_u(ph, uh, g0, g1, g2);
  double lmin = dt_source_control_1div(pn, u, src), lmax = 0.0;
  const double ivol = 1.0 / vol;
  const double pfact = STAGE ? 0.5 : 1.0, phfact = STAGE ? 0.5 : 0.0, ffact = STAGE ? 0.5 : 1.0;
#pragma unroll
  for (int v = 0; v < NPRIM; v++) {
    const double ddt = (sfl[v * NT + t + 1] - sfl[v * NT + t]) * ivol - src[v];
    u[v] = pfact * u[v] + phfact * uh[v] - ffact * dt * ddt;
  }
  double pf[NPRIM];
  const double irho = 1.0 / u[RHO];
  const double w1 = u[U1] * irho, w2 = u[U2] * irho, w3 = u[U3] * irho;
  pf[RHO] = u[RHO];
  pf[U1] = gc0 * w1;
  pf[U2] = gc1 * w2;
  pf[U3] = gc2 * w3;
  pf[UU] = u[UU] - 0.5 * pf[RHO] * (w1 * pf[U1] + w2 * pf[U2] + w3 * pf[U3]);
  if (P.floors) {
    pf[RHO] = fmax(pf[RHO], P.rho_floor);
    pf[UU] = fmax(pf[UU], P.e_floor);
  }
#pragma unroll
  for (int v = 0; v < NPRIM; v++) out.v[v][cell] = pf[v];
  flag_nonfinite(pf, tm);
  if (STAGE == 1) {
    const double cs = sqrt(P.gam * press / ph[RHO]);
    lmax = (fabs(pf[U1]) + cs / s00) / P.dx0;
  }
  return make_double2(lmin, lmax);
}

// Resident 64-thread-equivalents per SM the register allocation is bounded for (0: none).
// The kernel waits mostly on global loads (state pencils, FP32 weights), so occupancy
// pays: on the 2048-problem ensemble 16 x 64 threads per SM (64 registers, a few spilled
// bytes) ran 1.18x faster than 12 x 64 (80 registers) and 1.41x faster than the unbounded
// 114-register build (8 x 64); 20 x 64 (48 registers) was slower again (spills).
#ifndef MDG_MIX_MINB64
#define MDG_MIX_MINB64 16
#endif

// TAB: the launch's problems read the Romberg tables (ProbDev::geo_tab: a non-uniform
// coordinate map or monopole gravity); the solver and the server put their tiles in a
// list of their own, so the closed-form instantiation carries none of that code.
template <int NT, int STAGE, bool TAB>
__global__ void __launch_bounds__(NT, MDG_MIX_MINB64 * 64 / NT)
stage1d_mixed_kernel(const ProbDev *__restrict__ probs, ProbTime *__restrict__ times,
                     const Tile *__restrict__ tiles, WorkQueue *__restrict__ q, bool use_queue,
                     Tables tb, StateSoA sst, StateSoA sn, StateSoA out)
{
  __shared__ double sv[6][NT + 2];     // stage-state pencil: 5 primitives + pressure
  // FP32 right-face offset of each reconstructed zone (face value = zone average + offset,
  // formed in FP64 by the reader: half the shared memory of storing the FP64 face values,
  // which leaves more of the SM's L1 to the register spills)
  __shared__ float sdr[6][NT];
  __shared__ double sfl[NPRIM][NT];    // face fluxes
  __shared__ double sred[32];
  __shared__ int s_item;
  const int t = threadIdx.x;
  const double *rc = tb.rc0;
  const int64_t rcs = tb.rc0_stride;
  const int64_t gs = tb.geo_stride;
  const int ntiles = q->ntiles;

  int item;
  if (use_queue) {
    // the other stage's counter is idle while this kernel runs: reset it for its next launch
    if (blockIdx.x == 0 && t == 0) q->head[1 - STAGE] = 0u;
    if (t == 0) s_item = (int)atomicAdd(&q->head[STAGE], 1u);
    __syncthreads();
    item = s_item;
  } else {
    item = blockIdx.x;
  }

  while (item < ntiles) {
    const Tile tile = tiles[item];
    if (times[tile.prob].done) {       // past tmax: the time loop has ended (CTA-uniform)
      if (!use_queue) break;
      __syncthreads();                  // every thread has read the current s_item
      if (t == 0) s_item = (int)atomicAdd(&q->head[STAGE], 1u);
      __syncthreads();
      item = s_item;
      continue;
    }
    const ProbDev &P = probs[tile.prob];
    const double dt = times[tile.prob].dt;
    const double t_bc = STAGE ? times[tile.prob].t_bc1 : times[tile.prob].t;
    const int n1 = P.n1;
    const int z = tile.i0 - 1 + t;
    {
      double w[6];
      load_cell_1d(P, sst, rc, rcs, z, t_bc, w);
#pragma unroll
      for (int v = 0; v < 6; v++) sv[v][t + 1] = w[v];
      if (t == 0) {
        load_cell_1d(P, sst, rc, rcs, tile.i0 - 2, t_bc, w);
#pragma unroll
        for (int v = 0; v < 6; v++) sv[v][0] = w[v];
      }
      if (t == NT - 1) {
        load_cell_1d(P, sst, rc, rcs, tile.i0 + NT - 1, t_bc, w);
#pragma unroll
        for (int v = 0; v < 6; v++) sv[v][NT + 1] = w[v];
      }
    }
    __syncthreads();
    // fetch the next work item while this one is processed (read after later barriers)
    if (use_queue && t == 0) s_item = (int)atomicAdd(&q->head[STAGE], 1u);

    // FP32 reconstruction of zone z; FP64 face values a + da
    double al[6];
    {
      const int zc = z < -1 ? -1 : (z > n1 ? n1 : z);
      const MixW w = load_mixw(tb.mx + P.geo_off + zc + NG, gs);
#pragma unroll
      for (int v = 0; v < 6; v++) {
        const double a = sv[v][t + 1];
        float dl, dr;
        mixed_recon((float)(a - sv[v][t]), (float)(sv[v][t + 2] - a), w, dl, dr);
        al[v] = a + (double)dl;
        sdr[v][t] = dr;
      }
    }
    __syncthreads();

    double lmin = 1.0e300, lmax = 0.0;
    float smax = 0.0f;
    if (t >= 1) {
      double pl[6], flux[NPRIM];
      float sig;
#pragma unroll
      for (int v = 0; v < 6; v++) pl[v] = sv[v][t] + (double)sdr[v][t - 1];   // zone z-1: average sv[v][t]
      const int zf = z < 0 ? 0 : (z > n1 ? n1 : z);
      const FaceGeom<double> fg = TAB ? face_geom_tab(tb.geo, gs, P.geo_off + zf + NG) : face_geom_1d(P, zf);
      const GamConst<float> gc = gam_const<float>((float)P.gam);
      int isshock_unused;
      if (riemann_hllc_mixed<0>(pl, al, fg, gc, flux, sig, isshock_unused)) {
#pragma unroll
        for (int v = 0; v < NPRIM; v++) sfl[v][t] = flux[v];
      } else {
        const int zm = z - 1 < -1 ? -1 : (z - 1 > n1 ? n1 : z - 1);
        const int zc = z < -1 ? -1 : (z > n1 ? n1 : z);
        sig = face_fp64(&sv[0][t - 1], NT + 2, rc + P.geo_off + zm + NG, rc + P.geo_off + zc + NG, rcs, P.gam,
                        fg.area, fg.scale, fg.g0, fg.g1, fg.g2, &sfl[0][t], NT);
      }
      if (z >= 0 && z <= n1) smax = fmaxf(smax, sig);
    }
    __syncthreads();

    // push() for zone z in FP64 (step.c:380-470)
    if (t >= 1 && t <= NT - 2 && z >= 0 && z < n1) {
      const int64_t cell = P.cell_off + z;
      if (TAB) {
        const double2 r = push_zone_tab<STAGE, NT>(P, tb, z, t, dt, &sv[0][0], &sfl[0][0], sn, out, cell,
                                                   &times[tile.prob]);
        lmin = r.x;
        lmax = r.y;
      } else {
        // the uniform maps: gcov[0][0] = gcon[0] = scale[0][0] = 1
        double ph[NPRIM], pn[NPRIM], u[NPRIM], uh[NPRIM], src[NPRIM];
  #pragma unroll
        for (int v = 0; v < NPRIM; v++) ph[v] = sv[v][t + 1];
        if (STAGE == 0) {
  #pragma unroll
          for (int v = 0; v < NPRIM; v++) pn[v] = ph[v];
        } else {
  #pragma unroll
          for (int v = 0; v < NPRIM; v++) pn[v] = sn.v[v][cell];
        }
        const ZoneGeo1 zg = zone_geom_1d(P, z);
        if (P.has_src) {
          geo_sources_closed(P, zg, ph, sv[5][t + 1], src);
        } else {
  #pragma unroll
          for (int v = 0; v < NPRIM; v++) src[v] = 0.0;
        }
        if (P.grav_on) add_fixed_gravity(ph, P.grav, 1.0, zg.g1, zg.g2, 1, src);
        p_to_u(pn, u, 1.0, zg.g1, zg.g2);
        p_to_u(ph, uh, 1.0, zg.g1, zg.g2);
        lmin = dt_source_control_1div(pn, u, src);
        const double ivol = 1.0 / zg.vol;
        const double pfact = STAGE ? 0.5 : 1.0, phfact = STAGE ? 0.5 : 0.0, ffact = STAGE ? 0.5 : 1.0;
  #pragma unroll
        for (int v = 0; v < NPRIM; v++) {
          const double ddt = (sfl[v][t + 1] - sfl[v][t]) * ivol - src[v];
          u[v] = pfact * u[v] + phfact * uh[v] - ffact * dt * ddt;
        }
        // hydro_u_to_p (fluid.c:27-53) with one division
        double pf[NPRIM];
        const double irho = 1.0 / u[RHO];
        const double w1 = u[U1] * irho, w2 = u[U2] * irho, w3 = u[U3] * irho;
        pf[RHO] = u[RHO];
        pf[U1] = w1;
        pf[U2] = zg.gc1 * w2;
        pf[U3] = zg.gc2 * w3;
        pf[UU] = u[UU] - 0.5 * pf[RHO] * (w1 * pf[U1] + w2 * pf[U2] + w3 * pf[U3]);
        if (P.floors) {   // ENFORCE_FLOORS, fluid.c:43-46
          pf[RHO] = fmax(pf[RHO], P.rho_floor);
          pf[UU] = fmax(pf[UU], P.e_floor);
        }
  #pragma unroll
        for (int v = 0; v < NPRIM; v++) out.v[v][cell] = pf[v];
        flag_nonfinite(pf, &times[tile.prob]);
        if (STAGE == 1) {
          // zone term of the next estimate_dt (step.c:177-187)
          const double cs = sqrt(P.gam * sv[5][t + 1] / ph[RHO]);
          lmax = (fabs(pf[U1]) + cs) / P.dx0;
        }
      }
    }
    lmin = fmin(lmin, P.dx0 / (double)smax);
    if (STAGE == 1) lmin = fmin(lmin, 1.0 / lmax);
    block_min_to(lmin, &times[tile.prob].minacc, sred);
    if (!use_queue) break;
    __syncthreads();
    item = s_item;
  }
}

template <int NT, bool TAB>
static void launch_mixed_nt(int stage, int grid, bool use_queue, const ProbDev *probs, ProbTime *times,
                            const Tile *tiles, WorkQueue *q, const Tables &tb, StateSoA sst, StateSoA sn,
                            StateSoA out, cudaStream_t st)
{
  if (stage == 0)
    stage1d_mixed_kernel<NT, 0, TAB><<<grid, NT, 0, st>>>(probs, times, tiles, q, use_queue, tb, sst, sn, out);
  else
    stage1d_mixed_kernel<NT, 1, TAB><<<grid, NT, 0, st>>>(probs, times, tiles, q, use_queue, tb, sst, sn, out);
}

template <bool TAB>
static void launch_mixed_tab(int stage, int nt, int grid, bool use_queue, const ProbDev *probs, ProbTime *times,
                             const Tile *tiles, WorkQueue *q, const Tables &tb, StateSoA sst, StateSoA sn,
                             StateSoA out, cudaStream_t st)
{
  switch (nt) {
    case 64: launch_mixed_nt<64, TAB>(stage, grid, use_queue, probs, times, tiles, q, tb, sst, sn, out, st); break;
    case 256: launch_mixed_nt<256, TAB>(stage, grid, use_queue, probs, times, tiles, q, tb, sst, sn, out, st); break;
    default: launch_mixed_nt<128, TAB>(stage, grid, use_queue, probs, times, tiles, q, tb, sst, sn, out, st); break;
  }
}

void launch_stage1d_mixed(int stage, int nt, int grid, bool use_queue, const ProbDev *probs, ProbTime *times,
                          const Tile *tiles, WorkQueue *q, const Tables &tb, StateSoA sst, StateSoA sn,
                          StateSoA out, cudaStream_t st, bool tab)
{
  if (grid <= 0) return;
  if (tab) launch_mixed_tab<true>(stage, nt, grid, use_queue, probs, times, tiles, q, tb, sst, sn, out, st);
  else launch_mixed_tab<false>(stage, nt, grid, use_queue, probs, times, tiles, q, tb, sst, sn, out, st);
}

int mixed_max_ctas_per_sm(int nt)
{
  int n = 0;
  cudaError_t e;
  switch (nt) {
    case 64: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, stage1d_mixed_kernel<64, 1, false>, 64, 0); break;
    case 256: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, stage1d_mixed_kernel<256, 1, false>, 256, 0); break;
    default: e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, stage1d_mixed_kernel<128, 1, false>, 128, 0); break;
  }
  return e == cudaSuccess ? n : 0;
}

}  // namespace mdg
