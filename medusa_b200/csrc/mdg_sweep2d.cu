// 2-D RK stage kernels (plain FP64, Cartesian, no dendritic levels).
//
// The reference computes one stage of the directionally unsplit update as one face loop
// that reconstructs every zone twice per direction and writes SoA face fluxes
// (prim_to_fluxes2, step.c:659-764), followed by push() (step.c:327-478).  Here a stage
// is two kernels, each reconstructing every zone once:
//
//  x-kernel (direction 0): a CTA owns 128 consecutive columns and TIX rows; each thread
//    marches down its column with the stencil in registers (rows r-1, r, r+1; row r+2
//    prefetched), reconstructs zone (r, j), solves face (r, j) against the right state
//    of zone r-1, and writes the direction-0 part of the flux difference of zone (r-1, j)
//    -- (0 + F(r)) - F(r-1), the first two terms of push()'s divF sum in the reference's
//    order -- plus the face's shock bit.  No shared memory, no barriers.
//  y-kernel (direction 1 + push): a CTA owns TIY rows x 126 columns; per row the
//    130-zone pencil is staged in shared memory, each zone is reconstructed once, right
//    states are exchanged, faces are solved (HLLE or HLLC by the shock rule below), and
//    push() completes divF = ((acc + G(j+1)) - G(j)), applies the RK combine and writes
//    the new state.
//
// Traffic per zone: x reads the stage state (40 B) and writes the accumulator (40 B);
// y reads the stage state and the accumulator and writes the state (+ the base state in
// the second stage): 200 B per zone in the first stage, 240 B in the second.
//
// Shock tagging (HLLE in direction 1 next to a direction-0 shock) follows the serial
// order of the reference's CPU loop exactly (cells in i-major order, each cell doing its
// direction-0 face before its direction-1 face, step.c:676-760; transverse_shock,
// fluid.c:189-210): a direction-1 face (i,j) uses HLLE iff
//    - j is a boundary face (0 or n2): the flags it reads belong to ghost cells, which
//      are zero-filled at allocation (utils.c:164-174) and never reset, i.e. "shock"; or
//    - the direction-0 face (i,j) or (i,j-1) is a shock in the current stage (the only
//      current-stage marks already made when the reference reaches cell (i,j)); or
//    - in the second stage, cell (i,j) or (i,j-1) was marked in the first stage by any of
//      the direction-0 faces i, i+1, i+2 (set_shock_flag(0) runs once per step).
// Direction-0 shock bits are kept per stage in byte arrays: s0 (first stage, read again
// in the second) and s1 (second stage).
//
// Cartesian metric: gcov = gcon = scale = 1, so the metric multiplications and divisions
// (exact identities) are compiled out (UNIT = true).
// The per-variable reconstruction loops are not unrolled here (one inlined copy of
// para_recon per loop): 7.5 % faster on the 2048^2 Kelvin-Helmholtz grid on a B200 than
// unrolled, and faster than an out-of-line call there (same results).
#ifndef MDG_RECON_UNROLL
#define MDG_RECON_UNROLL 1
#endif
#include "mdg_hydro.cuh"
#include "mdg_kernels.cuh"
#include "mdg_mixed.cuh"

namespace mdg {

// Zone (i, j) of a 2-D problem, with the direction-0 and direction-1 boundary kinds of
// reset_boundaries_gpu applied as index maps (corners are never read by the sweep and
// are mapped to the nearest interior zone).  Primitives only.
__device__ __forceinline__ void load_prim_2d(const ProbDev &P, const StateSoA &s, int i, int j, double *w)
{
  const int n1 = P.n1, n2 = P.n2;
  const int64_t base = P.cell_off;
  i = i < -NG ? -NG : (i > n1 + NG - 1 ? n1 + NG - 1 : i);
  j = j < -NG ? -NG : (j > n2 + NG - 1 ? n2 + NG - 1 : j);
  auto rd = [&](int a, int b, double *o) {
    const int64_t c = base + (int64_t)a * n2 + b;
#pragma unroll
    for (int v = 0; v < NPRIM; v++) o[v] = s.v[v][c];
  };
  const bool iin = (i >= 0 && i < n1), jin = (j >= 0 && j < n2);
  if (iin && jin) {
    rd(i, j, w);
  } else if (!iin && !jin) {
    rd(i < 0 ? 0 : n1 - 1, j < 0 ? 0 : n2 - 1, w);
  } else if (!iin) {
    if (i < 0) {
      switch (P.bc_lo0) {
        case BC_REFLECT: rd(-1 - i, j, w); w[U1] *= -1.0; break;
        case BC_PERIODIC: rd(i + n1, j, w); break;
        case BC_EXTRAP: {
          double a[NPRIM], b[NPRIM];
          rd(0, j, a); rd(1, j, b);
#pragma unroll
          for (int v = 0; v < NPRIM; v++) w[v] = a[v] + i * (b[v] - a[v]);
        } break;
        default: rd(0, j, w); break;
      }
    } else {
      switch (P.bc_hi0) {
        case BC_REFLECT: rd(2 * n1 - i - 1, j, w); w[U1] *= -1.0; break;
        case BC_PERIODIC: rd(i - n1, j, w); break;
        case BC_EXTRAP: {
          double a[NPRIM], b[NPRIM];
          rd(n1 - 1, j, a); rd(n1 - 2, j, b);
#pragma unroll
          for (int v = 0; v < NPRIM; v++) w[v] = a[v] + (i - n1 + 1) * (a[v] - b[v]);
        } break;
        default: rd(n1 - 1, j, w); break;
      }
    }
  } else {
    if (j < 0) {
      switch (P.bc_lo1) {
        case BC_REFLECT: rd(i, -1 - j, w); w[U2] *= -1.0; break;
        case BC_PERIODIC: rd(i, j + n2, w); break;
        default: rd(i, 0, w); break;
      }
    } else {
      switch (P.bc_hi1) {
        case BC_REFLECT: rd(i, 2 * n2 - 1 - j, w); w[U2] *= -1.0; break;
        case BC_PERIODIC: rd(i, j - n2, w); break;
        default: rd(i, n2 - 1, w); break;
      }
    }
  }
}

// ------------------------------------------------------------------ direction 0
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// FP64 re-solve of a direction-DIR face that the mixed solver declined (MIX_COND_MAX):
// both face states reconstructed in FP64 from the stencil values a[0..3] (zones either side
// of the face and their outer neighbours) and the reconstruction columns of the two zones.
template <int DIR, typename GM, typename GZ>
__device__ __noinline__ void face2d_fp64(int order, const double (&a)[6][4], const GM &gm, const GZ &gz, double gam,
                                         const FaceGeom<double> &fg, double *f, double &sig)
{
  double pl[7], pr[7];
  for (int v = 0; v < 6; v++) {
    double lo, hi;
    recon_zone<double>(order, a[v][0], a[v][1], a[v][2], gm, lo, hi);
    pl[v] = hi;
    recon_zone<double>(order, a[v][1], a[v][2], a[v][3], gz, lo, hi);
    pr[v] = lo;
  }
  pl[6] = gam;
  pr[6] = gam;
  riemann_hllc<DIR, true, double>(pl, pr, fg, gam_const(gam), f, sig);
}

// MIX: the mixed-precision variant (FP32 difference-form reconstruction with the FP32
// weights of each zone, FP32 HLLC wave speeds and star-state increments, FP64 fluxes,
// accumulation, update and dt); faces the FP32 solver declines are re-solved in FP64,
// which needs the zone before the face's left zone: the column ring keeps 5 rows.
template <int STAGE, bool MIX>
__global__ void __launch_bounds__(NTX2, MDG_XMINB)
xsweep2d_kernel(const ProbDev *__restrict__ probs, ProbTime *__restrict__ times,
                const Tile *__restrict__ tiles, Tables tb, StateSoA sst, StateSoA acc,
                unsigned char *__restrict__ shock)
{
  constexpr int RING = MIX ? 5 : 4;
  // column stencil ring (rows r-1 .. r+2 of this thread's column), fed by cp.async
  __shared__ double ring[RING][6][NTX2];
  // direction-0 reconstruction coefficients of rows i0-1 .. i0+TIX2
  __shared__ double xrc[RC_NFIELDS][TIX2 + 2];
  __shared__ float xmx[MIX ? MX_NFIELDS : 1][TIX2 + 2];
  __shared__ double sred[32];
  const Tile tile = tiles[blockIdx.x];
  if (times[tile.prob].done) return;   // past tmax: the time loop has ended (CTA-uniform)
  const ProbDev &P = probs[tile.prob];
  const int n1 = P.n1, n2 = P.n2;
  const int t = threadIdx.x;
  const int j = tile.j0 + t;
  const int i0 = tile.i0;
  const int ilast = min(i0 + TIX2, n1);           // last face row of this tile (<= n1)
  const bool col_ok = j < n2;
  const int order = P.interp_order;
  const GamConst<double> gc = gam_const(P.gam);
  const FaceGeom<double> fg{P.area0, 1.0, 1.0, 1.0, 1.0};
  unsigned char *sh = shock + P.sh_off;
  double smax = 0.0;                               // max |signal speed| of this thread's faces
  // ring slot of a row (rows >= i0-2)
  auto slot = [&](int row) { return MIX ? (row - i0 + 2) % RING : (row & 3); };

  for (int k = t; k < RC_NFIELDS * (TIX2 + 2); k += NTX2) {
    const int f = k / (TIX2 + 2), rr = k - f * (TIX2 + 2);
    const int row = min(i0 - 1 + rr, n1);
    xrc[f][rr] = __ldg(tb.rc0 + f * tb.rc0_stride + P.geo_off + row + NG);
  }
  if (MIX) {
    for (int k = t; k < MX_NFIELDS * (TIX2 + 2); k += NTX2) {
      const int f = k / (TIX2 + 2), rr = k - f * (TIX2 + 2);
      const int row = min(i0 - 1 + rr, n1);
      xmx[f][rr] = __ldg(tb.mx + f * tb.rc0_stride + P.geo_off + row + NG);
    }
  }
  __syncthreads();

  if (col_ok) {
    // rows inside the grid arrive by cp.async; boundary rows are produced by the
    // boundary index maps and stored directly.  One commit group per row.
    auto stage_row = [&](int row) {
      double *dst0 = &ring[slot(row)][0][t];
      if (row >= 0 && row < n1) {
        const int64_t c = P.cell_off + (int64_t)row * n2 + j;
#pragma unroll
        for (int v = 0; v < NPRIM; v++) cp_async8(dst0 + v * NTX2, sst.v[v] + c);
      } else {
        double w[NPRIM];
        load_prim_2d(P, sst, row, j, w);
#pragma unroll
        for (int v = 0; v < NPRIM; v++) dst0[v * NTX2] = w[v];
      }
      cp_async_commit();
    };
    // pressure (eos_gamma.c:7 / eos_poly.c:7) of a landed row, stored as variable 5
    auto press_row = [&](int row) {
      double *d = &ring[slot(row)][0][t];
      d[5 * NTX2] = eos_press(P.eos, P.gam, P.Kpoly, d[RHO * NTX2], d[UU * NTX2]);
    };
    stage_row(i0 - 2);
    stage_row(i0 - 1);
    stage_row(i0);
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");   // rows i0-2, i0-1 have landed
    press_row(i0 - 2);
    press_row(i0 - 1);
    double xr_prev[6], f_prev[NPRIM];
#pragma unroll
    for (int v = 0; v < NPRIM; v++) f_prev[v] = 0.0;
#pragma unroll
    for (int v = 0; v < 6; v++) xr_prev[v] = 0.0;
    for (int r = i0 - 1; r <= ilast; r++) {
      if (r + 2 <= ilast + 1) stage_row(r + 2);
      else cp_async_commit();
      cp_async_wait1();                            // rows up to r+1 have landed
      press_row(r + 1);
      // reconstruct zone (r, j) along direction 0
      double xl[7], xr[6];
      if (MIX) {
        const MixW w = load_mixw_any(&xmx[0][r - i0 + 1], TIX2 + 2);
#pragma unroll
        for (int v = 0; v < 6; v++) {
          const double a = ring[slot(r)][v][t];
          float dl, dr;
          mixed_recon((float)(a - ring[slot(r - 1)][v][t]), (float)(ring[slot(r + 1)][v][t] - a), w, dl, dr);
          xl[v] = a + (double)dl;
          xr[v] = a + (double)dr;
        }
        xl[6] = P.gam;
      } else {
        const RcView<double, false> g{&xrc[0][r - i0 + 1], TIX2 + 2};
#pragma unroll kReconUnroll
        for (int v = 0; v < 6; v++)
          recon_zone<double>(order, ring[slot(r - 1)][v][t], ring[slot(r)][v][t], ring[slot(r + 1)][v][t], g,
                             xl[v], xr[v]);
        xl[6] = P.gam;
      }
      if (r >= i0) {
        // face (r, j): left state = right face value of zone r-1
        double pl[7], f[NPRIM], sig;
#pragma unroll
        for (int v = 0; v < 6; v++) pl[v] = xr_prev[v];
        pl[6] = P.gam;
        int sb;
        if (MIX) {
          float sgf;
          if (riemann_hllc_mixed<0>(pl, xl, fg, gam_const<float>((float)P.gam), f, sgf, sb)) {
            sig = (double)sgf;
          } else {
            double a[6][4];
#pragma unroll
            for (int v = 0; v < 6; v++)
              for (int q = 0; q < 4; q++) a[v][q] = ring[slot(r - 2 + q)][v][t];
            const RcView<double, false> gm{&xrc[0][r - i0], TIX2 + 2}, gz{&xrc[0][r - i0 + 1], TIX2 + 2};
            face2d_fp64<0>(order, a, gm, gz, P.gam, fg, f, sig);   // sb: the FP32 estimate's flag
          }
        } else {
          sb = riemann_hllc<0, true, double>(pl, xl, fg, gc, f, sig);
        }
        smax = tmax(smax, fabs(sig));
        sh[(int64_t)r * n2 + j] = (unsigned char)sb;
        // direction-0 part of divF of zone (r-1, j): (0 + F(r)) - F(r-1)
        if (r > i0) {
          const int64_t cell = P.cell_off + (int64_t)(r - 1) * n2 + j;
#pragma unroll
          for (int v = 0; v < NPRIM; v++) {
            double d = 0.0;
            d += f[v];
            d -= f_prev[v];
            acc.v[v][cell] = d;
          }
        }
#pragma unroll
        for (int v = 0; v < NPRIM; v++) f_prev[v] = f[v];
      }
#pragma unroll
      for (int v = 0; v < 6; v++) xr_prev[v] = xr[v];
    }
  }
  // min over this thread's faces of dx[0]/|sig| (step.c:718)
  block_min_to(P.dx0 / smax, &times[tile.prob].minacc, sred);
}

// ------------------------------------------------------------------ direction 1 + push
template <int STAGE, bool MIX>
__global__ void __launch_bounds__(NTY2, MDG_YMINB)
ysweep2d_kernel(const ProbDev *__restrict__ probs, ProbTime *__restrict__ times,
                const Tile *__restrict__ tiles, Tables tb, StateSoA sst, StateSoA sn, StateSoA acc,
                StateSoA out, const unsigned char *__restrict__ shock0, const unsigned char *__restrict__ shock1)
{
  __shared__ double sv[6][NTY2 + 2];
  __shared__ double syr[6][NTY2];
  __shared__ double sfy[NPRIM][NTY2];
  __shared__ double yrc[RC_NFIELDS][NTY2];    // direction-1 coefficients of each thread's column
  __shared__ float ymx[MIX ? MX_NFIELDS : 1][NTY2];
  __shared__ unsigned char sflag[NTY2];
  __shared__ double sred[32];

  const Tile tile = tiles[blockIdx.x];
  if (times[tile.prob].done) return;   // past tmax: the time loop has ended (CTA-uniform)
  const ProbDev &P = probs[tile.prob];
  const double dt = times[tile.prob].dt;
  const int t = threadIdx.x;
  const int n1 = P.n1, n2 = P.n2;
  const int j0 = tile.j0;
  const int jx = j0 - 1 + t;
  const double gam = P.gam;
  const int order = P.interp_order;
  const GamConst<double> gc = gam_const(gam);
  const FaceGeom<double> fg{P.area1, 1.0, 1.0, 1.0, 1.0};
  const unsigned char *s0 = shock0 + P.sh_off;
  const unsigned char *s1 = shock1 + P.sh_off;
  const bool real_col = (jx >= 0) && (jx < n2);
  const bool out_col = (t >= 1) && (t <= NTY2 - 2) && (jx < n2);
  const int iend = min(tile.i0 + TIY2, n1);
  double smax = 0.0;      // max |signal speed| of this thread's faces
  double nmin = 1.0e300;  // min numerator of the source-term limits (zero sources)
  double lsrc = 1.0e300;  // min source-term limit (fixed gravity)
  double lmax = 0.0;      // max local_dt of the next estimate_dt's zone terms
  {
    const int jc = jx < -1 ? -1 : (jx > n2 ? n2 : jx);
    for (int f = 0; f < RC_NFIELDS; f++) yrc[f][t] = __ldg(tb.rc1 + f * tb.rc1_stride + P.rc1_off + jc + NG);
    if (MIX)
      for (int f = 0; f < MX_NFIELDS; f++) ymx[f][t] = __ldg(tb.mx1 + f * tb.rc1_stride + P.rc1_off + jc + NG);
  }

  for (int r = tile.i0; r < iend; r++) {
    __syncthreads();
    {
      double w[NPRIM];
      load_prim_2d(P, sst, r, jx, w);
#pragma unroll
      for (int v = 0; v < NPRIM; v++) sv[v][t + 1] = w[v];
      sv[5][t + 1] = eos_press(P.eos, gam, P.Kpoly, w[RHO], w[UU]);
      if (t == 0) {
        load_prim_2d(P, sst, r, j0 - 2, w);
#pragma unroll
        for (int v = 0; v < NPRIM; v++) sv[v][0] = w[v];
        sv[5][0] = eos_press(P.eos, gam, P.Kpoly, w[RHO], w[UU]);
      }
      if (t == NTY2 - 1) {
        load_prim_2d(P, sst, r, jx + 1, w);
#pragma unroll
        for (int v = 0; v < NPRIM; v++) sv[v][NTY2 + 1] = w[v];
        sv[5][NTY2 + 1] = eos_press(P.eos, gam, P.Kpoly, w[RHO], w[UU]);
      }
    }
    // flag of zone (r, jx): current-stage mark by its own direction-0 face, and in the
    // second stage any first-stage mark by the direction-0 faces r, r+1, r+2
    unsigned char fl = 0;
    if (real_col) {
      const int64_t b = (int64_t)r * n2 + jx;
      if (STAGE == 0) fl = s0[b];
      else fl = s1[b] | s0[b] | s0[b + n2] | s0[b + 2 * (int64_t)n2];
    }
    sflag[t] = fl;
    double accv[NPRIM], pn[NPRIM];
    const int64_t cell = P.cell_off + (int64_t)r * n2 + jx;
    if (out_col) {
#pragma unroll
      for (int v = 0; v < NPRIM; v++) accv[v] = acc.v[v][cell];
      if (STAGE == 1) {
#pragma unroll
        for (int v = 0; v < NPRIM; v++) pn[v] = sn.v[v][cell];
      }
    }
    __syncthreads();
    // reconstruct zone (r, jx) along direction 1
    double yl[7];
    if (MIX) {
      const MixW w = load_mixw_any(&ymx[0][t], NTY2);
#pragma unroll
      for (int v = 0; v < 6; v++) {
        const double a = sv[v][t + 1];
        float dl, dr;
        mixed_recon((float)(a - sv[v][t]), (float)(sv[v][t + 2] - a), w, dl, dr);
        yl[v] = a + (double)dl;
        syr[v][t] = a + (double)dr;
      }
      yl[6] = gam;
    } else {
      const RcView<double, false> g{&yrc[0][t], NTY2};
      double yr[6];
#pragma unroll kReconUnroll
      for (int v = 0; v < 6; v++) recon_zone<double>(order, sv[v][t], sv[v][t + 1], sv[v][t + 2], g, yl[v], yr[v]);
#pragma unroll
      for (int v = 0; v < 6; v++) syr[v][t] = yr[v];
      yl[6] = gam;
    }
    __syncthreads();
    if (t >= 1) {
      double pl[7], fy[NPRIM], sig;
#pragma unroll
      for (int v = 0; v < 6; v++) pl[v] = syr[v][t - 1];
      pl[6] = gam;
      const bool hlle = (jx == 0) || (jx == n2) || sflag[t] || sflag[t - 1];
      if (hlle) {
        riemann_hlle<1, true, double>(pl, yl, fg, gc, fy, sig);
      } else if (!MIX) {
        riemann_hllc<1, true, double>(pl, yl, fg, gc, fy, sig);
      } else {
        float sgf;
        int sb;
        if (riemann_hllc_mixed<1>(pl, yl, fg, gam_const<float>((float)gam), fy, sgf, sb)) {
          sig = (double)sgf;
        } else {
          double a[6][4];
#pragma unroll
          for (int v = 0; v < 6; v++)
            for (int q = 0; q < 4; q++) a[v][q] = sv[v][t - 1 + q];
          const RcView<double, false> gm{&yrc[0][t - 1], NTY2}, gz{&yrc[0][t], NTY2};
          face2d_fp64<1>(order, a, gm, gz, gam, fg, fy, sig);
        }
      }
#pragma unroll
      for (int v = 0; v < NPRIM; v++) sfy[v][t] = fy[v];
      if (jx >= 0 && jx <= n2) smax = tmax(smax, fabs(sig));
    }
    __syncthreads();
    // push() of zone (r, jx), step.c:380-470 (Cartesian: no sources, unit metric)
    if (out_col) {
      double ph[NPRIM], u[NPRIM], uh[NPRIM], pf[NPRIM];
      double src[NPRIM] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int v = 0; v < NPRIM; v++) ph[v] = sv[v][t + 1];
      if (STAGE == 0) {
#pragma unroll
        for (int v = 0; v < NPRIM; v++) pn[v] = ph[v];
      }
      p_to_u(pn, u, 1.0, 1.0, 1.0);
      p_to_u(ph, uh, 1.0, 1.0, 1.0);
      if (P.grav_on) {
        // sources of the stage state: fixed gravity (the Cartesian geometric ones are 0)
        add_fixed_gravity(ph, P.grav, 1.0, 1.0, 1.0, 2, src);
        lsrc = tmin(lsrc, dt_source_control(pn, u, src));
      } else {
        nmin = tmin(nmin, src_dt_numerator_min(pn, u));   // dt_source_control, step.c:393
      }
      const double pfact = STAGE ? 0.5 : 1.0, phfact = STAGE ? 0.5 : 0.0, ffact = STAGE ? 0.5 : 1.0;
#pragma unroll
      for (int v = 0; v < NPRIM; v++) {
        double divF = accv[v];
        divF += sfy[v][t + 1];
        divF -= sfy[v][t];
        double ddt = divF / P.vol - src[v];
        u[v] = pfact * u[v] + phfact * uh[v] - ffact * dt * ddt;
      }
      u_to_p(u, pf, 1.0, 1.0, 1.0, P.floors != 0, P.rho_floor, P.e_floor);
#pragma unroll
      for (int v = 0; v < NPRIM; v++) out.v[v][cell] = pf[v];
      flag_nonfinite(pf, &times[tile.prob]);
      if (STAGE == 1) {
        // zone terms of the next estimate_dt (step.c:177-187): new velocities, sound
        // speed of the stage state
        const double cs = sqrt(gam * sv[5][t + 1] / ph[RHO]);
        // (the partial sum after direction 0 never gives the smaller 1/local_dt: the
        // direction-1 term is non-negative)
        double local_dt = 0.0;
        local_dt += (fabs(pf[U1]) + cs) / P.dx0;
        local_dt += (fabs(pf[U2]) + cs) / P.dx1;
        lmax = tmax(lmax, local_dt);
      }
    }
  }
  double lmin = tmin(1 * P.dx1 / smax, src_dt_from_numerator(nmin));
  lmin = tmin(lmin, lsrc);
  if (STAGE == 1) lmin = tmin(lmin, 1.0 / lmax);
  block_min_to(lmin, &times[tile.prob].minacc, sred);
}

void launch_stage2d(int stage, bool mixed, const ProbDev *probs, ProbTime *times, const Tile *xtiles, int nxt,
                    const Tile *ytiles, int nyt, const Tables &tb, StateSoA sst, StateSoA sn, StateSoA acc,
                    StateSoA out, unsigned char *shock0, unsigned char *shock1, cudaStream_t st)
{
  if (nxt <= 0 || nyt <= 0) return;
  if (stage == 0 && !mixed) {
    xsweep2d_kernel<0, false><<<nxt, NTX2, 0, st>>>(probs, times, xtiles, tb, sst, acc, shock0);
    ysweep2d_kernel<0, false><<<nyt, NTY2, 0, st>>>(probs, times, ytiles, tb, sst, sn, acc, out, shock0, shock1);
  } else if (!mixed) {
    xsweep2d_kernel<1, false><<<nxt, NTX2, 0, st>>>(probs, times, xtiles, tb, sst, acc, shock1);
    ysweep2d_kernel<1, false><<<nyt, NTY2, 0, st>>>(probs, times, ytiles, tb, sst, sn, acc, out, shock0, shock1);
  } else if (stage == 0) {
    xsweep2d_kernel<0, true><<<nxt, NTX2, 0, st>>>(probs, times, xtiles, tb, sst, acc, shock0);
    ysweep2d_kernel<0, true><<<nyt, NTY2, 0, st>>>(probs, times, ytiles, tb, sst, sn, acc, out, shock0, shock1);
  } else {
    xsweep2d_kernel<1, true><<<nxt, NTX2, 0, st>>>(probs, times, xtiles, tb, sst, acc, shock1);
    ysweep2d_kernel<1, true><<<nyt, NTY2, 0, st>>>(probs, times, ytiles, tb, sst, sn, acc, out, shock0, shock1);
  }
}

}  // namespace mdg
