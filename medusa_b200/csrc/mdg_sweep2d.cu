// Fused 2-D RK stage kernel (plain FP64, Cartesian, no dendritic levels).
//
// The reference computes one stage of the directionally unsplit update in three passes
// over memory: a face loop that reconstructs every zone twice per direction and writes
// SoA face fluxes (prim_to_fluxes2, step.c:659-764), then push() (step.c:327-478).  Here
// one kernel does the whole stage and each zone crosses HBM once per stage:
//
//  * a CTA owns a tile of TI2 = 32 rows x TJ2 = 126 columns and marches down the rows
//    (direction 0 = i, the slow index).  Thread t owns column j0-1+t;
//  * a 4-row ring of the stage state (5 primitives + pressure, 130 columns incl. the
//    direction-1 ghost halo) lives in shared memory; row r+3 is prefetched into
//    registers at the top of iteration r and parked in the ring after the row it
//    replaces has been consumed;
//  * direction 0: each thread reconstructs zone (r, j) once from the ring column and
//    solves face (r, j) with the right state of zone r-1 kept in registers;
//  * direction 1: each thread reconstructs zone (r, j) once from the ring row, exchanges
//    right states through shared memory and solves face (r, j);
//  * push() of zone (r-1, j) follows as soon as its last face flux exists.
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
// First-stage direction-0 shock bits are kept in a byte array for the second stage.
#include "mdg_hydro.cuh"
#include "mdg_kernels.cuh"

namespace mdg {

// Zone (i, j) of a 2-D problem, with the direction-0 and direction-1 boundary kinds of
// reset_boundaries_gpu applied as index maps (corners are never read by the sweep and
// are mapped to the nearest interior zone).
__device__ __forceinline__ void load_cell_2d(const ProbDev &P, const StateSoA &s, int i, int j, double *w)
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
  w[5] = eos_press(P.eos, P.gam, P.Kpoly, w[RHO], w[UU]);
}

template <int STAGE>
__global__ void __launch_bounds__(NT2, 2)
stage2d_kernel(const ProbDev *__restrict__ probs, ProbTime *__restrict__ times,
               const Tile *__restrict__ tiles, Tables tb, StateSoA sst, StateSoA sn, StateSoA out,
               unsigned char *__restrict__ shock0)
{
  __shared__ double ring[4][6][NT2 + 2];
  __shared__ double syr[6][NT2];
  __shared__ double sfy[NPRIM][NT2];
  __shared__ unsigned char sflag[NT2];
  __shared__ double sred[32];

  const Tile tile = tiles[blockIdx.x];
  const ProbDev &P = probs[tile.prob];
  const double dt = times[tile.prob].dt;
  const int t = threadIdx.x;
  const int n1 = P.n1, n2 = P.n2;
  const int i0 = tile.i0, j0 = tile.j0;
  const int jx = j0 - 1 + t;
  const int ilast = i0 + TI2;                     // last x-face row of this tile
  const double gam = P.gam;
  const int order = P.interp_order;
  unsigned char *sh0 = shock0 + P.sh_off;         // first-stage shock bits, rows 0..n1+2

  // direction-1 reconstruction coefficients of this thread's column (constant along the march)
  Rc<double> gy;
  {
    int jc = jx < -1 ? -1 : (jx > n2 ? n2 : jx);
    load_rc(gy, tb.rc1, tb.rc1_stride, P.rc1_off + jc + NG);
  }
  FaceGeom<double> fgx{P.area0, 1.0, 1.0, 1.0, 1.0};
  FaceGeom<double> fgy{P.area1, 1.0, 1.0, 1.0, 1.0};

  // prologue: rows i0-2 .. i0+1
  for (int r = i0 - 2; r <= i0 + 1; r++) {
    double w[6];
    load_cell_2d(P, sst, r, jx, w);
#pragma unroll
    for (int v = 0; v < 6; v++) ring[r & 3][v][t + 1] = w[v];
    if (t == 0) {
      load_cell_2d(P, sst, r, j0 - 2, w);
#pragma unroll
      for (int v = 0; v < 6; v++) ring[r & 3][v][0] = w[v];
    }
    if (t == NT2 - 1) {
      load_cell_2d(P, sst, r, jx + 1, w);
#pragma unroll
      for (int v = 0; v < 6; v++) ring[r & 3][v][NT2 + 1] = w[v];
    }
  }

  double xr_prev[6], fx_prev[NPRIM], fy_lo[NPRIM], fy_hi[NPRIM];
#pragma unroll
  for (int v = 0; v < NPRIM; v++) { fx_prev[v] = 0.0; fy_lo[v] = 0.0; fy_hi[v] = 0.0; }
#pragma unroll
  for (int v = 0; v < 6; v++) xr_prev[v] = 0.0;
  double lmin = 1.0e300;
  const bool out_col = (t >= 1) && (t <= NT2 - 2) && (jx < n2);
  const bool real_xcol = (jx >= 0) && (jx < n2);

  for (int r = i0 - 1; r <= ilast; r++) {
    __syncthreads();
    // prefetch row r+3 (needed from iteration r+2 on)
    const bool pre = (r + 3 <= ilast + 1);
    double pw[6], pw2[6];
    if (pre) {
      load_cell_2d(P, sst, r + 3, jx, pw);
      if (t == 0) load_cell_2d(P, sst, r + 3, j0 - 2, pw2);
      if (t == NT2 - 1) load_cell_2d(P, sst, r + 3, jx + 1, pw2);
    }
    double pn[NPRIM];
    const bool do_upd = (r - 1 >= i0) && (r - 1 < n1) && out_col;
    if (STAGE == 1 && do_upd) {
      const int64_t cell = P.cell_off + (int64_t)(r - 1) * n2 + jx;
#pragma unroll
      for (int v = 0; v < NPRIM; v++) pn[v] = sn.v[v][cell];
    }

    // ---- direction 0: reconstruct zone (r, jx), face (r, jx)
    double xl[7], xr[7];
    {
      Rc<double> gx;
      int rc = r < -1 ? -1 : (r > n1 ? n1 : r);
      load_rc(gx, tb.rc0, tb.rc0_stride, P.geo_off + rc + NG);
#pragma unroll
      for (int v = 0; v < 6; v++)
        recon_zone<double>(order, ring[(r - 1) & 3][v][t + 1], ring[r & 3][v][t + 1], ring[(r + 1) & 3][v][t + 1],
                           gx, xl[v], xr[v]);
      xl[6] = gam; xr[6] = gam;
    }
    int sh = 0;
    double fx[NPRIM];
    if (r >= i0) {
      double sig;
      double pl[7];
#pragma unroll
      for (int v = 0; v < 7; v++) pl[v] = (v < 6) ? xr_prev[v] : gam;
      sh = riemann_hllc<0, double>(pl, xl, fgx, fx, sig);
      if (real_xcol && r <= n1) {
        lmin = tmin(lmin, P.dx0 / fabs(sig));
        if (STAGE == 0) sh0[(int64_t)r * n2 + jx] = (unsigned char)sh;
      }
      // ---- push() of zone (r-1, jx): all four face fluxes exist now
      if (do_upd) {
        double ph[NPRIM], u[NPRIM], uh[NPRIM], divF[NPRIM], pf[NPRIM];
        const double src[NPRIM] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int v = 0; v < NPRIM; v++) ph[v] = ring[(r - 1) & 3][v][t + 1];
        if (STAGE == 0) {
#pragma unroll
          for (int v = 0; v < NPRIM; v++) pn[v] = ph[v];
        }
        p_to_u(pn, u, 1.0, 1.0, 1.0);
        p_to_u(ph, uh, 1.0, 1.0, 1.0);
        lmin = tmin(lmin, dt_source_control(pn, u, src));
#pragma unroll
        for (int v = 0; v < NPRIM; v++) {
          divF[v] = 0.0;
          divF[v] += fx[v];
          divF[v] -= fx_prev[v];
          divF[v] += fy_hi[v];
          divF[v] -= fy_lo[v];
        }
        const double pfact = STAGE ? 0.5 : 1.0, phfact = STAGE ? 0.5 : 0.0, ffact = STAGE ? 0.5 : 1.0;
#pragma unroll
        for (int v = 0; v < NPRIM; v++) {
          double ddt = divF[v] / P.vol - src[v];
          u[v] = pfact * u[v] + phfact * uh[v] - ffact * dt * ddt;
        }
        u_to_p(u, pf, 1.0, 1.0, 1.0);
        const int64_t cell = P.cell_off + (int64_t)(r - 1) * n2 + jx;
#pragma unroll
        for (int v = 0; v < NPRIM; v++) out.v[v][cell] = pf[v];
        if (STAGE == 1) {
          // zone terms of the next estimate_dt (step.c:177-187): new velocities, sound
          // speed of the stage state
          const double cs = sqrt(gam * ring[(r - 1) & 3][5][t + 1] / ph[RHO]);
          double local_dt = 0.0;
          local_dt += (fabs(pf[U1]) + cs) / P.dx0;
          lmin = tmin(lmin, 1.0 / local_dt);
          local_dt += (fabs(pf[U2]) + cs) / P.dx1;
          lmin = tmin(lmin, 1.0 / local_dt);
        }
      }
    }

    const bool ywork = (r >= i0) && (r < ilast);    // CTA-uniform
    if (ywork) {
      // ---- direction 1: reconstruct zone (r, jx), face (r, jx)
      double yl[7], yr[6];
#pragma unroll
      for (int v = 0; v < 6; v++)
        recon_zone<double>(order, ring[r & 3][v][t], ring[r & 3][v][t + 1], ring[r & 3][v][t + 2], gy, yl[v], yr[v]);
      yl[6] = gam;
#pragma unroll
      for (int v = 0; v < 6; v++) syr[v][t] = yr[v];
      unsigned char fl = 0;
      if (real_xcol && r < n1) {
        fl = (unsigned char)sh;
        if (STAGE == 1) {
          const int64_t b = (int64_t)r * n2 + jx;
          fl |= sh0[b] | sh0[b + n2] | sh0[b + 2 * (int64_t)n2];
        }
      }
      sflag[t] = fl;
      __syncthreads();
      if (t >= 1) {
        double pl[7], fy[NPRIM], sig;
#pragma unroll
        for (int v = 0; v < 6; v++) pl[v] = syr[v][t - 1];
        pl[6] = gam;
        const bool hlle = (jx == 0) || (jx == n2) || sflag[t] || sflag[t - 1];
        if (hlle) riemann_hlle<1, double>(pl, yl, fgy, fy, sig);
        else riemann_hllc<1, double>(pl, yl, fgy, fy, sig);
#pragma unroll
        for (int v = 0; v < NPRIM; v++) sfy[v][t] = fy[v];
        if (jx >= 0 && jx <= n2 && r < n1) lmin = tmin(lmin, 1 * P.dx1 / fabs(sig));
      }
      __syncthreads();
      if (t >= 1) {
#pragma unroll
        for (int v = 0; v < NPRIM; v++) fy_lo[v] = sfy[v][t];
      }
      if (t <= NT2 - 2) {
#pragma unroll
        for (int v = 0; v < NPRIM; v++) fy_hi[v] = sfy[v][t + 1];
      }
    } else {
      __syncthreads();
    }
    // park row r+3 in the slot of row r-1 (consumed by now)
    if (pre) {
      const int sl = (r + 3) & 3;
#pragma unroll
      for (int v = 0; v < 6; v++) ring[sl][v][t + 1] = pw[v];
      if (t == 0) {
#pragma unroll
        for (int v = 0; v < 6; v++) ring[sl][v][0] = pw2[v];
      }
      if (t == NT2 - 1) {
#pragma unroll
        for (int v = 0; v < 6; v++) ring[sl][v][NT2 + 1] = pw2[v];
      }
    }
#pragma unroll
    for (int v = 0; v < 6; v++) xr_prev[v] = xr[v];
    if (r >= i0) {
#pragma unroll
      for (int v = 0; v < NPRIM; v++) fx_prev[v] = fx[v];
    }
  }
  block_min_to(lmin, &times[tile.prob].minacc, sred);
}

void launch_stage2d(int stage, const ProbDev *probs, ProbTime *times, const Tile *tiles, int ntiles,
                    const Tables &tb, StateSoA sst, StateSoA sn, StateSoA out, unsigned char *shock0,
                    cudaStream_t st)
{
  if (ntiles <= 0) return;
  if (stage == 0) stage2d_kernel<0><<<ntiles, NT2, 0, st>>>(probs, times, tiles, tb, sst, sn, out, shock0);
  else stage2d_kernel<1><<<ntiles, NT2, 0, st>>>(probs, times, tiles, tb, sst, sn, out, shock0);
}

}  // namespace mdg
