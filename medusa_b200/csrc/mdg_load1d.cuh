// Boundary handling of 1-D problems, shared by the FP64 and mixed-precision sweeps:
// reset_boundaries_gpu (bc.c:705-1422) applied as index maps when a zone is loaded.
#pragma once
#include "mdg_hydro.cuh"
#include "mdg_kernels.cuh"

namespace mdg {

// Noh inflow boundary, problems/init_spherical_noh.c:63-79 (ijk_to_r of
// metric_spherical_general.c:483-496: r = r(beta0/Gamma0), rhat0 = dr/dx = 1).
__device__ __forceinline__ void prob_bounds_noh(double gam, double b0, double g0, double t, double *w)
{
  double x = b0 / g0;
  double r = fabs(x);
  w[RHO] = 1.;
  w[UU] = 1.e-6 / (gam - 1.);
  w[U1] = -1. / 1.0;
  w[U2] = 0.;
  w[U3] = 0.;
  w[RHO] += t / r;
  w[RHO] *= w[RHO];
}

// Zone i (may be a ghost, i in [-NG, n1+NG)) of a 1-D problem: 5 primitives + pressure.
__device__ __forceinline__ void load_cell_1d(const ProbDev &P, const StateSoA &s, const double *__restrict__ rc,
                                             int64_t rcs, int i, double t_bc, double *w)
{
  const int n = P.n1;
  const int64_t base = P.cell_off;
  if (i < -NG) i = -NG;
  if (i > n + NG - 1) i = n + NG - 1;
  auto rd = [&](int k, double *o) {
#pragma unroll
    for (int v = 0; v < NPRIM; v++) o[v] = s.v[v][base + k];
  };
  if (i >= 0 && i < n) {
    rd(i, w);
  } else if (i < 0) {
    switch (P.bc_lo0) {
      case BC_REFLECT: rd(-1 - i, w); w[U1] *= -1.0; break;
      case BC_SPHERICAL_ORIGIN: rd(-1 - i, w); w[U1] *= -1.0; w[U3] *= -1.0; break;
      case BC_PERIODIC: rd(i + n, w); break;
      case BC_EXTRAP: {
        double a[NPRIM], b[NPRIM];
        rd(0, a); rd(1, b);
#pragma unroll
        for (int v = 0; v < NPRIM; v++) w[v] = a[v] + i * (b[v] - a[v]);
      } break;
      case BC_PROB:
        prob_bounds_noh(P.gam, __ldg(rc + RC_B0 * rcs + P.geo_off + i + NG),
                        __ldg(rc + RC_G0 * rcs + P.geo_off + i + NG), t_bc, w);
        break;
      default: rd(0, w); break;   // OUTFLOW
    }
  } else {
    switch (P.bc_hi0) {
      case BC_REFLECT: rd(2 * n - i - 1, w); w[U1] *= -1.0; break;
      case BC_PERIODIC: rd(i - n, w); break;
      case BC_EXTRAP: {
        double a[NPRIM], b[NPRIM];
        rd(n - 1, a); rd(n - 2, b);
#pragma unroll
        for (int v = 0; v < NPRIM; v++) w[v] = a[v] + (i - n + 1) * (a[v] - b[v]);
      } break;
      case BC_PROB:
        if (P.prob_kind == MDG_PROB_DUST) {
          // outflow, with v^r = -1/sqrt(r) / scale[0][0] of the ghost zone (init_dustcollapse.c:104-113)
          rd(n - 1, w);
          w[U1] = P.u1_hi[i - n];
        } else {
          prob_bounds_noh(P.gam, __ldg(rc + RC_B0 * rcs + P.geo_off + i + NG),
                          __ldg(rc + RC_G0 * rcs + P.geo_off + i + NG), t_bc, w);
        }
        break;
      default: rd(n - 1, w); break;   // OUTFLOW
    }
  }
  w[5] = eos_press(P.eos, P.gam, P.Kpoly, w[RHO], w[UU]);
}

// Geometric source terms of zone gi from its stage state ph and pressure
// (get_geom_src_terms, rad_fluid.c:164-192; hydro_stress_tensor, fluid.c:56-73):
// src[U1+m] = sum over l, n of T[l][n] conn[l][m][n], T[l][m] = rho v^m v_l + p delta_lm.
// With sparse_conn only the nine coefficients that the spherical metric fills are read;
// the others are exactly zero and their products add nothing, so the sum is unchanged.
__device__ __forceinline__ void geo_sources_1d(const double *__restrict__ geo, int64_t gs, int64_t gi,
                                               bool sparse_conn, const double *ph, double press, double gc0,
                                               double gc1, double gc2, double *src)
{
  const double vcov[3] = {gc0 * ph[U1], gc1 * ph[U2], gc2 * ph[U3]};
  double T[3][3];
#pragma unroll
  for (int l = 0; l < 3; l++) {
#pragma unroll
    for (int m = 0; m < 3; m++) T[l][m] = ph[RHO] * ph[U1 + m] * vcov[l];
    T[l][l] += press;
  }
  src[RHO] = 0.0;
  src[UU] = 0.0;
  auto c = [&](int k) { return __ldg(geo + (GF_CONN + k) * gs + gi); };
  if (sparse_conn) {
    // (l,m,n) = (1,0,1) (2,0,2) | (0,1,1) (1,1,0) (2,1,2) | (0,2,2) (1,2,2) (2,2,0) (2,2,1)
    src[U1] = 0.0; src[U1] += T[1][1] * c(10); src[U1] += T[2][2] * c(20);
    src[U2] = 0.0; src[U2] += T[0][1] * c(4);  src[U2] += T[1][0] * c(12); src[U2] += T[2][2] * c(23);
    src[U3] = 0.0; src[U3] += T[0][2] * c(8);  src[U3] += T[1][2] * c(17); src[U3] += T[2][0] * c(24);
    src[U3] += T[2][1] * c(25);
  } else {
    src[U1] = 0.0; src[U2] = 0.0; src[U3] = 0.0;
#pragma unroll
    for (int l = 0; l < 3; l++)
#pragma unroll
      for (int m = 0; m < 3; m++)
#pragma unroll
        for (int n = 0; n < 3; n++) src[U1 + m] += T[l][n] * c(l * 9 + m * 3 + n);
  }
}

}  // namespace mdg
