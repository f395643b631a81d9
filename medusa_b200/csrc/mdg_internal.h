// Internal data structures shared by the host code (mdg_capi.cu, mdg_geometry.cpp) and
// the sweep kernels.  Not part of the public ABI.
#pragma once
#include <stdint.h>
#include "../../include/medusa_b200.h"

#ifdef __CUDACC__
#define MDG_HD __host__ __device__
#else
#define MDG_HD
#endif

namespace mdg {

constexpr int NG = 2;       // ghost layers (decs.h:61)
constexpr int NPRIM = 5;    // rho, u, v1, v2, v3 (decs.h:57)
enum { RHO = 0, UU = 1, U1 = 2, U2 = 3, U3 = 4 };
enum { BC_OUTFLOW = 0, BC_REFLECT = 1, BC_EXTRAP = 2, BC_PERIODIC = 3, BC_PROB = 4,
       BC_SPHERICAL_ORIGIN = 5 };

// Problems on the dendritic spherical grid (DENDRITIC_GRID=TRUE with GEOM=SPHERICAL):
// every 3-D problem, and 2-D problems in spherical (r, theta) coordinates.
inline bool is_dendritic(const mdg_problem_desc &d)
{
  return d.ndim == 3 || (d.ndim == 2 && d.geom == MDG_SPHERICAL);
}

// Per-zone reconstruction coefficients along one direction: the geometry-only
// sub-expressions of para_recon (reconstruct.c:151-157,174-175) and lin_recon
// (reconstruct.c:100-104), precomputed on the host in the reference's operation order.
enum ReconField {
  RC_AM, RC_A0, RC_AP,        // alpha[i-1], alpha[i], alpha[i+1]
  RC_BM, RC_B0, RC_BP,        // beta
  RC_GM, RC_G0, RC_GP,        // Gamma
  RC_XL, RC_XR,               // x[i], x[i+1] (zone edges)
  RC_DEN1,                    // 1/(a0b1g2 + a1b2g0 + a2b0g1 - a0b2g1 - a1b0g2 - a2b1g0)
  RC_DEN2,                    // 1/((x[i]-x[i+1])*(alpha[i] + Gamma[i]x[i]x[i+1] - beta[i](x[i]+x[i+1])))
  RC_XLR,                     // x[i]-x[i+1]
  RC_XL2, RC_XR2,             // SQR(x[i]), SQR(x[i+1])
  RC_XMID,                    // 0.5*(x[i]+x[i+1])
  RC_DMR, RC_DML,             // alpha + xhi*(Gamma*xhi - 2 beta), alpha + xlo*(Gamma*xlo - 2 beta)
  RC_LSM, RC_LSP, RC_LSC,     // lin_recon denominators x0-0.5(x[i]+xm), 0.5(x[i+1]+xp)-x0, xp-xm
  RC_NFIELDS
};

// FP32 reconstruction weights of one zone for the mixed-precision sweep: para_recon
// rewritten on the differences dqm = a[i]-a[i-1], dqp = a[i+1]-a[i] (the same parabola,
// well conditioned in FP32), with the geometry folded into weights computed in FP64:
//   al - a = WLM dqm + WLP dqp,  ar - a = WRM dqm + WRP dqp          (reconstruct.c:151-163)
//   second fit  A2 = EAL dl + EAR dr,  B2' = EBL dl + EBR dr  (x measured from x[i]),
//   extremum at s = -B2'/(2 A2), inside when 0 < s < DXZ, "right" when s > DXZ/2;
//   moved faces  al = a + MR dr,  ar = a + ML dl                      (reconstruct.c:174-200)
enum MixField {
  MX_WLM, MX_WLP, MX_WRM, MX_WRP, MX_EAL, MX_EAR, MX_EBL, MX_EBR, MX_DXZ, MX_MR, MX_ML,
  MX_NFIELDS
};

// Per-face and per-zone geometry of 1-D problems (one record per index i+NG).
enum GeoField {
  GF_AREA,                    // face i: area[0]
  GF_FSCALE,                  // face i: scale[1][0]
  GF_FG0, GF_FG1, GF_FG2,     // face i: gcov[1][0..2]
  GF_VOL,                     // zone i: volume
  GF_G0, GF_G1, GF_G2,        // zone i: gcov[0][0..2]
  GF_GC0, GF_GC1, GF_GC2,     // zone i: gcon[0..2]
  GF_S00,                     // zone i: scale[0][0]
  GF_CONN,                    // zone i: conn[l][m][n], 27 consecutive fields
  GF_RE2 = GF_CONN + 27,      // edge i (lower edge of zone i): SQR(redge[i]) (init_coords)
  GF_DRDX,                    // edge i: dr_dx(startx[0] + i*dx[0])
  GF_NFIELDS
};

// The connection coefficients conn[l][m][n] (index l*9+m*3+n) that the 1-D spherical
// metric can make non-zero; with every other entry exactly 0.0 the source sum over these
// nine alone, in the same order, is bit-identical to the full 27-term sum.
constexpr int NSPARSE_CONN = 9;
constexpr int SPARSE_CONN[NSPARSE_CONN] = {4, 8, 10, 12, 17, 20, 23, 24, 25};

// Device-side description of one problem.
struct ProbDev {
  int ndim, geom, eos, interp_order;
  int n1, n2;
  int bc_lo0, bc_hi0, bc_lo1, bc_hi1;
  int prob_kind;
  int has_src;              // spherical: geometric source terms are computed
  int sparse_conn;          // 1-D: only the 9 connection coefficients of SPARSE_CONN are non-zero
  int floors;               // ENFORCE_FLOORS: u_to_p clamps rho and u to the floors below
  int grav_on;              // GRAV=FIXED_GRAV: the fixed acceleration grav[] is applied
  int mono;                 // GRAV=SPHERICAL_MONOPOLE_GRAV: self-gravity, monopole approximation
  int geo_tab;              // mixed 1-D sweep: geometry from the Romberg tables (a non-uniform
                            // coordinate map), not in closed form
  int64_t mono_off;         // first zone of this problem in the monopole acceleration array
  int64_t cell_off;         // first zone of this problem in the state arrays
  int64_t ncell;            // interior zones (n1*n2 on 1-D/2-D grids; the dendritic count in 3-D)
  int64_t geo_off;          // first record (i=-NG) in the 1-D geometry tables
  int64_t rc1_off;          // first record (j=-NG) of the direction-1 recon table (2-D)
  int64_t sh_off;           // first byte of the first-stage shock bits (2-D)
  double gam, Kpoly;
  double dx0, dx1;
  double area0, area1, vol; // Cartesian 2-D constants
  double cfl, dt_init_safety, dt_grow_safety, initial_dt, dtmax, dtmin, tmax;
  double rho_floor, e_floor;
  double grav[3];           // contravariant g0
  double u1_hi[2];          // MDG_PROB_DUST: v^1 of the outer ghost zones n1, n1+1
  // 1-D geometry in closed form (mixed-precision sweep): lower edge of zone 0 and the
  // angular integrals of the 1-D spherical metric (spherical_1d_constants)
  double x0, gk_area, gk_th1, gk_th2, gk_tc;
};

// Time bookkeeping of one problem, resident on the device.
struct ProbTime {
  double t;          // time of the state
  double dt;         // dt of the step in progress / last step
  double dtold;      // main.c dtold
  double t_bc1;      // t + dt: time seen by the second-stage boundaries (bc.c:721)
  double t_next;     // ((t + dt) - dt) + dt, the reference's t after the step
  unsigned long long minacc;   // order-preserving encoding of the running min_dt
  int istep;
  int dt_ready;      // dt of the next step already finalized
  int done;          // t >= tmax: the main.c loop (main.c:206) has ended; steps leave it unchanged
  int err;           // MDG_ERR_NONFINITE once its estimate dropped below dtmin (main.c:229-238)
};

// Order-preserving map from double to uint64 so atomicMin on the integer is a min on
// the double (negative values and infinities included).
MDG_HD inline unsigned long long dbl_to_ord(double x) {
  union { double d; unsigned long long u; } c; c.d = x;
  return (c.u & 0x8000000000000000ULL) ? ~c.u : (c.u | 0x8000000000000000ULL);
}
MDG_HD inline double ord_to_dbl(unsigned long long u) {
  union { double d; unsigned long long u; } c;
  c.u = (u & 0x8000000000000000ULL) ? (u & 0x7FFFFFFFFFFFFFFFULL) : ~u;
  return c.d;
}

}  // namespace mdg
