// Fused 1-D RK stage kernel (plain FP64).
//
// One CTA advances one tile of TILE1 = 126 zones of one problem through a whole RK
// stage: it stages the 130-zone pencil (tile + 2 ghost zones each side) in shared
// memory, reconstructs every zone ONCE (the reference reconstructs each zone twice,
// once per adjacent face: step.c:501-547), solves the 127 face Riemann problems, and
// applies push() (step.c:380-470) to its 126 zones.  Boundary zones are never stored:
// they are produced on load by the boundary kinds of reset_boundaries_gpu (bc.c:705-1422)
// as index maps.  The CFL minimum (face terms step.c:560, source terms step.c:393, and in
// the second stage the zone terms of the next estimate_dt, step.c:177-187) is reduced
// per CTA with warp shuffles and folded into the problem's accumulator with one atomic.
//
// Many problems of different sizes are advanced by one launch: the grid is a list of
// (problem, tile) work items.
//
// Small problems (at most 16 tiles, 2016 zones) can instead be advanced by the resident
// stepper: one thread-block cluster per problem, one CTA per tile, runs the whole step
// sequence of many steps in one launch -- the dt rules, both RK stages and the time
// update, separated by cluster barriers -- where the per-phase path pays four dependent
// launches per step.  It runs the same tile code, so the two paths agree bit for bit.
// The FP64 reconstruction is called out of line here (one copy of para_recon in the
// kernel instead of six): the kernel is bound by instruction fetch and load latency, and
// the smaller code ran the 2048-problem ensemble 18 % faster on a B200 (same results).
#define MDG_RECON_OUTLINE 1
#include "mdg_hydro.cuh"
#include "mdg_kernels.cuh"
#include "mdg_load1d.cuh"
#include "mdg_tma.cuh"
#include "mdg_timeloop.cuh"
#include <cooperative_groups.h>

namespace mdg {

// TMA: the tile's reconstruction coefficients (all RC_TMA_ROWS rows) and face/zone geometry
// (GF_TMA_ROWS rows) arrive in shared memory by two tensor loads issued at the start,
// which overlap the state loads; otherwise every field is read from the tables in HBM
// when used.  The results are the same.
// One RK stage of one tile (run by the NT1 threads of a CTA).  tm: the tensor maps of
// the tables (a __grid_constant__ kernel parameter; not read without TMA).
template <int STAGE, bool TMA>
__device__ __forceinline__ void stage1d_tile(const ProbDev *__restrict__ probs, ProbTime *__restrict__ times,
                                             const Tile tile, const Tables &tb, const StateSoA &sst,
                                             const StateSoA &sn, const StateSoA &out, const TmaTables1d &tm)
{
  __shared__ double sv[6][NT1 + 2];     // stage-state pencil: 5 primitives + pressure
  __shared__ double sred[32];
  __shared__ __align__(128) double s_rc[TMA ? RC_TMA_ROWS : 1][TMA ? TMA_COLS1 : 1];
  __shared__ __align__(128) double s_geo[TMA ? GF_TMA_ROWS : 1][TMA ? TMA_COLS1 : 1];
  __shared__ __align__(8) uint64_t s_bar;
  // right face values of each reconstructed zone and the face fluxes; with TMA they
  // reuse the reconstruction rows, which are dead once every zone is reconstructed
  __shared__ double sar_own[TMA ? 1 : 6][NT1];
  __shared__ double sfl_own[TMA ? 1 : NPRIM][NT1];
  static_assert(!TMA || (6 + NPRIM) * NT1 <= RC_TMA_ROWS * TMA_COLS1, "exchange buffers fit the recon rows");
  double (*sar)[NT1] = TMA ? reinterpret_cast<double(*)[NT1]>(&s_rc[0][0]) : sar_own;
  double (*sfl)[NT1] = TMA ? reinterpret_cast<double(*)[NT1]>(&s_rc[0][0] + 6 * NT1) : sfl_own;

  if (times[tile.prob].done) return;   // past tmax: the time loop has ended (CTA-uniform)
  const ProbDev &P = probs[tile.prob];
  const double dt = times[tile.prob].dt;
  const double t_bc = STAGE ? times[tile.prob].t_bc1 : times[tile.prob].t;
  const int t = threadIdx.x;
  const int n1 = P.n1;
  const int z = tile.i0 - 1 + t;           // zone reconstructed by this thread
  const double *rc = tb.rc0;
  const int64_t rcs = tb.rc0_stride;
  const double *geo = tb.geo;
  const int64_t gs = tb.geo_stride;
  // first table column of the box: the column of zone i0-1 rounded down to even (TMA
  // start coordinates are 16-byte aligned); a table column c sits at box column c - bx
  const int64_t bx = (P.geo_off + NG + tile.i0 - 1) & ~int64_t(1);
  if (TMA) {
    if (t == 0) mbar_init(&s_bar, 1);
    __syncthreads();
    if (t == 0) {
      mbar_arrive_expect_tx(&s_bar, (unsigned)((RC_TMA_ROWS + GF_TMA_ROWS) * TMA_COLS1 * sizeof(double)));
      tma_load_2d(&s_rc[0][0], &tm.rc, (int)bx, 0, &s_bar);
      tma_load_2d(&s_geo[0][0], &tm.geo, (int)bx, 0, &s_bar);
    }
  }
  // geometry field f of table column c (faces and zones of this tile)
  auto gf = [&](int f, int64_t c) -> double {
    if (TMA) return s_geo[f][c - bx];
    return __ldg(geo + f * gs + c);
  };

  double w[6];
  load_cell_1d(P, sst, rc, rcs, z, t_bc, w);
#pragma unroll
  for (int v = 0; v < 6; v++) sv[v][t + 1] = w[v];
  if (t == 0) {
    double w2[6];
    load_cell_1d(P, sst, rc, rcs, tile.i0 - 2, t_bc, w2);
#pragma unroll
    for (int v = 0; v < 6; v++) sv[v][0] = w2[v];
  }
  if (t == NT1 - 1) {
    double w2[6];
    load_cell_1d(P, sst, rc, rcs, tile.i0 + NT1 - 1, t_bc, w2);
#pragma unroll
    for (int v = 0; v < 6; v++) sv[v][NT1 + 1] = w2[v];
  }
  if (TMA) {
    // the tables have landed (bounded wait: a copy that never completes flags the
    // problem and the CTA leaves after waiting once more, as bounded)
    const bool ok = mbar_wait(&s_bar, 0);
    if (__syncthreads_or(!ok)) {
      if (t == 0) times[tile.prob].err = MDG_ERR_INTERNAL;
      mbar_wait(&s_bar, 0);
      return;
    }
  }
  __syncthreads();

  // reconstruct zone z once (interp(), reconstruct.c:225-279); Gamma is the constant
  // adiabatic index, which every order reconstructs to itself.
  double al[7], ar[7];
  {
    int zc = z < -1 ? -1 : (z > n1 ? n1 : z);
    const int64_t c = P.geo_off + zc + NG;
    const RcView<double, !TMA> g{TMA ? &s_rc[0][c - bx] : rc + c, TMA ? (int64_t)TMA_COLS1 : rcs};
#pragma unroll kReconUnroll
    for (int v = 0; v < 6; v++) recon_zone<double>(P.interp_order, sv[v][t], sv[v][t + 1], sv[v][t + 2], g, al[v], ar[v]);
    al[6] = P.gam; ar[6] = P.gam;
  }
  if (TMA) __syncthreads();   // every zone reconstructed: the recon rows may be overwritten
#pragma unroll
  for (int v = 0; v < 6; v++) sar[v][t] = ar[v];
  __syncthreads();

  double lmin = 1.0e300;
  double smax = 0.0, nmin = 1.0e300, lmax = 0.0;
  const GamConst<double> gc = gam_const(P.gam);
  // face z: between zones z-1 and z (pl = right state of z-1, pr = left state of z)
  const bool face_ok = (t >= 1) && (z >= 0) && (z <= n1);
  if (t >= 1) {
    double pl[7], flux[NPRIM], sig;
#pragma unroll
    for (int v = 0; v < 6; v++) pl[v] = sar[v][t - 1];
    pl[6] = P.gam;
    FaceGeom<double> fg;
    int zf = z < 0 ? 0 : (z > n1 ? n1 : z);
    const int64_t gi = P.geo_off + zf + NG;
    fg.area = gf(GF_AREA, gi);
    fg.scale = gf(GF_FSCALE, gi);
    fg.g0 = gf(GF_FG0, gi);
    fg.g1 = gf(GF_FG1, gi);
    fg.g2 = gf(GF_FG2, gi);
    riemann_hllc<0, false, double>(pl, al, fg, gc, flux, sig);
#pragma unroll
    for (int v = 0; v < NPRIM; v++) sfl[v][t] = flux[v];
    if (face_ok) smax = tmax(smax, fabs(sig));
  }
  __syncthreads();

  // push() for zone z (step.c:380-470)
  if (t >= 1 && t <= NT1 - 2 && z >= 0 && z < n1) {
    const int64_t gi = P.geo_off + z + NG;
    const int64_t cell = P.cell_off + z;
    double ph[NPRIM], pn[NPRIM], u[NPRIM], uh[NPRIM], src[NPRIM], divF[NPRIM], pf[NPRIM];
#pragma unroll
    for (int v = 0; v < NPRIM; v++) ph[v] = sv[v][t + 1];
    if (STAGE == 0) {
#pragma unroll
      for (int v = 0; v < NPRIM; v++) pn[v] = ph[v];
    } else {
#pragma unroll
      for (int v = 0; v < NPRIM; v++) pn[v] = sn.v[v][cell];
    }
    const double gc0 = gf(GF_G0, gi), gc1 = gf(GF_G1, gi), gc2 = gf(GF_G2, gi);
    // geometric source terms from the stage state (rad_fluid.c:164-192, fluid.c:56-73)
    if (P.has_src) {
      geo_sources_1d(geo, gs, gi, P.sparse_conn != 0, ph, sv[5][t + 1], gc0, gc1, gc2, src);
    } else {
#pragma unroll
      for (int v = 0; v < NPRIM; v++) src[v] = 0.0;
    }
    if (P.grav_on) add_fixed_gravity(ph, P.grav, gc0, gc1, gc2, 1, src);
    if (P.mono) {
      // mass flux density at the outer and inner face (gravity.c:380-401)
      double vr = 0.0, area = 0.0;
      vr += sfl[RHO][t + 1];
      area += gf(GF_AREA, gi + 1) + 1.0e-16;
      vr /= area;
      const double vl = sfl[RHO][t] / (gf(GF_AREA, gi) + 1.0e-16);
      add_monopole_gravity(ph[RHO], tb.gmono[P.mono_off + z], vl, vr, P.x0 + z * P.dx0, P.dx0,
                           __ldg(rc + RC_B0 * rcs + gi), __ldg(rc + RC_G0 * rcs + gi), src);
    }
    p_to_u(pn, u, gc0, gc1, gc2);
    p_to_u(ph, uh, gc0, gc1, gc2);
    if (P.has_src || P.grav_on || P.mono) lmin = tmin(lmin, dt_source_control(pn, u, src));
    else nmin = tmin(nmin, src_dt_numerator_min(pn, u));   // zero sources: shared denominator
#pragma unroll
    for (int v = 0; v < NPRIM; v++) { divF[v] = 0.0; divF[v] += sfl[v][t + 1]; divF[v] -= sfl[v][t]; }
    const double vol = gf(GF_VOL, gi);
    const double pfact = STAGE ? 0.5 : 1.0, phfact = STAGE ? 0.5 : 0.0, ffact = STAGE ? 0.5 : 1.0;
#pragma unroll
    for (int v = 0; v < NPRIM; v++) {
      double ddt = divF[v] / vol - src[v];
      u[v] = pfact * u[v] + phfact * uh[v] - ffact * dt * ddt;
    }
    u_to_p(u, pf, gf(GF_GC0, gi), gf(GF_GC1, gi), gf(GF_GC2, gi), P.floors != 0, P.rho_floor, P.e_floor);
#pragma unroll
    for (int v = 0; v < NPRIM; v++) out.v[v][cell] = pf[v];
    flag_nonfinite(pf, &times[tile.prob]);
    if (STAGE == 1) {
      // zone term of the next estimate_dt (step.c:177-187): velocity of the new state,
      // sound speed of the stage state (sim_eos was last filled from sim_ph)
      const double cs = sqrt(P.gam * sv[5][t + 1] / ph[RHO]);
      double local_dt = 0.0;
      local_dt += (fabs(pf[U1]) + cs / gf(GF_S00, gi)) / P.dx0;
      lmax = tmax(lmax, local_dt);
    }
  }
  // min of dx/|sig| over faces, of the zero-source limits and of 1/local_dt, each taken
  // on its numerator or denominator (monotone division, see src_dt_numerator_min)
  lmin = tmin(lmin, P.dx0 / smax);
  lmin = tmin(lmin, src_dt_from_numerator(nmin));
  if (STAGE == 1) lmin = tmin(lmin, 1.0 / lmax);
  block_min_to(lmin, &times[tile.prob].minacc, sred);
}

template <int STAGE, bool TMA>
__global__ void __launch_bounds__(NT1)
stage1d_kernel(const ProbDev *__restrict__ probs, ProbTime *__restrict__ times,
               const Tile *__restrict__ tiles, Tables tb, StateSoA sst, StateSoA sn, StateSoA out,
               const __grid_constant__ TmaTables1d tm)
{
  stage1d_tile<STAGE, TMA>(probs, times, tiles[blockIdx.x], tb, sst, sn, out, tm);
}

// The resident stepper: nsteps steps of every problem, cluster c advancing problem c with
// CTA r on the tile of zones [126 r, 126 r + 126) (CTAs past the last zone only take part
// in the barriers).  Each step: the dt rules (one thread), stage 0 (p -> ph), stage 1
// (ph, p -> p), the time update (one thread); a cluster barrier after the dt rules and
// after each stage orders the state, the time record and the CFL accumulator between the
// CTAs (release/acquire at cluster scope).  Every CTA of a cluster takes the same
// barriers: the loop runs nsteps iterations unless the problem's loop has ended (t >=
// tmax), which every CTA reads from the time record after the same barrier -- the next
// write of that flag comes two barriers later -- so all leave together; the lead then
// closes the step as the time update would (a step past the end changes nothing else).
__global__ void __launch_bounds__(NT1)
resident1d_kernel(const ProbDev *__restrict__ probs, ProbTime *__restrict__ times, Tables tb, StateSoA p,
                  StateSoA ph, int nsteps, int *err, const __grid_constant__ TmaTables1d none)
{
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int m = (int)(blockIdx.x / cl.num_blocks());
  const Tile tile{m, rank * TILE1, 0, 0};
  const bool active = tile.i0 < probs[m].n1;
  const bool lead = rank == 0 && threadIdx.x == 0;
  for (int k = 0; k < nsteps; k++) {
    if (lead) dt_finalize_one(probs[m], times + m, err);
    cl.sync();
    if (times[m].done) {
      if (lead) finish_one(times + m);
      break;
    }
    if (active) stage1d_tile<0, false>(probs, times, tile, tb, p, p, ph, none);
    cl.sync();
    if (active) stage1d_tile<1, false>(probs, times, tile, tb, ph, p, p, none);
    cl.sync();
    if (lead) finish_one(times + m);
  }
}

static cudaLaunchConfig_t resident1d_config(int cs, int nprob, cudaStream_t st, cudaLaunchAttribute *attr)
{
  cudaLaunchConfig_t c = {};
  c.gridDim = dim3((unsigned)(cs * nprob), 1, 1);
  c.blockDim = dim3(NT1, 1, 1);
  c.dynamicSmemBytes = 0;
  c.stream = st;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  c.attrs = attr;
  c.numAttrs = 1;
  return c;
}

int resident1d_cluster_size(int max_tiles)
{
  if (max_tiles < 1 || max_tiles > RESIDENT1D_MAX_TILES) return 0;
  int cs = 1;
  while (cs < max_tiles) cs <<= 1;
  if (cs > 8 && cudaFuncSetAttribute(resident1d_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                    cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cudaLaunchAttribute attr[1];
  const cudaLaunchConfig_t c = resident1d_config(cs, 1, nullptr, attr);
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, (const void *)resident1d_kernel, &c) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n >= 1 ? cs : 0;
}

cudaError_t launch_resident1d(int cs, int nprob, const ProbDev *probs, ProbTime *times, const Tables &tb,
                              StateSoA p, StateSoA ph, int nsteps, int *err, cudaStream_t st)
{
  if (nsteps <= 0 || nprob <= 0) return cudaSuccess;
  cudaLaunchAttribute attr[1];
  const cudaLaunchConfig_t c = resident1d_config(cs, nprob, st, attr);
  static const TmaTables1d none{};
  return cudaLaunchKernelEx(&c, resident1d_kernel, probs, times, tb, p, ph, nsteps, err, none);
}

void launch_stage1d(int stage, const ProbDev *probs, ProbTime *times, const Tile *tiles, int ntiles,
                    const Tables &tb, StateSoA sst, StateSoA sn, StateSoA out, cudaStream_t st,
                    const TmaTables1d *tm)
{
  if (ntiles <= 0) return;
  static const TmaTables1d none{};
  const bool tma = tm && tm->valid;
  const TmaTables1d &m = tma ? *tm : none;
  if (stage == 0 && tma) stage1d_kernel<0, true><<<ntiles, NT1, 0, st>>>(probs, times, tiles, tb, sst, sn, out, m);
  else if (stage == 0) stage1d_kernel<0, false><<<ntiles, NT1, 0, st>>>(probs, times, tiles, tb, sst, sn, out, m);
  else if (tma) stage1d_kernel<1, true><<<ntiles, NT1, 0, st>>>(probs, times, tiles, tb, sst, sn, out, m);
  else stage1d_kernel<1, false><<<ntiles, NT1, 0, st>>>(probs, times, tiles, tb, sst, sn, out, m);
}

}  // namespace mdg
