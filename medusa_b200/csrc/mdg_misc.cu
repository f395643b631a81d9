// Small kernels around the sweep: time-step control (estimate_dt + main.c rules), time
// bookkeeping, the first estimate before step 0, and AoS <-> SoA staging of the state.
#include "mdg_hydro.cuh"
#include "mdg_kernels.cuh"
#include "mdg_timeloop.cuh"

namespace mdg {

// estimate_dt() + the main.c dt rules (dt_finalize_one), one thread per problem.
__global__ void dt_finalize_kernel(const ProbDev *__restrict__ probs, ProbTime *__restrict__ times, int nprob,
                                   int *err)
{
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nprob) return;
  dt_finalize_one(probs[m], times + m, err);
}

// estimate_dt() (step.c:192-198) alone: what it leaves in the reference's global dt.
__global__ void raw_estimate_kernel(const ProbDev *__restrict__ probs, const ProbTime *__restrict__ times, int nprob,
                                    double *__restrict__ out)
{
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nprob) return;
  const ProbDev &P = probs[m];
  const ProbTime &T = times[m];
  double min_dt = ord_to_dbl(T.minacc);
  if (T.istep == 0) min_dt = tmin(min_dt, P.initial_dt);
  min_dt = tmin(min_dt, P.dtmax);
  min_dt *= P.cfl;
  out[m] = min_dt;
}

// The time record of one step() with a dt chosen by the host's own time loop: the
// boundary times of reset_boundaries_gpu (bc.c:721, 1418) and main.c's t += dt.
__global__ void set_dt_kernel(ProbTime *__restrict__ times, int nprob, const double *__restrict__ dts)
{
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nprob) return;
  ProbTime T = times[m];
  const double dt = dts[m];
  T.dt = dt;
  T.dtold = dt;
  T.t_bc1 = T.t + dt;
  T.t_next = (T.t_bc1 - dt) + dt;
  T.minacc = dbl_to_ord(1.0e100);
  T.done = 0;
  T.dt_ready = 1;
  times[m] = T;
}

void launch_raw_estimate(const ProbDev *probs, const ProbTime *times, int nprob, double *out, cudaStream_t st)
{
  raw_estimate_kernel<<<(nprob + 127) / 128, 128, 0, st>>>(probs, times, nprob, out);
}

void launch_set_dt(ProbTime *times, int nprob, const double *dt, cudaStream_t st)
{
  set_dt_kernel<<<(nprob + 127) / 128, 128, 0, st>>>(times, nprob, dt);
}

__global__ void finish_kernel(ProbTime *__restrict__ times, int nprob)
{
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nprob) return;
  finish_one(times + m);
}

// monopole_gravity_start/finish (gravity.c:145-425, GR_MONOPOLE=FALSE) of a 1-D problem,
// one thread per problem, in the reference's serial order: shell masses vol*rho of the
// stage state, enclosed mass mr at the radial edges, g = -G mr / r^2 dr/dx there
// (g = 0 at the inner edge), interpolated linearly to each zone centroid.
__global__ void monopole1d_kernel(const ProbDev *__restrict__ probs, ProbTime *__restrict__ times, int nprob,
                                  Tables tb, StateSoA s)
{
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nprob) return;
  const ProbDev &P = probs[m];
  if (!P.mono || times[m].done) return;
  const double *geo = tb.geo;
  const int64_t gs = tb.geo_stride, rcs = tb.rc0_stride;
  double mr = 0.0, gl = 0.0;
  for (int ii = 0; ii < P.n1; ii++) {
    const int64_t gi = P.geo_off + ii + NG;
    double ms = 0.0;
    ms += __ldg(geo + GF_VOL * gs + gi) * s.v[RHO][P.cell_off + ii];
    mr = mr + ms;
    const double gr = -GNEWT * mr / __ldg(geo + GF_RE2 * gs + gi + 1) * __ldg(geo + GF_DRDX * gs + gi + 1);
    const double x0l = P.x0 + ii * P.dx0;
    tb.gmono[P.mono_off + ii] = monopole_centroid(gl, gr, x0l, P.dx0, __ldg(tb.rc0 + RC_B0 * rcs + gi),
                                                  __ldg(tb.rc0 + RC_G0 * rcs + gi));
    gl = gr;
  }
}

void launch_monopole1d(const ProbDev *probs, ProbTime *times, int nprob, const Tables &tb, StateSoA s,
                       cudaStream_t st)
{
  monopole1d_kernel<<<(nprob + 127) / 128, 128, 0, st>>>(probs, times, nprob, tb, s);
}

// First estimate_dt() of a problem (step.c:171-187 with firstc): zone terms of the
// initial state with its own EOS (main.c:180-182 fills sim_eos from sim_p).
__device__ __forceinline__ void initial_estimate_block(const ProbDev *__restrict__ probs,
                                                      ProbTime *__restrict__ times, int m, const Tables &tb,
                                                      const StateSoA &s)
{
  __shared__ double sred[32];
  const ProbDev &P = probs[m];
  const int64_t ncell = P.ncell;
  const int64_t z = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double lmin = 1.0e300;
  if (z < ncell) {
    const int64_t c = P.cell_off + z;
    const double rho = s.v[RHO][c], uu = s.v[UU][c];
    const double press = eos_press(P.eos, P.gam, P.Kpoly, rho, uu);
    const double cs = sqrt(P.gam * press / rho);
    double local_dt = 0.0;
    if (P.ndim == 1) {
      const double s00 = __ldg(tb.geo + GF_S00 * tb.geo_stride + P.geo_off + z + NG);
      local_dt += (fabs(s.v[U1][c]) + cs / s00) / P.dx0;
      lmin = tmin(lmin, 1.0 / local_dt);
    } else {
      local_dt += (fabs(s.v[U1][c]) + cs) / P.dx0;
      lmin = tmin(lmin, 1.0 / local_dt);
      local_dt += (fabs(s.v[U2][c]) + cs) / P.dx1;
      lmin = tmin(lmin, 1.0 / local_dt);
    }
  }
  block_min_to(lmin, &times[m].minacc, sred);
}

__global__ void initial_estimate_kernel(const ProbDev *__restrict__ probs, ProbTime *__restrict__ times, int m,
                                        Tables tb, StateSoA s)
{
  initial_estimate_block(probs, times, m, tb, s);
}

// The same for problems m0 .. m0+gridDim.y-1 at once (blocks beyond a problem's zones
// return as a whole, before any barrier).
__global__ void initial_estimate_many_kernel(const ProbDev *__restrict__ probs, ProbTime *__restrict__ times,
                                             int m0, Tables tb, StateSoA s)
{
  const int m = m0 + blockIdx.y;
  const ProbDev &P = probs[m];
  if ((int64_t)blockIdx.x * blockDim.x >= P.ncell) return;
  initial_estimate_block(probs, times, m, tb, s);
}

__global__ void reset_time_all_kernel(ProbTime *times, int nprob)
{
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nprob) return;
  ProbTime T;
  T.t = 0.0; T.dt = 0.0; T.dtold = 1.0e100; T.t_bc1 = 0.0; T.t_next = 0.0;
  T.minacc = dbl_to_ord(1.0e100);
  T.istep = 0; T.dt_ready = 0; T.done = 0; T.err = 0;
  times[m] = T;
}

__global__ void reset_time_kernel(ProbTime *times, int m)
{
  ProbTime T;
  T.t = 0.0; T.dt = 0.0; T.dtold = 1.0e100; T.t_bc1 = 0.0; T.t_next = 0.0;
  T.minacc = dbl_to_ord(1.0e100);
  T.istep = 0; T.dt_ready = 0; T.done = 0; T.err = 0;
  times[m] = T;
}

__global__ void aos_to_soa_kernel(const double *__restrict__ aos, StateSoA s, int64_t off, int64_t n)
{
  const int64_t z = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= n) return;
#pragma unroll
  for (int v = 0; v < NPRIM; v++) s.v[v][off + z] = aos[z * NPRIM + v];
}

__global__ void soa_to_aos_kernel(StateSoA s, int64_t off, int64_t n, double *__restrict__ aos)
{
  const int64_t z = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= n) return;
#pragma unroll
  for (int v = 0; v < NPRIM; v++) aos[z * NPRIM + v] = s.v[v][off + z];
}

// EOS record of each zone (PRESS, CS, TEMP, ENT, GAMMA), eos_gamma.c:45-58 / eos_poly.c:56-69
__device__ __forceinline__ void eos_record(const StateSoA &s, const ProbDev &P, int64_t off, int64_t z,
                                           double *__restrict__ aos)
{
  const double rho = s.v[RHO][off + z], uu = s.v[UU][off + z];
  const double press = eos_press(P.eos, P.gam, P.Kpoly, rho, uu);
  const double cs = sqrt(P.gam * press / rho);
  const double kb = 1.3806488e-16, mp = 1.67262158e-24, me = 9.10938291e-28;
  const double tp = (P.eos == 0) ? press / (2.0 * rho * kb) * (mp + me) : press / (rho * kb) * mp;
  aos[z * 5 + 0] = press;
  aos[z * 5 + 1] = cs;
  aos[z * 5 + 2] = tp;
  aos[z * 5 + 3] = 0.0;
  aos[z * 5 + 4] = P.gam;
}

__global__ void eos_aos_kernel(StateSoA s, const ProbDev *__restrict__ probs, int m, int64_t off, int64_t n,
                               double *__restrict__ aos)
{
  const int64_t z = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= n) return;
  eos_record(s, probs[m], off, z, aos);
}

// The same with the EOS source chosen on the device: the stage state PH once a step has
// been taken (sim_eos was last filled by update_eos(sim_ph)), else the state P.
__global__ void eos_aos_sel_kernel(StateSoA p, StateSoA ph, const ProbDev *__restrict__ probs,
                                   const ProbTime *__restrict__ times, int m, int64_t off, int64_t n,
                                   double *__restrict__ aos)
{
  const int64_t z = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= n) return;
  eos_record(times[m].istep > 0 ? ph : p, probs[m], off, z, aos);
}

void launch_eos_aos_sel(StateSoA p, StateSoA ph, const ProbDev *probs, const ProbTime *times, int m, int64_t off,
                        int64_t n, double *aos, cudaStream_t st)
{
  if (n <= 0) return;
  eos_aos_sel_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(p, ph, probs, times, m, off, n, aos);
}

// Neumaier's compensated summation: s + c carries the sum of the added terms with an
// error independent of their number (to first order).
__device__ __forceinline__ void neumaier_add(double &s, double &c, double x)
{
  const double t = s + x;
  if (fabs(s) >= fabs(x)) c += (s - t) + x;
  else c += (x - t) + s;
  s = t;
}

// Mass and total energy of each problem (one CTA per problem): the integrands of
// calculate_total_mass / calculate_total_energy (utils.c:2337-2361, 2581-2612) summed
// with compensation per thread and then over the threads in a fixed order.
__global__ void conserved_totals_kernel(const ProbDev *__restrict__ probs, Tables tb, StateSoA s,
                                        double *__restrict__ out)
{
  __shared__ double sh[4][256];
  const int m = blockIdx.x;
  const int t = threadIdx.x;
  const ProbDev &P = probs[m];
  const int64_t n = P.ncell;
  double ms = 0.0, mc = 0.0, es = 0.0, ec = 0.0;
  for (int64_t z = t; z < n; z += blockDim.x) {
    const int64_t c = P.cell_off + z;
    double p[NPRIM], u[NPRIM];
#pragma unroll
    for (int v = 0; v < NPRIM; v++) p[v] = s.v[v][c];
    double vol = P.vol, g0 = 1.0, g1 = 1.0, g2 = 1.0;
    if (P.ndim == 1) {
      const int64_t gi = P.geo_off + z + NG;
      vol = tb.geo[GF_VOL * tb.geo_stride + gi];
      g0 = tb.geo[GF_G0 * tb.geo_stride + gi];
      g1 = tb.geo[GF_G1 * tb.geo_stride + gi];
      g2 = tb.geo[GF_G2 * tb.geo_stride + gi];
    }
    p_to_u(p, u, g0, g1, g2);
    neumaier_add(ms, mc, p[RHO] * vol);
    neumaier_add(es, ec, u[UU] * vol);
  }
  sh[0][t] = ms; sh[1][t] = mc; sh[2][t] = es; sh[3][t] = ec;
  __syncthreads();
  if (t == 0) {
    double S = 0.0, C = 0.0, E = 0.0, D = 0.0;
    for (int k = 0; k < (int)blockDim.x; k++) {
      neumaier_add(S, C, sh[0][k]); C += sh[1][k];
      neumaier_add(E, D, sh[2][k]); D += sh[3][k];
    }
    out[2 * m] = S + C;
    out[2 * m + 1] = E + D;
  }
}

void launch_conserved_totals(const ProbDev *probs, int nprob, const Tables &tb, StateSoA s, double *out,
                             cudaStream_t st)
{
  if (nprob <= 0) return;
  conserved_totals_kernel<<<nprob, 256, 0, st>>>(probs, tb, s, out);
}

void launch_dt_finalize(const ProbDev *probs, ProbTime *times, int nprob, int *err, cudaStream_t st)
{
  dt_finalize_kernel<<<(nprob + 127) / 128, 128, 0, st>>>(probs, times, nprob, err);
}

void launch_finish(ProbTime *times, int nprob, cudaStream_t st)
{
  finish_kernel<<<(nprob + 127) / 128, 128, 0, st>>>(times, nprob);
}

void launch_reset_time(ProbTime *times, int m, cudaStream_t st)
{
  reset_time_kernel<<<1, 1, 0, st>>>(times, m);
}

void launch_initial_estimate_one(const ProbDev *probs, ProbTime *times, int m, int64_t ncell,
                                 const Tables &tb, StateSoA s, cudaStream_t st)
{
  const int nb = (int)((ncell + 255) / 256);
  initial_estimate_kernel<<<nb, 256, 0, st>>>(probs, times, m, tb, s);
}

void launch_reset_time_all(ProbTime *times, int nprob, cudaStream_t st)
{
  if (nprob > 0) reset_time_all_kernel<<<(nprob + 127) / 128, 128, 0, st>>>(times, nprob);
}

void launch_initial_estimate_all(const ProbDev *probs, ProbTime *times, int nprob, int64_t max_cells,
                                 const Tables &tb, StateSoA s, cudaStream_t st)
{
  const unsigned nb = (unsigned)((max_cells + 255) / 256);
  for (int m0 = 0; m0 < nprob; m0 += 65535) {
    const int k = (nprob - m0 < 65535) ? nprob - m0 : 65535;
    initial_estimate_many_kernel<<<dim3(nb, k), 256, 0, st>>>(probs, times, m0, tb, s);
  }
}

void launch_aos_to_soa(const double *aos, StateSoA s, int64_t off, int64_t n, cudaStream_t st)
{
  if (n <= 0) return;
  aos_to_soa_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(aos, s, off, n);
}

void launch_soa_to_aos(StateSoA s, int64_t off, int64_t n, double *aos, cudaStream_t st)
{
  if (n <= 0) return;
  soa_to_aos_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(s, off, n, aos);
}

void launch_eos_aos_m(StateSoA s, const ProbDev *probs, int m, int64_t off, int64_t n, double *aos, cudaStream_t st)
{
  if (n <= 0) return;
  eos_aos_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(s, probs, m, off, n, aos);
}

}  // namespace mdg
