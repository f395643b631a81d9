// mdg_advance_1d_noalloc: the 1-D sweep for callers that cannot allocate device memory.
//
// Who needs this: code that runs where cudaMalloc is not available or not allowed --
// a host that has handed all device memory to its own pool allocator and forbids other
// allocations, a real-time or interrupt-driven control loop in which cudaMalloc's
// implicit device synchronisation and unbounded latency are unacceptable, or an
// embedding that must not grow the process's device footprint after start-up.  Such a
// caller owns its input and output buffers; everything else the sweep needs between its
// kernels (the RK stage state, the geometry tables, the per-problem time and CFL
// accumulators, the tile list) lives in ONE file-scope device array below, which every
// GPU that loads this library holds until the process exits.
//
// Limits and rules (also stated in include/medusa_b200.h):
//  * one 1-D problem per call, at most MDG_NOALLOC_MAX_ZONES zones, plain FP64;
//  * the scratch array is shared by every call in the process: calls whose work overlaps
//    on the GPU (different streams, different host threads) race and corrupt each other;
//  * the first call on a device resolves the array's device address with
//    cudaGetSymbolAddress (device set-up); make that first call before any stream capture;
//  * the array keeps the previous call's contents: each call re-initialises everything it
//    reads (time record, error flag, tables, tile list) before use;
//  * every call waits for its own work on the stream before it returns: it reads back the
//    problem's time record and error flag and reports a non-finite state or a dt below
//    dtmin as MDG_ERR_NONFINITE, as mdg_synchronize does for the allocating path;
//  * the host-side staging of the tables is one process-wide set, held under a lock from
//    the table build until its copies have landed, so calls from different host threads
//    (on one GPU or on several) never share it while it is in use.
// This entry point calls no cudaMalloc, cudaFree or other allocating library routine.
#include <cuda_runtime.h>
#include <cstring>
#include <mutex>
#include "mdg_internal.h"
#include "mdg_kernels.cuh"

namespace mdg {
void make_probdev(const mdg_problem_desc &d, ProbDev &P);
void build_recon_table_into(const mdg_problem_desc &d, int dir, double *tab, int64_t stride, int64_t off,
                            double *al, double *be, double *ga);
void build_geo_1d(const mdg_problem_desc &d, double *tab, int64_t stride, int64_t off);
int conn_is_sparse(const double *tab, int64_t stride, int64_t off, int nrec);
}

using namespace mdg;

namespace {

constexpr int64_t NMAX = MDG_NOALLOC_MAX_ZONES;
constexpr int64_t NCOL = NMAX + 2 * NG;                    // table columns (zones + ghosts)
constexpr int64_t MAX_TILES = (NMAX + TILE1 - 1) / TILE1;

// byte layout of the scratch array (every block 256-byte aligned)
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t OFF_PH = 0;                                                  // stage state [5][NMAX]
constexpr size_t OFF_RC = align256(OFF_PH + sizeof(double) * NPRIM * NMAX);   // RC_NFIELDS x NCOL
constexpr size_t OFF_GEO = align256(OFF_RC + sizeof(double) * RC_NFIELDS * NCOL);  // GF_NFIELDS x NCOL
constexpr size_t OFF_PROB = align256(OFF_GEO + sizeof(double) * GF_NFIELDS * NCOL);
constexpr size_t OFF_TIME = align256(OFF_PROB + sizeof(ProbDev));
constexpr size_t OFF_TILES = align256(OFF_TIME + sizeof(ProbTime));
constexpr size_t OFF_ERR = align256(OFF_TILES + sizeof(Tile) * MAX_TILES);
constexpr size_t SCRATCH_BYTES = align256(OFF_ERR + sizeof(int));

}  // namespace

// The scratch: ~4.4 MB per device for MDG_NOALLOC_MAX_ZONES = 8192.
static __device__ __align__(256) unsigned char mdg_noalloc_scratch[SCRATCH_BYTES];

namespace {

constexpr int MAX_DEVICES = 64;
unsigned char *g_scratch[MAX_DEVICES] = {nullptr};
std::mutex g_setup_mutex;
std::mutex g_staging_mutex;   // held while the host staging below is filled and copied

// Host staging of the tables (host memory reserved at load time, not allocated per call).
double h_rc[RC_NFIELDS * NCOL];
double h_geo[GF_NFIELDS * NCOL];
Tile h_tiles[MAX_TILES];
double h_al[NCOL], h_be[NCOL], h_ga[NCOL];
// Failures are reported by status code only (the message text documents the cause).
int fail(int code, const char *why)
{
  (void)why;
  return code;
}

int check_desc(const mdg_problem_desc &d)
{
  if (d.ndim != 1) return fail(MDG_ERR_INVALID, "mdg_advance_1d_noalloc: ndim must be 1");
  if (d.n1 < 2) return fail(MDG_ERR_INVALID, "mdg_advance_1d_noalloc: n1 must be at least 2");
  if (d.n1 > NMAX)
    return fail(MDG_ERR_OUTOFMEM, "mdg_advance_1d_noalloc: n1 exceeds MDG_NOALLOC_MAX_ZONES: does not fit the scratch");
  if (d.geom != MDG_CARTESIAN && d.geom != MDG_SPHERICAL) return fail(MDG_ERR_INVALID, "mdg_advance_1d_noalloc: geom");
  if (d.eos != MDG_GAMMA_LAW && d.eos != MDG_POLYTROPIC) return fail(MDG_ERR_INVALID, "mdg_advance_1d_noalloc: eos");
  if (d.hydro_interp_order < 1 || d.hydro_interp_order > 3)
    return fail(MDG_ERR_INVALID, "mdg_advance_1d_noalloc: hydro_interp_order");
  if (!(d.dx[0] > 0.0) || !(d.gam > 1.0) || !(d.cfl > 0.0))
    return fail(MDG_ERR_INVALID, "mdg_advance_1d_noalloc: dx, gam or cfl");
  const int lo = d.bc_lo[0], hi = d.bc_hi[0];
  const bool sph = d.geom == MDG_SPHERICAL, noh = d.prob_kind == MDG_PROB_NOH;
  const bool lo_ok = lo == MDG_BC_OUTFLOW || lo == MDG_BC_REFLECT || lo == MDG_BC_EXTRAP ||
                     lo == MDG_BC_PERIODIC || (lo == MDG_BC_PROB && sph && noh) ||
                     (lo == MDG_BC_SPHERICAL_ORIGIN && sph);
  const bool hi_ok = hi == MDG_BC_OUTFLOW || hi == MDG_BC_REFLECT || hi == MDG_BC_EXTRAP ||
                     hi == MDG_BC_PERIODIC || (hi == MDG_BC_PROB && sph && noh);
  if (!lo_ok || !hi_ok) return fail(MDG_ERR_NOTIMPL, "mdg_advance_1d_noalloc: boundary kinds");
  if ((lo == MDG_BC_PERIODIC) != (hi == MDG_BC_PERIODIC))
    return fail(MDG_ERR_INVALID, "mdg_advance_1d_noalloc: periodic boundaries must be paired");
  if (d.rcoord != MDG_RCOORD_UNIFORM && d.rcoord != MDG_RCOORD_SINH && d.rcoord != MDG_RCOORD_SINH_MODIFIED)
    return fail(MDG_ERR_INVALID, "mdg_advance_1d_noalloc: rcoord");
  if (d.thcoord != MDG_THCOORD_UNIFORM && (d.thcoord != MDG_THCOORD_POLYTH || !sph || !(d.poly_xt > 0.0) ||
                                           !(d.poly_alpha >= 1.0)))
    return fail(MDG_ERR_INVALID, "mdg_advance_1d_noalloc: thcoord");
  if (d.rcoord == MDG_RCOORD_SINH_MODIFIED && !(d.rfact[2] != 0.0))
    return fail(MDG_ERR_INVALID, "mdg_advance_1d_noalloc: factc");
  if (d.monopole != 0 || d.prob_kind == MDG_PROB_DUST)
    return fail(MDG_ERR_NOTIMPL, "mdg_advance_1d_noalloc: monopole gravity and the dust-collapse hook are not built here");
  if (d.rcoord != MDG_RCOORD_UNIFORM && (!sph || !(d.rtrans > 0.0) || lo == MDG_BC_PROB || hi == MDG_BC_PROB))
    return fail(MDG_ERR_INVALID, "mdg_advance_1d_noalloc: the SINH radial map needs a spherical grid, rtrans > 0 "
                                 "and no PROB boundary");
  return MDG_OK;
}

// Device set-up, once per device, with that device current.
int scratch_of_current_device(unsigned char **out)
{
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(MDG_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= MAX_DEVICES) return fail(MDG_ERR_INVALID, "mdg_advance_1d_noalloc: device ordinal");
  std::lock_guard<std::mutex> lk(g_setup_mutex);
  if (!g_scratch[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, mdg_noalloc_scratch);
    if (e != cudaSuccess || !p) return fail(MDG_ERR_CUDA, "cudaGetSymbolAddress(mdg_noalloc_scratch) failed");
    g_scratch[dev] = static_cast<unsigned char *>(p);
  }
  *out = g_scratch[dev];
  return MDG_OK;
}

}  // namespace

extern "C" int mdg_advance_1d_noalloc(const mdg_problem_desc *desc, const double *prim_in, double *prim_out,
                                      int nsteps, void *stream, double *t_out, double *dt_out)
{
  if (!desc || !prim_in || !prim_out) return fail(MDG_ERR_INVALID, "mdg_advance_1d_noalloc: null argument");
  if (nsteps < 0) return fail(MDG_ERR_INVALID, "mdg_advance_1d_noalloc: nsteps < 0");
  int rc = check_desc(*desc);
  if (rc != MDG_OK) return rc;
  unsigned char *base = nullptr;
  rc = scratch_of_current_device(&base);
  if (rc != MDG_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const mdg_problem_desc &d = *desc;
  const int n1 = d.n1;

  // problem record, tables and tiles (host staging, copied into the scratch)
  ProbDev P;
  make_probdev(d, P);
  P.cell_off = 0;
  P.mono_off = 0;
  P.geo_off = 0;
  const int64_t ncol = n1 + 2 * NG;

  double *ph = reinterpret_cast<double *>(base + OFF_PH);
  double *rcd = reinterpret_cast<double *>(base + OFF_RC);
  double *geo = reinterpret_cast<double *>(base + OFF_GEO);
  ProbDev *probs = reinterpret_cast<ProbDev *>(base + OFF_PROB);
  ProbTime *times = reinterpret_cast<ProbTime *>(base + OFF_TIME);
  Tile *tiles = reinterpret_cast<Tile *>(base + OFF_TILES);
  int *err = reinterpret_cast<int *>(base + OFF_ERR);

#define CKN(call)                                                            \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess) return fail(MDG_ERR_CUDA, cudaGetErrorString(e_)); \
  } while (0)
  int ntiles = 0;
  {
    // the staging is shared by all host threads: hold it until the copies have landed
    std::lock_guard<std::mutex> lk(g_staging_mutex);
    build_recon_table_into(d, 0, h_rc, ncol, 0, h_al, h_be, h_ga);
    build_geo_1d(d, h_geo, ncol, 0);
    P.sparse_conn = conn_is_sparse(h_geo, ncol, 0, (int)ncol);
    for (int i0 = 0; i0 < n1; i0 += TILE1) h_tiles[ntiles++] = Tile{0, i0, 0, 0};
    CKN(cudaMemcpyAsync(rcd, h_rc, sizeof(double) * RC_NFIELDS * ncol, cudaMemcpyHostToDevice, st));
    CKN(cudaMemcpyAsync(geo, h_geo, sizeof(double) * GF_NFIELDS * ncol, cudaMemcpyHostToDevice, st));
    CKN(cudaMemcpyAsync(probs, &P, sizeof P, cudaMemcpyHostToDevice, st));
    CKN(cudaMemcpyAsync(tiles, h_tiles, sizeof(Tile) * ntiles, cudaMemcpyHostToDevice, st));
    CKN(cudaMemsetAsync(err, 0, sizeof(int), st));        // the error flag must start at zero
    if (prim_out != prim_in)
      CKN(cudaMemcpyAsync(prim_out, prim_in, sizeof(double) * NPRIM * n1, cudaMemcpyDeviceToDevice, st));
    CKN(cudaStreamSynchronize(st));
  }

  Tables tb{};
  tb.rc0 = rcd; tb.rc0_stride = ncol;
  tb.geo = geo; tb.geo_stride = ncol;
  StateSoA S{}, PH{};
  for (int v = 0; v < NPRIM; v++) { S.v[v] = prim_out + (int64_t)v * n1; PH.v[v] = ph + (int64_t)v * n1; }

  launch_reset_time(times, 0, st);
  launch_initial_estimate_one(probs, times, 0, n1, tb, S, st);
  for (int k = 0; k < nsteps; k++) {
    launch_dt_finalize(probs, times, 1, err, st);
    launch_stage1d(0, probs, times, tiles, ntiles, tb, S, S, PH, st);
    launch_stage1d(1, probs, times, tiles, ntiles, tb, PH, S, S, st);
    launch_finish(times, 1, st);
  }
  CKN(cudaGetLastError());
  // the outcome: the time record (non-finite state, dt below dtmin) and the error word
  ProbTime T;
  int errw = 0;
  CKN(cudaMemcpyAsync(&T, times, sizeof T, cudaMemcpyDeviceToHost, st));
  CKN(cudaMemcpyAsync(&errw, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CKN(cudaStreamSynchronize(st));
  if (t_out) *t_out = T.t;
  if (dt_out) *dt_out = T.dt;
  if (errw) return fail(errw, "mdg_advance_1d_noalloc: a time step estimate dropped below dtmin");
  if (T.err) return fail(T.err, "mdg_advance_1d_noalloc: non-finite state or dt below dtmin");
#undef CKN
  return MDG_OK;
}
