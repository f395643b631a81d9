// Solve server: a request loop that keeps 1-D and 2-D problems resident on one GPU and
// advances every admitted problem together (continuous batching).
//
// No counterpart in the reference, whose executable advances one problem per process
// through the main.c time loop (main.c:206-313).  Each request here is such a run: a
// problem description, its initial state and its end time (desc.tmax); the loop steps it
// with exactly the main.c rules until t >= tmax, after which the stage kernels leave it
// untouched (ProbTime::done), so a result does not depend on when it is collected nor on
// the other problems in the batch.
//
// Device memory is two sets of arenas sized at creation from HBM budgets.  The unit arena
// holds the 1-D states (P, PH), the reconstruction and geometry tables and the FP32
// weights, all indexed by zone units; 2-D requests keep their two reconstruction tables
// there too (n1 + 2*NG units of direction 0, then n2 + 2*NG of direction 1).  The cell
// arena holds the 2-D states (P, PH and the direction-0 accumulator) and the two shock-bit
// arrays, indexed by cells.  The mixed 1-D sweep's tables are built on the device at
// admission (mdg_tables.cu); the FP64 sweeps', which must be the reference's Romberg
// values, in the submitting thread.  A request is admitted when a slot and contiguous
// ranges of both arenas are free (first fit, coalescing on release): the HBM footprint
// is the admission test.  Between rounds of steps_per_round steps the loop admits queued
// requests (back-filling smaller ones when the oldest does not fit), rebuilds the
// (problem, tile) lists, runs the round and retires the problems that reached their end
// time.  A round is, per step, the dt reduction, the two RK stages of the 1-D lane on the
// main stream and of the 2-D lane (plain FP64 split sweep) on a second stream forked
// from it, and the time update after both lanes joined.  For the mixed 1-D sweep the
// round is one CUDA graph: the persistent, work-queue fed stage launches never change
// their arguments because the tile count lives in device memory; the graph is captured
// again only when the 2-D tile counts change.
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>
#include "mdg_internal.h"
#include "mdg_kernels.cuh"

namespace mdg {
int report_error(int code, const std::string &msg);
int validate_desc(const mdg_problem_desc &d, int ndim0, std::string &why);
void make_probdev(const mdg_problem_desc &d, ProbDev &P);
void build_recon_table(const mdg_problem_desc &d, int dir, double *tab, int64_t stride, int64_t off);
void build_geo_1d(const mdg_problem_desc &d, double *tab, int64_t stride, int64_t off);
void build_mixed_table(const mdg_problem_desc &d, int dir, float *tab, int64_t stride, int64_t off);
int conn_is_sparse(const double *tab, int64_t stride, int64_t off, int nrec);
}

using namespace mdg;

namespace {

using Clock = std::chrono::steady_clock;

// failures are reported like the solver's: the message is read by mdg_last_error_message
int sfail(int code, const std::string &msg) { return report_error(code, msg); }

#define SCK(call)                                                                      \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return sfail(e_ == cudaErrorMemoryAllocation ? MDG_ERR_OUTOFMEM : MDG_ERR_CUDA,  \
                   std::string(#call) + ": " + cudaGetErrorString(e_));                \
  } while (0)

// First-fit allocator over [0, cap) with coalescing of released ranges.
class RangeAlloc {
 public:
  void reset(int64_t cap)
  {
    free_.clear();
    if (cap > 0) free_[0] = cap;
  }
  int64_t alloc(int64_t n)
  {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      const int64_t off = it->first, len = it->second;
      free_.erase(it);
      if (len > n) free_[off + n] = len - n;
      return off;
    }
    return -1;
  }
  void release(int64_t off, int64_t n)
  {
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
 private:
  std::map<int64_t, int64_t> free_;
};

struct Request {
  long long id = 0;
  mdg_problem_desc desc{};
  std::vector<double> ic;       // [zone][5]
  std::vector<double> result;   // [zone][5] once finished
  std::vector<double> rc, geo;  // FP64 sweeps: the reference's tables, built at submission
  std::vector<float> mx;        // mixed 2-D: FP32 weights of both directions, laid out as rc
  int sparse = 0;
  int status = MDG_REQ_QUEUED;
  int err = MDG_OK;
  int slot = -1;
  int64_t seg = -1, units = 0;  // range of the unit arena
  int64_t seg2 = -1, cells = 0; // range of the cell arena (2-D)
  int64_t ncell = 0;            // zones of the problem
  Sweep3 *s3 = nullptr;         // 3-D: its own grid tables, face fluxes and shock bits
  double *d_state3 = nullptr;   // 3-D: state P then PH, 5 arrays of ncell each
  int64_t bytes3 = 0;           // 3-D: device memory held (counted against hbm_bytes_3d)
  double t = 0.0;
  int istep = 0;
  Clock::time_point t_submit, t_admit, t_done;
};

double seconds(Clock::time_point a, Clock::time_point b)
{
  return std::chrono::duration<double>(b - a).count();
}

}  // namespace

struct mdg_server {
  mdg_server_config cfg{};
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  int64_t units = 0;
  int max_probs = 0, max_tiles = 0, tile_len = 0;
  ProbDev *d_probs = nullptr;
  ProbTime *d_times = nullptr;
  Tile *d_tiles = nullptr;
  WorkQueue *d_queue = nullptr;   // [2]: closed-form 1-D tiles, tiles reading the Romberg tables
  WorkQueue h_queue[2] = {};
  int *d_err = nullptr;
  double *d_state = nullptr, *d_rc0 = nullptr, *d_geo = nullptr, *d_stage = nullptr;
  double *d_gmono = nullptr;   // monopole gravity per zone unit
  float *d_mx = nullptr;
  StateSoA P{}, PH{};
  Tables tb{};
  ProbTime *h_times = nullptr;   // pinned
  double *h_ret = nullptr;       // pinned return buffer of finished states
  size_t ret_cap = 0;
  std::vector<Request *> slots;
  RangeAlloc alloc;
  int64_t units_in_use = 0;
  int ntiles = 0;
  bool tiles_dirty = true;
  bool mono1d = false;                      // a resident 1-D request has monopole gravity
  int graph_mono1d = -1;                    // mono1d when the graph was captured
  int ntab1d = 0;                           // the last ntab1d 1-D tiles: requests reading the Romberg tables
  int graph_tab1d = -1;                     // ntab1d > 0 when the graph was captured
  // 2-D lane: cell arena, shock bits, tile lists (x tiles then y tiles), second stream
  int64_t cells = 0;
  RangeAlloc alloc2;
  int64_t cells_in_use = 0;
  double *d_state2 = nullptr;
  unsigned char *d_shock0 = nullptr, *d_shock1 = nullptr;
  StateSoA P2{}, PH2{}, ACC2{};
  Tile *d_tiles2 = nullptr;
  int tiles2_cap = 0, ntx2 = 0, nty2 = 0;
  // 2-D lane; 3-D lane: resident dendritic requests spread over NS3 streams, so that
  // several grids (each too small to fill the GPU alone) run side by side
#ifndef MDG_SERVER_NS3
#define MDG_SERVER_NS3 32
#endif
  static constexpr int NS3 = MDG_SERVER_NS3;
  cudaStream_t stream2 = nullptr, stream3[NS3] = {};
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_join3[NS3] = {};
  int graph_ntx2 = -1, graph_nty2 = -1;   // 2-D tile counts the graph was captured with
  // 3-D lane: resident 3-D requests (each with its own grid), on the second stream
  std::vector<Request *> jobs3;
  int64_t bytes3_in_use = 0;
  int jobs3_version = 0, graph_jobs3_version = -1;
  cudaGraphExec_t graph = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // requests
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Request *> queue;
  std::unordered_map<long long, Request *> reqs;
  long long next_id = 1;
  long long submitted = 0;
  // loop
  std::mutex loop_mu;
  std::thread th;
  std::atomic<bool> running{false};
  int loop_rc = MDG_OK;
  std::string loop_msg;
  // statistics of finished requests
  long long completed = 0, failed = 0, rounds = 0;
  std::atomic<long long> launches{0};
  double zone_updates = 0.0, device_ms = 0.0;
  std::vector<double> latency, wait;
};

namespace {

void free_server(mdg_server *s)
{
  if (s->graph) cudaGraphExecDestroy(s->graph);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  if (s->ev_fork) cudaEventDestroy(s->ev_fork);
  if (s->ev_join) cudaEventDestroy(s->ev_join);
  for (int q = 0; q < mdg_server::NS3; q++) {
    if (s->ev_join3[q]) cudaEventDestroy(s->ev_join3[q]);
    if (s->stream3[q]) cudaStreamDestroy(s->stream3[q]);
  }
  cudaFree(s->d_probs); cudaFree(s->d_times); cudaFree(s->d_tiles); cudaFree(s->d_queue); cudaFree(s->d_err);
  cudaFree(s->d_state); cudaFree(s->d_rc0); cudaFree(s->d_geo); cudaFree(s->d_stage); cudaFree(s->d_mx);
  cudaFree(s->d_gmono);
  cudaFree(s->d_state2); cudaFree(s->d_shock0); cudaFree(s->d_shock1); cudaFree(s->d_tiles2);
  if (s->h_times) cudaFreeHost(s->h_times);
  if (s->h_ret) cudaFreeHost(s->h_ret);
  if (s->stream2) cudaStreamDestroy(s->stream2);
  if (s->stream) cudaStreamDestroy(s->stream);
  for (auto &kv : s->reqs) {
    sweep3_destroy(kv.second->s3);
    cudaFree(kv.second->d_state3);
    delete kv.second;
  }
}

StateSoA soa3(const Request *r, int which)
{
  StateSoA q;
  for (int v = 0; v < NPRIM; v++) q.v[v] = r->d_state3 + (int64_t)(which * NPRIM + v) * r->ncell;
  return q;
}

// bytes of device memory per zone unit: state P and PH, RC and GF tables, FP32 weights
int64_t bytes_per_unit(int precision)
{
  // state P and PH, the RC and GF tables, the monopole gravity per zone and the FP32
  // weights (mixed)
  return 2 * NPRIM * 8 + RC_NFIELDS * 8 + GF_NFIELDS * 8 + 8 + (precision == MDG_PREC_MIXED ? MX_NFIELDS * 4 : 0);
}

// bytes per cell of the 2-D arena: state P, PH and accumulator, two shock bytes
int64_t bytes_per_cell_2d() { return 3 * NPRIM * 8 + 2; }

// Unit-arena and cell-arena footprints of a request: the 1-D state and tables, or the
// two 2-D reconstruction tables and the 2-D state with its shock bits ((n1 + 3) x n2
// bytes each: the face count of set_shock_flag, as in the solver's layout).
void footprint(const mdg_problem_desc &d, int64_t &units, int64_t &cells)
{
  if (d.ndim == 2 && !is_dendritic(d)) {
    units = (int64_t)d.n1 + 2 * NG + d.n2 + 2 * NG;
    cells = (int64_t)(d.n1 + 3) * d.n2;
  } else {
    units = (int64_t)d.n1 + 2 * NG;
    cells = 0;
  }
}

int persistent_grid(const mdg_server *s)
{
  int k = mixed_max_ctas_per_sm(s->cfg.threads);
  if (k <= 0) k = 1;
  if (s->cfg.ctas_per_sm > 0 && s->cfg.ctas_per_sm < k) k = s->cfg.ctas_per_sm;
  return k * s->num_sms;
}

int queue_round(mdg_server *s, int nsteps)
{
  const bool mixed = s->cfg.precision == MDG_PREC_MIXED;
  const int grid = mixed ? persistent_grid(s) : 0;
  const bool lane2 = s->ntx2 > 0, lane3 = !s->jobs3.empty();
  for (int k = 0; k < nsteps; k++) {
    launch_dt_finalize(s->d_probs, s->d_times, s->max_probs, s->d_err, s->stream);
    if (lane2 || lane3) SCK(cudaEventRecord(s->ev_fork, s->stream));
    if (lane2) SCK(cudaStreamWaitEvent(s->stream2, s->ev_fork, 0));
    const int n3s = lane3 ? std::min<int>(mdg_server::NS3, (int)s->jobs3.size()) : 0;
    for (int q = 0; q < n3s; q++) SCK(cudaStreamWaitEvent(s->stream3[q], s->ev_fork, 0));
    if (mixed) {
      // monopole gravity of the 1-D requests that have it, from each stage's state (only
      // while such a request is resident)
      // closed-form tiles, then (while such requests are resident) the tiles of requests
      // that read the Romberg tables, each with its own work queue
      const int nu = s->ntiles - s->ntab1d;
      if (s->mono1d) launch_monopole1d(s->d_probs, s->d_times, s->max_probs, s->tb, s->P, s->stream);
      launch_stage1d_mixed(0, s->cfg.threads, grid, true, s->d_probs, s->d_times, s->d_tiles, s->d_queue, s->tb,
                           s->P, s->P, s->PH, s->stream, false);
      if (s->ntab1d > 0)
        launch_stage1d_mixed(0, s->cfg.threads, grid, true, s->d_probs, s->d_times, s->d_tiles + nu, s->d_queue + 1,
                             s->tb, s->P, s->P, s->PH, s->stream, true);
      if (s->mono1d) launch_monopole1d(s->d_probs, s->d_times, s->max_probs, s->tb, s->PH, s->stream);
      launch_stage1d_mixed(1, s->cfg.threads, grid, true, s->d_probs, s->d_times, s->d_tiles, s->d_queue, s->tb,
                           s->PH, s->P, s->P, s->stream, false);
      if (s->ntab1d > 0)
        launch_stage1d_mixed(1, s->cfg.threads, grid, true, s->d_probs, s->d_times, s->d_tiles + nu, s->d_queue + 1,
                             s->tb, s->PH, s->P, s->P, s->stream, true);
    } else {
      // monopole gravity of the 1-D requests that have it (one thread per slot; the others
      // return at once), from each stage's state
      launch_monopole1d(s->d_probs, s->d_times, s->max_probs, s->tb, s->P, s->stream);
      launch_stage1d(0, s->d_probs, s->d_times, s->d_tiles, s->ntiles, s->tb, s->P, s->P, s->PH, s->stream);
      launch_monopole1d(s->d_probs, s->d_times, s->max_probs, s->tb, s->PH, s->stream);
      launch_stage1d(1, s->d_probs, s->d_times, s->d_tiles, s->ntiles, s->tb, s->PH, s->P, s->P, s->stream);
    }
    if (lane2) {
      launch_stage2d(0, mixed, s->d_probs, s->d_times, s->d_tiles2, s->ntx2, s->d_tiles2 + s->ntx2, s->nty2, s->tb,
                     s->P2, s->P2, s->ACC2, s->PH2, s->d_shock0, s->d_shock1, s->stream2);
      launch_stage2d(1, mixed, s->d_probs, s->d_times, s->d_tiles2, s->ntx2, s->d_tiles2 + s->ntx2, s->nty2, s->tb,
                     s->PH2, s->P2, s->ACC2, s->P2, s->d_shock0, s->d_shock1, s->stream2);
      SCK(cudaEventRecord(s->ev_join, s->stream2));
      SCK(cudaStreamWaitEvent(s->stream, s->ev_join, 0));
    }
    if (lane3) {
      for (size_t n = 0; n < s->jobs3.size(); n++) {
        Request *r = s->jobs3[n];
        cudaStream_t st = s->stream3[n % mdg_server::NS3];
        ProbDev *pr = s->d_probs + r->slot;
        ProbTime *tr = s->d_times + r->slot;
        launch_stage3d(0, mixed, r->s3, pr, tr, soa3(r, 0), soa3(r, 0), soa3(r, 1), st);
        launch_stage3d(1, mixed, r->s3, pr, tr, soa3(r, 1), soa3(r, 0), soa3(r, 0), st);
      }
      for (int q = 0; q < n3s; q++) {
        SCK(cudaEventRecord(s->ev_join3[q], s->stream3[q]));
        SCK(cudaStreamWaitEvent(s->stream, s->ev_join3[q], 0));
      }
    }
    launch_finish(s->d_times, s->max_probs, s->stream);
  }
  return MDG_OK;
}

// Upload tables, record, state and time of request r into slot r->slot, units r->seg...
int admit(mdg_server *s, Request *r)
{
  const mdg_problem_desc &d = r->desc;
  const int64_t w = r->units, seg = r->seg;
  ProbDev P;
  make_probdev(d, P);
  if (is_dendritic(d)) {
    // its own grid (built at submission); the AoS initial state is staged in PH
    P.n2 = d.n2;
    P.ncell = r->ncell;
    SCK(cudaMemcpyAsync(s->d_probs + r->slot, &P, sizeof P, cudaMemcpyHostToDevice, s->stream));
    double *stage = r->d_state3 + (int64_t)NPRIM * r->ncell;
    SCK(cudaMemcpyAsync(stage, r->ic.data(), sizeof(double) * NPRIM * r->ncell, cudaMemcpyHostToDevice, s->stream));
    launch_aos_to_soa(stage, soa3(r, 0), 0, r->ncell, s->stream);
    launch_reset_time(s->d_times, r->slot, s->stream);
    launch_initial_estimate3(r->s3, s->d_probs + r->slot, s->d_times + r->slot, soa3(r, 0), s->stream);
    SCK(cudaGetLastError());
    s->launches += 3;
    s->jobs3.push_back(r);
    s->jobs3_version++;
    return MDG_OK;
  }
  P.cell_off = seg;
  P.geo_off = seg;
  P.mono_off = seg;
  P.sparse_conn = r->sparse;
  // a mixed 1-D request on a non-uniform coordinate map reads its Romberg tables
  if (s->cfg.precision == MDG_PREC_MIXED && d.ndim == 1 && !r->geo.empty()) P.geo_tab = 1;
  if (d.ndim == 2) {
    P.cell_off = r->seg2;
    P.rc1_off = seg + d.n1 + 2 * NG;
    P.sh_off = r->seg2;
  }
  // stream-ordered copies from pageable memory return once the source has been staged,
  // so nothing here waits for the device
  SCK(cudaMemcpyAsync(s->d_probs + r->slot, &P, sizeof P, cudaMemcpyHostToDevice, s->stream));
  if (d.ndim == 2) {
    // both reconstruction tables in one copy; the shock bits start zero-filled, as the
    // reference's calloc'd flag arrays (utils.c:164-174)
    SCK(cudaMemcpy2DAsync(s->d_rc0 + seg, sizeof(double) * s->units, r->rc.data(), sizeof(double) * w,
                          sizeof(double) * w, RC_NFIELDS, cudaMemcpyHostToDevice, s->stream));
    if (!r->mx.empty())
      SCK(cudaMemcpy2DAsync(s->d_mx + seg, sizeof(float) * s->units, r->mx.data(), sizeof(float) * w,
                            sizeof(float) * w, MX_NFIELDS, cudaMemcpyHostToDevice, s->stream));
    SCK(cudaMemsetAsync(s->d_shock0 + r->seg2, 0, r->cells, s->stream));
    SCK(cudaMemsetAsync(s->d_shock1 + r->seg2, 0, r->cells, s->stream));
    SCK(cudaMemcpyAsync(s->d_stage, r->ic.data(), sizeof(double) * NPRIM * r->ncell, cudaMemcpyHostToDevice,
                        s->stream));
    launch_aos_to_soa(s->d_stage, s->P2, r->seg2, r->ncell, s->stream);
    launch_reset_time(s->d_times, r->slot, s->stream);
    launch_initial_estimate_one(s->d_probs, s->d_times, r->slot, r->ncell, s->tb, s->P2, s->stream);
    SCK(cudaGetLastError());
    s->launches += 3;
    return MDG_OK;
  }
  if (s->cfg.precision == MDG_PREC_MIXED && r->geo.empty()) {
    launch_build_tables_1d(s->d_probs, r->slot, d.n1, s->d_rc0, s->d_geo, s->d_mx, s->units, s->stream);
  } else {
    const size_t pitch = sizeof(double) * s->units;
    SCK(cudaMemcpy2DAsync(s->d_rc0 + seg, pitch, r->rc.data(), sizeof(double) * w, sizeof(double) * w, RC_NFIELDS,
                          cudaMemcpyHostToDevice, s->stream));
    SCK(cudaMemcpy2DAsync(s->d_geo + seg, pitch, r->geo.data(), sizeof(double) * w, sizeof(double) * w,
                          GF_NFIELDS, cudaMemcpyHostToDevice, s->stream));
    if (!r->mx.empty())
      SCK(cudaMemcpy2DAsync(s->d_mx + seg, sizeof(float) * s->units, r->mx.data(), sizeof(float) * w,
                            sizeof(float) * w, MX_NFIELDS, cudaMemcpyHostToDevice, s->stream));
  }
  SCK(cudaMemcpyAsync(s->d_stage, r->ic.data(), sizeof(double) * NPRIM * d.n1, cudaMemcpyHostToDevice, s->stream));
  launch_aos_to_soa(s->d_stage, s->P, seg, d.n1, s->stream);
  launch_reset_time(s->d_times, r->slot, s->stream);
  launch_initial_estimate_one(s->d_probs, s->d_times, r->slot, d.n1, s->tb, s->P, s->stream);
  SCK(cudaGetLastError());
  s->launches += (s->cfg.precision == MDG_PREC_MIXED) ? 4 : 3;
  return MDG_OK;
}

// Retire the finished problems of a round: one strided copy of each state (5 rows of
// n1 or n1 x n2 doubles) into the pinned return buffer, one wait, then the [zone][5]
// results.
int retire_all(mdg_server *s, const std::vector<int> &fin)
{
  if (fin.empty()) return MDG_OK;
  size_t need = 0;
  for (int k : fin) need += (size_t)NPRIM * s->slots[k]->ncell;
  if (need > s->ret_cap) {
    if (s->h_ret) cudaFreeHost(s->h_ret);
    s->h_ret = nullptr;
    s->ret_cap = 0;
    SCK(cudaMallocHost(&s->h_ret, sizeof(double) * need));
    s->ret_cap = need;
  }
  size_t off = 0;
  for (int k : fin) {
    Request *r = s->slots[k];
    const int64_t n = r->ncell;
    const bool two = r->desc.ndim == 2 && !is_dendritic(r->desc);
    const double *src = two ? s->P2.v[0] + r->seg2 : s->P.v[0] + r->seg;
    size_t pitch = sizeof(double) * (two ? s->cells : s->units);
    if (is_dendritic(r->desc)) {
      src = r->d_state3;
      pitch = sizeof(double) * n;
    }
    SCK(cudaMemcpy2DAsync(s->h_ret + off, sizeof(double) * n, src, pitch, sizeof(double) * n, NPRIM,
                          cudaMemcpyDeviceToHost, s->stream));
    off += (size_t)NPRIM * n;
  }
  SCK(cudaStreamSynchronize(s->stream));
  const Clock::time_point now = Clock::now();
  off = 0;
  for (int k : fin) {
    Request *r = s->slots[k];
    const ProbTime &T = s->h_times[k];
    const int64_t n = r->ncell;
    r->result.resize((size_t)NPRIM * n);
    for (int64_t z = 0; z < n; z++)
      for (int v = 0; v < NPRIM; v++) r->result[(size_t)z * NPRIM + v] = s->h_ret[off + (size_t)v * n + z];
    off += (size_t)NPRIM * n;
    r->t = T.t;
    r->istep = T.istep;
    r->err = T.err;
    r->t_done = now;
    s->slots[k] = nullptr;
    if (is_dendritic(r->desc)) {
      // the round has ended (retire_all waited for the stream): give its memory back
      s->jobs3.erase(std::find(s->jobs3.begin(), s->jobs3.end(), r));
      s->jobs3_version++;
      sweep3_destroy(r->s3);
      r->s3 = nullptr;
      cudaFree(r->d_state3);
      r->d_state3 = nullptr;
      s->bytes3_in_use -= r->bytes3;
    } else {
      s->alloc.release(r->seg, r->units);
      s->units_in_use -= r->units;
    }
    if (r->cells > 0) {
      s->alloc2.release(r->seg2, r->cells);
      s->cells_in_use -= r->cells;
    }
    r->slot = -1;
    std::lock_guard<std::mutex> lk(s->mu);
    r->status = T.err ? MDG_REQ_FAILED : MDG_REQ_DONE;
    if (T.err) s->failed++;
    else s->completed++;
    s->zone_updates += (double)n * T.istep;
    s->latency.push_back(seconds(r->t_submit, r->t_done));
    s->wait.push_back(seconds(r->t_submit, r->t_admit));
  }
  s->tiles_dirty = true;
  s->cv.notify_all();
  return MDG_OK;
}

// One scheduling round: admit, rebuild the tile list, step, retire.
int round_once(mdg_server *s, int *active_out)
{
  std::lock_guard<std::mutex> lk(s->loop_mu);
  SCK(cudaSetDevice(s->cfg.device));
  // 1. admission (back-filling: a request that does not fit does not block smaller ones)
  std::vector<Request *> adm;
  {
    std::lock_guard<std::mutex> ql(s->mu);
    for (auto it = s->queue.begin(); it != s->queue.end();) {
      Request *r = *it;
      int slot = -1;
      for (int k = 0; k < s->max_probs; k++)
        if (!s->slots[k]) { slot = k; break; }
      if (slot < 0) break;
      if (is_dendritic(r->desc)) {
        if (s->bytes3_in_use + r->bytes3 > s->cfg.hbm_bytes_3d) { ++it; continue; }
        s->bytes3_in_use += r->bytes3;
        r->slot = slot;
        s->slots[slot] = r;
        r->status = MDG_REQ_RUNNING;
        r->t_admit = Clock::now();
        adm.push_back(r);
        it = s->queue.erase(it);
        continue;
      }
      const int64_t seg = s->alloc.alloc(r->units);
      if (seg < 0) { ++it; continue; }
      int64_t seg2 = -1;
      if (r->cells > 0) {
        seg2 = s->alloc2.alloc(r->cells);
        if (seg2 < 0) {
          s->alloc.release(seg, r->units);
          ++it;
          continue;
        }
        s->cells_in_use += r->cells;
      }
      r->slot = slot;
      r->seg = seg;
      r->seg2 = seg2;
      s->slots[slot] = r;
      s->units_in_use += r->units;
      r->status = MDG_REQ_RUNNING;
      r->t_admit = Clock::now();
      adm.push_back(r);
      it = s->queue.erase(it);
    }
  }
  for (Request *r : adm) {
    int rc = admit(s, r);
    if (rc != MDG_OK) return rc;
    s->tiles_dirty = true;
  }
  // 2. the (problem, tile) list of the resident problems
  int active = 0;
  for (int k = 0; k < s->max_probs; k++) active += s->slots[k] != nullptr;
  if (s->tiles_dirty) {
    std::vector<Tile> tl, tl_tab, xt, yt;
    s->mono1d = false;
    const bool mixed1d = s->cfg.precision == MDG_PREC_MIXED;
    for (int k = 0; k < s->max_probs; k++) {
      const Request *r = s->slots[k];
      if (!r || is_dendritic(r->desc)) continue;   // dendritic problems run on their own grids
      if (r->desc.ndim == 1 && r->desc.monopole) s->mono1d = true;
      if (r->desc.ndim == 1 && mixed1d && !r->geo.empty()) {
        // a mixed request that reads the Romberg tables: the second 1-D list
        for (int i0 = 0; i0 < r->desc.n1; i0 += s->tile_len) tl_tab.push_back(Tile{k, i0, 0, 0});
        continue;
      }
      if (r->desc.ndim == 2) {
        // the solver's 2-D tiling: direction-0 tiles of TIX2 rows x NTX2 columns,
        // direction-1 tiles of TIY2 rows x TJY2 columns
        for (int i0 = 0; i0 < r->desc.n1; i0 += TIX2)
          for (int j0 = 0; j0 < r->desc.n2; j0 += NTX2) xt.push_back(Tile{k, i0, j0, 0});
        for (int i0 = 0; i0 < r->desc.n1; i0 += TIY2)
          for (int j0 = 0; j0 < r->desc.n2; j0 += TJY2) yt.push_back(Tile{k, i0, j0, 0});
      } else {
        for (int i0 = 0; i0 < r->desc.n1; i0 += s->tile_len) tl.push_back(Tile{k, i0, 0, 0});
      }
    }
    s->ntab1d = (int)tl_tab.size();
    const int nu = (int)tl.size();
    tl.insert(tl.end(), tl_tab.begin(), tl_tab.end());
    if ((int)tl.size() > s->max_tiles) return sfail(MDG_ERR_INTERNAL, "tile list exceeds its capacity");
    if (!tl.empty())
      SCK(cudaMemcpyAsync(s->d_tiles, tl.data(), sizeof(Tile) * tl.size(), cudaMemcpyHostToDevice, s->stream));
    s->h_queue[0] = WorkQueue{{0u, 0u}, nu, 0};
    s->h_queue[1] = WorkQueue{{0u, 0u}, s->ntab1d, 0};
    SCK(cudaMemcpyAsync(s->d_queue, s->h_queue, sizeof s->h_queue, cudaMemcpyHostToDevice, s->stream));
    s->ntiles = (int)tl.size();
    const int n2d = (int)(xt.size() + yt.size());
    if (n2d > s->tiles2_cap) {
      // grow the 2-D tile list (the previous round has ended: round_once waits for it)
      const int cap = std::max(n2d, 2 * s->tiles2_cap + 1024);
      cudaFree(s->d_tiles2);
      s->d_tiles2 = nullptr;
      s->tiles2_cap = 0;
      SCK(cudaMalloc(&s->d_tiles2, sizeof(Tile) * cap));
      s->tiles2_cap = cap;
      s->graph_ntx2 = -1;   // the graph holds the old list's address
    }
    xt.insert(xt.end(), yt.begin(), yt.end());
    if (!xt.empty())
      SCK(cudaMemcpyAsync(s->d_tiles2, xt.data(), sizeof(Tile) * xt.size(), cudaMemcpyHostToDevice, s->stream));
    s->ntx2 = n2d > 0 ? n2d - (int)yt.size() : 0;
    s->nty2 = (int)yt.size();
    s->tiles_dirty = false;
  }
  // 3. the round of steps
  if (active > 0) {
    const int K = s->cfg.steps_per_round;
    SCK(cudaEventRecord(s->ev0, s->stream));
    if (s->cfg.precision == MDG_PREC_MIXED) {
      if (s->graph && (s->graph_ntx2 != s->ntx2 || s->graph_nty2 != s->nty2 ||
                       s->graph_jobs3_version != s->jobs3_version || s->graph_mono1d != (int)s->mono1d ||
                       s->graph_tab1d != (int)(s->ntab1d > 0))) {
        cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
      }
      if (!s->graph) {
        cudaGraph_t g = nullptr;
        SCK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        const int qrc = queue_round(s, K);
        const cudaError_t e = cudaStreamEndCapture(s->stream, &g);
        if (qrc != MDG_OK) {
          if (g) cudaGraphDestroy(g);
          return qrc;
        }
        if (e != cudaSuccess) return sfail(MDG_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(e));
        const cudaError_t ei = cudaGraphInstantiate(&s->graph, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) {
          s->graph = nullptr;
          return sfail(MDG_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
        }
        s->graph_ntx2 = s->ntx2;
        s->graph_nty2 = s->nty2;
        s->graph_jobs3_version = s->jobs3_version;
        s->graph_mono1d = (int)s->mono1d;
        s->graph_tab1d = (int)(s->ntab1d > 0);
      }
      SCK(cudaGraphLaunch(s->graph, s->stream));
    } else {
      const int qrc = queue_round(s, K);
      if (qrc != MDG_OK) return qrc;
    }
    SCK(cudaEventRecord(s->ev1, s->stream));
    SCK(cudaGetLastError());
    // per step: dt reduction, two 1-D stages, time update; four 2-D direction sweeps
    long long per_step = 4 + (s->ntx2 > 0 ? 4 : 0);
    for (size_t q = 0; q < s->jobs3.size(); q++) per_step += 8;
    s->launches += (long long)K * per_step;
  }
  // 4. retire the problems that reached their end time (or failed)
  SCK(cudaMemcpyAsync(s->h_times, s->d_times, sizeof(ProbTime) * s->max_probs, cudaMemcpyDeviceToHost, s->stream));
  SCK(cudaStreamSynchronize(s->stream));
  if (active > 0) {
    float ms = 0.f;
    SCK(cudaEventElapsedTime(&ms, s->ev0, s->ev1));
    s->device_ms += ms;
    s->rounds++;
  }
  std::vector<int> fin;
  for (int k = 0; k < s->max_probs; k++)
    if (s->slots[k] && (s->h_times[k].done || s->h_times[k].err)) fin.push_back(k);
  int rc = retire_all(s, fin);
  if (rc != MDG_OK) return rc;
  active -= (int)fin.size();
  if (active_out) *active_out = active;
  return MDG_OK;
}

void loop_main(mdg_server *s)
{
  while (s->running.load()) {
    int active = 0;
    const int rc = round_once(s, &active);
    if (rc != MDG_OK) {
      std::lock_guard<std::mutex> lk(s->mu);
      s->loop_rc = rc;
      s->loop_msg = mdg_last_error_message();
      s->running = false;
      s->cv.notify_all();
      return;
    }
    if (active == 0) {
      std::unique_lock<std::mutex> lk(s->mu);
      if (s->queue.empty())
        s->cv.wait_for(lk, std::chrono::milliseconds(1), [&] { return !s->queue.empty() || !s->running.load(); });
    }
  }
}

double percentile(std::vector<double> v, double q)
{
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * (v.size() - 1);
  const size_t i = (size_t)pos;
  const double f = pos - i;
  return (i + 1 < v.size()) ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

}  // namespace

extern "C" {

int mdg_server_create(const mdg_server_config *cfg, mdg_server **out)
{
  if (!cfg || !out) return sfail(MDG_ERR_INVALID, "cfg/out");
  *out = nullptr;
  const mdg_server_config &c = *cfg;
  if (c.precision != MDG_PREC_FP64 && c.precision != MDG_PREC_MIXED) return sfail(MDG_ERR_INVALID, "precision");
  if (c.max_problems < 1 || c.max_problems > (1 << 20)) return sfail(MDG_ERR_INVALID, "max_problems out of [1, 2^20]");
  if (c.max_zones < 8 || c.max_zones > (1 << 26)) return sfail(MDG_ERR_INVALID, "max_zones out of [8, 2^26]");
  if (c.steps_per_round < 1 || c.steps_per_round > 100000) return sfail(MDG_ERR_INVALID, "steps_per_round out of [1, 1e5]");
  if (c.precision == MDG_PREC_MIXED && c.threads != 64 && c.threads != 128 && c.threads != 256)
    return sfail(MDG_ERR_INVALID, "threads must be 64, 128 or 256");
  const int64_t bpu = bytes_per_unit(c.precision);
  const int64_t units = c.hbm_bytes / bpu;
  if (units < c.max_zones + 2 * NG) return sfail(MDG_ERR_INVALID, "hbm_bytes too small for one problem of max_zones");
  if (c.hbm_bytes_2d < 0) return sfail(MDG_ERR_INVALID, "hbm_bytes_2d must not be negative");
  if (c.hbm_bytes_3d < 0) return sfail(MDG_ERR_INVALID, "hbm_bytes_3d must not be negative");
  const int64_t cells = c.hbm_bytes_2d / bytes_per_cell_2d();
  if (cells > 0) {
    if (c.max_cells_2d < 4 || c.max_cells_2d > (1 << 30))
      return sfail(MDG_ERR_INVALID, "max_cells_2d out of [4, 2^30]");
    if (cells < 2 * (int64_t)c.max_cells_2d)
      return sfail(MDG_ERR_INVALID, "hbm_bytes_2d too small for one 2-D problem of max_cells_2d");
  }
  int ndev = 0;
  SCK(cudaGetDeviceCount(&ndev));
  if (c.device < 0 || c.device >= ndev) return sfail(MDG_ERR_INVALID, "device ordinal out of range");
  SCK(cudaSetDevice(c.device));
  mdg_server *s = new mdg_server();
  s->cfg = c;
  s->units = units;
  s->max_probs = c.max_problems;
  s->tile_len = (c.precision == MDG_PREC_MIXED) ? c.threads - 2 : TILE1;
  s->max_tiles = (int)(units / s->tile_len + c.max_problems + 1);
  s->slots.assign(c.max_problems, nullptr);
  s->alloc.reset(units);
  s->cells = cells;
  s->alloc2.reset(cells);
  auto bail = [&](int rc) { free_server(s); delete s; return rc; };
#define SCKB(call)                                                                         \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return bail(sfail(e_ == cudaErrorMemoryAllocation ? MDG_ERR_OUTOFMEM : MDG_ERR_CUDA, \
                        std::string(#call) + ": " + cudaGetErrorString(e_)));              \
  } while (0)
  SCKB(cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, c.device));
  SCKB(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  SCKB(cudaStreamCreateWithFlags(&s->stream2, cudaStreamNonBlocking));
  for (int q = 0; q < mdg_server::NS3; q++) SCKB(cudaStreamCreateWithFlags(&s->stream3[q], cudaStreamNonBlocking));
  SCKB(cudaEventCreate(&s->ev0));
  SCKB(cudaEventCreate(&s->ev1));
  SCKB(cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming));
  SCKB(cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming));
  for (int q = 0; q < mdg_server::NS3; q++) SCKB(cudaEventCreateWithFlags(&s->ev_join3[q], cudaEventDisableTiming));
  SCKB(cudaMalloc(&s->d_probs, sizeof(ProbDev) * s->max_probs));
  SCKB(cudaMalloc(&s->d_times, sizeof(ProbTime) * s->max_probs));
  SCKB(cudaMalloc(&s->d_tiles, sizeof(Tile) * s->max_tiles));
  SCKB(cudaMalloc(&s->d_queue, 2 * sizeof(WorkQueue)));
  SCKB(cudaMalloc(&s->d_err, sizeof(int)));
  SCKB(cudaMalloc(&s->d_state, sizeof(double) * 2 * NPRIM * units));
  SCKB(cudaMalloc(&s->d_rc0, sizeof(double) * RC_NFIELDS * units));
  SCKB(cudaMalloc(&s->d_geo, sizeof(double) * GF_NFIELDS * units));
  SCKB(cudaMalloc(&s->d_stage, sizeof(double) * NPRIM * std::max<int64_t>(c.max_zones, cells > 0 ? c.max_cells_2d : 0)));
  if (c.precision == MDG_PREC_MIXED) SCKB(cudaMalloc(&s->d_mx, sizeof(float) * MX_NFIELDS * units));
  SCKB(cudaMalloc(&s->d_gmono, sizeof(double) * units));
  if (cells > 0) {
    SCKB(cudaMalloc(&s->d_state2, sizeof(double) * 3 * NPRIM * cells));
    SCKB(cudaMalloc(&s->d_shock0, cells));
    SCKB(cudaMalloc(&s->d_shock1, cells));
    SCKB(cudaMemset(s->d_state2, 0, sizeof(double) * 3 * NPRIM * cells));
  }
  SCKB(cudaMallocHost(&s->h_times, sizeof(ProbTime) * s->max_probs));
  // empty slots: a zero record has tmax = 0, so the time loop treats it as finished
  SCKB(cudaMemset(s->d_probs, 0, sizeof(ProbDev) * s->max_probs));
  SCKB(cudaMemset(s->d_times, 0, sizeof(ProbTime) * s->max_probs));
  SCKB(cudaMemset(s->d_queue, 0, 2 * sizeof(WorkQueue)));
  SCKB(cudaMemset(s->d_err, 0, sizeof(int)));
  SCKB(cudaMemset(s->d_state, 0, sizeof(double) * 2 * NPRIM * units));
#undef SCKB
  for (int v = 0; v < NPRIM; v++) {
    s->P.v[v] = s->d_state + (int64_t)v * units;
    s->PH.v[v] = s->d_state + (int64_t)(NPRIM + v) * units;
  }
  for (int v = 0; v < NPRIM && cells > 0; v++) {
    s->P2.v[v] = s->d_state2 + (int64_t)v * cells;
    s->PH2.v[v] = s->d_state2 + (int64_t)(NPRIM + v) * cells;
    s->ACC2.v[v] = s->d_state2 + (int64_t)(2 * NPRIM + v) * cells;
  }
  // a 2-D problem's direction-1 table sits in the same arena, after its direction-0 one
  s->tb.rc0 = s->d_rc0; s->tb.rc0_stride = units;
  s->tb.rc1 = s->d_rc0; s->tb.rc1_stride = units;
  s->tb.geo = s->d_geo; s->tb.geo_stride = units;
  s->tb.gmono = s->d_gmono;
  s->tb.mx = s->d_mx;
  s->tb.mx1 = s->d_mx;   // direction 1 of a 2-D request, after its direction-0 weights
  *out = s;
  return MDG_OK;
}

int mdg_server_submit(mdg_server *s, const mdg_problem_desc *desc, const double *prim, long long *id)
{
  if (!s || !desc || !prim) return sfail(MDG_ERR_INVALID, "server/desc/prim");
  std::string why;
  const int ndim = (desc->ndim == 2 || desc->ndim == 3) ? desc->ndim : 1;
  int rc = validate_desc(*desc, ndim, why);
  if (rc != MDG_OK) return sfail(rc, "request: " + why);
  if (!(desc->tmax > 0.0) || !(desc->tmax < 1.0e99))
    return sfail(MDG_ERR_INVALID, "request: tmax must state a finite end time");
  if (is_dendritic(*desc)) {
    // 3-D requests and 2-D spherical (r, theta) requests: the dendritic lane
    if (s->cfg.hbm_bytes_3d <= 0) return sfail(MDG_ERR_NOTIMPL, "request: the server takes no dendritic-grid requests");
    if (s->cfg.precision == MDG_PREC_MIXED && desc->hydro_interp_order != 3)
      return sfail(MDG_ERR_NOTIMPL, "request: the mixed-precision sweep is built for parabolic reconstruction");
    // its grid tables, face fluxes and state, built here in the submitting thread
    SCK(cudaSetDevice(s->cfg.device));
    Request *r = new Request();
    r->desc = *desc;
    rc = sweep3_create(*desc, &r->s3, why);
    if (rc != MDG_OK) {
      delete r;
      return sfail(rc, "request: dendritic grid: " + why);
    }
    r->ncell = sweep3_ncell(r->s3);
    const cudaError_t e = cudaMalloc(&r->d_state3, sizeof(double) * 2 * NPRIM * r->ncell);
    r->bytes3 = sweep3_bytes(r->s3) + (int64_t)sizeof(double) * 2 * NPRIM * r->ncell;
    if (e != cudaSuccess || r->bytes3 > s->cfg.hbm_bytes_3d) {
      sweep3_destroy(r->s3);
      if (e == cudaSuccess) cudaFree(r->d_state3);
      delete r;
      return sfail(MDG_ERR_OUTOFMEM, "request: the dendritic-grid problem does not fit in hbm_bytes_3d");
    }
    r->ic.assign(prim, prim + (size_t)NPRIM * r->ncell);
    r->t_submit = Clock::now();
    {
      std::lock_guard<std::mutex> lk(s->mu);
      r->id = s->next_id++;
      s->reqs[r->id] = r;
      s->queue.push_back(r);
      s->submitted++;
    }
    s->cv.notify_all();
    if (id) *id = r->id;
    return MDG_OK;
  }
  if (ndim == 2) {
    if (s->cells == 0) return sfail(MDG_ERR_NOTIMPL, "request: the server was created without a 2-D arena");
    if ((int64_t)desc->n1 * desc->n2 > s->cfg.max_cells_2d)
      return sfail(MDG_ERR_OUTOFMEM, "request: n1 x n2 exceeds the server's max_cells_2d");
    if ((int64_t)desc->n1 + desc->n2 + 4 * NG > s->units)
      return sfail(MDG_ERR_OUTOFMEM, "request: its tables exceed the unit arena");
  } else if (desc->n1 > s->cfg.max_zones) {
    return sfail(MDG_ERR_OUTOFMEM, "request: n1 exceeds the server's max_zones");
  }
  if (s->cfg.precision == MDG_PREC_MIXED && ndim == 1) {
    if (desc->hydro_interp_order != 3)
      return sfail(MDG_ERR_NOTIMPL, "request: the mixed-precision sweep is built for parabolic reconstruction");
    if (desc->geom == MDG_SPHERICAL && !(desc->startx[0] >= 0.0))
      return sfail(MDG_ERR_NOTIMPL, "request: the mixed-precision sweep needs a spherical grid starting at r >= 0");
  }
  Request *r = new Request();
  r->desc = *desc;
  r->ncell = (int64_t)desc->n1 * (ndim == 2 ? desc->n2 : 1);
  r->ic.assign(prim, prim + (size_t)NPRIM * r->ncell);
  footprint(*desc, r->units, r->cells);
  if (ndim == 2) {
    // the reference's Romberg tables of both directions, side by side: direction 0 at
    // columns 0 .. n1+2NG-1, direction 1 after it
    r->rc.assign((size_t)RC_NFIELDS * r->units, 0.0);
    build_recon_table(r->desc, 0, r->rc.data(), r->units, 0);
    build_recon_table(r->desc, 1, r->rc.data(), r->units, desc->n1 + 2 * NG);
    if (s->cfg.precision == MDG_PREC_MIXED) {
      r->mx.assign((size_t)MX_NFIELDS * r->units, 0.0f);
      build_mixed_table(r->desc, 0, r->mx.data(), r->units, 0);
      build_mixed_table(r->desc, 1, r->mx.data(), r->units, desc->n1 + 2 * NG);
    }
  } else if (s->cfg.precision == MDG_PREC_FP64 || desc->rcoord != MDG_RCOORD_UNIFORM ||
             desc->thcoord != MDG_THCOORD_UNIFORM || desc->monopole) {
    // the reference's Romberg tables, built here in the submitting thread so that the
    // request loop does not spend its time on them (the mixed sweep reads them, with
    // FP32 weights from the same moments, on a non-uniform coordinate map or with
    // monopole gravity)
    r->rc.assign((size_t)RC_NFIELDS * r->units, 0.0);
    r->geo.assign((size_t)GF_NFIELDS * r->units, 0.0);
    build_recon_table(r->desc, 0, r->rc.data(), r->units, 0);
    build_geo_1d(r->desc, r->geo.data(), r->units, 0);
    r->sparse = conn_is_sparse(r->geo.data(), r->units, 0, (int)r->units);
    if (s->cfg.precision == MDG_PREC_MIXED) {
      r->mx.assign((size_t)MX_NFIELDS * r->units, 0.0f);
      build_mixed_table(r->desc, 0, r->mx.data(), r->units, 0);
    }
  }
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    r->id = s->next_id++;
    s->reqs[r->id] = r;
    s->queue.push_back(r);
    s->submitted++;
  }
  s->cv.notify_all();
  if (id) *id = r->id;
  return MDG_OK;
}

int mdg_server_run(mdg_server *s, int rounds, int *active)
{
  if (!s) return sfail(MDG_ERR_INVALID, "server");
  if (s->running.load()) return sfail(MDG_ERR_LOGICAL, "the request loop is running on its own thread");
  int act = 0;
  for (int k = 0; rounds <= 0 || k < rounds; k++) {
    int rc = round_once(s, &act);
    if (rc != MDG_OK) return rc;
    if (rounds <= 0) {
      std::lock_guard<std::mutex> lk(s->mu);
      if (act == 0 && s->queue.empty()) break;
    }
  }
  if (active) *active = act;
  return MDG_OK;
}

int mdg_server_start(mdg_server *s)
{
  if (!s) return sfail(MDG_ERR_INVALID, "server");
  if (s->running.load()) return MDG_OK;
  s->loop_rc = MDG_OK;
  s->running = true;
  s->th = std::thread(loop_main, s);
  return MDG_OK;
}

int mdg_server_stop(mdg_server *s)
{
  if (!s) return sfail(MDG_ERR_INVALID, "server");
  s->running = false;
  s->cv.notify_all();
  if (s->th.joinable()) s->th.join();
  if (s->loop_rc != MDG_OK) return sfail(s->loop_rc, "request loop: " + s->loop_msg);
  return MDG_OK;
}

int mdg_server_poll(mdg_server *s, long long id, int *status)
{
  if (!s || !status) return sfail(MDG_ERR_INVALID, "server/status");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return sfail(MDG_ERR_NOTFOUND, "no such request");
  *status = it->second->status;
  return MDG_OK;
}

int mdg_server_wait(mdg_server *s, long long id, double timeout_s, int *status)
{
  if (!s) return sfail(MDG_ERR_INVALID, "server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return sfail(MDG_ERR_NOTFOUND, "no such request");
  Request *r = it->second;
  const auto until = Clock::now() + std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 0.0);
  s->cv.wait_until(lk, until, [&] {
    return r->status == MDG_REQ_DONE || r->status == MDG_REQ_FAILED || !s->running.load();
  });
  if (status) *status = r->status;
  return MDG_OK;
}

int mdg_server_result(mdg_server *s, long long id, double *prim, double *t, int *istep, double *latency_s)
{
  if (!s) return sfail(MDG_ERR_INVALID, "server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return sfail(MDG_ERR_NOTFOUND, "no such request");
  Request *r = it->second;
  if (r->status != MDG_REQ_DONE && r->status != MDG_REQ_FAILED)
    return sfail(MDG_ERR_LOGICAL, "request has not finished");
  if (prim) std::memcpy(prim, r->result.data(), sizeof(double) * r->result.size());
  if (t) *t = r->t;
  if (istep) *istep = r->istep;
  if (latency_s) *latency_s = seconds(r->t_submit, r->t_done);
  const int err = r->err;
  s->reqs.erase(it);
  delete r;
  return err ? sfail(err, "request stopped: non-finite state or time step below dtmin") : MDG_OK;
}

int mdg_server_get_stats(mdg_server *s, mdg_server_stats *st)
{
  if (!s || !st) return sfail(MDG_ERR_INVALID, "server/stats");
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(st, 0, sizeof *st);
  st->submitted = s->submitted;
  st->completed = s->completed;
  st->failed = s->failed;
  st->queued = (long long)s->queue.size();
  long long running = 0;
  for (auto &kv : s->reqs) running += kv.second->status == MDG_REQ_RUNNING;
  st->running = running;
  st->rounds = s->rounds;
  st->zone_updates = s->zone_updates;
  st->device_seconds = s->device_ms * 1e-3;
  st->latency_p50 = percentile(s->latency, 0.50);
  st->latency_p99 = percentile(s->latency, 0.99);
  st->wait_p50 = percentile(s->wait, 0.50);
  st->wait_p99 = percentile(s->wait, 0.99);
  const int64_t bpu = bytes_per_unit(s->cfg.precision);
  st->hbm_capacity = (double)s->units * bpu + (double)s->cells * bytes_per_cell_2d() + (double)s->cfg.hbm_bytes_3d;
  st->hbm_in_use = (double)s->units_in_use * bpu + (double)s->cells_in_use * bytes_per_cell_2d() +
                   (double)s->bytes3_in_use;
  st->kernel_launches = s->launches.load();
  return MDG_OK;
}

int mdg_server_destroy(mdg_server *s)
{
  if (!s) return MDG_OK;
  mdg_server_stop(s);
  cudaSetDevice(s->cfg.device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  free_server(s);
  delete s;
  return MDG_OK;
}

}  // extern "C"
