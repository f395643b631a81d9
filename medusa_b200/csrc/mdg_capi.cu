// C ABI of medusa_b200 (include/medusa_b200.h): solver lifetime, state transfer and the
// per-step launch sequence.
#include <cuda_runtime.h>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include "mdg_internal.h"
#include "mdg_kernels.cuh"
#include "mdg_tma.cuh"
#include "mdg_grid3d.cuh"

namespace mdg {
void build_recon_table(const mdg_problem_desc &d, int dir, double *tab, int64_t stride, int64_t off);
void build_geo_1d(const mdg_problem_desc &d, double *tab, int64_t stride, int64_t off);
double radial_coordinate(const mdg_problem_desc &d, double x);
void dust_ghost_u1(const mdg_problem_desc &d, double *u1);
void cartesian_2d_constants(const mdg_problem_desc &d, double &vol, double &area0, double &area1);
void build_mixed_table(const mdg_problem_desc &d, int dir, float *tab, int64_t stride, int64_t off);
int conn_is_sparse(const double *tab, int64_t stride, int64_t off, int nrec);
void spherical_1d_constants(double &area_k, double &th1, double &th2, double &tc);
void build_grid3(const mdg_problem_desc &d, Grid3Host &h);
void dendritic_zone_counts(const mdg_problem_desc &d, Grid3Host &h);
int64_t dendritic_refine_errors(const Grid3Host &h);
}

using namespace mdg;

struct mdg_solver {
  int device = 0;
  int ndim = 1;
  int nprob = 0;
  int precision = MDG_PREC_FP64;
  cudaStream_t stream = nullptr;
  std::vector<mdg_problem_desc> descs;
  std::vector<ProbDev> hprobs;
  ProbDev *d_probs = nullptr;
  ProbTime *d_times = nullptr;
  Tile *d_tiles = nullptr;
  int ntiles = 0;
  int ntx = 0, nty = 0;           // 2-D: direction-0 tiles first, then direction-1 tiles
  StateSoA ACC{};                 // 2-D: direction-0 part of the flux difference
  unsigned char *d_shock1 = nullptr;
  double *d_rc0 = nullptr, *d_rc1 = nullptr, *d_geo = nullptr;
  Tables tb{};
  TmaTables1d tm1{};              // 1-D FP64: tensor maps of rc0/geo (tile staging by TMA)
  double *d_state = nullptr;      // 10 arrays: P (5) then PH (5)
  StateSoA P{}, PH{};
  int64_t ncell_total = 0;
  unsigned char *d_shock0 = nullptr;
  double *d_stage = nullptr;      // AoS staging buffer, 5 doubles per zone of the largest problem
  double *d_stage_all = nullptr;  // AoS staging of every problem (mdg_upload_all / mdg_download_all)
  int64_t max_cells = 0;
  Sweep3 *s3 = nullptr;           // 3-D: the dendritic sweep of the single problem
  // output path: an asynchronous snapshot of one problem (state and EOS records, [zone][5]
  // each, then its time) taken on the solver's stream and copied to pinned host memory on
  // a copy stream while later steps run
  double *d_snap = nullptr, *h_snap = nullptr;
  size_t snap_cap = 0;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_snap = nullptr, ev_snap_done = nullptr;
  int snap_prob = -1;
  int64_t snap_n = 0;
  bool snap_pending = false;
  int *d_err = nullptr;
  // mixed precision: FP32 weights, the work queue and its tile list (tile = threads-2 zones)
  float *d_mx = nullptr, *d_mx1 = nullptr;   // FP32 weights (mixed): 1-D or 2-D direction 0; 2-D direction 1
  double *d_gmono = nullptr;      // monopole gravity at the zone centroids of the 1-D problems
  double *d_dtbuf = nullptr;      // per-problem dt of mdg_estimate_dt_raw / mdg_step_dt
  bool any_mono = false;          // a 1-D problem has monopole gravity
  WorkQueue *d_queue = nullptr;
  Tile *d_mtiles = nullptr;
  int mtiles_cap = 0, nmtiles = 0;
  int nmtab = 0;                  // mixed tiles of problems reading the Romberg tables (all lanes)
  // mixed 1-D sweep in lanes (mdg_launch_config::lanes): lane l advances problems
  // [m0, m1), whose tiles are d_mtiles[t0, t0+ntu) (closed-form geometry, queue 2l) and
  // [t0+ntu, t0+ntu+ntt) (Romberg tables, queue 2l+1); lane 0 runs on `stream`
  struct Lane { int m0 = 0, m1 = 0, t0 = 0, ntu = 0, ntt = 0; };
  Lane lane[MDG_MAX_LANES];
  int nlanes = 1;
  cudaStream_t lane_st[MDG_MAX_LANES] = {};
  cudaEvent_t lane_ev[MDG_MAX_LANES] = {};
  cudaEvent_t ev_fork = nullptr;
  int num_sms = 0;
  mdg_launch_config cfg{128, 0, 10, 16, 1, 1};
  // plain FP64 1-D solvers without monopole gravity whose problems have at most
  // RESIDENT1D_MAX_TILES tiles: CTAs per problem of the resident stepper (0: none)
  int res_cs = 0;
  // CUDA graph of cfg.steps_per_graph steps (rebuilt when the launch shape changes)
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  double *d_totals = nullptr;
  bool timing = false;
  cudaEvent_t ev[MDG_NTIMERS][2] = {};
  double tms[MDG_NTIMERS] = {0, 0, 0, 0};
  long long tcalls[MDG_NTIMERS] = {0, 0, 0, 0};
};

static thread_local std::string g_msg;

static int fail(int code, const std::string &msg)
{
  g_msg = msg;
  return code;
}

#define CK(call)                                                                   \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess)                                                         \
      return fail(MDG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace mdg {
int report_error(int code, const std::string &msg) { return fail(code, msg); }
int validate_desc(const mdg_problem_desc &d, int ndim0, std::string &why);
void make_probdev(const mdg_problem_desc &d, ProbDev &P);
}

// Checks of one problem description (shared with the solve server).
int mdg::validate_desc(const mdg_problem_desc &d, int ndim0, std::string &why)
{
  char buf[256];
  auto bad = [&](const char *m) { why = m; return MDG_ERR_INVALID; };
  if (d.ndim != 1 && d.ndim != 2 && d.ndim != 3) return bad("ndim must be 1, 2 or 3");
  if (d.ndim != ndim0) return bad("all problems of a solver must have the same ndim");
  if (d.rcoord != MDG_RCOORD_UNIFORM && d.rcoord != MDG_RCOORD_SINH && d.rcoord != MDG_RCOORD_SINH_MODIFIED &&
      d.rcoord != MDG_RCOORD_LOG)
    return bad("unknown radial map (rcoord)");
  if (d.thcoord != MDG_THCOORD_UNIFORM && d.thcoord != MDG_THCOORD_POLYTH) return bad("unknown theta map (thcoord)");
  if (d.thcoord != MDG_THCOORD_UNIFORM) {
    if (d.geom != MDG_SPHERICAL) return bad("theta maps apply to spherical grids");
    if (!(d.poly_xt > 0.0 && d.poly_xt < 1.0e300) || !(d.poly_alpha >= 1.0 && d.poly_alpha < 1.0e3))
      return bad("POLYTH needs poly_xt > 0 and poly_alpha >= 1");
  }
  if (d.rcoord == MDG_RCOORD_SINH_MODIFIED &&
      (!(d.rfact[2] != 0.0) || !std::isfinite(d.rfact[0]) || !std::isfinite(d.rfact[1]) || !std::isfinite(d.rfact[2])))
    return bad("SINH_MODIFIED needs finite facta, factb and a non-zero factc");
  if (d.monopole != 0 && d.monopole != 1) return bad("monopole must be 0 or 1");
  if (d.monopole) {
    if (d.geom != MDG_SPHERICAL) return bad("monopole gravity needs a spherical grid");
    if (d.grav[0] != 0.0 || d.grav[1] != 0.0 || d.grav[2] != 0.0)
      return bad("monopole and fixed gravity are exclusive (one GRAV switch)");
  }
  if (d.prob_kind < MDG_PROB_NONE || d.prob_kind > MDG_PROB_DUST) return bad("unknown prob_kind");
  if (d.rcoord != MDG_RCOORD_UNIFORM) {
    if (d.geom != MDG_SPHERICAL) return bad("radial maps apply to spherical grids");
    if (!(d.rtrans > 0.0) || !(d.rtrans < 1.0e300)) return bad("rtrans must be positive and finite");
    if ((d.bc_lo[0] == MDG_BC_PROB || d.bc_hi[0] == MDG_BC_PROB) && d.prob_kind == MDG_PROB_NOH) {
      why = "the Noh inflow boundary is built for the uniform radial map";
      return MDG_ERR_NOTIMPL;
    }
  }
  if (is_dendritic(d)) {
    // the dendritic spherical grid of prim_to_fluxes3 (3-D) or prim_to_fluxes2 (2-D,
    // step.c:659-764) over the whole sphere; a 2-D grid has one phi zone of width 2 pi
    // (init_coords, metric_spherical_general.c:570-572)
    const bool three = d.ndim == 3;
    auto pow2 = [](int n) { return n > 0 && (n & (n - 1)) == 0; };
    if (d.geom != MDG_SPHERICAL) { why = "3-D grids are spherical (dendritic) in this version"; return MDG_ERR_NOTIMPL; }
    if (d.n1 < 2 || d.n1 > (1 << 16)) return bad("n1 out of range [2, 2^16]");
    if (!pow2(d.n2) || d.n2 < 2 || d.n2 > (1 << 12)) return bad("n2 must be a power of two in [2, 4096]");
    if (three && (!pow2(d.n3) || d.n3 < 4 || d.n3 > (1 << 13))) return bad("n3 must be a power of two in [4, 8192]");
    if (!three && d.n3 != 1) return bad("a 2-D spherical grid has n3 = 1");
    if (!(d.dx[0] > 0.0 && d.dx[1] > 0.0 && d.dx[2] > 0.0)) return bad("dx must be positive");
    if (!(d.startx[0] >= 0.0)) return bad("the radial grid must start at r >= 0");
    if (d.startx[1] != -1.0 || std::fabs(d.startx[1] + d.n2 * d.dx[1] - 1) >= 1.0e-15)
      return bad("theta must cover the whole sphere (x1 from -1 to 1)");
    if (d.startx[2] != 0.0 || std::fabs(d.n3 * d.dx[2] - 2.0 * M_PI) > 1.0e-12)
      return bad("phi must cover [0, 2 pi)");
    if (d.eos != MDG_GAMMA_LAW && d.eos != MDG_POLYTROPIC) return bad("eos must be gamma-law or polytrope");
    if (d.hydro_interp_order < 1 || d.hydro_interp_order > 3) return bad("hydro_interp_order must be 1, 2 or 3");
    if (!(d.gam > 1.0)) return bad("gam must exceed 1");
    if (!(d.cfl > 0.0)) return bad("cfl must be positive");
    if (d.enforce_floors != 0 && d.enforce_floors != 1) return bad("enforce_floors must be 0 or 1");
    const bool ok = (d.bc_lo[0] == MDG_BC_REFLECT || d.bc_lo[0] == MDG_BC_SPHERICAL_ORIGIN) &&
                    (d.bc_hi[0] == MDG_BC_OUTFLOW || d.bc_hi[0] == MDG_BC_REFLECT);
    auto okj = [](int k) { return k == MDG_BC_REFLECT || k == MDG_BC_SPHERICAL_ORIGIN || k == MDG_BC_OUTFLOW; };
    auto okk = [](int k) { return k == MDG_BC_PERIODIC || k == MDG_BC_REFLECT || k == MDG_BC_OUTFLOW; };
    if (!ok || !okj(d.bc_lo[1]) || !okj(d.bc_hi[1]) || (three && (!okk(d.bc_lo[2]) || !okk(d.bc_hi[2])))) {
      why = "unsupported dendritic-grid boundary kinds";
      return MDG_ERR_NOTIMPL;
    }
    if (three && (d.bc_lo[2] == MDG_BC_PERIODIC) != (d.bc_hi[2] == MDG_BC_PERIODIC))
      return bad("periodic boundaries must be paired");
    if (three) {
      // the reference's init_dendritic exits on 4-to-1 phi refinement (utils.c:548-586)
      Grid3Host h;
      dendritic_zone_counts(d, h);
      const int64_t cells = dendritic_refine_errors(h);
      if (cells > 0) {
        snprintf(buf, sizeof buf,
                 "the dendritic grid refines 4-to-1 in phi in %lld cells (the reference's init_dendritic "
                 "rejects it): the radius grows too fast for 2-to-1 coarsening near r = r(startx)",
                 (long long)cells);
        why = buf;
        return MDG_ERR_INVALID;
      }
    }
    return MDG_OK;
  }
  if (d.n1 < 2 || d.n1 > (1 << 28)) return bad("n1 out of range [2, 2^28]");
  if (d.ndim == 2 && (d.n2 < 2 || (int64_t)d.n1 * d.n2 > (int64_t)1 << 31)) return bad("n2 out of range");
  if (d.eos != MDG_GAMMA_LAW && d.eos != MDG_POLYTROPIC) return bad("eos must be gamma-law or polytrope");
  if (d.hydro_interp_order < 1 || d.hydro_interp_order > 3) return bad("hydro_interp_order must be 1, 2 or 3");
  if (!(d.dx[0] > 0.0) || (d.ndim == 2 && !(d.dx[1] > 0.0))) return bad("dx must be positive");
  if (!(d.gam > 1.0)) return bad("gam must exceed 1");
  if (!(d.cfl > 0.0)) return bad("cfl must be positive");
  if (d.enforce_floors != 0 && d.enforce_floors != 1) return bad("enforce_floors must be 0 or 1");
  if (d.ndim == 1) {
    if (d.geom != MDG_CARTESIAN && d.geom != MDG_SPHERICAL) return bad("1-D geometry must be Cartesian or spherical");
    int lo = d.bc_lo[0], hi = d.bc_hi[0];
    bool lo_ok = lo == MDG_BC_OUTFLOW || lo == MDG_BC_REFLECT || lo == MDG_BC_EXTRAP || lo == MDG_BC_PERIODIC ||
                 (lo == MDG_BC_PROB && d.geom == MDG_SPHERICAL && d.prob_kind == MDG_PROB_NOH) ||
                 (lo == MDG_BC_SPHERICAL_ORIGIN && d.geom == MDG_SPHERICAL);
    bool hi_ok = hi == MDG_BC_OUTFLOW || hi == MDG_BC_REFLECT || hi == MDG_BC_EXTRAP || hi == MDG_BC_PERIODIC ||
                 (hi == MDG_BC_PROB && d.geom == MDG_SPHERICAL &&
                  (d.prob_kind == MDG_PROB_NOH || d.prob_kind == MDG_PROB_DUST));
    if (!lo_ok || !hi_ok) {
      snprintf(buf, sizeof buf, "unsupported 1-D boundary kinds lo=%d hi=%d for geom=%d", lo, hi, d.geom);
      why = buf;
      return MDG_ERR_NOTIMPL;
    }
    if ((lo == MDG_BC_PERIODIC) != (hi == MDG_BC_PERIODIC)) return bad("periodic boundaries must be paired");
    if (d.geom == MDG_SPHERICAL && (d.startx[0] != d.startx[0])) return bad("bad startx");
  } else {
    if (d.geom != MDG_CARTESIAN) {
      why = "2-D grids are Cartesian or dendritic spherical";
      return MDG_ERR_NOTIMPL;
    }
    for (int dir = 0; dir < 2; dir++) {
      int lo = d.bc_lo[dir], hi = d.bc_hi[dir];
      auto ok = [&](int k) {
        return k == MDG_BC_OUTFLOW || k == MDG_BC_REFLECT || k == MDG_BC_PERIODIC || (dir == 0 && k == MDG_BC_EXTRAP);
      };
      if (!ok(lo) || !ok(hi)) {
        snprintf(buf, sizeof buf, "unsupported 2-D boundary kinds in direction %d: lo=%d hi=%d", dir, lo, hi);
        why = buf;
        return MDG_ERR_NOTIMPL;
      }
      if ((lo == MDG_BC_PERIODIC) != (hi == MDG_BC_PERIODIC)) return bad("periodic boundaries must be paired");
    }
  }
  return MDG_OK;
}

// Tile list of the mixed sweep for nt threads per CTA (tiles of nt-2 zones) in `lanes`
// lanes (contiguous problem ranges of about equal zone count): per lane the tiles of
// problems with closed-form geometry, then those of problems reading the Romberg tables
// (each part has its own launch and work queue).  Caller has synchronized the solver's
// stream.
static int build_mixed_tiles(mdg_solver *s, int nt, int lanes)
{
  const int tl = nt - 2;
  std::vector<Tile> t;
  int ntab = 0;
  // lane boundaries: cut the problem list where the running zone count passes l/lanes
  int64_t total = 0, run = 0;
  for (int m = 0; m < s->nprob; m++) total += s->hprobs[m].n1;
  int nl = 0, m0 = 0;
  for (int m = 0; m <= s->nprob && nl < lanes; m++) {
    const bool last = (nl == lanes - 1);
    if (m == s->nprob || (!last && m > m0 && run * lanes >= total * (nl + 1))) {
      if (m == m0) break;
      mdg_solver::Lane &L = s->lane[nl];
      L.m0 = m0;
      L.m1 = m;
      L.t0 = (int)t.size();
      for (int pass = 0; pass < 2; pass++) {
        for (int q = m0; q < m; q++)
          if ((s->hprobs[q].geo_tab != 0) == (pass == 1))
            for (int i0 = 0; i0 < s->hprobs[q].n1; i0 += tl) t.push_back(Tile{q, i0, 0, 0});
        (pass == 0 ? L.ntu : L.ntt) = (int)t.size() - L.t0 - (pass == 0 ? 0 : L.ntu);
      }
      ntab += L.ntt;
      nl++;
      m0 = m;
      if (m == s->nprob) break;
    }
    if (m < s->nprob) run += s->hprobs[m].n1;
  }
  s->nlanes = nl;
  if ((int)t.size() > s->mtiles_cap) {
    cudaFree(s->d_mtiles);
    s->d_mtiles = nullptr;
    s->mtiles_cap = 0;
    cudaError_t e = cudaMalloc(&s->d_mtiles, sizeof(Tile) * t.size());
    if (e != cudaSuccess) return fail(MDG_ERR_OUTOFMEM, std::string("tile list: ") + cudaGetErrorString(e));
    s->mtiles_cap = (int)t.size();
  }
  CK(cudaMemcpy(s->d_mtiles, t.data(), sizeof(Tile) * t.size(), cudaMemcpyHostToDevice));
  s->nmtiles = (int)t.size();
  s->nmtab = ntab;
  WorkQueue q[2 * MDG_MAX_LANES] = {};
  for (int l = 0; l < s->nlanes; l++) {
    q[2 * l].ntiles = s->lane[l].ntu;
    q[2 * l + 1].ntiles = s->lane[l].ntt;
  }
  CK(cudaMemcpy(s->d_queue, q, sizeof q, cudaMemcpyHostToDevice));
  // streams and events of the extra lanes, created once
  if (s->nlanes > 1 && !s->ev_fork) {
    CK(cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming));
    for (int l = 1; l < MDG_MAX_LANES; l++) {
      CK(cudaStreamCreateWithFlags(&s->lane_st[l], cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&s->lane_ev[l], cudaEventDisableTiming));
    }
  }
  return MDG_OK;
}

// CTAs of one mixed-sweep launch over ntiles tiles: one per tile, or ctas_per_sm
// persistent CTAs per SM (bounded by the occupancy of the kernel and by the tile count)
static int mixed_grid(const mdg_solver *s, int ntiles)
{
  if (s->cfg.ctas_per_sm <= 0) return ntiles;
  int k = mixed_max_ctas_per_sm(s->cfg.threads);
  if (k <= 0) k = 1;
  if (s->cfg.ctas_per_sm < k) k = s->cfg.ctas_per_sm;
  const int64_t g = (int64_t)k * s->num_sms;
  return (int)(g < ntiles ? g : ntiles);
}

// Device record of one problem from its description (offsets left at zero).
void mdg::make_probdev(const mdg_problem_desc &d, ProbDev &P)
{
  memset(&P, 0, sizeof P);
  P.ndim = d.ndim; P.geom = d.geom; P.eos = d.eos; P.interp_order = d.hydro_interp_order;
  P.n1 = d.n1; P.n2 = (d.ndim > 1) ? d.n2 : 1;
  P.ncell = (int64_t)P.n1 * P.n2;
  P.bc_lo0 = d.bc_lo[0]; P.bc_hi0 = d.bc_hi[0]; P.bc_lo1 = d.bc_lo[1]; P.bc_hi1 = d.bc_hi[1];
  P.prob_kind = d.prob_kind;
  P.has_src = (d.geom == MDG_SPHERICAL);
  P.gam = d.gam; P.Kpoly = d.Kpoly;
  P.dx0 = d.dx[0]; P.dx1 = d.dx[1];
  if (d.ndim == 2) cartesian_2d_constants(d, P.vol, P.area0, P.area1);
  P.cfl = d.cfl; P.dt_init_safety = d.dt_init_safety; P.dt_grow_safety = d.dt_grow_safety;
  P.initial_dt = d.initial_dt; P.dtmax = d.dtmax; P.dtmin = d.dtmin; P.tmax = d.tmax;
  P.floors = d.enforce_floors; P.rho_floor = d.rho_floor; P.e_floor = d.e_floor;
  P.grav[0] = d.grav[0]; P.grav[1] = d.grav[1]; P.grav[2] = d.grav[2];
  P.grav_on = (d.grav[0] != 0.0 || d.grav[1] != 0.0 || d.grav[2] != 0.0);
  P.x0 = d.startx[0];
  P.mono = d.monopole;
  if (d.ndim == 1 && d.geom == MDG_SPHERICAL) spherical_1d_constants(P.gk_area, P.gk_th1, P.gk_th2, P.gk_tc);
  if (d.ndim == 1 && d.prob_kind == MDG_PROB_DUST) dust_ghost_u1(d, P.u1_hi);
}

static void free_all(mdg_solver *s)
{
  if (!s) return;
  for (int k = 0; k < MDG_NTIMERS; k++)
    for (int e = 0; e < 2; e++)
      if (s->ev[k][e]) cudaEventDestroy(s->ev[k][e]);
  cudaFree(s->d_probs); cudaFree(s->d_times); cudaFree(s->d_tiles);
  cudaFree(s->d_rc0); cudaFree(s->d_rc1); cudaFree(s->d_geo);
  cudaFree(s->d_state); cudaFree(s->d_shock0); cudaFree(s->d_shock1); cudaFree(s->d_stage); cudaFree(s->d_err);
  cudaFree(s->d_mx); cudaFree(s->d_mx1); cudaFree(s->d_queue); cudaFree(s->d_mtiles); cudaFree(s->d_totals); cudaFree(s->d_stage_all);
  cudaFree(s->d_gmono);
  cudaFree(s->d_dtbuf);
  sweep3_destroy(s->s3);
  s->s3 = nullptr;
  if (s->copy_stream) cudaStreamSynchronize(s->copy_stream);
  cudaFree(s->d_snap);
  if (s->h_snap) cudaFreeHost(s->h_snap);
  if (s->ev_snap) cudaEventDestroy(s->ev_snap);
  if (s->ev_snap_done) cudaEventDestroy(s->ev_snap_done);
  if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
  if (s->graph) cudaGraphExecDestroy(s->graph);
  for (int l = 0; l < MDG_MAX_LANES; l++) {
    if (s->lane_ev[l]) cudaEventDestroy(s->lane_ev[l]);
    if (s->lane_st[l]) cudaStreamDestroy(s->lane_st[l]);
  }
  if (s->ev_fork) cudaEventDestroy(s->ev_fork);
  if (s->stream) cudaStreamDestroy(s->stream);
}

// A solver of one dendritic spherical problem, 3-D or 2-D (validated by the caller): the
// grid tables of mdg_sweep3d.cu, state P and PH of ncell zones in the reference's zone
// order.  Its solver runs the dendritic lane (ndim 3 inside the solver) whatever the
// problem's own ndim.
static int create_3d(const mdg_problem_desc &d, int precision, int device, mdg_solver **out)
{
  mdg_solver *s = new mdg_solver();
  s->device = device;
  s->ndim = 3;
  s->nprob = 1;
  s->precision = precision;
  s->descs.assign(1, d);
  std::string why;
  int rc = sweep3_create(d, &s->s3, why);
  if (rc != MDG_OK) {
    delete s;
    return fail(rc, "3-D grid: " + why);
  }
  const int64_t n = sweep3_ncell(s->s3);
  ProbDev P;
  make_probdev(d, P);
  P.n2 = d.n2;
  P.ncell = n;
  P.cell_off = 0;
  s->hprobs.push_back(P);
  s->ncell_total = n;
  s->max_cells = n;
  auto cleanup_fail = [&](cudaError_t e, const char *what) {
    fail(e == cudaErrorMemoryAllocation ? MDG_ERR_OUTOFMEM : MDG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    free_all(s);
    delete s;
    return e == cudaErrorMemoryAllocation ? MDG_ERR_OUTOFMEM : MDG_ERR_CUDA;
  };
#define CK3(call)                                   \
  do {                                              \
    cudaError_t e_ = (call);                        \
    if (e_ != cudaSuccess) return cleanup_fail(e_, #call); \
  } while (0)
  CK3(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  CK3(cudaMalloc(&s->d_probs, sizeof(ProbDev)));
  CK3(cudaMalloc(&s->d_times, sizeof(ProbTime)));
  CK3(cudaMalloc(&s->d_state, sizeof(double) * 2 * NPRIM * n));
  CK3(cudaMalloc(&s->d_stage, sizeof(double) * NPRIM * n));
  CK3(cudaMalloc(&s->d_err, sizeof(int)));
  CK3(cudaMalloc(&s->d_totals, sizeof(double) * 2));
  CK3(cudaMalloc(&s->d_queue, sizeof(WorkQueue)));
  CK3(cudaMemset(s->d_queue, 0, sizeof(WorkQueue)));
  CK3(cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device));
  CK3(cudaMemcpy(s->d_probs, &P, sizeof(ProbDev), cudaMemcpyHostToDevice));
  CK3(cudaMemset(s->d_state, 0, sizeof(double) * 2 * NPRIM * n));
  CK3(cudaMemset(s->d_err, 0, sizeof(int)));
  CK3(cudaMemset(s->d_times, 0, sizeof(ProbTime)));
  for (int v = 0; v < NPRIM; v++) {
    s->P.v[v] = s->d_state + (int64_t)v * n;
    s->PH.v[v] = s->d_state + (int64_t)(NPRIM + v) * n;
  }
#undef CK3
  *out = s;
  return MDG_OK;
}

extern "C" {

int mdg_version(void) { return 100; }

int mdg_grid3d_counts(const mdg_problem_desc *desc, int *nj, int *nk, long long *ncell)
{
  if (!desc) return fail(MDG_ERR_INVALID, "desc");
  std::string why;
  int rc = validate_desc(*desc, desc->ndim, why);
  if (rc == MDG_OK && !is_dendritic(*desc)) {
    rc = MDG_ERR_NOTIMPL;
    why = "not a dendritic spherical grid";
  }
  if (rc != MDG_OK) return fail(rc, why);
  Grid3Host h;
  build_grid3(*desc, h);
  int64_t c = 0;
  for (int i = 0; i < h.n1; i++) {
    if (nj) nj[i] = h.njr(i);
    for (int j = 0; j < h.njr(i); j++) {
      if (nk) nk[c] = h.nk[h.row(i, j)];
      c++;
    }
  }
  if (ncell) *ncell = h.ncell;
  return MDG_OK;
}

int mdg_grid3d_geometry(const mdg_problem_desc *desc, double *rows, long long *nrows)
{
  if (!desc) return fail(MDG_ERR_INVALID, "desc");
  std::string why;
  int rc = validate_desc(*desc, desc->ndim, why);
  if (rc == MDG_OK && !is_dendritic(*desc)) {
    rc = MDG_ERR_NOTIMPL;
    why = "not a dendritic spherical grid";
  }
  if (rc != MDG_OK) return fail(rc, why);
  Grid3Host h;
  build_grid3(*desc, h);
  if (nrows) *nrows = h.nij;
  if (rows)
    for (int64_t r = 0; r < h.nij; r++)
      for (int f = 0; f < G3_NFIELDS; f++) rows[r * G3_NFIELDS + f] = h.geo[(size_t)f * h.nij + r];
  return MDG_OK;
}

const char *mdg_error_string(int code)
{
  switch (code) {
    case MDG_OK: return "ok";
    case MDG_ERR_INVALID: return "invalid argument";
    case MDG_ERR_INDEX: return "index out of range";
    case MDG_ERR_NOTFOUND: return "not found";
    case MDG_ERR_IO: return "i/o error";
    case MDG_ERR_NOTIMPL: return "not implemented";
    case MDG_ERR_OUTOFMEM: return "out of device memory";
    case MDG_ERR_PARFILE: return "parameter error";
    case MDG_ERR_LOGICAL: return "logical error";
    case MDG_ERR_INTERNAL: return "internal error";
    case MDG_ERR_CUDA: return "CUDA runtime error";
    case MDG_ERR_NONFINITE: return "time step dropped below dtmin";
    default: return "unknown status";
  }
}

const char *mdg_last_error_message(void) { return g_msg.c_str(); }

int mdg_create(const mdg_problem_desc *descs, int nprob, int precision, int device, mdg_solver **out)
{
  if (!descs || nprob <= 0 || !out) return fail(MDG_ERR_INVALID, "descs/nprob/out");
  if (precision != MDG_PREC_FP64 && precision != MDG_PREC_MIXED) return fail(MDG_ERR_INVALID, "precision");
  *out = nullptr;
  const int ndim = descs[0].ndim;
  for (int m = 0; m < nprob; m++) {
    std::string why;
    int rc = validate_desc(descs[m], ndim, why);
    if (rc != MDG_OK) return fail(rc, "problem " + std::to_string(m) + ": " + why);
    if (precision == MDG_PREC_MIXED && descs[m].hydro_interp_order != 3)
      return fail(MDG_ERR_NOTIMPL, "problem " + std::to_string(m) +
                                       ": the mixed-precision sweeps are built for parabolic reconstruction");
    if (precision == MDG_PREC_MIXED && descs[m].geom == MDG_SPHERICAL && !(descs[m].startx[0] >= 0.0))
      return fail(MDG_ERR_NOTIMPL, "problem " + std::to_string(m) +
                                       ": the mixed-precision sweep needs a spherical grid starting at r >= 0");
  }
  const bool dendritic = is_dendritic(descs[0]);
  if (dendritic && nprob != 1) return fail(MDG_ERR_NOTIMPL, "a dendritic-grid solver advances one problem");
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(MDG_ERR_INVALID, "device ordinal out of range");
  CK(cudaSetDevice(device));
  if (dendritic) return create_3d(descs[0], precision, device, out);

  mdg_solver *s = new mdg_solver();
  s->device = device;
  s->ndim = ndim;
  s->nprob = nprob;
  s->precision = precision;
  s->descs.assign(descs, descs + nprob);

  // layout: state offsets, table offsets, tiles
  std::vector<Tile> tiles, ytiles;
  int64_t cell = 0, rc0 = 0, rc1 = 0, sh = 0;
  for (int m = 0; m < nprob; m++) {
    const mdg_problem_desc &d = descs[m];
    ProbDev P;
    make_probdev(d, P);
    P.cell_off = cell;
    P.mono_off = cell;
    P.geo_off = rc0;
    P.rc1_off = rc1;
    P.sh_off = sh;
    s->hprobs.push_back(P);
    if (d.monopole) s->any_mono = true;
    const int64_t nc = (int64_t)P.n1 * P.n2;
    if (nc > s->max_cells) s->max_cells = nc;
    cell += nc;
    rc0 += P.n1 + 2 * NG;
    if (d.ndim == 2) {
      rc1 += P.n2 + 2 * NG;
      sh += (int64_t)(P.n1 + 3) * P.n2;
      for (int i0 = 0; i0 < P.n1; i0 += TIX2)
        for (int j0 = 0; j0 < P.n2; j0 += NTX2) tiles.push_back(Tile{m, i0, j0, 0});
      for (int i0 = 0; i0 < P.n1; i0 += TIY2)
        for (int j0 = 0; j0 < P.n2; j0 += TJY2) ytiles.push_back(Tile{m, i0, j0, 0});
    } else {
      for (int i0 = 0; i0 < P.n1; i0 += TILE1) tiles.push_back(Tile{m, i0, 0, 0});
    }
  }
  rc0 += rc0 & 1;                     // an even table stride: 16-byte rows for the TMA maps
  s->ncell_total = cell;
  s->ntx = (int)tiles.size();
  s->nty = (int)ytiles.size();
  tiles.insert(tiles.end(), ytiles.begin(), ytiles.end());
  s->ntiles = (int)tiles.size();
  const int nstate = (ndim == 2) ? 3 : 2;   // P, PH (+ ACC in 2-D)

  // host tables of the FP64 sweeps (Romberg moments, bit-identical to the reference's);
  // 1-D mixed: tables built on the device from closed-form moments on the uniform maps,
  // host Romberg tables otherwise; 2-D mixed: the FP64 tables (for declined faces) plus
  // host-built FP32 weights of both directions
  const bool dev_tables = precision == MDG_PREC_MIXED && ndim == 1;
  const size_t n_rc0 = (size_t)RC_NFIELDS * rc0, n_geo = (ndim == 2) ? 0 : (size_t)GF_NFIELDS * rc0;
  std::vector<double> h_rc0, h_rc1, h_geo;
  if (!dev_tables) h_rc0.assign(n_rc0, 0.0);
  if (ndim == 2) h_rc1.assign((size_t)RC_NFIELDS * rc1, 0.0);
  else if (!dev_tables) h_geo.assign(n_geo, 0.0);
  // mixed 1-D problems on a non-uniform coordinate map, or with monopole gravity (whose
  // enclosed-mass solve reads the edge radii of the tables), read the Romberg tables
  // (built here, columns of the problem only) instead of the closed-form geometry
  struct HostCols { int m; std::vector<double> rc, geo; std::vector<float> mx; };
  std::vector<HostCols> tab_probs;
  for (int m = 0; m < nprob && dev_tables; m++) {
    if (descs[m].rcoord == MDG_RCOORD_UNIFORM && descs[m].thcoord == MDG_THCOORD_UNIFORM && !descs[m].monopole)
      continue;
    const int64_t ncol = descs[m].n1 + 2 * NG;
    HostCols hc;
    hc.m = m;
    hc.rc.assign((size_t)RC_NFIELDS * ncol, 0.0);
    hc.geo.assign((size_t)GF_NFIELDS * ncol, 0.0);
    hc.mx.assign((size_t)MX_NFIELDS * ncol, 0.0f);
    build_recon_table(descs[m], 0, hc.rc.data(), ncol, 0);
    build_geo_1d(descs[m], hc.geo.data(), ncol, 0);
    build_mixed_table(descs[m], 0, hc.mx.data(), ncol, 0);
    s->hprobs[m].geo_tab = 1;
    s->hprobs[m].sparse_conn = conn_is_sparse(hc.geo.data(), ncol, 0, (int)ncol);
    tab_probs.push_back(std::move(hc));
  }
  for (int m = 0; m < nprob && !dev_tables; m++) {
    build_recon_table(descs[m], 0, h_rc0.data(), rc0, s->hprobs[m].geo_off);
    if (ndim == 2) {
      build_recon_table(descs[m], 1, h_rc1.data(), rc1, s->hprobs[m].rc1_off);
    } else {
      build_geo_1d(descs[m], h_geo.data(), rc0, s->hprobs[m].geo_off);
      s->hprobs[m].sparse_conn = conn_is_sparse(h_geo.data(), rc0, s->hprobs[m].geo_off, descs[m].n1 + 2 * NG);
    }
  }

  auto cleanup_fail = [&](int code) { free_all(s); delete s; return code; };
#define CKC(call)                                                                     \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      fail(e_ == cudaErrorMemoryAllocation ? MDG_ERR_OUTOFMEM : MDG_ERR_CUDA,         \
           std::string(#call) + ": " + cudaGetErrorString(e_));                       \
      return cleanup_fail(e_ == cudaErrorMemoryAllocation ? MDG_ERR_OUTOFMEM : MDG_ERR_CUDA); \
    }                                                                                 \
  } while (0)

  CKC(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  CKC(cudaMalloc(&s->d_probs, sizeof(ProbDev) * nprob));
  CKC(cudaMalloc(&s->d_times, sizeof(ProbTime) * nprob));
  CKC(cudaMalloc(&s->d_tiles, sizeof(Tile) * s->ntiles));
  CKC(cudaMalloc(&s->d_rc0, sizeof(double) * n_rc0));
  if (ndim == 2) CKC(cudaMalloc(&s->d_rc1, sizeof(double) * h_rc1.size()));
  else CKC(cudaMalloc(&s->d_geo, sizeof(double) * n_geo));
  CKC(cudaMalloc(&s->d_state, sizeof(double) * nstate * NPRIM * cell));
  if (s->any_mono) CKC(cudaMalloc(&s->d_gmono, sizeof(double) * cell));
  CKC(cudaMalloc(&s->d_stage, sizeof(double) * NPRIM * s->max_cells));
  CKC(cudaMalloc(&s->d_err, sizeof(int)));
  CKC(cudaMalloc(&s->d_totals, sizeof(double) * 2 * nprob));
  CKC(cudaMalloc(&s->d_queue, 2 * MDG_MAX_LANES * sizeof(WorkQueue)));
  CKC(cudaMemset(s->d_queue, 0, 2 * MDG_MAX_LANES * sizeof(WorkQueue)));
  if (precision == MDG_PREC_MIXED) CKC(cudaMalloc(&s->d_mx, sizeof(float) * MX_NFIELDS * rc0));
  if (precision == MDG_PREC_MIXED && ndim == 2) {
    CKC(cudaMalloc(&s->d_mx1, sizeof(float) * MX_NFIELDS * rc1));
    std::vector<float> m0((size_t)MX_NFIELDS * rc0, 0.0f), m1((size_t)MX_NFIELDS * rc1, 0.0f);
    for (int m = 0; m < nprob; m++) {
      build_mixed_table(descs[m], 0, m0.data(), rc0, s->hprobs[m].geo_off);
      build_mixed_table(descs[m], 1, m1.data(), rc1, s->hprobs[m].rc1_off);
    }
    CKC(cudaMemcpy(s->d_mx, m0.data(), sizeof(float) * m0.size(), cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(s->d_mx1, m1.data(), sizeof(float) * m1.size(), cudaMemcpyHostToDevice));
  }
  CKC(cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, device));
  if (ndim == 2) CKC(cudaMalloc(&s->d_shock0, sh > 0 ? sh : 1));
  if (ndim == 2) CKC(cudaMalloc(&s->d_shock1, sh > 0 ? sh : 1));

  CKC(cudaMemcpy(s->d_probs, s->hprobs.data(), sizeof(ProbDev) * nprob, cudaMemcpyHostToDevice));
  CKC(cudaMemcpy(s->d_tiles, tiles.data(), sizeof(Tile) * s->ntiles, cudaMemcpyHostToDevice));
  if (dev_tables) {
    for (int m = 0; m < nprob; m++)
      if (!s->hprobs[m].geo_tab)
        launch_build_tables_1d(s->d_probs, m, descs[m].n1, s->d_rc0, s->d_geo, s->d_mx, rc0, s->stream);
    CKC(cudaGetLastError());
    CKC(cudaStreamSynchronize(s->stream));
    for (const HostCols &hc : tab_probs) {
      const int64_t ncol = descs[hc.m].n1 + 2 * NG, off = s->hprobs[hc.m].geo_off;
      CKC(cudaMemcpy2D(s->d_rc0 + off, sizeof(double) * rc0, hc.rc.data(), sizeof(double) * ncol,
                       sizeof(double) * ncol, RC_NFIELDS, cudaMemcpyHostToDevice));
      CKC(cudaMemcpy2D(s->d_geo + off, sizeof(double) * rc0, hc.geo.data(), sizeof(double) * ncol,
                       sizeof(double) * ncol, GF_NFIELDS, cudaMemcpyHostToDevice));
      CKC(cudaMemcpy2D(s->d_mx + off, sizeof(float) * rc0, hc.mx.data(), sizeof(float) * ncol,
                       sizeof(float) * ncol, MX_NFIELDS, cudaMemcpyHostToDevice));
    }
  } else {
    CKC(cudaMemcpy(s->d_rc0, h_rc0.data(), sizeof(double) * n_rc0, cudaMemcpyHostToDevice));
    if (ndim != 2) CKC(cudaMemcpy(s->d_geo, h_geo.data(), sizeof(double) * n_geo, cudaMemcpyHostToDevice));
  }
  if (ndim == 2) CKC(cudaMemcpy(s->d_rc1, h_rc1.data(), sizeof(double) * h_rc1.size(), cudaMemcpyHostToDevice));
  CKC(cudaMemset(s->d_state, 0, sizeof(double) * nstate * NPRIM * cell));
  CKC(cudaMemset(s->d_err, 0, sizeof(int)));
  if (ndim == 2) CKC(cudaMemset(s->d_shock0, 0, sh > 0 ? sh : 1));
  if (ndim == 2) CKC(cudaMemset(s->d_shock1, 0, sh > 0 ? sh : 1));
  CKC(cudaMemset(s->d_times, 0, sizeof(ProbTime) * nprob));
  for (int v = 0; v < NPRIM; v++) {
    s->P.v[v] = s->d_state + (int64_t)v * cell;
    s->PH.v[v] = s->d_state + (int64_t)(NPRIM + v) * cell;
    if (ndim == 2) s->ACC.v[v] = s->d_state + (int64_t)(2 * NPRIM + v) * cell;
  }
  s->tb.rc0 = s->d_rc0; s->tb.rc0_stride = rc0;
  s->tb.rc1 = s->d_rc1; s->tb.rc1_stride = rc1;
  s->tb.geo = s->d_geo; s->tb.geo_stride = rc0;
  s->tb.mx = s->d_mx;
  s->tb.mx1 = s->d_mx1;
  s->tb.gmono = s->d_gmono;
  if (ndim == 1 && precision == MDG_PREC_FP64) {
    // tile staging of the FP64 tables by TMA; without the driver's encoder the kernel
    // reads the tables directly (same results)
    std::string why;
    const uint64_t row = sizeof(double) * (uint64_t)rc0;
    s->tm1.valid = tma_encode_2d_f64(&s->tm1.rc, s->d_rc0, rc0, RC_NFIELDS, row, TMA_COLS1, RC_TMA_ROWS, &why) &&
                   tma_encode_2d_f64(&s->tm1.geo, s->d_geo, rc0, GF_NFIELDS, row, TMA_COLS1, GF_TMA_ROWS, &why);
  }
#undef CKC
  if (precision == MDG_PREC_MIXED && ndim == 1) {
    int rc = build_mixed_tiles(s, s->cfg.threads, s->cfg.lanes);
    if (rc != MDG_OK) { free_all(s); delete s; return rc; }
  }
  if (precision == MDG_PREC_FP64 && ndim == 1 && !s->any_mono) {
    int max_tiles = 0;
    for (const ProbDev &P : s->hprobs) max_tiles = std::max(max_tiles, (P.n1 + TILE1 - 1) / TILE1);
    s->res_cs = resident1d_cluster_size(max_tiles);
  }
  *out = s;
  return MDG_OK;
}

int mdg_upload_state(mdg_solver *s, int prob, const double *prim)
{
  if (!s || !prim) return fail(MDG_ERR_INVALID, "solver/prim");
  if (prob < 0 || prob >= s->nprob) return fail(MDG_ERR_INDEX, "problem index out of range");
  CK(cudaSetDevice(s->device));
  const ProbDev &P = s->hprobs[prob];
  const int64_t n = P.ncell;
  CK(cudaMemcpyAsync(s->d_stage, prim, sizeof(double) * NPRIM * n, cudaMemcpyHostToDevice, s->stream));
  launch_aos_to_soa(s->d_stage, s->P, P.cell_off, n, s->stream);
  launch_reset_time(s->d_times, prob, s->stream);
  if (s->ndim == 3) launch_initial_estimate3(s->s3, s->d_probs, s->d_times, s->P, s->stream);
  else launch_initial_estimate_one(s->d_probs, s->d_times, prob, n, s->tb, s->P, s->stream);
  CK(cudaGetLastError());
  return MDG_OK;
}

static int stage_all(mdg_solver *s)
{
  if (!s->d_stage_all) CK(cudaMalloc(&s->d_stage_all, sizeof(double) * NPRIM * s->ncell_total));
  return MDG_OK;
}

int mdg_upload_all(mdg_solver *s, const double *prim)
{
  if (!s || !prim) return fail(MDG_ERR_INVALID, "solver/prim");
  CK(cudaSetDevice(s->device));
  int rc = stage_all(s);
  if (rc != MDG_OK) return rc;
  CK(cudaMemcpyAsync(s->d_stage_all, prim, sizeof(double) * NPRIM * s->ncell_total, cudaMemcpyHostToDevice,
                     s->stream));
  launch_aos_to_soa(s->d_stage_all, s->P, 0, s->ncell_total, s->stream);
  launch_reset_time_all(s->d_times, s->nprob, s->stream);
  if (s->ndim == 3) launch_initial_estimate3(s->s3, s->d_probs, s->d_times, s->P, s->stream);
  else launch_initial_estimate_all(s->d_probs, s->d_times, s->nprob, s->max_cells, s->tb, s->P, s->stream);
  CK(cudaGetLastError());
  return MDG_OK;
}

int mdg_download_all(mdg_solver *s, double *prim)
{
  if (!s || !prim) return fail(MDG_ERR_INVALID, "solver/prim");
  CK(cudaSetDevice(s->device));
  int rc = stage_all(s);
  if (rc != MDG_OK) return rc;
  launch_soa_to_aos(s->P, 0, s->ncell_total, s->d_stage_all, s->stream);
  CK(cudaMemcpyAsync(prim, s->d_stage_all, sizeof(double) * NPRIM * s->ncell_total, cudaMemcpyDeviceToHost,
                     s->stream));
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaGetLastError());
  return MDG_OK;
}

static cudaError_t ensure_dt_buffer(mdg_solver *s)
{
  if (s->d_dtbuf) return cudaSuccess;
  return cudaMalloc(&s->d_dtbuf, sizeof(double) * s->nprob);
}

static int queue_steps(mdg_solver *s, int nsteps)
{
  auto mark = [&](int k, int e) { if (s->timing) cudaEventRecord(s->ev[k][e], s->stream); };
  const bool mix3 = s->ndim == 3 && s->precision == MDG_PREC_MIXED;
  const bool mix2 = s->ndim == 2 && s->precision == MDG_PREC_MIXED;
  const bool mixed = s->ndim == 1 && s->precision == MDG_PREC_MIXED;   // the batched 1-D mixed sweep
  const bool queue = s->cfg.ctas_per_sm > 0;
  // the mixed stage launches of every lane (each lane's two tile lists), on stream st
  auto mixed_stage = [&](int stage, int l, cudaStream_t st) {
    const mdg_solver::Lane &L = s->lane[l];
    const StateSoA sst = stage ? s->PH : s->P, out = stage ? s->P : s->PH;
    launch_stage1d_mixed(stage, s->cfg.threads, mixed_grid(s, L.ntu), queue, s->d_probs, s->d_times,
                         s->d_mtiles + L.t0, s->d_queue + 2 * l, s->tb, sst, s->P, out, st, false);
    launch_stage1d_mixed(stage, s->cfg.threads, mixed_grid(s, L.ntt), queue, s->d_probs, s->d_times,
                         s->d_mtiles + L.t0 + L.ntu, s->d_queue + 2 * l + 1, s->tb, sst, s->P, out, st, true);
  };
  if (mixed && s->nlanes > 1 && !s->timing) {
    // lanes: each lane's whole step sequence on its own stream (its problems' time
    // records, dt and sweeps touch nothing of the other lanes)
    CK(cudaEventRecord(s->ev_fork, s->stream));
    for (int l = 1; l < s->nlanes; l++) CK(cudaStreamWaitEvent(s->lane_st[l], s->ev_fork, 0));
    for (int k = 0; k < nsteps; k++) {
      for (int l = 0; l < s->nlanes; l++) {
        const mdg_solver::Lane &L = s->lane[l];
        cudaStream_t st = l ? s->lane_st[l] : s->stream;
        const int n = L.m1 - L.m0;
        launch_dt_finalize(s->d_probs + L.m0, s->d_times + L.m0, n, s->d_err, st);
        if (s->any_mono) launch_monopole1d(s->d_probs + L.m0, s->d_times + L.m0, n, s->tb, s->P, st);
        mixed_stage(0, l, st);
        if (s->any_mono) launch_monopole1d(s->d_probs + L.m0, s->d_times + L.m0, n, s->tb, s->PH, st);
        mixed_stage(1, l, st);
        launch_finish(s->d_times + L.m0, n, st);
      }
    }
    for (int l = 1; l < s->nlanes; l++) {
      CK(cudaEventRecord(s->lane_ev[l], s->lane_st[l]));
      CK(cudaStreamWaitEvent(s->stream, s->lane_ev[l], 0));
    }
    CK(cudaGetLastError());
    return MDG_OK;
  }
  for (int k = 0; k < nsteps; k++) {
    mark(MDG_TIMER_DT, 0);
    launch_dt_finalize(s->d_probs, s->d_times, s->nprob, s->d_err, s->stream);
    mark(MDG_TIMER_DT, 1);
    mark(MDG_TIMER_STAGE0, 0);
    if (mixed && s->any_mono) launch_monopole1d(s->d_probs, s->d_times, s->nprob, s->tb, s->P, s->stream);
    if (mixed) {
      for (int l = 0; l < s->nlanes; l++) mixed_stage(0, l, s->stream);
    }
    else if (s->ndim == 3)
      launch_stage3d(0, mix3, s->s3, s->d_probs, s->d_times, s->P, s->P, s->PH, s->stream);
    else if (s->ndim == 1) {
      if (s->any_mono) launch_monopole1d(s->d_probs, s->d_times, s->nprob, s->tb, s->P, s->stream);
      launch_stage1d(0, s->d_probs, s->d_times, s->d_tiles, s->ntiles, s->tb, s->P, s->P, s->PH, s->stream,
                     &s->tm1);
    }
    else
      launch_stage2d(0, mix2, s->d_probs, s->d_times, s->d_tiles, s->ntx, s->d_tiles + s->ntx, s->nty, s->tb,
                     s->P, s->P, s->ACC, s->PH, s->d_shock0, s->d_shock1, s->stream);
    mark(MDG_TIMER_STAGE0, 1);
    mark(MDG_TIMER_STAGE1, 0);
    if (mixed && s->any_mono) launch_monopole1d(s->d_probs, s->d_times, s->nprob, s->tb, s->PH, s->stream);
    if (mixed) {
      for (int l = 0; l < s->nlanes; l++) mixed_stage(1, l, s->stream);
    }
    else if (s->ndim == 3)
      launch_stage3d(1, mix3, s->s3, s->d_probs, s->d_times, s->PH, s->P, s->P, s->stream);
    else if (s->ndim == 1) {
      if (s->any_mono) launch_monopole1d(s->d_probs, s->d_times, s->nprob, s->tb, s->PH, s->stream);
      launch_stage1d(1, s->d_probs, s->d_times, s->d_tiles, s->ntiles, s->tb, s->PH, s->P, s->P, s->stream,
                     &s->tm1);
    }
    else
      launch_stage2d(1, mix2, s->d_probs, s->d_times, s->d_tiles, s->ntx, s->d_tiles + s->ntx, s->nty, s->tb,
                     s->PH, s->P, s->ACC, s->P, s->d_shock0, s->d_shock1, s->stream);
    mark(MDG_TIMER_STAGE1, 1);
    mark(MDG_TIMER_FINISH, 0);
    launch_finish(s->d_times, s->nprob, s->stream);
    mark(MDG_TIMER_FINISH, 1);
    if (s->timing) {
      CK(cudaStreamSynchronize(s->stream));
      for (int t = 0; t < MDG_NTIMERS; t++) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, s->ev[t][0], s->ev[t][1]));
        s->tms[t] += ms;
        s->tcalls[t] += 1;
      }
    }
  }
  CK(cudaGetLastError());
  return MDG_OK;
}

int mdg_estimate_dt(mdg_solver *s, double *dt_out)
{
  if (!s) return fail(MDG_ERR_INVALID, "solver");
  CK(cudaSetDevice(s->device));
  launch_dt_finalize(s->d_probs, s->d_times, s->nprob, s->d_err, s->stream);
  CK(cudaGetLastError());
  if (dt_out) {
    std::vector<ProbTime> T(s->nprob);
    CK(cudaMemcpyAsync(T.data(), s->d_times, sizeof(ProbTime) * s->nprob, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    for (int m = 0; m < s->nprob; m++) dt_out[m] = T[m].dt;
  }
  return MDG_OK;
}

int mdg_estimate_dt_raw(mdg_solver *s, double *dt_out)
{
  if (!s || !dt_out) return fail(MDG_ERR_INVALID, "solver/dt_out");
  CK(cudaSetDevice(s->device));
  CK(ensure_dt_buffer(s));
  launch_raw_estimate(s->d_probs, s->d_times, s->nprob, s->d_dtbuf, s->stream);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(dt_out, s->d_dtbuf, sizeof(double) * s->nprob, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return MDG_OK;
}

int mdg_step_dt(mdg_solver *s, const double *dt)
{
  if (!s || !dt) return fail(MDG_ERR_INVALID, "solver/dt");
  for (int m = 0; m < s->nprob; m++)
    if (!(dt[m] > 0.0) || !(dt[m] < 1.0e300)) return fail(MDG_ERR_INVALID, "dt must be positive and finite");
  CK(cudaSetDevice(s->device));
  CK(ensure_dt_buffer(s));
  // the copy is staged from pageable memory before the call returns
  CK(cudaMemcpyAsync(s->d_dtbuf, dt, sizeof(double) * s->nprob, cudaMemcpyHostToDevice, s->stream));
  launch_set_dt(s->d_times, s->nprob, s->d_dtbuf, s->stream);
  return queue_steps(s, 1);
}

// Capture cfg.steps_per_graph steps of the launch sequence into a CUDA graph (once per
// launch shape).  Every kernel argument is fixed for the solver's life; what changes from
// step to step (dt, times, the work queue) lives in device memory.
static int ensure_graph(mdg_solver *s)
{
  const int k = s->cfg.steps_per_graph;
  if (s->graph && s->graph_steps == k) return MDG_OK;
  if (s->graph) {
    cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
  }
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
  const int rc = queue_steps(s, k);
  const cudaError_t e = cudaStreamEndCapture(s->stream, &g);
  if (rc != MDG_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return fail(MDG_ERR_CUDA, std::string("stream capture: ") + cudaGetErrorString(e));
  const cudaError_t ei = cudaGraphInstantiate(&s->graph, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) {
    s->graph = nullptr;
    return fail(MDG_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
  }
  s->graph_steps = k;
  return MDG_OK;
}

static void drop_graph(mdg_solver *s)
{
  if (s->graph) cudaGraphExecDestroy(s->graph);
  s->graph = nullptr;
  s->graph_steps = 0;
}

// mdg_step advances the solver with the resident stepper (launches of at most
// RESIDENT_STEPS steps each) rather than the per-phase launches
static bool uses_resident(const mdg_solver *s)
{
  return s->res_cs > 0 && s->cfg.resident && !s->timing;
}
constexpr int RESIDENT_STEPS = 256;

int mdg_step(mdg_solver *s, int nsteps)
{
  if (!s) return fail(MDG_ERR_INVALID, "solver");
  if (nsteps < 0) return fail(MDG_ERR_INVALID, "nsteps < 0");
  CK(cudaSetDevice(s->device));
  if (uses_resident(s)) {
    for (int left = nsteps; left > 0; left -= RESIDENT_STEPS)
      CK(launch_resident1d(s->res_cs, s->nprob, s->d_probs, s->d_times, s->tb, s->P, s->PH,
                           std::min(left, RESIDENT_STEPS), s->d_err, s->stream));
    return MDG_OK;
  }
  const int k = s->cfg.steps_per_graph;
  if (s->timing || k <= 0 || nsteps < k) return queue_steps(s, nsteps);
  int rc = ensure_graph(s);
  if (rc != MDG_OK) return rc;
  for (int g = 0; g < nsteps / k; g++) CK(cudaGraphLaunch(s->graph, s->stream));
  return queue_steps(s, nsteps % k);
}

int mdg_run_host(mdg_solver *const *solvers, int n, const double *const *h_in, double *const *h_out, int nsteps,
                 float *elapsed_ms)
{
  if (!solvers || !h_in || !h_out || n < 1) return fail(MDG_ERR_INVALID, "solvers/buffers");
  if (nsteps < 0) return fail(MDG_ERR_INVALID, "nsteps < 0");
  for (int i = 0; i < n; i++) {
    if (!solvers[i] || !h_in[i] || !h_out[i]) return fail(MDG_ERR_INVALID, "null solver or buffer");
    if (solvers[i]->device != solvers[0]->device) return fail(MDG_ERR_INVALID, "solvers on different devices");
    if (solvers[i]->timing) return fail(MDG_ERR_INVALID, "event timers are on (mdg_set_timing)");
  }
  CK(cudaSetDevice(solvers[0]->device));
  // everything that allocates or captures happens before the first copy
  for (int i = 0; i < n; i++) {
    mdg_solver *s = solvers[i];
    int rc = stage_all(s);
    if (rc != MDG_OK) return rc;
    if (!uses_resident(s) && s->cfg.steps_per_graph > 0 && nsteps >= s->cfg.steps_per_graph &&
        (rc = ensure_graph(s)) != MDG_OK)
      return rc;
  }
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::vector<cudaEvent_t> done(n, nullptr);
  auto cleanup = [&]() {
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (auto &e : done)
      if (e) cudaEventDestroy(e);
  };
#define CKR(call)                                                                      \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      cleanup();                                                                       \
      return fail(MDG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
    }                                                                                  \
  } while (0)
  CKR(cudaEventCreate(&ev0));
  CKR(cudaEventCreate(&ev1));
  for (int i = 0; i < n; i++) CKR(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming));
  cudaStream_t st0 = solvers[0]->stream;
  CKR(cudaEventRecord(ev0, st0));
  // the uploads first, in solver order (the copy engine serves them in turn), then every
  // solver's steps, each waiting only for its own upload on its own stream, then the
  // downloads
  for (int i = 0; i < n; i++) {
    mdg_solver *s = solvers[i];
    if (i > 0) CKR(cudaStreamWaitEvent(s->stream, ev0, 0));
    CKR(cudaMemcpyAsync(s->d_stage_all, h_in[i], sizeof(double) * NPRIM * s->ncell_total, cudaMemcpyHostToDevice,
                        s->stream));
    launch_aos_to_soa(s->d_stage_all, s->P, 0, s->ncell_total, s->stream);
    launch_reset_time_all(s->d_times, s->nprob, s->stream);
    if (s->ndim == 3) launch_initial_estimate3(s->s3, s->d_probs, s->d_times, s->P, s->stream);
    else launch_initial_estimate_all(s->d_probs, s->d_times, s->nprob, s->max_cells, s->tb, s->P, s->stream);
  }
  int rc = MDG_OK;
  for (int i = 0; i < n && rc == MDG_OK; i++) rc = mdg_step(solvers[i], nsteps);
  if (rc != MDG_OK) {
    for (int i = 0; i < n; i++) cudaStreamSynchronize(solvers[i]->stream);
    cleanup();
    return rc;
  }
  for (int i = 0; i < n; i++) {
    mdg_solver *s = solvers[i];
    launch_soa_to_aos(s->P, 0, s->ncell_total, s->d_stage_all, s->stream);
    CKR(cudaMemcpyAsync(h_out[i], s->d_stage_all, sizeof(double) * NPRIM * s->ncell_total, cudaMemcpyDeviceToHost,
                        s->stream));
    CKR(cudaEventRecord(done[i], s->stream));
    if (i > 0) CKR(cudaStreamWaitEvent(st0, done[i], 0));
  }
  CKR(cudaEventRecord(ev1, st0));
  CKR(cudaEventSynchronize(ev1));
  CKR(cudaGetLastError());
  if (elapsed_ms) CKR(cudaEventElapsedTime(elapsed_ms, ev0, ev1));
#undef CKR
  cleanup();
  return MDG_OK;
}

int mdg_get_launch_config(mdg_solver *s, mdg_launch_config *cfg)
{
  if (!s || !cfg) return fail(MDG_ERR_INVALID, "solver/cfg");
  *cfg = s->cfg;
  return MDG_OK;
}

int mdg_resident_cluster(mdg_solver *s, int *ctas)
{
  if (!s || !ctas) return fail(MDG_ERR_INVALID, "solver/ctas");
  *ctas = s->res_cs;
  return MDG_OK;
}

int mdg_set_launch_config(mdg_solver *s, const mdg_launch_config *cfg)
{
  if (!s || !cfg) return fail(MDG_ERR_INVALID, "solver/cfg");
  if (cfg->threads != 64 && cfg->threads != 128 && cfg->threads != 256)
    return fail(MDG_ERR_INVALID, "threads must be 64, 128 or 256");
  if (cfg->ctas_per_sm < 0 || cfg->ctas_per_sm > 64) return fail(MDG_ERR_INVALID, "ctas_per_sm out of [0, 64]");
  if (cfg->steps_per_graph < 0 || cfg->steps_per_graph > 10000)
    return fail(MDG_ERR_INVALID, "steps_per_graph out of [0, 10000]");
  if (cfg->run_length < 1 || cfg->run_length > 64) return fail(MDG_ERR_INVALID, "run_length out of [1, 64]");
  if (cfg->lanes < 1 || cfg->lanes > MDG_MAX_LANES) return fail(MDG_ERR_INVALID, "lanes out of [1, 4]");
  if (cfg->resident != 0 && cfg->resident != 1) return fail(MDG_ERR_INVALID, "resident must be 0 or 1");
  CK(cudaSetDevice(s->device));
  CK(cudaStreamSynchronize(s->stream));
  if (s->ndim == 3 && cfg->run_length != s->cfg.run_length) {
    std::string why;
    const int rc = sweep3_set_run_length(s->s3, cfg->run_length, why);
    if (rc != MDG_OK) return fail(rc, "run_length: " + why);
    drop_graph(s);
  }
  const bool reshape = cfg->threads != s->cfg.threads || cfg->lanes != s->cfg.lanes;
  const bool batched = s->precision == MDG_PREC_MIXED && s->ndim == 1;
  if (batched) {
    // rebuilds the tile lists (a new shape) or just resets every work queue
    int rc = build_mixed_tiles(s, cfg->threads, cfg->lanes);
    if (rc != MDG_OK) return rc;
  }
  if (reshape || cfg->ctas_per_sm != s->cfg.ctas_per_sm || cfg->steps_per_graph != s->cfg.steps_per_graph)
    drop_graph(s);
  s->cfg = *cfg;
  return MDG_OK;
}

int mdg_autotune(mdg_solver *s, int trial_steps, mdg_launch_config *best, double *ms_per_step)
{
  if (!s) return fail(MDG_ERR_INVALID, "solver");
  if (trial_steps < 1) return fail(MDG_ERR_INVALID, "trial_steps < 1");
  const bool dendritic = s->ndim == 3;
  if (!dendritic && (s->precision != MDG_PREC_MIXED || s->ndim != 1))
    return fail(MDG_ERR_NOTIMPL, "only the batched 1-D mixed sweep and the dendritic sweeps have tunable launch shapes");
  CK(cudaSetDevice(s->device));
  CK(cudaStreamSynchronize(s->stream));
  // the trials advance the state: keep a copy of everything a step changes
  const size_t sbytes = sizeof(double) * 2 * NPRIM * s->ncell_total;
  double *bk = nullptr;
  ProbTime *bt = nullptr;
  int berr = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = MDG_OK;
  auto restore = [&]() -> int {
    CK(cudaMemcpyAsync(s->d_state, bk, sbytes, cudaMemcpyDeviceToDevice, s->stream));
    CK(cudaMemcpyAsync(s->d_times, bt, sizeof(ProbTime) * s->nprob, cudaMemcpyDeviceToDevice, s->stream));
    CK(cudaMemcpyAsync(s->d_err, &berr, sizeof(int), cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return MDG_OK;
  };
  const mdg_launch_config orig = s->cfg;
  mdg_launch_config bestc = orig;
  double bestms = 1.0e300;
  do {
    if (cudaMalloc(&bk, sbytes) != cudaSuccess || cudaMalloc(&bt, sizeof(ProbTime) * s->nprob) != cudaSuccess) {
      rc = fail(MDG_ERR_OUTOFMEM, "autotune: no room for the state copy");
      break;
    }
    if (cudaMemcpy(bk, s->d_state, sbytes, cudaMemcpyDeviceToDevice) != cudaSuccess ||
        cudaMemcpy(bt, s->d_times, sizeof(ProbTime) * s->nprob, cudaMemcpyDeviceToDevice) != cudaSuccess ||
        cudaMemcpy(&berr, s->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
      rc = fail(MDG_ERR_CUDA, "autotune: set-up");
      break;
    }
    // candidate shapes: (threads, ctas_per_sm) of the mixed 1-D sweep, or the run length
    // of a dendritic sweep
    std::vector<mdg_launch_config> cand;
    const int k = orig.steps_per_graph;
    if (dendritic) {
      for (int len : {4, 8, 16, 32})
        cand.push_back(mdg_launch_config{orig.threads, orig.ctas_per_sm, k, len, 1, orig.resident});
    } else {
      for (int nt : {64, 128, 256}) {
        const int occ = mixed_max_ctas_per_sm(nt);
        for (int c : {0, 1, 2, 3, 4, 6, 8, 12, 16})
          if (c <= occ) cand.push_back(mdg_launch_config{nt, c, k, orig.run_length, 1, orig.resident});
      }
    }
    const int steps = (k > 0) ? ((trial_steps + k - 1) / k) * k : trial_steps;
    // one trial: the state restored, a warm-up (and graph capture), then `steps` timed steps
    auto trial = [&](const mdg_launch_config &c) -> int {
      int r = mdg_set_launch_config(s, &c);
      if (r == MDG_OK) r = restore();
      if (r == MDG_OK) r = mdg_step(s, k > 0 ? k : 1);
      if (r != MDG_OK) return r;
      float ms = 0.f;
      cudaError_t ce = cudaEventRecord(e0, s->stream);
      if (ce == cudaSuccess && (r = mdg_step(s, steps)) != MDG_OK) return r;
      if (ce == cudaSuccess) ce = cudaEventRecord(e1, s->stream);
      if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
      if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
      if (ce != cudaSuccess) return fail(MDG_ERR_CUDA, std::string("autotune timing: ") + cudaGetErrorString(ce));
      const double per = ms / steps;
      if (per < bestms) { bestms = per; bestc = c; }
      return MDG_OK;
    };
    for (size_t ci = 0; ci < cand.size() && rc == MDG_OK; ci++) rc = trial(cand[ci]);
    // the mixed 1-D sweep: lanes with the best (threads, ctas_per_sm)
    if (!dendritic) {
      const mdg_launch_config shape = bestc;
      for (int nl : {2, 4}) {
        if (rc != MDG_OK) break;
        mdg_launch_config c = shape;
        c.lanes = nl;
        rc = trial(c);
      }
    }
    if (rc == MDG_OK) rc = mdg_set_launch_config(s, &bestc);
    else mdg_set_launch_config(s, &orig);
    const int rc2 = restore();
    if (rc == MDG_OK) rc = rc2;
  } while (0);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(bk);
  cudaFree(bt);
  if (rc != MDG_OK) return rc;
  if (best) *best = bestc;
  if (ms_per_step) *ms_per_step = bestms;
  return MDG_OK;
}

int mdg_conserved_totals(mdg_solver *s, double *mass, double *energy)
{
  if (!s) return fail(MDG_ERR_INVALID, "solver");
  CK(cudaSetDevice(s->device));
  if (s->ndim == 3) launch_totals3(s->s3, s->P, s->d_totals, s->stream);
  else launch_conserved_totals(s->d_probs, s->nprob, s->tb, s->P, s->d_totals, s->stream);
  CK(cudaGetLastError());
  std::vector<double> h(2 * (size_t)s->nprob);
  CK(cudaMemcpyAsync(h.data(), s->d_totals, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  for (int m = 0; m < s->nprob; m++) {
    if (mass) mass[m] = h[2 * m];
    if (energy) energy[m] = h[2 * m + 1];
  }
  return MDG_OK;
}

int mdg_download_state(mdg_solver *s, int prob, double *prim, double *eos)
{
  if (!s || !prim) return fail(MDG_ERR_INVALID, "solver/prim");
  if (prob < 0 || prob >= s->nprob) return fail(MDG_ERR_INDEX, "problem index out of range");
  CK(cudaSetDevice(s->device));
  const ProbDev &P = s->hprobs[prob];
  const int64_t n = P.ncell;
  launch_soa_to_aos(s->P, P.cell_off, n, s->d_stage, s->stream);
  CK(cudaMemcpyAsync(prim, s->d_stage, sizeof(double) * NPRIM * n, cudaMemcpyDeviceToHost, s->stream));
  if (eos) {
    ProbTime T;
    CK(cudaMemcpyAsync(&T, s->d_times + prob, sizeof(ProbTime), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    // the reference's sim_eos holds the EOS of the last stage state (update_eos(sim_ph))
    launch_eos_aos_m(T.istep > 0 ? s->PH : s->P, s->d_probs, prob, P.cell_off, n, s->d_stage, s->stream);
    CK(cudaMemcpyAsync(eos, s->d_stage, sizeof(double) * NPRIM * n, cudaMemcpyDeviceToHost, s->stream));
  }
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaGetLastError());
  return MDG_OK;
}

int mdg_snapshot(mdg_solver *s, int prob)
{
  if (!s) return fail(MDG_ERR_INVALID, "solver");
  if (prob < 0 || prob >= s->nprob) return fail(MDG_ERR_INDEX, "problem index out of range");
  CK(cudaSetDevice(s->device));
  if (s->snap_pending) CK(cudaEventSynchronize(s->ev_snap_done));   // one snapshot in flight
  const ProbDev &P = s->hprobs[prob];
  const int64_t n = P.ncell;
  const size_t need = (size_t)2 * NPRIM * n + sizeof(ProbTime) / sizeof(double) + 1;
  if (need > s->snap_cap) {
    cudaFree(s->d_snap);
    s->d_snap = nullptr;
    if (s->h_snap) cudaFreeHost(s->h_snap);
    s->h_snap = nullptr;
    s->snap_cap = 0;
    CK(cudaMalloc(&s->d_snap, sizeof(double) * need));
    CK(cudaMallocHost(&s->h_snap, sizeof(double) * need));
    s->snap_cap = need;
  }
  if (!s->copy_stream) {
    CK(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&s->ev_snap, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&s->ev_snap_done, cudaEventDisableTiming));
  }
  // device-side copies on the solver's stream (the next step waits only for these)
  launch_soa_to_aos(s->P, P.cell_off, n, s->d_snap, s->stream);
  launch_eos_aos_sel(s->P, s->PH, s->d_probs, s->d_times, prob, P.cell_off, n, s->d_snap + NPRIM * n, s->stream);
  CK(cudaMemcpyAsync(s->d_snap + 2 * NPRIM * n, s->d_times + prob, sizeof(ProbTime), cudaMemcpyDeviceToDevice,
                     s->stream));
  CK(cudaEventRecord(s->ev_snap, s->stream));
  // the host copy overlaps whatever the solver's stream does next
  CK(cudaStreamWaitEvent(s->copy_stream, s->ev_snap, 0));
  CK(cudaMemcpyAsync(s->h_snap, s->d_snap, sizeof(double) * need, cudaMemcpyDeviceToHost, s->copy_stream));
  CK(cudaEventRecord(s->ev_snap_done, s->copy_stream));
  CK(cudaGetLastError());
  s->snap_prob = prob;
  s->snap_n = n;
  s->snap_pending = true;
  return MDG_OK;
}

static int snap_wait(mdg_solver *s)
{
  if (!s->snap_pending) return fail(MDG_ERR_LOGICAL, "no snapshot has been taken");
  CK(cudaSetDevice(s->device));
  CK(cudaEventSynchronize(s->ev_snap_done));
  return MDG_OK;
}

int mdg_snapshot_read(mdg_solver *s, double *prim, double *eos, double *t)
{
  if (!s) return fail(MDG_ERR_INVALID, "solver");
  int rc = snap_wait(s);
  if (rc != MDG_OK) return rc;
  const int64_t n = s->snap_n;
  if (prim) std::memcpy(prim, s->h_snap, sizeof(double) * NPRIM * n);
  if (eos) std::memcpy(eos, s->h_snap + NPRIM * n, sizeof(double) * NPRIM * n);
  if (t) {
    ProbTime T;
    std::memcpy(&T, s->h_snap + 2 * NPRIM * n, sizeof T);
    *t = T.t;
  }
  return MDG_OK;
}

int mdg_snapshot_write_ascii1(mdg_solver *s, const char *path)
{
  if (!s || !path) return fail(MDG_ERR_INVALID, "solver/path");
  int rc = snap_wait(s);
  if (rc != MDG_OK) return rc;
  const mdg_problem_desc &d = s->descs[s->snap_prob];
  if (d.ndim != 1) return fail(MDG_ERR_NOTIMPL, "dump_ascii1 writes 1-D problems");
  const int64_t n = s->snap_n;
  const double *prim = s->h_snap, *eos = s->h_snap + NPRIM * n;
  ProbTime T;
  std::memcpy(&T, s->h_snap + 2 * NPRIM * n, sizeof T);
  // the reference's zone geometry (volume, scale[0][0]) from its Romberg tables
  const int64_t w = d.n1 + 2 * NG;
  std::vector<double> geo((size_t)GF_NFIELDS * w, 0.0);
  build_geo_1d(d, geo.data(), w, 0);
  FILE *fp = std::fopen(path, "w");
  if (!fp) return fail(MDG_ERR_IO, std::string("cannot open ") + path);
  // dump_ascii1 (io.c:111-220): "# t", then per zone x (r on spherical grids), the
  // primitives with the velocity in physical units (scale[0][0] v^1), the EOS record, the
  // enclosed mass at the zone centre and the two lapse columns (1 without GR_MONOPOLE)
  std::fprintf(fp, "# %g\n", T.t);
  double mass = 0.0;
  for (int64_t i = 0; i < n; i++) {
    double x = d.startx[0] + (i + 0.5) * d.dx[0];
    if (d.geom == MDG_SPHERICAL) x = radial_coordinate(d, x);
    const double s00 = geo[(size_t)GF_S00 * w + i + NG], vol = geo[(size_t)GF_VOL * w + i + NG];
    std::fprintf(fp, "%16.14e ", x);
    const double *p = prim + NPRIM * i;
    const double scale[NPRIM] = {1.0, 1.0, s00, 1.0, 1.0};
    for (int v = 0; v < NPRIM; v++) std::fprintf(fp, "%16.14e ", p[v] * scale[v]);
    for (int v = 0; v < NPRIM; v++) std::fprintf(fp, "%16.15e ", eos[NPRIM * i + v]);
    const double dm = vol * p[RHO];
    std::fprintf(fp, "%16.15e ", mass + 0.5 * dm);
    mass += dm;
    std::fprintf(fp, "%16.15e %16.15e ", 1.0, 1.0);
    std::fprintf(fp, "\n");
  }
  const bool ok = std::ferror(fp) == 0;
  std::fclose(fp);
  if (!ok) return fail(MDG_ERR_IO, std::string("write failed: ") + path);
  return MDG_OK;
}

int mdg_dump_ascii1(mdg_solver *s, int prob, const char *path)
{
  int rc = mdg_snapshot(s, prob);
  if (rc != MDG_OK) return rc;
  return mdg_snapshot_write_ascii1(s, path);
}

int mdg_get_time(mdg_solver *s, int prob, double *t, double *dt_last, int *istep)
{
  if (!s) return fail(MDG_ERR_INVALID, "solver");
  if (prob < 0 || prob >= s->nprob) return fail(MDG_ERR_INDEX, "problem index out of range");
  CK(cudaSetDevice(s->device));
  ProbTime T;
  CK(cudaMemcpyAsync(&T, s->d_times + prob, sizeof(ProbTime), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  if (t) *t = T.t;
  if (dt_last) *dt_last = T.dt;
  if (istep) *istep = T.istep;
  return MDG_OK;
}

int mdg_set_time(mdg_solver *s, int prob, double t, int istep)
{
  if (!s) return fail(MDG_ERR_INVALID, "solver");
  if (prob < 0 || prob >= s->nprob) return fail(MDG_ERR_INDEX, "problem index out of range");
  if (!std::isfinite(t) || istep < 0) return fail(MDG_ERR_INVALID, "t must be finite and istep >= 0");
  CK(cudaSetDevice(s->device));
  ProbTime T;
  CK(cudaMemcpyAsync(&T, s->d_times + prob, sizeof(ProbTime), cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  // the record a run resumed from a restart starts with: Time and Step of the file, no
  // step of this process yet (dtold = 1e100, main.c:194); the running min_dt holds the
  // zone terms of the uploaded state (estimate_dt's first call, step.c:171-174)
  T.t = t;
  T.istep = istep;
  T.dt = 0.0;
  T.dtold = 1.0e100;
  T.t_bc1 = 0.0;
  T.t_next = 0.0;
  T.dt_ready = 0;
  T.done = 0;
  CK(cudaMemcpyAsync(s->d_times + prob, &T, sizeof(ProbTime), cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return MDG_OK;
}

namespace {
// restart file: this header, then ncell x 5 doubles in the [zone][var] order of sim_p
struct RestartHeader {
  char magic[8];       // "MDGRST1" and a NUL
  int32_t ndim, n1, n2, n3;
  int32_t istep, reserved;
  int64_t ncell;
  double t;
};
const char kRestartMagic[8] = {'M', 'D', 'G', 'R', 'S', 'T', '1', '\0'};
}  // namespace

int mdg_restart_write(mdg_solver *s, int prob, const char *path)
{
  if (!s || !path) return fail(MDG_ERR_INVALID, "solver/path");
  if (prob < 0 || prob >= s->nprob) return fail(MDG_ERR_INDEX, "problem index out of range");
  const mdg_problem_desc &d = s->descs[prob];
  const int64_t n = s->hprobs[prob].ncell;
  std::vector<double> prim((size_t)NPRIM * n);
  int rc = mdg_download_state(s, prob, prim.data(), nullptr);
  if (rc != MDG_OK) return rc;
  RestartHeader h{};
  std::memcpy(h.magic, kRestartMagic, 8);
  h.ndim = d.ndim; h.n1 = d.n1; h.n2 = d.ndim > 1 ? d.n2 : 1; h.n3 = d.ndim > 2 ? d.n3 : 1;
  h.ncell = n;
  rc = mdg_get_time(s, prob, &h.t, nullptr, &h.istep);
  if (rc != MDG_OK) return rc;
  FILE *f = std::fopen(path, "wb");
  if (!f) return fail(MDG_ERR_IO, std::string("cannot open ") + path);
  const bool ok = std::fwrite(&h, sizeof h, 1, f) == 1 &&
                  std::fwrite(prim.data(), sizeof(double), prim.size(), f) == prim.size();
  if (std::fclose(f) != 0 || !ok) return fail(MDG_ERR_IO, std::string("cannot write ") + path);
  return MDG_OK;
}

int mdg_restart_read(mdg_solver *s, int prob, const char *path)
{
  if (!s || !path) return fail(MDG_ERR_INVALID, "solver/path");
  if (prob < 0 || prob >= s->nprob) return fail(MDG_ERR_INDEX, "problem index out of range");
  const mdg_problem_desc &d = s->descs[prob];
  const int64_t n = s->hprobs[prob].ncell;
  FILE *f = std::fopen(path, "rb");
  if (!f) return fail(MDG_ERR_IO, std::string("cannot open ") + path);
  RestartHeader h{};
  std::vector<double> prim((size_t)NPRIM * n);
  bool ok = std::fread(&h, sizeof h, 1, f) == 1;
  const bool same = ok && std::memcmp(h.magic, kRestartMagic, 8) == 0 && h.ndim == d.ndim && h.n1 == d.n1 &&
                    h.n2 == (d.ndim > 1 ? d.n2 : 1) && h.n3 == (d.ndim > 2 ? d.n3 : 1) && h.ncell == n;
  if (same) ok = std::fread(prim.data(), sizeof(double), prim.size(), f) == prim.size();
  std::fclose(f);
  if (!ok) return fail(MDG_ERR_IO, std::string("cannot read ") + path);
  if (!same) return fail(MDG_ERR_INVALID, std::string(path) + ": not a restart file of this problem's grid");
  int rc = mdg_upload_state(s, prob, prim.data());
  if (rc != MDG_OK) return rc;
  return mdg_set_time(s, prob, h.t, h.istep);
}

int mdg_get_stream(mdg_solver *s, void **stream)
{
  if (!s || !stream) return fail(MDG_ERR_INVALID, "solver/stream");
  *stream = (void *)s->stream;
  return MDG_OK;
}

int mdg_synchronize(mdg_solver *s)
{
  if (!s) return fail(MDG_ERR_INVALID, "solver");
  CK(cudaSetDevice(s->device));
  CK(cudaStreamSynchronize(s->stream));
  int err = 0;
  CK(cudaMemcpy(&err, s->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) return fail(err, "a time step estimate dropped below dtmin");
  // non-finite states flagged by the update kernels, per problem
  std::vector<ProbTime> T(s->nprob);
  CK(cudaMemcpy(T.data(), s->d_times, sizeof(ProbTime) * s->nprob, cudaMemcpyDeviceToHost));
  for (int m = 0; m < s->nprob; m++)
    if (T[m].err) return fail(T[m].err, "problem " + std::to_string(m) + ": non-finite state or dt below dtmin");
  return MDG_OK;
}

int mdg_set_timing(mdg_solver *s, int enable)
{
  if (!s) return fail(MDG_ERR_INVALID, "solver");
  CK(cudaSetDevice(s->device));
  if (enable && !s->ev[0][0]) {
    for (int k = 0; k < MDG_NTIMERS; k++)
      for (int e = 0; e < 2; e++) CK(cudaEventCreate(&s->ev[k][e]));
  }
  s->timing = enable != 0;
  for (int k = 0; k < MDG_NTIMERS; k++) { s->tms[k] = 0.0; s->tcalls[k] = 0; }
  return MDG_OK;
}

int mdg_get_timers(mdg_solver *s, double *ms, long long *calls)
{
  if (!s) return fail(MDG_ERR_INVALID, "solver");
  for (int k = 0; k < MDG_NTIMERS; k++) {
    if (ms) ms[k] = s->tms[k];
    if (calls) calls[k] = s->tcalls[k];
  }
  return MDG_OK;
}

int mdg_write_timers(mdg_solver *s, int prob, const char *path)
{
  if (!s || !path) return fail(MDG_ERR_INVALID, "solver/path");
  double t = 0.0;
  int istep = 0;
  int rc = mdg_get_time(s, prob, &t, nullptr, &istep);
  if (rc != MDG_OK) return rc;
  static const char *names[MDG_NTIMERS] = {"estimate_dt", "stage0", "stage1", "finish"};
  FILE *probe = std::fopen(path, "r");
  const bool fresh = probe == nullptr;
  if (probe) std::fclose(probe);
  FILE *f = std::fopen(path, "a");
  if (!f) return fail(MDG_ERR_IO, std::string("cannot open ") + path);
  bool ok = true;
  if (fresh) ok = std::fprintf(f, "timer,time,step,ncycle,max,min,avg\n") > 0;
  for (int k = 0; k < MDG_NTIMERS && ok; k++) {
    // one process: the maximum, minimum and mean over ranks are its own total, in seconds
    const double sec = s->tms[k] * 1.0e-3;
    ok = std::fprintf(f, "%s,%f,%d,%lu,%f,%f,%f\n", names[k], t, istep, (unsigned long)s->tcalls[k], sec, sec,
                      sec) > 0;
  }
  if (std::fclose(f) != 0 || !ok) return fail(MDG_ERR_IO, std::string("cannot write ") + path);
  return MDG_OK;
}

struct mdg_eos_table {
  int device = 0;
  int num_sms = 0;
  mdg_eos_grid g{};
  double2 *d_f = nullptr;
  cudaStream_t stream = nullptr;
  EosTableDev dev() const
  {
    return EosTableDev{d_f, g.ny, g.nr, g.nt, g.r1, g.r2, g.t1, g.t2, g.y1, g.y2, g.const_hack};
  }
};

int mdg_eos_table_destroy(mdg_eos_table *t)
{
  if (!t) return MDG_OK;
  cudaSetDevice(t->device);
  if (t->stream) cudaStreamSynchronize(t->stream);
  cudaFree(t->d_f);
  if (t->stream) cudaStreamDestroy(t->stream);
  delete t;
  return MDG_OK;
}

int mdg_eos_table_create(const mdg_eos_grid *grid, const double *table, int device, mdg_eos_table **out)
{
  if (!grid || !table || !out) return fail(MDG_ERR_INVALID, "grid/table/out");
  *out = nullptr;
  const mdg_eos_grid &g = *grid;
  if (g.nrec < 12 || g.ny < 2 || g.nr < 2 || g.nt < 2)
    return fail(MDG_ERR_INVALID, "the table needs nrec >= 12 and at least 2 points per axis");
  if (!(g.r2 > g.r1) || !(g.t2 > g.t1) || !(g.y2 > g.y1) || !std::isfinite(g.const_hack))
    return fail(MDG_ERR_INVALID, "table bounds must be finite and increasing");
  int ndev = 0;
  CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(MDG_ERR_INVALID, "device ordinal out of range");
  CK(cudaSetDevice(device));
  const size_t npt = (size_t)g.ny * g.nr * g.nt;
  // records 1, 2, 3, 12 (energy, log pressure, entropy, Gamma_1) interleaved per grid point
  std::vector<double> hf(4 * npt);
  const double *e = table, *lp = table + 1 * npt, *en = table + 2 * npt, *g1 = table + 11 * npt;
  for (size_t k = 0; k < npt; k++) {
    hf[4 * k + 0] = e[k];
    hf[4 * k + 1] = lp[k];
    hf[4 * k + 2] = en[k];
    hf[4 * k + 3] = g1[k];
  }
  mdg_eos_table *t = new mdg_eos_table();
  t->device = device;
  t->g = g;
  auto bail = [&](cudaError_t e) {
    mdg_eos_table_destroy(t);
    if (e == cudaErrorMemoryAllocation) return fail(MDG_ERR_OUTOFMEM, "no device memory for the EOS table");
    return fail(MDG_ERR_CUDA, std::string("EOS table: ") + cudaGetErrorString(e));
  };
  cudaError_t ce = cudaDeviceGetAttribute(&t->num_sms, cudaDevAttrMultiProcessorCount, device);
  if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking);
  if (ce == cudaSuccess) ce = cudaMalloc(&t->d_f, sizeof(double) * 4 * npt);
  if (ce == cudaSuccess) ce = cudaMemcpy(t->d_f, hf.data(), sizeof(double) * 4 * npt, cudaMemcpyHostToDevice);
  if (ce != cudaSuccess) return bail(ce);
  *out = t;
  return MDG_OK;
}

int mdg_eos_given_rex(mdg_eos_table *t, long long n, const double *rho, const double *u, const double *ye,
                      double *temp, double *press, double *cs, double *ent, double *gam1, void *stream)
{
  if (!t) return fail(MDG_ERR_INVALID, "table");
  if (n < 0) return fail(MDG_ERR_INVALID, "n < 0");
  if (n > 0 && (!rho || !u || !ye || !temp || !press || !cs || !ent || !gam1))
    return fail(MDG_ERR_INVALID, "null zone array");
  CK(cudaSetDevice(t->device));
  launch_eos_rex(t->dev(), n, rho, u, ye, temp, press, cs, ent, gam1, t->num_sms, (cudaStream_t)stream);
  CK(cudaGetLastError());
  return MDG_OK;
}

int mdg_eos_given_rex_host(mdg_eos_table *t, long long n, const double *rho, const double *u, const double *ye,
                           double *temp, double *press, double *cs, double *ent, double *gam1)
{
  if (!t) return fail(MDG_ERR_INVALID, "table");
  if (n < 0) return fail(MDG_ERR_INVALID, "n < 0");
  if (n == 0) return MDG_OK;
  if (!rho || !u || !ye || !temp || !press || !cs || !ent || !gam1) return fail(MDG_ERR_INVALID, "null zone array");
  CK(cudaSetDevice(t->device));
  const size_t b = sizeof(double) * (size_t)n;
  double *d = nullptr;
  CK(cudaMalloc(&d, 8 * b));
  double *dz[8];
  for (int k = 0; k < 8; k++) dz[k] = d + (size_t)k * (size_t)n;
  const double *hin[4] = {rho, u, ye, temp};
  double *hout[5] = {temp, press, cs, ent, gam1};
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < 4 && e == cudaSuccess; k++)
    e = cudaMemcpyAsync(dz[k], hin[k], b, cudaMemcpyHostToDevice, t->stream);
  if (e == cudaSuccess) {
    launch_eos_rex(t->dev(), n, dz[0], dz[1], dz[2], dz[3], dz[4], dz[5], dz[6], dz[7], t->num_sms, t->stream);
    e = cudaGetLastError();
  }
  double *dout[5] = {dz[3], dz[4], dz[5], dz[6], dz[7]};
  for (int k = 0; k < 5 && e == cudaSuccess; k++)
    e = cudaMemcpyAsync(hout[k], dout[k], b, cudaMemcpyDeviceToHost, t->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(t->stream);
  cudaFree(d);
  if (e != cudaSuccess) return fail(MDG_ERR_CUDA, std::string("mdg_eos_given_rex_host: ") + cudaGetErrorString(e));
  return MDG_OK;
}

int mdg_destroy(mdg_solver *s)
{
  if (!s) return MDG_OK;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  free_all(s);
  delete s;
  return MDG_OK;
}

}  // extern "C"
