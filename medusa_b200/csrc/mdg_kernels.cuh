// Shared declarations of the sweep kernels and their launch helpers.
#pragma once
#include <cuda_runtime.h>
#include <string>
#include "mdg_internal.h"

namespace mdg {

// Structure-of-arrays state of all problems of a solver: v[var][zone], zones of problem m
// at [cell_off, cell_off + n1*n2), i-major, no ghost storage (boundaries are applied on
// the fly as index maps).
struct StateSoA { double *v[NPRIM]; };

struct Tables {
  const double *rc0;     // direction-0 reconstruction table, RC_NFIELDS x rc0_stride
  int64_t rc0_stride;
  const double *rc1;     // direction-1 reconstruction table (2-D)
  int64_t rc1_stride;
  const double *geo;     // 1-D face/zone geometry, GF_NFIELDS x geo_stride
  int64_t geo_stride;
  const float *mx;       // FP32 reconstruction weights (mixed precision), MX_NFIELDS x geo_stride: 1-D problems,
                         // and direction 0 of 2-D problems (indexed like rc0)
  const float *mx1;      // direction-1 FP32 weights of 2-D problems, indexed like rc1
  double *gmono;         // monopole gravity at the zone centroids of 1-D problems (ProbDev::mono_off)
};

// Device work queue of the persistent mixed-precision sweep: one head counter per RK
// stage (each stage resets the other's head, so a step needs no reset launch) and the
// number of (problem, tile) items in the tile list.
struct WorkQueue { unsigned int head[2]; int ntiles; int pad; };

// One work tile: problem, first output row i0, first output column j0 (2-D).
struct Tile { int prob; int i0; int j0; int pad; };

constexpr int NT1 = 128;          // threads per 1-D tile (126 output zones)
constexpr int TILE1 = NT1 - 2;
// 2-D tile shapes and occupancy targets (compile-time tunables)
#ifndef MDG_TIX2
#define MDG_TIX2 32
#endif
#ifndef MDG_TIY2
#define MDG_TIY2 16
#endif
#ifndef MDG_XMINB
#define MDG_XMINB 4
#endif
#ifndef MDG_YMINB
#define MDG_YMINB 4
#endif
constexpr int NTX2 = 128;         // threads (= columns) per direction-0 tile
constexpr int TIX2 = MDG_TIX2;    // rows per direction-0 tile
constexpr int NTY2 = 128;         // threads per direction-1 tile (126 output columns)
constexpr int TJY2 = NTY2 - 2;
constexpr int TIY2 = MDG_TIY2;    // rows per direction-1 tile

struct TmaTables1d;
// Tabulated EOS on the device (mdg_eos_table.cu): the records f[jy][jr][jt] = {e, log p,
// s, Gamma_1} as two double2 per grid point; grid sizes and bounds as the reference's
// DEFINE_EOSCONST_1.
struct EosTableDev {
  const double2 *f;
  int ny, nr, nt;
  double r1, r2, t1, t2, y1, y2, const_hack;
};
void launch_eos_rex(const EosTableDev &d, long long n, const double *rho, const double *u, const double *ye,
                    double *temp, double *press, double *cs, double *ent, double *gam1, int num_sms,
                    cudaStream_t st);
// The resident 1-D stepper (plain FP64): CTAs per problem for problems of at most
// max_tiles tiles (a power of two), or 0 when it cannot run (more than
// RESIDENT1D_MAX_TILES tiles, or such a cluster does not fit this device); the launch of
// nsteps steps of nprob problems with that cluster size.
constexpr int RESIDENT1D_MAX_TILES = 16;
int resident1d_cluster_size(int max_tiles);
cudaError_t launch_resident1d(int cs, int nprob, const ProbDev *probs, ProbTime *times, const Tables &tb,
                              StateSoA p, StateSoA ph, int nsteps, int *err, cudaStream_t st);
// One RK stage of the plain FP64 1-D sweep; tm (may be NULL): tensor maps of tb's rc0 and
// geo tables, with which each tile's tables are staged into shared memory by TMA.
void launch_stage1d(int stage, const ProbDev *probs, ProbTime *times, const Tile *tiles, int ntiles,
                    const Tables &tb, StateSoA stage_state, StateSoA state_n, StateSoA out,
                    cudaStream_t st, const TmaTables1d *tm = nullptr);
void launch_stage2d(int stage, bool mixed, const ProbDev *probs, ProbTime *times, const Tile *xtiles, int nxt,
                    const Tile *ytiles, int nyt, const Tables &tb, StateSoA stage_state, StateSoA state_n,
                    StateSoA acc, StateSoA out, unsigned char *shock0, unsigned char *shock1, cudaStream_t st);
// Mixed-precision 1-D stage: nt threads per CTA (tile = nt-2 zones), grid CTAs; with
// use_queue the CTAs are persistent and pull tiles from q, else CTA b takes tile b.  tab:
// the tiles' problems read the Romberg tables (ProbDev::geo_tab), the others' geometry is
// evaluated in closed form.
void launch_stage1d_mixed(int stage, int nt, int grid, bool use_queue, const ProbDev *probs, ProbTime *times,
                          const Tile *tiles, WorkQueue *q, const Tables &tb, StateSoA stage_state,
                          StateSoA state_n, StateSoA out, cudaStream_t st, bool tab);
int mixed_max_ctas_per_sm(int nt);
// Monopole self-gravity of every 1-D problem with ProbDev::mono from its stage state:
// the acceleration at each zone centroid into tb.gmono (gravity.c:145-425).
void launch_monopole1d(const ProbDev *probs, ProbTime *times, int nprob, const Tables &tb, StateSoA stage_state,
                       cudaStream_t st);
void launch_conserved_totals(const ProbDev *probs, int nprob, const Tables &tb, StateSoA s, double *out,
                             cudaStream_t st);
// Reconstruction, geometry and FP32-weight tables of 1-D problem m, built on the device
// from closed-form moments (the mixed-precision sweep's tables), at columns geo_off..+n1+3.
void launch_build_tables_1d(const ProbDev *probs, int m, int n1, double *rc, double *geo, float *mx,
                            int64_t stride, cudaStream_t st);
// 3-D dendritic spherical sweep (mdg_sweep3d.cu): one problem, in slot 0.
struct Sweep3;
int sweep3_create(const mdg_problem_desc &d, Sweep3 **out, std::string &why);
void sweep3_destroy(Sweep3 *w);
int64_t sweep3_ncell(const Sweep3 *w);
int64_t sweep3_bytes(const Sweep3 *w);   // device memory of the grid tables, face fluxes and bits
// Faces per work item of the radial and theta run kernels (1..64); rebuilds the work lists.
int sweep3_set_run_length(Sweep3 *w, int run_length, std::string &why);
void launch_stage3d(int stage, bool mixed, Sweep3 *w, const ProbDev *probs, ProbTime *times,
                    StateSoA stage_state, StateSoA state_n, StateSoA out, cudaStream_t st);
void launch_initial_estimate3(Sweep3 *w, const ProbDev *probs, ProbTime *times, StateSoA s, cudaStream_t st);
void launch_totals3(Sweep3 *w, StateSoA s, double *out, cudaStream_t st);
void launch_dt_finalize(const ProbDev *probs, ProbTime *times, int nprob, int *err, cudaStream_t st);
void launch_finish(ProbTime *times, int nprob, cudaStream_t st);
// estimate_dt() alone into out[m]; and the time record of a step with the host's dt[m]
void launch_raw_estimate(const ProbDev *probs, const ProbTime *times, int nprob, double *out, cudaStream_t st);
void launch_set_dt(ProbTime *times, int nprob, const double *dt, cudaStream_t st);
void launch_reset_time(ProbTime *times, int m, cudaStream_t st);
void launch_initial_estimate_one(const ProbDev *probs, ProbTime *times, int m, int64_t ncell,
                                 const Tables &tb, StateSoA s, cudaStream_t st);
void launch_reset_time_all(ProbTime *times, int nprob, cudaStream_t st);
void launch_initial_estimate_all(const ProbDev *probs, ProbTime *times, int nprob, int64_t max_cells,
                                 const Tables &tb, StateSoA s, cudaStream_t st);
void launch_aos_to_soa(const double *aos, StateSoA s, int64_t off, int64_t n, cudaStream_t st);
void launch_soa_to_aos(StateSoA s, int64_t off, int64_t n, double *aos, cudaStream_t st);
void launch_eos_aos_sel(StateSoA p, StateSoA ph, const ProbDev *probs, const ProbTime *times, int m, int64_t off,
                        int64_t n, double *aos, cudaStream_t st);
void launch_eos_aos_m(StateSoA s, const ProbDev *probs, int m, int64_t off, int64_t n, double *aos,
                      cudaStream_t st);

}  // namespace mdg
