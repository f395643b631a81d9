/*
 * medusa_b200 -- C ABI of the B200 hydrodynamic sweep.
 *
 * This is the drop-in boundary for the reference's hot path.  The reference's time
 * loop (main.c:206-313) calls three functions with global state:
 *
 *   void estimate_dt(void);   step.c:163-203   (declared decs.h:756)
 *   void step(void);          step.c:28-129    (declared decs.h:755)
 *   void update_cpu(void);    step.c:16-24     (declared decs.h:754)
 *
 * and establishes device residency in the upload block main.c:129-165.  The entry
 * points below replace those with handle-based calls: one handle (a "solver") holds
 * one or more independent problems of the same dimensionality that advance together.
 * All arguments are plain C types; no call allocates on behalf of the caller except
 * mdg_create (device state) and none calls exit().  Every call returns an MDG_*
 * status; the reference's own error codes (decs.h:89-98) map onto the same values.
 *
 * Semantics follow the reference exactly: the primitive state (rho, internal energy
 * density u, contravariant velocities v1 v2 v3) lives on the device between calls; one
 * mdg_step is one pass of the main.c time loop: estimate_dt() + the dt safety/clip
 * rules of main.c:228-251 + the two-stage step() + t += dt.
 */
#ifndef MEDUSA_B200_H_
#define MEDUSA_B200_H_

#ifdef __cplusplus
extern "C" {
#endif

/* status codes: same numbering as decs.h:89-98 */
#define MDG_OK             0
#define MDG_ERR_INVALID    1
#define MDG_ERR_INDEX      2
#define MDG_ERR_NOTFOUND   3
#define MDG_ERR_IO         4
#define MDG_ERR_NOTIMPL    5
#define MDG_ERR_OUTOFMEM   6
#define MDG_ERR_PARFILE    7
#define MDG_ERR_LOGICAL    8
#define MDG_ERR_INTERNAL   9
#define MDG_ERR_CUDA       10   /* a CUDA runtime call failed; see mdg_last_error_message */
#define MDG_ERR_NONFINITE  11   /* a non-finite time step was produced (dt < dtmin, main.c:229) */

/* geometry (decs.h:669-671), EOS (decs.h:674-675), boundary kinds (decs.h:64-69) */
#define MDG_CARTESIAN 0
#define MDG_SPHERICAL 1
#define MDG_GAMMA_LAW 0
#define MDG_POLYTROPIC 1
#define MDG_BC_OUTFLOW 0
#define MDG_BC_REFLECT 1
#define MDG_BC_EXTRAP 2
#define MDG_BC_PERIODIC 3
#define MDG_BC_PROB 4
#define MDG_BC_SPHERICAL_ORIGIN 5
/* PROB boundary hooks restated on the device (the reference's prob_bounds callbacks) */
#define MDG_PROB_NONE 0
#define MDG_PROB_NOH 1   /* problems/init_spherical_noh.c:63-79 */
#define MDG_PROB_DUST 2  /* problems/init_dustcollapse.c:77-113: outflow, v^r = -1/sqrt(r) in the ghost zones */
/* radial coordinate maps r(x) of spherical grids (RCOORD, metric_spherical_general.c:149-219) */
#define MDG_RCOORD_UNIFORM 0   /* r = |x| */
#define MDG_RCOORD_SINH 1      /* r = rtrans sinh(|x| / rtrans): zones of width dx near the
                                  centre, growing geometrically outside rtrans */
#define MDG_RCOORD_SINH_MODIFIED 2  /* the SINH map minus facta [sigmoid((|x| - factb) / factc)
                                       - sigmoid(-factb / factc)] (the reference's default) */
#define MDG_RCOORD_LOG 3       /* r = rtrans exp(|x| / rtrans): zones log-spaced outwards from
                                  r = rtrans at x = 0 (inner zone width dx there).  Not one of
                                  the reference's maps: added in the form of its SINH branch
                                  for grids that start away from the origin */
/* theta maps th(x), x in [-1, 1] (THCOORD, metric_spherical_general.c:222-290) */
#define MDG_THCOORD_UNIFORM 0  /* th = pi (x + 1) / 2 */
#define MDG_THCOORD_POLYTH 1   /* th = poly_norm x (1 + (x/poly_xt)^poly_alpha / (poly_alpha + 1)) + pi/2,
                                  zones concentrated at the equator (the reference's default) */

/* arithmetic of the sweep */
#define MDG_PREC_FP64 0   /* plain: FP64 throughout, the reference's operation order */
#define MDG_PREC_MIXED 1  /* FP32 reconstruction/limiting/Riemann, FP64 accumulation,
                             sources, geometry and dt */

/*
 * One problem.  Replaces the compile-time switches of setup.mk/build.h (NDIM, GEOM,
 * EOS, ENFORCE_FLOORS; Makefile:157-212), the run-time keys of the input.* file that
 * the sweep reads (io.c:4979-5785: n1 n2 n3 cfl dt_init_safety dt_grow_safety
 * initial_dt dtmax dtmin tmax hydro_interp_order) and what the problem hooks set
 * (init_grid: startx, dx; init_problem: gam/Kpoly, bc[], rho_floor/e_floor;
 * prob_bounds).  The geometry tables that the reference builds in init_geometry()
 * (geometry.c:4-63) are rebuilt from these fields by the library, bit-identically.
 */
typedef struct mdg_problem_desc {
  int ndim;                 /* 1, 2 or 3 */
  int geom;                 /* MDG_CARTESIAN (1-D, 2-D) or MDG_SPHERICAL (1-D; 2-D and 3-D on
                               the dendritic grid, DENDRITIC_GRID=TRUE) */
  int eos;                  /* MDG_GAMMA_LAW or MDG_POLYTROPIC */
  int n1, n2, n3;           /* interior zones; n2 = n3 = 1 in 1-D */
  double startx[3];         /* lower coordinate edge of zone 0 */
  double dx[3];             /* coordinate spacing */
  double gam;               /* adiabatic index */
  double Kpoly;             /* polytropic constant (MDG_POLYTROPIC) */
  int bc_lo[3], bc_hi[3];   /* boundary kind per direction */
  int prob_kind;            /* MDG_PROB_* used by MDG_BC_PROB boundaries */
  double cfl, dt_init_safety, dt_grow_safety, initial_dt, dtmax, dtmin, tmax;
  int hydro_interp_order;   /* 1, 2 (linear) or 3 (parabolic) */
  int enforce_floors;       /* the ENFORCE_FLOORS build switch (fluid.c:43-46): 0 or 1 */
  double rho_floor, e_floor;/* floors set by the problem hook (io.c:5081-5082 defaults -1) */
  double grav[3];           /* fixed contravariant gravitational acceleration g0 (the GRAV=FIXED_GRAV
                               build, gravity.c:38-64; init_rt.c:57-59); all zero: NO_GRAV */
  int rcoord;               /* MDG_RCOORD_* radial map of a spherical grid (the RCOORD build switch) */
  double rtrans;            /* transition radius of the SINH map (rx_info.rtrans; problem hooks
                               set it with rtrans_solve, e.g. problems/init_sedov.c:20) */
  double rfact[3];          /* facta, factb, factc of MDG_RCOORD_SINH_MODIFIED (rx_info; parse_input
                               sets 1e6, 1.5e6, 5e5, io.c:5008-5010) */
  int thcoord;              /* MDG_THCOORD_* theta map of a spherical grid (the THCOORD build switch) */
  double poly_xt, poly_alpha;  /* MDG_THCOORD_POLYTH parameters (thx_info; parse_input sets 1.2, 4) */
  int monopole;             /* 1: self-gravity in the monopole approximation, the
                               GRAV=SPHERICAL_MONOPOLE_GRAV build with GR_MONOPOLE=FALSE
                               (gravity.c:145-425); spherical grids, grav[] all zero */
} mdg_problem_desc;

typedef struct mdg_solver mdg_solver;   /* opaque */

/* Create a solver for nprob problems (all of the same ndim) and allocate their
 * device state.  Replaces the allocation + upload block main.c:129-165.
 * precision: MDG_PREC_FP64 or MDG_PREC_MIXED.  device: CUDA ordinal. */
int mdg_create(const mdg_problem_desc *descs, int nprob, int precision, int device,
               mdg_solver **out);

/* Copy the interior primitive state of problem `prob` to the device, from host memory
 * laid out [zone][5] in the reference's zone order (ZLOOP: i-major, then j), and reset
 * its time to t=0, istep=0 (main.c:172-176, 180-182). */
int mdg_upload_state(mdg_solver *s, int prob, const double *prim);

/* mdg_upload_state / mdg_download_state for every problem at once (one copy and a few
 * launches instead of several per problem): prim holds the problems' states one after
 * the other in problem order, each [zone][5].  The first call allocates a staging buffer
 * of the whole state on the device. */
int mdg_upload_all(mdg_solver *s, const double *prim);
int mdg_download_all(mdg_solver *s, double *prim);

/* No counterpart in the reference (its executable holds one problem in host memory).
 * Advance several solvers from host buffers with their transfers overlapping each other's
 * steps: solver i uploads h_in[i] (every problem's state, as mdg_upload_all), takes nsteps
 * steps (mdg_step) and downloads into h_out[i] (as mdg_download_all), each on its own
 * stream; the uploads are issued in solver order, so solver i's upload runs while earlier
 * solvers step and their downloads run while later ones step.  A caller with one large
 * batch of independent problems splits it into a few solvers to hide the copies.  Host
 * buffers must be page-locked for the copies to overlap.  Returns when every result is in
 * host memory; *elapsed_ms (may be NULL) receives the device time from the start of the
 * first upload to the end of the last download.  All solvers on one device, event timers
 * off. */
int mdg_run_host(mdg_solver *const *solvers, int n, const double *const *h_in, double *const *h_out, int nsteps,
                 float *elapsed_ms);

/* The next time step of every problem as estimate_dt() + main.c:239-251 would produce
 * it; written to dt_out[nprob] (may be NULL).  Idempotent until the next mdg_step. */
int mdg_estimate_dt(mdg_solver *s, double *dt_out);

/* Advance every problem by nsteps passes of the main.c time loop.  Asynchronous with
 * respect to the host (work is queued on the solver's stream): the per-phase launches
 * (replayed from CUDA graphs of mdg_launch_config::steps_per_graph steps), or for small
 * plain-FP64 1-D problems the resident stepper (mdg_launch_config::resident). */
int mdg_step(mdg_solver *s, int nsteps);

/* For a host that runs the main.c time loop itself (its own dump/pdump/tmax clipping of
 * dt, main.c:228-251):
 *   mdg_estimate_dt_raw  what estimate_dt() (step.c:163-203) leaves in the global dt:
 *                        cfl * min(CFL and source limits of the last step or, before the
 *                        first step, of the state; initial_dt at step 0; dtmax), one per
 *                        problem in dt_out[nprob].  Synchronous; changes nothing.
 *   mdg_step_dt          one step() (step.c:28-129) of every problem with the host's
 *                        dt[nprob]; each problem's t advances by dt as main.c's t += dt
 *                        does.  Asynchronous. */
int mdg_estimate_dt_raw(mdg_solver *s, double *dt_out);
int mdg_step_dt(mdg_solver *s, const double *dt);

/* update_cpu() equivalent: copy problem `prob`'s interior primitives ([zone][5]) and,
 * if eos != NULL, its EOS record ([zone][5]: PRESS, CS, TEMP, ENT(=0), GAMMA; the EOS
 * of the most recent stage state, as the reference's sim_eos holds) to host memory. */
int mdg_download_state(mdg_solver *s, int prob, double *prim, double *eos);

/* Time bookkeeping of problem `prob` after all queued work: t, the dt of the last
 * step and the step count. */
int mdg_get_time(mdg_solver *s, int prob, double *t, double *dt_last, int *istep);

/* Checkpoint / resume (the reference's restart_dump_v2 / restart_read_v2, io.c:3237-3583,
 * 4318-4936, whose files are HDF5; these are a flat binary file of the same content for
 * the hydro state: a 48-byte header -- "MDGRST1\0", int32 ndim, n1, n2, n3, istep, 0,
 * int64 zone count, double t -- then the zones' 5 primitives in sim_p's [zone][var]
 * order).  mdg_set_time gives problem `prob` the time record of a run resumed from a
 * restart: Time and Step of the file and, as a new reference process has, no step of its
 * own yet (dtold = 1e100, main.c:194, so the first step's dt is not limited by the
 * growth factor); call it after mdg_upload_state, whose state the first estimate_dt of
 * the resumed run uses (step.c:171-174).  mdg_restart_read checks that the file belongs
 * to the problem's grid (MDG_ERR_INVALID otherwise) and does both. */
int mdg_set_time(mdg_solver *s, int prob, double t, int istep);
int mdg_restart_write(mdg_solver *s, int prob, const char *path);
int mdg_restart_read(mdg_solver *s, int prob, const char *path);

/* The CUDA stream all work of this solver is queued on (a cudaStream_t). */
int mdg_get_stream(mdg_solver *s, void **stream);

/* Wait for all queued work; returns the first asynchronous error, if any. */
int mdg_synchronize(mdg_solver *s);

/* Free the solver and its device memory. */
int mdg_destroy(mdg_solver *s);

/* Static description of a status code, and the message of the last failure in this
 * thread (a CUDA error string or the validation that failed). */
const char *mdg_error_string(int code);
const char *mdg_last_error_message(void);

/* Per-kernel timers, the counterpart of the reference's TIMER_START/TIMER_STOP
 * instrumentation (decs.h:717-746, timer.c) and its timing.csv (io.c:51-108).  With
 * timing enabled every queued launch is bracketed by CUDA events and each mdg_step
 * waits for its step to finish; ms[k] and calls[k] accumulate per timer k: */
#define MDG_TIMER_DT        0   /* estimate_dt + main.c dt rules */
#define MDG_TIMER_STAGE0    1   /* first RK stage (fused sweep) */
#define MDG_TIMER_STAGE1    2   /* second RK stage (fused sweep) */
#define MDG_TIMER_FINISH    3   /* t += dt bookkeeping */
#define MDG_NTIMERS         4
int mdg_set_timing(mdg_solver *s, int enable);
int mdg_get_timers(mdg_solver *s, double *ms, long long *calls);
/* Append the timers to the CSV file `path` in the columns of the reference's timing.csv
 * (output_timers, io.c:51-108: timer, time, step, ncycle, max, min, avg; seconds; the
 * header row when the file is new), with t and the step count of problem `prob`.  Timer
 * names: estimate_dt, stage0, stage1, finish (as Solver.timers).  (The reference's
 * single-process path writes the first timer's total in every row; here each row has its
 * own timer's.) */
int mdg_write_timers(mdg_solver *s, int prob, const char *path);

/*
 * No counterpart in the reference (its launch shapes are compile-time constants).
 * Launch shape of a solver's step sequence:
 *   threads          mixed 1-D sweep: threads per CTA, 64, 128 or 256; a tile holds
 *                    threads-2 zones (the FP64 sweeps ignore it: 128);
 *   ctas_per_sm      mixed 1-D sweep: 0 = one CTA per tile; k > 0 = k persistent CTAs
 *                    per SM that pull (problem, tile) items from a device work queue;
 *   steps_per_graph  steps captured in one CUDA graph and replayed by mdg_step
 *                    (0 = direct launches; timing enabled always launches directly);
 *   run_length       dendritic (3-D and 2-D spherical) sweeps: radial and theta faces
 *                    one thread walks per work item, 1..64 (default 16); the results do
 *                    not depend on it;
 *   lanes            mixed 1-D sweep: the problems split into 1..4 groups of about equal
 *                    zone count, each group's steps queued on a stream of its own, so that
 *                    one group's short kernels and kernel tails overlap another's stage
 *                    kernels (default 1); the results do not depend on it;
 *   resident         plain FP64 1-D solvers without monopole gravity whose problems have at
 *                    most 16 tiles (2016 zones): 1 (default) = mdg_step runs the whole
 *                    step sequence -- dt rules, both RK stages, time update -- in one launch
 *                    per 256 steps, one thread-block cluster of CTAs per problem (the
 *                    per-phase path launches four dependent kernels per step); 0 = the
 *                    per-phase launches.  Other solvers ignore it; the results do not
 *                    depend on it.  mdg_resident_cluster reports whether it applies.
 */
#define MDG_MAX_LANES 4
typedef struct mdg_launch_config {
  int threads;
  int ctas_per_sm;
  int steps_per_graph;
  int run_length;
  int lanes;
  int resident;
} mdg_launch_config;
int mdg_get_launch_config(mdg_solver *s, mdg_launch_config *cfg);
int mdg_set_launch_config(mdg_solver *s, const mdg_launch_config *cfg);
/* CTAs per problem of the resident stepper (mdg_launch_config::resident) for this solver,
 * 0 when mdg_step cannot use it (other solvers, a problem of more than 16 tiles, or such
 * a cluster does not fit the device).  With resident = 1 and *ctas > 0, mdg_step(s, n)
 * queues ceil(n / 256) kernel launches. */
int mdg_resident_cluster(mdg_solver *s, int *ctas);

/* Time every admissible launch shape over trial_steps steps of the solver's own
 * problems, keep the fastest and restore the state, times and error flag as they were:
 * (threads, ctas_per_sm) of the batched 1-D mixed sweep and then its lanes (1, 2, 4) with
 * the best of those, run_length (4, 8, 16, 32) of a dendritic-grid solver of either
 * precision.  best/ms_per_step may be NULL.
 * MDG_ERR_NOTIMPL for the FP64 1-D and 2-D Cartesian solvers, whose shapes are fixed. */
int mdg_autotune(mdg_solver *s, int trial_steps, mdg_launch_config *best, double *ms_per_step);

/* Conserved totals of every problem after all queued work: mass[m] = sum rho dV and
 * energy[m] = sum (rho v.v/2 + u) dV over the interior zones, each summed in FP64 with
 * compensated (Neumaier) summation.  The integrands of calculate_total_mass and
 * calculate_total_energy (utils.c:2337-2361, 2581-2612; without the gravitational
 * term), which the reference sums in plain serial order. */
int mdg_conserved_totals(mdg_solver *s, double *mass, double *energy);

/*
 * No counterpart in the reference.  A 1-D advance that allocates nothing, for callers
 * that cannot call cudaMalloc: hosts whose device memory is owned by their own pool
 * allocator, real-time loops that cannot afford cudaMalloc's implicit synchronisation,
 * embeddings that must not grow their device footprint after start-up.
 *
 * Advances one 1-D problem (desc->ndim == 1, desc->n1 <= MDG_NOALLOC_MAX_ZONES) by
 * nsteps passes of the reference time loop, exactly as mdg_create + mdg_upload_state +
 * mdg_step would, starting from t = 0.  prim_in and prim_out are DEVICE pointers owned
 * by the caller, laid out [var][zone] (5 x n1 doubles; they may be the same buffer);
 * work is queued on `stream` (a cudaStream_t, 0 for the legacy default stream).  The
 * call waits for that work to finish before it returns; it then stores the final time
 * and the last dt in t_out/dt_out (when non-NULL) and returns MDG_ERR_NONFINITE, as
 * mdg_synchronize does, when the state became non-finite or a dt estimate dropped below
 * desc->dtmin.
 *
 * Everything else the sweep needs lives in one file-scope device array of fixed size
 * (about 4.4 MB, held by every GPU that loads this library until exit).  Rules:
 *   - n1 > MDG_NOALLOC_MAX_ZONES is rejected with MDG_ERR_OUTOFMEM (does not fit);
 *   - the first call on a device performs the device set-up (it looks up the array's
 *     device address);
 *   - no call can be captured into a CUDA graph: each waits on its stream before it
 *     returns (the host tables must outlive their copies);
 *   - all calls share the array: calls whose work overlaps on the GPU race;
 *   - the array keeps the last call's contents; each call re-initialises what it uses;
 *   - the tables are built in one process-wide host buffer under a lock, so calls from
 *     several host threads wait for each other while their tables are copied.
 * Calls no cudaMalloc, cudaFree or other allocating routine.
 */
#define MDG_NOALLOC_MAX_ZONES 8192
int mdg_advance_1d_noalloc(const mdg_problem_desc *desc, const double *prim_in, double *prim_out,
                           int nsteps, void *stream, double *t_out, double *dt_out);

/*
 * Solve server.  No counterpart in the reference, whose executable advances one problem
 * per process.  A server keeps 1-D and 2-D problems resident on one GPU and advances
 * every admitted problem together, batching their uneven grids into the same stage
 * launches (1-D, for MDG_PREC_MIXED: persistent CTAs fed from a device work queue, each
 * round of steps_per_round steps replayed from one CUDA graph; 2-D: the split sweep in
 * the server's precision, on a second stream that runs beside the 1-D launches; 3-D
 * dendritic spherical problems on that stream too, each with its own grid, in the
 * server's precision).  A
 * request is a problem description, its initial state ([zone][5], as mdg_upload_state)
 * and its end time desc->tmax; it runs the main.c time loop until t >= tmax and is then
 * retired.
 *
 * Admission is by device-memory footprint: the arenas are sized once from hbm_bytes
 * (1-D states and every request's tables) and hbm_bytes_2d (2-D states), a 3-D request
 * holds its own grid and state counted against hbm_bytes_3d, and a queued
 * request is admitted between rounds when a slot and contiguous ranges of n1 + 4 zone
 * units (2-D: n1 + n2 + 8 table units and (n1 + 3) x n2 cells) are free (requests that do
 * not fit yet wait; smaller ones behind them may go first).  A finished problem's state
 * is left unchanged by later rounds, so every result is the same whatever else shares
 * the GPU and whenever it is collected.
 *
 * The request loop runs either on a thread of the server (mdg_server_start/stop), while
 * other threads submit, poll and collect, or in the caller's thread (mdg_server_run).
 */
typedef struct mdg_server mdg_server;   /* opaque */
typedef struct mdg_server_config {
  int device;               /* CUDA ordinal */
  int precision;            /* MDG_PREC_MIXED or MDG_PREC_FP64 */
  long long hbm_bytes;      /* device memory for resident problems: the admission budget */
  int max_problems;         /* resident problems at most */
  int max_zones;            /* largest n1 a request may have */
  int steps_per_round;      /* steps between two scheduling points */
  int threads;              /* mixed sweep: threads per CTA, 64, 128 or 256 */
  int ctas_per_sm;          /* mixed sweep: persistent CTAs per SM (0: as many as fit) */
  long long hbm_bytes_2d;   /* device memory for resident 2-D states (0: 2-D requests refused) */
  int max_cells_2d;         /* largest n1 x n2 a 2-D request may have */
  long long hbm_bytes_3d;   /* device memory for resident 3-D problems, state and grid
                               (0: 3-D requests refused) */
} mdg_server_config;

#define MDG_REQ_QUEUED  0
#define MDG_REQ_RUNNING 1
#define MDG_REQ_DONE    2
#define MDG_REQ_FAILED  3   /* its time step dropped below dtmin (main.c:229-238) */

typedef struct mdg_server_stats {
  long long submitted, completed, failed, queued, running, rounds;
  double zone_updates;      /* sum over finished requests of zones (n1 or n1 x n2) x steps */
  double device_seconds;    /* device time of the step rounds */
  double latency_p50, latency_p99;   /* seconds from submission to completion */
  double wait_p50, wait_p99;         /* seconds from submission to admission */
  double hbm_capacity, hbm_in_use;   /* bytes of the arenas, bytes held by resident problems */
  long long kernel_launches;         /* this library's kernels launched (graph replays included) */
} mdg_server_stats;

int mdg_server_create(const mdg_server_config *cfg, mdg_server **out);
/* Queue a 1-D, 2-D Cartesian or dendritic (3-D, 2-D spherical) request (thread-safe);
 * *id identifies it in the calls below. */
int mdg_server_submit(mdg_server *s, const mdg_problem_desc *desc, const double *prim, long long *id);
/* Run `rounds` scheduling rounds in the calling thread (rounds <= 0: until nothing is
 * queued or running); *active = problems resident after the last round. */
int mdg_server_run(mdg_server *s, int rounds, int *active);
/* Run the request loop on a thread of the server / stop it (returns the loop's error). */
int mdg_server_start(mdg_server *s);
int mdg_server_stop(mdg_server *s);
int mdg_server_poll(mdg_server *s, long long id, int *status);
/* Wait up to timeout_s seconds for a request to finish (its status in *status). */
int mdg_server_wait(mdg_server *s, long long id, double timeout_s, int *status);
/* Copy a finished request's final state ([zone][5]), time, step count and seconds from
 * submission to completion, and forget the request. */
int mdg_server_result(mdg_server *s, long long id, double *prim, double *t, int *istep, double *latency_s);
int mdg_server_get_stats(mdg_server *s, mdg_server_stats *st);
int mdg_server_destroy(mdg_server *s);

/*
 * Output path (the reference's update_cpu() + dump, main.c:289-291; its ASCII dump
 * dump_ascii1, io.c:111-220, written for restarts at main.c:271).
 *   mdg_snapshot           queues, on the solver's stream, a copy of problem `prob`'s
 *                          state and EOS records ([zone][5] each, as mdg_download_state)
 *                          and its time, then a copy to pinned host memory on a second
 *                          stream; returns at once, and later mdg_step calls overlap the
 *                          host copy (one snapshot in flight: a new one waits for the last);
 *   mdg_snapshot_read      waits for the snapshot and copies it out (any pointer may be NULL);
 *   mdg_snapshot_write_ascii1  waits and writes it as dump_ascii1 does (1-D problems):
 *                          "# t", then per zone x (r on spherical grids), rho, u,
 *                          scale[0][0] v^1, v^2, v^3, the EOS record, the enclosed mass at
 *                          the zone centre and the two lapse columns, in its printf formats;
 *   mdg_dump_ascii1        snapshot + write.
 */
int mdg_snapshot(mdg_solver *s, int prob);
int mdg_snapshot_read(mdg_solver *s, double *prim, double *eos, double *t);
int mdg_snapshot_write_ascii1(mdg_solver *s, const char *path);
int mdg_dump_ascii1(mdg_solver *s, int prob, const char *path);

/*
 * 3-D dendritic spherical grids (ndim = 3; the grid of DENDRITIC_GRID=TRUE builds,
 * utils.c:181-525).  Radial row i has nj[i] theta zones and row (i, j) nk phi zones; the
 * state of a 3-D problem is passed in the reference's zone order (ZLOOP: i, then j, then
 * k).  Host-only calls (no device work):
 *   mdg_grid3d_counts   nj[i] for i in [0, n1) (nj may be NULL), nk of every interior
 *                       row in zone order (nk may be NULL; sum(nj) entries), *ncell the
 *                       interior zone count;
 *   mdg_grid3d_geometry the per-row zone geometry for every row i in [-2, n1+2),
 *                       j in [-2, nj[i]+2) (ghost rows included), MDG_GEO3_FIELDS doubles
 *                       each: volume, area[3], gcov[4][3], gcon[3], scale[4][3], then
 *                       conn[l][m][n] for (lmn) = 000 011 022 101 110 111 122 202 220 212
 *                       221 (the coefficients the spherical metric sets, init_conn);
 *                       rows may be NULL, *nrows the row count.
 * A 3-D solver advances one problem, plain FP64 (MDG_PREC_FP64).
 */
#define MDG_GEO3_FIELDS 42
int mdg_grid3d_counts(const mdg_problem_desc *desc, int *nj, int *nk, long long *ncell);
int mdg_grid3d_geometry(const mdg_problem_desc *desc, double *rows, long long *nrows);

/*
 * Tabulated (nuclear) EOS: the zone update of the reference's production EOS,
 * eos_given_rex_per_zone (eos/burrows/eos_stuff.c:768-902, called per zone by
 * eos_given_rex_tianshu, :507-640): from density, internal energy density, Ye and a
 * temperature guess to temperature, pressure, sound speed, entropy and Gamma_1.
 *
 * mdg_eos_grid holds what the reference fixes in DEFINE_EOSCONST_1 (eos_stuff.c:8-21:
 * nrec = 16 records of ny = 50 x nr = 300 x nt = 300, log10 rho in [1, 15.5], log10 T
 * (MeV) in [-2, 2], Ye in [0.035, 0.56]) and const_hack (0 there).  mdg_eos_table_create
 * copies a table in the reference's layout (TAB_ELEM, eos_stuff.c:7: [nrec][ny][nr][nt],
 * jt fastest; records 1, 2, 3 and 12 -- energy, log pressure, entropy, Gamma_1 -- are
 * used, so nrec >= 12) to the device, rearranged for the gathers (the four records
 * interleaved per grid point, 32 B: 144 MB at the reference's sizes).  Results agree with the reference's to a few
 * ulps (CUDA's log10, exp and pow; everything else in the reference's operation order).
 * Indices the reference would take outside the table (inputs outside its range) are
 * clamped to it.
 */
typedef struct mdg_eos_grid {
  int nrec, ny, nr, nt;
  double r1, r2;            /* log10 rho range */
  double t1, t2;            /* log10 T (MeV) range */
  double y1, y2;            /* Ye range */
  double const_hack;        /* subtracted from the specific energy (eos_stuff.c:784) */
} mdg_eos_grid;
typedef struct mdg_eos_table mdg_eos_table;   /* opaque */
int mdg_eos_table_create(const mdg_eos_grid *grid, const double *table, int device, mdg_eos_table **out);
int mdg_eos_table_destroy(mdg_eos_table *t);
/* n zones, DEVICE pointers: rho, u (internal energy density), ye in; temp in (the guess,
 * eos[TEMP] before the call) and out; press, cs, ent, gam1 out.  Queued on `stream` (a
 * cudaStream_t, 0 for the legacy default stream). */
int mdg_eos_given_rex(mdg_eos_table *t, long long n, const double *rho, const double *u, const double *ye,
                      double *temp, double *press, double *cs, double *ent, double *gam1, void *stream);
/* The same from HOST buffers: copies in, the update, copies out; returns when done. */
int mdg_eos_given_rex_host(mdg_eos_table *t, long long n, const double *rho, const double *u, const double *ye,
                           double *temp, double *press, double *cs, double *ent, double *gam1);

/* Library version as major*10000 + minor*100 + patch. */
int mdg_version(void);

#ifdef __cplusplus
}
#endif
#endif /* MEDUSA_B200_H_ */
