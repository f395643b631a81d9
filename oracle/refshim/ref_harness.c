/*
 * TEST INFRASTRUCTURE ONLY -- never linked into, called by, or shipped with the
 * medusa_b200 product path.
 *
 * Drives the UNMODIFIED reference hydro sweep (step.c, reconstruct.c, riemann.c,
 * fluid.c, rad_fluid.c, bc.c, eos.c, utils.c, geometry.c, mpi.c and the metric
 * compiled from the reference tree by oracle/build_ref.py) and exposes a small C API
 * that Python loads with ctypes.  Everything here is glue that the reference leaves
 * to files this build cannot compile (io.c needs HDF5; the tabulated EOS needs table
 * files; the gamma-law/polytrope EOS and the problem files use a removed API):
 *
 *   - the init sequence restates main.c:56-192 (minus dumps, tracers, MPI types);
 *   - the time-step control restates main.c:226-264;
 *   - eos_fill_tianshu / eos_fill_ghost_tianshu loop like
 *     eos/burrows/eos_stuff.c:521-532,668-683 with the gamma-law arithmetic of
 *     eos/gamma/eos_gamma.c:5-12,45-58 or the polytrope of eos/polytropic/eos_poly.c:5-11,56-69;
 *   - init_grid / init_problem take the grid and the initial primitive state from the
 *     caller (the problem files problems/init_sod.c, init_kh.c, init_sedov.c and
 *     init_spherical_noh.c are restated on the Python side), prob_bounds restates
 *     problems/init_spherical_noh.c:63-79;
 *   - output_timers restates io.c:51-108 (timing.csv) for builds with DO_TIMING=TRUE;
 *     the other io.c entry points that the hot path references are no-ops.
 */
#include "decs.h"
#include "defs.h"
#include "constants.h"

#define REF_API __attribute__((visibility("default")))

/* ---- parameters handed in by the caller ---- */
typedef struct {
  int n1, n2, n3;
  double startx[3];
  double dx[3];
  double gam;
  double Kpoly;
  int eos_kind;        /* 0 gamma law, 1 polytrope */
  int bc_lo[3], bc_hi[3];
  int prob_kind;       /* 0 none, 1 spherical Noh inflow */
  double cfl;
  double dt_init_safety, dt_grow_safety;
  double initial_dt, dtmax, dtmin;
  double tmax;
  double rtrans;
  int hydro_interp_order;
  int enforce_floors;  /* must match the ENFORCE_FLOORS of the build */
  double rho_floor, e_floor;
  double grav[3];     /* fixed gravitational acceleration g0 (GRAV=FIXED_GRAV builds) */
  int rcoord;         /* radial map; must match the RCOORD of the build (rtrans above) */
  double rfact[3];    /* rx_info.facta/b/c (SINH_MODIFIED) */
  int thcoord;        /* theta map; must match the THCOORD of the build */
  double poly_xt, poly_alpha;   /* thx_info (POLYTH) */
} ref_params;

static ref_params g_prm;
static const double *g_ic = NULL;   /* interior primitives, [cell][NPRIM], i-major */
static double g_dtold = 1.0e100;

/* ---------------- io.c entry points referenced by the hot path ---------------- */
void parse_input(char *name) { (void)name; }
void run_log() {}
/* io.c:51-108: append the reference's timers (TIMER_START/TIMER_STOP, decs.h:717-746)
 * to timing.csv in the working directory, with the header row when the file is new.
 * One process: max, min and avg are the timer's own total (the reference's serial path
 * writes the first timer's total in every row). */
void output_timers()
{
#if DO_TIMING==TRUE
  const char *fname = "timing.csv";
  FILE *probe = fopen(fname, "r");
  const int fresh = probe == NULL;
  if (probe) fclose(probe);
  FILE *fp = fopen(fname, "a");
  if (!fp) return;
  if (fresh) fprintf(fp, "timer,time,step,ncycle,max,min,avg\n");
  for (int k = 0; k < ntimers; ++k) {
    Timer *timer = get_timer(k);
    double total = 0.0;
    timer_get_total(timer, &total);
    fprintf(fp, "%s,%f,%d,%lu,%f,%f,%f\n", timer->name, t, istep, timer->ncycles, total, total, total);
  }
  fclose(fp);
#endif
}
void dump1() {}
void dump2() {}
void dump3() {}
void dump_ascii1(int is_restart) { (void)is_restart; }
void dump_tracers() {}
void restart_dump() {}
void restart_read() {}

/* ---------------- EOS (gamma law / polytrope) ---------------- */
static void fill_one(const double *p, double *eos)
{
  double press, cs, tp;
  if (g_prm.eos_kind == 0) {
    /* eos/gamma/eos_gamma.c:5-12 and :45-58 */
    press = (gam-1.0)*p[UU];
    cs = sqrt(gam*press/p[RHO]);
    tp = press/(2.0*p[RHO]*KBOLTZ)*(MP+ME);
  } else {
    /* eos/polytropic/eos_poly.c:5-11 and :56-69 */
    press = Kpoly*pow(p[RHO],gam);
    cs = sqrt(gam*press/p[RHO]);
    tp = press/(p[RHO]*KBOLTZ)*MP;
  }
  eos[PRESS] = press;
  eos[CS   ] = cs;
  eos[TEMP ] = tp;
  eos[GAMMA] = gam;
}

int eos_fill_tianshu(const double *table, double **p, double **eos)
{
  (void)table;
  for (int II=0; II<cell_count; II++) fill_one(p[II], eos[II]);
  return 1;
}

int eos_fill_ghost_tianshu(const double *table, double **p, double **eos)
{
  (void)table;
  for (int II=cell_count; II<cell_count_all; II++) fill_one(p[II], eos[II]);
  return 1;
}

/* ---------------- problem hooks ---------------- */
void init_grid()
{
  for (int d=0; d<3; d++) {
    startx[d] = g_prm.startx[d];
    dx[d] = g_prm.dx[d];
    periodic[d] = (g_prm.bc_lo[d] == PERIODIC);
  }
  rx_info.rtrans = g_prm.rtrans;
}

void init_problem()
{
  int ii=0, jj=0, kk=0, vv, dd, c=0;
  gam = g_prm.gam;
  Kpoly = g_prm.Kpoly;
  VLOOP {
    DLOOP {
      bc[vv].lo[dd] = g_prm.bc_lo[dd];
      bc[vv].hi[dd] = g_prm.bc_hi[dd];
    }
  }
  if (g_prm.prob_kind == 2) {
    /* problems/init_dustcollapse.c:77-86: outflow, with the PROB hook on v^r only */
    VLOOP bc[vv].hi[0] = OUTFLOW;
    bc[U1].hi[0] = PROB;
  }
  ZLOOP {
    for (vv=0; vv<NPRIM; vv++) NDP_ELEM_LINEAR(sim_p,ii,jj,kk,vv) = g_ic[NPRIM*c+vv];
    c++;
  }
}

void prob_bounds(int i, int j, int k, double *p)
{
  if (g_prm.prob_kind == 1) {
    /* problems/init_spherical_noh.c:63-79 */
    double r, rhat[SPACEDIM];
    p[RHO] = 1.;
    p[UU] = 1.e-6/(gam-1.);
    r = ijk_to_r(i,j,k,rhat);
    p[U1] = -1./rhat[0];
    p[U2] = 0.;
    p[U3] = 0.;
    p[RHO] += t/r;
    p[RHO] *= p[RHO];
  } else if (g_prm.prob_kind == 2) {
    /* problems/init_dustcollapse.c:104-113 */
    double r = r_of_x(rx_info, beta0[i]/Gamma0[i]);
    double vr = -1.0/sqrt(r);
    p[U1] = vr/ND_ELEM_LINEAR(geom,i,j,k).scale[0][0];
  }
}

void analysis_preloop() {}
void analysis_inloop() {}
void analysis_postloop() {}

/* ---------------- API ---------------- */

/* Restates the init sequence of main.c:56-192 (no dumps / tracers / MPI types).
 * ic: interior primitives [cell][NPRIM] in the reference's ZLOOP order. */
REF_API int ref_init(const ref_params *prm, const double *ic)
{
  g_prm = *prm;
  g_ic = ic;
#if (RCOORD == SINH)
  if (prm->rcoord != 1) { fprintf(stderr, "ref_init: this build has the SINH radial map\n"); return -1; }
#elif (RCOORD == SINH_MODIFIED)
  if (prm->rcoord != 2) { fprintf(stderr, "ref_init: this build has the SINH_MODIFIED radial map\n"); return -1; }
#elif (defined(LOG) && RCOORD == LOG)
  if (prm->rcoord != 3) { fprintf(stderr, "ref_init: this build has the LOG radial map\n"); return -1; }
#else
  if (prm->rcoord != 0) { fprintf(stderr, "ref_init: this build has the uniform radial map\n"); return -1; }
#endif
#if (THCOORD == POLYTH)
  if (prm->thcoord != 1) { fprintf(stderr, "ref_init: this build has the POLYTH theta map\n"); return -1; }
#else
  if (prm->thcoord != 0) { fprintf(stderr, "ref_init: this build has the uniform theta map\n"); return -1; }
#endif

  /* parse_input defaults, io.c:5000-5117, then the keys this build sets */
  rx_info.facta = prm->rfact[0];       /* io.c:5008-5010 defaults 1e6, 1.5e6, 5e5 */
  rx_info.factb = prm->rfact[1];
  rx_info.factc = prm->rfact[2];
  thx_info.nice_alpha = 1.01;
  thx_info.poly_xt = prm->poly_xt;      /* io.c:5014-5015 defaults 1.2, 4 */
  thx_info.poly_alpha = prm->poly_alpha;
  Nskip = 1;
  n1 = prm->n1; n2 = prm->n2; n3 = prm->n3;
  cfl = prm->cfl;
  dt_grow_safety = prm->dt_grow_safety;
  dt_init_safety = prm->dt_init_safety;
  dtmax = prm->dtmax;
  dtmin = prm->dtmin;
  initial_dt = prm->initial_dt;
  tmax = prm->tmax;
  ncomp = 0;
  hydro_interp_order = prm->hydro_interp_order;
#if (GRAV == FIXED_GRAV)
  g0[0] = prm->grav[0]; g0[1] = prm->grav[1]; g0[2] = prm->grav[2];   /* init_rt.c:57-59 */
#endif
  if (prm->enforce_floors != (ENFORCE_FLOORS == TRUE)) {
    fprintf(stderr, "ref_harness: enforce_floors=%d but this build has ENFORCE_FLOORS=%d\n",
            prm->enforce_floors, (int)(ENFORCE_FLOORS == TRUE));
    exit(3);
  }
  rad_interp_order = 2;
  dt_dump = 1.0e100;
  dt_pdump = dt_dump;
  dt_restart = 1.0e100;
  di_restart = INT_MAX/2;
  nstep_log = 100;
  nstep_analysis = 100;
  nstep_timing = INT_MAX;
  max_steps = 2147483647;
  e_floor = prm->e_floor;       /* io.c:5081-5082 defaults are -1; problem hooks set their own */
  rho_floor = prm->rho_floor;
  detect_tbounce = 0;
  dump_hdf = 0;
#if (NDIM==1)
  n2 = n3 = 1;
#elif (NDIM==2)
  n3 = 1;
#endif
  nhydro = NPRIM + ncomp;
  nvars = nhydro;
  ninterp = nvars + 2;

  init_fornax_rand();
  init_grid();
  init_coords();
  init_dendritic();
  init_mpi_setup();
  allocate_memory();
  init_geometry();

  t = 0.0;
  istep = 0;
  t_next_dump = dt_dump;
  t_next_pdump = dt_pdump;
  t_next_restart = dt_restart;
  i_next_restart = di_restart;

  init_problem();
  init_interp_order();

  update_eos(eostable, sim_p, sim_eos);
  g_dtold = 1.0e100;
  return cell_count_all;
}

/* One pass of the time loop of main.c:226-264 (dump clipping omitted: dt_dump is
 * infinite here).  Returns the dt that was used. */
REF_API double ref_advance_one(void)
{
  estimate_dt();
  if (istep==0) dt *= dt_init_safety;
  else dt = MIN(g_dtold*dt_grow_safety, dt);
  g_dtold = dt;
  if (t+Nskip*dt > tmax) {
    dt = 1.000000001*(tmax - t)/Nskip;
  }
  if (dt < dtmin) dt = dtmin;
  step();
  t += dt;
  istep++;
  return dt;
}

/* Lower-level hooks: estimate_dt() alone, step() alone with the caller's dt. */
REF_API double ref_estimate_dt(void) { estimate_dt(); return dt; }
REF_API void ref_step_with_dt(double dtin)
{
  dt = dtin;
  step();
  t += dt;
  istep++;
}

/* the timers of a DO_TIMING=TRUE build: zeroed (after warm-up steps) and written */
REF_API void ref_timers_reset(void)
{
#if DO_TIMING==TRUE
  for (int k = 0; k < ntimers; ++k) timer_reset(get_timer(k));
#endif
}
REF_API void ref_timers_write(void) { output_timers(); }
REF_API double ref_get_t(void) { return t; }
REF_API double ref_get_min_dt(void) { return min_dt; }
REF_API int ref_get_istep(void) { return istep; }
REF_API int ref_cell_count(void) { return cell_count; }
REF_API int ref_cell_count_all(void) { return cell_count_all; }

/* Interior state (ZLOOP order) of sim_p [cell][NPRIM] and sim_eos [cell][NEOS]. */
REF_API void ref_get_interior(double *prim, double *eos)
{
  int ii=0, jj=0, kk=0, vv, c=0;
  ZLOOP {
    for (vv=0; vv<NPRIM; vv++) prim[NPRIM*c+vv] = NDP_ELEM_LINEAR(sim_p,ii,jj,kk,vv);
    for (vv=0; vv<NEOS; vv++) eos[NEOS*c+vv] = NDP_ELEM_LINEAR(sim_eos,ii,jj,kk,vv);
    c++;
  }
}

/* Overwrite the interior primitive state (ZLOOP order). */
REF_API void ref_set_interior(const double *prim)
{
  int ii=0, jj=0, kk=0, vv, c=0;
  ZLOOP {
    for (vv=0; vv<NPRIM; vv++) NDP_ELEM_LINEAR(sim_p,ii,jj,kk,vv) = prim[NPRIM*c+vv];
    c++;
  }
}

/* 1-D volume moments alpha0/beta0/Gamma0 over i in [-NG, n1+NG). */
REF_API void ref_get_moments0(double *a, double *b, double *g)
{
  for (int i=-NG; i<n1+NG; i++) {
    a[i+NG] = alpha0[i];
    b[i+NG] = beta0[i];
    g[i+NG] = Gamma0[i];
  }
}

/* Per-zone geometry record of cell (i,j,k): volume, area[NDIM], gcov[0..NDIM][3],
 * gcon[3], scale[0..NDIM][3], conn[3][3][3], written in that order. */
REF_API int ref_get_geom(int i, int j, int k, double *out)
{
  zone_geom *g = &ND_ELEM_LINEAR(geom,i,j,k);
  int c = 0, d, l, m, n;
  (void)j; (void)k;
  out[c++] = g->volume;
  for (d=0; d<NDIM; d++) out[c++] = g->area[d];
  for (l=0; l<=NDIM; l++) for (m=0; m<SPACEDIM; m++) out[c++] = g->gcov[l][m];
  for (m=0; m<SPACEDIM; m++) out[c++] = g->gcon[m];
  for (l=0; l<=NDIM; l++) for (m=0; m<SPACEDIM; m++) out[c++] = g->scale[l][m];
  for (l=0; l<SPACEDIM; l++) for (m=0; m<SPACEDIM; m++) for (n=0; n<SPACEDIM; n++) out[c++] = g->conn[l][m][n];
  return c;
}

REF_API int ref_ndim(void) { return NDIM; }

/* Dendritic zone counts (utils.c:181-354): nj[i] for i in [-NG, n1+NG), then nk[i][j]
 * for each of those rows and j in [-NG, nj[i]+NG), row after row.  Returns the number
 * of nk entries written (call with nk == NULL to size the buffer). */
REF_API int ref_get_grid(int *njo, int *nko)
{
  int c = 0;
  for (int i=-NG; i<n1+NG; i++) {
#if (NDIM>1)
    int nji = n2/DJS(i);
#else
    int nji = 1;
#endif
    if (njo) njo[i+NG] = nji;
    for (int j=-NG; j<nji+NG; j++) {
#if (NDIM==3)
      if (nko) nko[c] = n3/DKS(i,j);
#else
      if (nko) nko[c] = 1;
#endif
      c++;
    }
  }
  return c;
}
