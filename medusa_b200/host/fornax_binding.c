/*
 * Drop-in binding of the reference's host code to libmedusa_b200.
 *
 * Compiled into the reference's own build in place of step.c: it defines the entry
 * points main.c calls from there -- estimate_dt(), step(), update_cpu() (step.c:16-203;
 * declared in decs.h:754-757) and set_tbounce() (step.c:133-155) -- on top of the C ABI of
 * include/medusa_b200.h.  Everything else stays the reference's: main.c's time loop
 * (main.c:206-320, with its own dt safety, growth and dump/tmax clipping of the global
 * dt), parse_input, the problem hooks, init_geometry, the dumps.  It reads the
 * reference's globals (decs.h / defs.h) and its build switches (build.h), so it is built
 * with the reference's include path:
 *
 *   gcc -std=gnu99 -I<build.h dir> -I<reference> -I<this repository>/include -c fornax_binding.c
 *
 * and linked with -lmedusa_b200.  Optional defines:
 *   MDG_BINDING_PROB_KIND   MDG_PROB_* of the problem's prob_bounds hook (default
 *                           MDG_PROB_NONE; MDG_PROB_NOH for problems/init_spherical_noh.c,
 *                           MDG_PROB_DUST for problems/init_dustcollapse.c)
 *   MDG_BINDING_PRECISION   MDG_PREC_FP64 (default) or MDG_PREC_MIXED
 *   MDG_BINDING_DEVICE      CUDA device ordinal (default 0)
 *
 * The state is handed over in the reference's collapsed layout: with one rank (no MPI
 * send cells) the interior cells lead sim_p/sim_eos, [cell][nvars] / [cell][NEOS] in
 * ZLOOP order (utils.c:1367-1375), nvars = 5 (ncomp = 0).  A failing call prints the
 * library's message and exits with status 1, as the reference does on its own errors.
 */
#include "decs.h"
#include "medusa_b200.h"

#ifndef MDG_BINDING_PROB_KIND
#define MDG_BINDING_PROB_KIND MDG_PROB_NONE
#endif
#ifndef MDG_BINDING_PRECISION
#define MDG_BINDING_PRECISION MDG_PREC_FP64
#endif
#ifndef MDG_BINDING_DEVICE
#define MDG_BINDING_DEVICE 0
#endif

static mdg_solver *g_mdg = NULL;

static void mdg_or_die(int rc, const char *where)
{
  if (rc != MDG_OK) {
    fprintf(stderr, "[%s] %s: %s\n", where, mdg_error_string(rc), mdg_last_error_message());
    exit(1);
  }
}

/* mdg_problem_desc from the reference's build switches and globals (after init_grid,
 * init_problem and init_interp_order, i.e. at the first estimate_dt of main.c:228) */
static void describe(mdg_problem_desc *d)
{
  int k;
  memset(d, 0, sizeof *d);
  d->ndim = NDIM;
  d->geom = (GEOM == SPHERICAL) ? MDG_SPHERICAL : MDG_CARTESIAN;
  d->eos = (EOS == POLYTROPIC) ? MDG_POLYTROPIC : MDG_GAMMA_LAW;
  d->n1 = n1;
  d->n2 = (NDIM > 1) ? n2 : 1;
  d->n3 = (NDIM > 2) ? n3 : 1;
  for (k = 0; k < 3; k++) {
    d->startx[k] = startx[k];
    d->dx[k] = dx[k];
  }
  d->gam = gam;
  d->Kpoly = Kpoly;
  /* one boundary kind per face: the density's (a PROB hook on single variables is
     described by the prob kind, e.g. the dust collapse's outer v^r) */
  for (k = 0; k < NDIM; k++) {
    d->bc_lo[k] = bc[RHO].lo[k];
    d->bc_hi[k] = bc[RHO].hi[k];
    if (bc[U1].hi[k] == PROB) d->bc_hi[k] = MDG_BC_PROB;
    if (bc[U1].lo[k] == PROB) d->bc_lo[k] = MDG_BC_PROB;
  }
  for (k = NDIM; k < 3; k++) d->bc_lo[k] = d->bc_hi[k] = MDG_BC_PERIODIC;
  d->prob_kind = MDG_BINDING_PROB_KIND;
  d->cfl = cfl;
  d->dt_init_safety = dt_init_safety;
  d->dt_grow_safety = dt_grow_safety;
  d->initial_dt = initial_dt;
  d->dtmax = dtmax;
  d->dtmin = dtmin;
  d->tmax = tmax;
  d->hydro_interp_order = hydro_interp_order;
  d->enforce_floors = (ENFORCE_FLOORS == TRUE);
  d->rho_floor = rho_floor;
  d->e_floor = e_floor;
#if (GRAV == FIXED_GRAV)
  for (k = 0; k < 3; k++) d->grav[k] = g0[k];
#endif
#if (GRAV == SPHERICAL_MONOPOLE_GRAV && GR_MONOPOLE == FALSE)
  d->monopole = 1;
#endif
#if (GEOM == SPHERICAL && RCOORD == SINH)
  d->rcoord = MDG_RCOORD_SINH;
#elif (GEOM == SPHERICAL && RCOORD == SINH_MODIFIED)
  d->rcoord = MDG_RCOORD_SINH_MODIFIED;
#elif (GEOM == SPHERICAL && defined(LOG) && RCOORD == LOG)
  d->rcoord = MDG_RCOORD_LOG;   /* the RCOORD=LOG build of the oracle's reference sources */
#else
  d->rcoord = MDG_RCOORD_UNIFORM;
#endif
  d->rtrans = rx_info.rtrans;
  d->rfact[0] = rx_info.facta;
  d->rfact[1] = rx_info.factb;
  d->rfact[2] = rx_info.factc;
#if (GEOM == SPHERICAL && THCOORD == POLYTH)
  d->thcoord = MDG_THCOORD_POLYTH;
#else
  d->thcoord = MDG_THCOORD_UNIFORM;
#endif
  d->poly_xt = thx_info.poly_xt;
  d->poly_alpha = thx_info.poly_alpha;
}

static void attach(void)
{
  mdg_problem_desc d;
  describe(&d);
  mdg_or_die(mdg_create(&d, 1, MDG_BINDING_PRECISION, MDG_BINDING_DEVICE, &g_mdg), "mdg_create");
  /* main.c:172-182: the state after init_problem at t = 0 */
  mdg_or_die(mdg_upload_state(g_mdg, 0, &sim_p[0][0]), "mdg_upload_state");
}

/* step.c:163-203: the CFL estimate into the global dt (main.c applies its own rules) */
void estimate_dt(void)
{
  double d;
  if (!g_mdg) attach();
  mdg_or_die(mdg_estimate_dt_raw(g_mdg, &d), "estimate_dt");
  min_dt = d;
  dt = d;
}

/* step.c:16-24: the device state (and its EOS record) back into sim_p / sim_eos */
void update_cpu(void)
{
  if (!g_mdg) return;
  mdg_or_die(mdg_synchronize(g_mdg), "update_cpu");
  mdg_or_die(mdg_download_state(g_mdg, 0, &sim_p[0][0], &sim_eos[0][0]), "update_cpu");
}

/* step.c:133-155: bounce time from the central density (of the state on the host) */
void set_tbounce(void)
{
  double rho_cent = 0.0;
  update_cpu();
  if (istart[0] == 0) rho_cent = sim_p[0][RHO];   /* zone (0, 0, 0) leads the interior */
  rho_cent = mpi_max(rho_cent);
  if (rho_cent > rho_cent_max) rho_cent_max = rho_cent;
  if (rho_cent < 0.95*rho_cent_max) {
    tbounce = t;
    if (mpi_io_proc()) fprintf(stderr, "[set_tbounce]:  Bounce detected! tbounce=%1.6f\n", tbounce);
  }
}

/* step.c:28-129: both RK stages with the global dt; main.c adds dt to t itself */
void step(void)
{
  if (!g_mdg) attach();
  mdg_or_die(mdg_step_dt(g_mdg, &dt), "step");
  if (detect_tbounce && tbounce < 0.0) set_tbounce();
}
