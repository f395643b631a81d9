/*
 * TEST INFRASTRUCTURE ONLY.
 *
 * Glue that lets the reference's UNMODIFIED main.c (main.c:9-346) run a problem end to
 * end in this container, where io.c (HDF5) and the problem files (written against a
 * removed API) do not compile.  oracle/build_ref.py links it twice with the same
 * reference sources: once with the reference's own step.c (the CPU run), once with
 * medusa_b200/host/fornax_binding.c instead of step.c (the drop-in GPU run).  Both read
 * the same input file, so the comparison of their final states tests the drop-in
 * boundary itself: main.c's loop, its dt rules and the problem hooks are the same
 * code in both.
 *
 *   - parse_input restates the key = value reader of io.c:4979-5785 for the keys the
 *     hydro run uses (defaults as io.c:5000-5117);
 *   - the problem hooks restate, in the current API, problems/init_sod.c:31-99
 *     (DROPIN_PROB 1), problems/init_dustcollapse.c:27-113 (DROPIN_PROB 2) and
 *     problems/init_sedov.c:3-164 on the 3-D dendritic grid (DROPIN_PROB 3; its outer
 *     PROB boundary, a fixed ambient state equal to the initial outer zones, is OUTFLOW
 *     here, the same ghost values until the blast reaches the outer radius);
 *   - the gamma-law EOS fill loops as eos/burrows/eos_stuff.c:521-532,668-683 with the
 *     arithmetic of eos/gamma/eos_gamma.c:5-12,45-58;
 *   - dumps, logs and restarts are no-ops; analysis_postloop brings the state to the
 *     host (update_cpu) and writes istep, t, the interior primitives and EOS records to
 *     $DROPIN_OUT (default dropin_final.bin).
 */
#include "decs.h"
#include "constants.h"

#ifndef DROPIN_PROB
#define DROPIN_PROB 1
#endif

/* ---------------- parse_input (io.c:4979-5785, the hydro keys) ---------------- */
static char *trim(char *s)
{
  char *e;
  while (*s == ' ' || *s == '\t') s++;
  e = s + strlen(s);
  while (e > s && (e[-1] == ' ' || e[-1] == '\t' || e[-1] == '\n' || e[-1] == '\r')) *--e = '\0';
  return s;
}

void parse_input(char *name)
{
  FILE *fp;
  char line[512];
  /* defaults (io.c:5000-5117) */
  rx_info.facta = 10*1e5;
  rx_info.factb = 15*1e5;
  rx_info.factc = 5*1e5;
  thx_info.nice_alpha = 1.01;
  thx_info.poly_xt = 1.2;
  thx_info.poly_alpha = 4;
  Nskip = 1;
  cfl = 0.9;
  n1 = 1024; n2 = 1; n3 = 1;
  dt_grow_safety = 1.1;
  dt_init_safety = 0.1;
  dtmax = 1.0e200;
  dtmin = 1.0e-200;
  initial_dt = 1.0e100;
  tmax = 1.0;
  ncomp = 0;
  hydro_interp_order = 3;
  rad_interp_order = 2;
  dt_dump = 1.0e100;
  dt_pdump = 1.0e100;
  dt_restart = 1.0e100;
  di_restart = INT_MAX/2;
  nstep_log = INT_MAX;
  nstep_analysis = INT_MAX;
  nstep_timing = INT_MAX;
  max_steps = 2147483647;
  max_wtime = 1.0e100;
  e_floor = -1.0;
  rho_floor = -1.0;
  detect_tbounce = 0;
  dump_hdf = 0;
  restart_from_hdf = 0;
  restart_create_1d = 0;

  fp = fopen(name, "r");
  if (!fp) {
    fprintf(stderr, "parse_input: cannot open %s\n", name);
    exit(1);
  }
  while (fgets(line, sizeof line, fp)) {
    char *eq, *lhs, *rhs, *hash = strchr(line, '#');
    if (hash) *hash = '\0';
    eq = strchr(line, '=');
    if (!eq) continue;
    *eq = '\0';
    lhs = trim(line);
    rhs = trim(eq + 1);
    if (strcmp(lhs, "n1") == 0) n1 = atoi(rhs);
    else if (strcmp(lhs, "n2") == 0) n2 = atoi(rhs);
    else if (strcmp(lhs, "n3") == 0) n3 = atoi(rhs);
    else if (strcmp(lhs, "cfl") == 0) cfl = atof(rhs);
    else if (strcmp(lhs, "tmax") == 0) tmax = atof(rhs);
    else if (strcmp(lhs, "dt_init_safety") == 0) dt_init_safety = atof(rhs);
    else if (strcmp(lhs, "dt_grow_safety") == 0) dt_grow_safety = atof(rhs);
    else if (strcmp(lhs, "initial_dt") == 0) initial_dt = atof(rhs);
    else if (strcmp(lhs, "dtmax") == 0) dtmax = atof(rhs);
    else if (strcmp(lhs, "dtmin") == 0) dtmin = atof(rhs);
    else if (strcmp(lhs, "hydro_interp_order") == 0) hydro_interp_order = atoi(rhs);
    else if (strcmp(lhs, "max_steps") == 0) max_steps = atoi(rhs);
    else if (strcmp(lhs, "dt_dump") == 0) dt_dump = atof(rhs);
    else if (strcmp(lhs, "nstep_log") == 0) nstep_log = atoi(rhs);
    else if (strcmp(lhs, "nstep_analysis") == 0) nstep_analysis = atoi(rhs);
  }
  fclose(fp);
#if (NDIM==1)
  n2 = n3 = 1;
#elif (NDIM==2)
  n3 = 1;
#endif
  /* io.c:5684-5693 */
  nhydro = NPRIM + ncomp;
  nvars = nhydro;
  ninterp = nvars + 2;
}

/* ---------------- io.c entry points: no-ops ---------------- */
void run_log() {}
void output_timers() {}
void dump1() {}
void dump2() {}
void dump3() {}
void dump_ascii1(int is_restart) { (void)is_restart; }
void dump_tracers() {}
void restart_dump() {}
void restart_read() {}

/* ---------------- EOS fill (gamma law) ---------------- */
static void fill_one(const double *p, double *eos)
{
  double press = (gam-1.0)*p[UU];
  eos[PRESS] = press;
  eos[CS   ] = sqrt(gam*press/p[RHO]);
  eos[TEMP ] = press/(2.0*p[RHO]*KBOLTZ)*(MP+ME);
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
#if (DROPIN_PROB == 1)
/* problems/init_sod.c:31-99 */
void init_grid()
{
  startx[0] = 0.0;
  dx[0] = 1.0/n1;
}

void init_problem()
{
  int ii=0, jj=0, kk=0, vv, dd;
  double xl, xr, rhol, el, ul, rhor, er, ur;
  gam = 1.4;
  rhol = 1.0; el = 1.0/(gam-1.0); ul = 0.0;
  rhor = 0.125; er = 0.1/(gam-1.0); ur = 0.0;
  VLOOP {
    bc[vv].lo[0] = OUTFLOW;
    bc[vv].hi[0] = OUTFLOW;
  }
  ZLOOP {
    xl = ii*dx[0];
    xr = xl+dx[0];
    if (xr < 0.5) {
      NDP_ELEM_LINEAR(sim_p,ii,jj,kk,RHO) = rhol;
      NDP_ELEM_LINEAR(sim_p,ii,jj,kk,UU ) = el;
      DLOOP { NDP_ELEM_LINEAR(sim_p,ii,jj,kk,U1+dd) = ul; }
    } else if (xl < 0.5) {
      NDP_ELEM_LINEAR(sim_p,ii,jj,kk,RHO) = rhol*(0.5-xl)/dx[0] + rhor*(xr-0.5)/dx[0];
      NDP_ELEM_LINEAR(sim_p,ii,jj,kk,UU ) = el*(0.5-xl)/dx[0] + er*(xr-0.5)/dx[0];
      DLOOP { NDP_ELEM_LINEAR(sim_p,ii,jj,kk,U1+dd) = ul*(0.5-xl)/dx[0] + ur*(xr-0.5)/dx[0]; }
    } else {
      NDP_ELEM_LINEAR(sim_p,ii,jj,kk,RHO) = rhor;
      NDP_ELEM_LINEAR(sim_p,ii,jj,kk,UU ) = er;
      DLOOP { NDP_ELEM_LINEAR(sim_p,ii,jj,kk,U1+dd) = ur; }
    }
    for (dd=NDIM; dd<SPACEDIM; dd++) NDP_ELEM_LINEAR(sim_p,ii,jj,kk,U1+dd) = 0.0;
  }
}

void prob_bounds(int i, int j, int k, double *p) { (void)i; (void)j; (void)k; (void)p; }

#elif (DROPIN_PROB == 2)
/* problems/init_dustcollapse.c:27-113 */
static double rho0 = 1.0e9;
static double r0   = 6.5e8;
static double t0   = 1.0;
static double Mach = 2.0;

void init_grid()
{
  startx[0] = 0.0;
  dx[0] = 5.0e4;
  rx_info.rtrans = rtrans_solve(dx[0], 7.0e8);
  periodic[0] = 0;
  periodic[1] = 0;
  periodic[2] = 1;
}

void init_problem()
{
  int ii=0, jj=0, kk=0, vv;
  double v0, p0, rm, rp;
  gam = 5.0/3.0;
  v0 = r0/t0;
  p0 = rho0*SQR(v0/Mach)/gam;
  rho_floor = 1.0e-5*rho0;
  e_floor = p0/(gam-1.0);
  VLOOP {
    bc[vv].lo[0] = SPHERICAL_ORIGIN;
    bc[vv].hi[0] = OUTFLOW;
  }
  bc[U1].hi[0] = PROB;
  ZLOOP {
    rm = r_of_x(rx_info, startx[0] + (ii  )*dx[0]);
    rp = r_of_x(rx_info, startx[0] + (ii+1)*dx[0]);
    if (rp < r0) {
      NDP_ELEM_LINEAR(sim_p,ii,jj,kk,RHO) = rho0;
    } else if (rm < r0) {
      NDP_ELEM_LINEAR(sim_p,ii,jj,kk,RHO) = rho0*(pow(r0,3) - pow(rm,3))/(pow(rp,3) - pow(rm,3));
    } else {
      NDP_ELEM_LINEAR(sim_p,ii,jj,kk,RHO) = rho_floor;
    }
    NDP_ELEM_LINEAR(sim_p,ii,jj,kk,UU) = p0/(gam-1.0);
    NDP_ELEM_LINEAR(sim_p,ii,jj,kk,U1) = 0.0;
    NDP_ELEM_LINEAR(sim_p,ii,jj,kk,U2) = 0.0;
    NDP_ELEM_LINEAR(sim_p,ii,jj,kk,U3) = 0.0;
  }
}

void prob_bounds(int i, int j, int k, double *p)
{
  double r = r_of_x(rx_info, beta0[i]/Gamma0[i]);
  double vr = -1.0/sqrt(r);
  p[U1] = vr/ND_ELEM_LINEAR(geom,i,j,k).scale[0][0];
}

#elif (DROPIN_PROB == 3)
/* problems/init_sedov.c:3-164 (3-D) */
void init_grid()
{
  startx[0] = 0.;
  startx[1] = -1.;
  startx[2] = 0.;
  dx[0] = 0.4*1.2/n1;
  dx[1] = 2./n2;
  dx[2] = 2.*M_PI/n3;
  rx_info.rtrans = rtrans_solve(dx[0], 1.2);
  periodic[0] = 0;
  periodic[1] = 0;
  periodic[2] = 1;
}

void init_problem()
{
  int ii=0, jj=0, kk=0, vv;
  double rho_amb = 1., e_amb = 1.e-12, u_amb = 0.;
  double E_expl = 0.851072, R_expl = 0.075, Edens;
  gam = 1.4;
  VLOOP {
    bc[vv].lo[0] = SPHERICAL_ORIGIN;
    bc[vv].hi[0] = OUTFLOW;
    bc[vv].lo[1] = REFLECT;
    bc[vv].hi[1] = REFLECT;
    bc[vv].lo[2] = PERIODIC;
    bc[vv].hi[2] = PERIODIC;
  }
  ZLOOP {
    NDP_ELEM_LINEAR(sim_p,ii,jj,kk,RHO) = rho_amb;
    NDP_ELEM_LINEAR(sim_p,ii,jj,kk,UU) = e_amb;
    NDP_ELEM_LINEAR(sim_p,ii,jj,kk,U1) = u_amb;
    NDP_ELEM_LINEAR(sim_p,ii,jj,kk,U2) = 0.;
    NDP_ELEM_LINEAR(sim_p,ii,jj,kk,U3) = 0.;
  }
  Edens = E_expl/(4./3.*M_PI*pow(R_expl,3.));
  if (redge[istart[0]] < R_expl) {
    for (ii=istart[0]; ii<istop[0]; ii++) {
      if (redge[ii+1] < R_expl) {
        JSLOOP(ii,jj) { KSLOOP(ii,jj,kk) { NDP_ELEM_LINEAR(sim_p,ii,jj,kk,UU) = Edens; } }
      } else if (redge[ii] < R_expl) {
        Edens *= (pow(R_expl,3.)-pow(redge[ii],3.))/(pow(redge[ii+1],3.)-pow(redge[ii],3.));
        JSLOOP(ii,jj) { KSLOOP(ii,jj,kk) { NDP_ELEM_LINEAR(sim_p,ii,jj,kk,UU) = Edens; } }
        break;
      } else {
        break;
      }
    }
  }
}

void prob_bounds(int i, int j, int k, double *p) { (void)i; (void)j; (void)k; (void)p; }
#endif

/* ---------------- analysis hooks ---------------- */
void analysis_preloop() {}
void analysis_inloop() {}

void analysis_postloop()
{
  const char *name = getenv("DROPIN_OUT");
  FILE *fp;
  int II;
  update_cpu();
  fp = fopen(name ? name : "dropin_final.bin", "wb");
  if (!fp) {
    fprintf(stderr, "analysis_postloop: cannot write the final state\n");
    exit(1);
  }
  fwrite(&istep, sizeof istep, 1, fp);
  fwrite(&t, sizeof t, 1, fp);
  for (II=0; II<cell_count; II++) fwrite(sim_p[II], sizeof(double), NPRIM, fp);
  for (II=0; II<cell_count; II++) fwrite(sim_eos[II], sizeof(double), NEOS, fp);
  fclose(fp);
}
