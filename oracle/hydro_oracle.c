/*
 * hydro_oracle.c -- CPU restatement of the reference hydrodynamic sweep.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for medusa_b200: only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, and only to
 * check or time; the product path never links or calls it.
 *
 * It restates, in plain C99 with runtime dimensionality (NDIM 1 or 2), the
 * algorithm of the reference's single-rank CPU build, function by function, in the
 * reference's floating-point operation order (build with -O2 -fno-fast-math
 * -ffp-contract=off):
 *   step()                          step.c:28-129
 *   estimate_dt() + main.c dt rules step.c:163-203, main.c:226-264
 *   dt_source_control()             step.c:205-223
 *   push()                          step.c:327-478
 *   prim_to_fluxes1()               step.c:482-567
 *   prim_to_fluxes2()/prolongate0() step.c:579-628, 659-764 (Cartesian, no dendritic level change)
 *   para_recon()/lin_recon()        reconstruct.c:89-213, interp() reconstruct.c:225-279
 *   riemann_flux_HLLC/HLLE, p_uflux, pflux   riemann.c:4-62, 178-499
 *   hydro_p_to_u/u_to_p             fluid.c:4-53
 *   hydro_stress_tensor, p_to_geom_src  fluid.c:56-73, rad_fluid.c:164-192
 *   set_shock_flag(0), transverse_shock  fluid.c:75-89, 189-210
 *   reset_boundaries_gpu            bc.c:705-1422 (OUTFLOW, REFLECT, EXTRAP, PERIODIC,
 *                                   SPHERICAL_ORIGIN, PROB) incl. the t+=dt / t-=dt shift
 *   gamma-law / polytrope EOS       eos/gamma/eos_gamma.c:5-12,45-58, eos/polytropic/eos_poly.c:5-11
 *   geometry                        metrics/metric_cartesian.c:47-295,
 *                                   metrics/metric_spherical_general.c:145-300, 558-1051 (RCOORD =
 *                                   UNIFORM, SINH, SINH_MODIFIED and LOG, THCOORD = UNIFORM
 *                                   and POLYTH; 1-D),
 *                                   utils.c:32-62 (romb)
 * Parity is pinned against the reference itself, built unmodified by
 * oracle/build_ref.py (tests/test_oracle_pin.py) and against the golden fixtures in
 * tests/golden/ that the same reference build produced.
 *
 * Layout: structure of arrays with NG=2 ghost layers, cell (i,j) at
 * (i+NG)*(n2+2NG)+(j+NG) (2-D) or i+NG (1-D).  Ghost "corner" cells exist and stay 0,
 * as the reference's calloc'ed arrays do.  Shock flags of ghost cells stay 0 ("shock")
 * for the whole run, exactly as in the reference (utils.c:164-174 zero-fills and
 * set_shock_flag(0) resets only interior cells).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

#define NG 2
#define NPRIM 5
#define RHO 0
#define UU 1
#define U1 2
#define U2 3
#define U3 4
#define PRESS 0
#define CS 1
#define TEMP 2
#define ENT 3
#define GAMMA 4
#define NINT 7   /* 5 primitives + pressure + Gamma */

#define OUTFLOW 0
#define REFLECT 1
#define EXTRAP 2
#define PERIODIC 3
#define PROB 4
#define SPHERICAL_ORIGIN 5

#define MIN(a,b) ((a) < (b) ? (a) : (b))
#define MAX(a,b) ((a) > (b) ? (a) : (b))
#define SQR(x) ((x)*(x))
#define CUBE(x) ((x)*(x)*(x))
#define SIGN(a) ((a) < 0.0 ? -1.0 : 1.0)
#define MINMOD(a,b) (0.5*(SIGN(a)+SIGN(b))*MIN(fabs(a),fabs(b)))

#define KBOLTZ 1.3806488e-16
#define MP 1.67262158e-24
#define ME 9.10938291e-28

/* same field order as ref_params in oracle/refshim/ref_harness.c */
typedef struct {
  int n1, n2, n3;
  double startx[3];
  double dx[3];
  double gam;
  double Kpoly;
  int eos_kind;
  int bc_lo[3], bc_hi[3];
  int prob_kind;
  double cfl;
  double dt_init_safety, dt_grow_safety;
  double initial_dt, dtmax, dtmin;
  double tmax;
  double rtrans;
  int hydro_interp_order;
  int enforce_floors;
  double rho_floor, e_floor;
  double grav[3];
  int rcoord;          /* radial map: 0 UNIFORM, 1 SINH, 2 SINH_MODIFIED, 3 LOG (the RCOORD build switch) */
  double rfact[3];     /* SINH_MODIFIED: facta, factb, factc */
  int thcoord;         /* theta map: 0 UNIFORM, 1 POLYTH (the THCOORD build switch) */
  double poly_xt, poly_alpha;   /* POLYTH */
} orc_params;

typedef struct {
  double area[2];
  double gcov[3][3];
  double gcon[3];
  double scale[3][3];
  double volume;
  double conn[3][3][3];
} orc_geom;

typedef struct {
  orc_params prm;
  int ndim, geom;         /* geom: 0 Cartesian, 1 spherical */
  int n1, n2, s1, s2;     /* interior sizes, padded sizes */
  int ncell;              /* padded cell count */
  double *p[NPRIM], *ph[NPRIM], *eos[5], *src[NPRIM];
  int *flag;
  double *f0[NPRIM], *f1[NPRIM];   /* face fluxes, indexed by the face's cell */
  orc_geom *g;
  double *alpha0, *beta0, *Gamma0;   /* [n1+2NG] */
  double *alpha1, *beta1, *Gamma1;   /* [n2+2NG] (2-D) */
  double t, dt, min_dt, dtold;
  int istep;
  int interp_order;
  int est_first;
  int grav_on;            /* GRAV=FIXED_GRAV: a non-zero fixed acceleration */
} orc_t;

static inline int C(const orc_t *o, int i, int j) { return (i+NG)*o->s2 + (o->ndim > 1 ? j+NG : j); }

/* ------------------------------------------------------------------ romb */
/* utils.c:16-62 (ROMBERG_MAX 15, TOL 1e-15, ATOL 1e-15) */
static double rtrap(double x0, double x1, int rstage, double (*f)(double))
{
  unsigned long long int nseg = 1ULL<<rstage, i;
  double dx = (x1-x0)/nseg, sum = 0.0;
  if (rstage == 0) return 0.5*dx*((*f)(x0) + (*f)(x1));
  for (i=0; i<(1ULL<<(rstage-1)); i++) sum += (*f)(x0 + (2*i+1)*dx);
  return dx*sum;
}

static double romb(double x0, double x1, double (*f)(double))
{
  double rvec[16], R0, R1;
  unsigned long long int fm;
  int rstage, m;
  rvec[0] = rtrap(x0,x1,0,f);
  for (rstage=1; rstage<=15; rstage++) {
    R0 = rvec[0];
    rvec[0] = 0.5*R0 + rtrap(x0,x1,rstage,f);
    for (m=1; m<=rstage; m++) {
      fm = 1ULL<<(2*m);
      R1 = rvec[m];
      rvec[m] = 1.0/(fm-1)*(fm*rvec[m-1] - R0);
      R0 = R1;
    }
    if (fabs((rvec[rstage]-rvec[rstage-1])/rvec[rstage]) < 1.e-15 ||
        (rstage > 2 && fabs(rvec[rstage]) < 1.e-15)) return rvec[rstage];
  }
  return rvec[15];
}

/* metric_spherical_general.c maps and integrands: r(x) for RCOORD = UNIFORM, SINH and
 * SINH_MODIFIED (r_of_x 149-178 with sigmoid 145-147, dr_dx 180-198, d2r_dx2 200-219),
 * the LOG map r = rtrans exp(|x|/rtrans) that the oracle's RCOORD=LOG reference builds add
 * in the form of the SINH branch, and th(x) for THCOORD = UNIFORM and POLYTH (th_of_x
 * 222-256, dth_dx 258-279, d2th_dx2 281-300, poly_norm as init_coords sets it, 568).
 * The maps are those of the problem being built (the integrands are plain functions
 * handed to romb). */
enum { RC_UNIFORM = 0, RC_SINH = 1, RC_SINH_MODIFIED = 2, RC_LOG = 3 };
enum { TH_UNIFORM = 0, TH_POLYTH = 1 };
static int g_rcoord = RC_UNIFORM, g_thcoord = TH_UNIFORM;
static double g_rtrans = 1.0, g_facta = 0.0, g_factb = 0.0, g_factc = 1.0;
static double g_poly_norm = 0.0, g_poly_xt = 1.0, g_poly_alpha = 0.0;
static double sigmoid(double x) { return 1.0/(1.0+exp(-x)); }
static double r_of_x(double x)
{
  if (g_rcoord == RC_SINH) return g_rtrans*sinh(fabs(x)/g_rtrans);
  if (g_rcoord == RC_SINH_MODIFIED)
    return g_rtrans*sinh(fabs(x)/g_rtrans) - g_facta*sigmoid((fabs(x)-g_factb)/g_factc)
           + g_facta*sigmoid(-g_factb/g_factc);
  if (g_rcoord == RC_LOG) return g_rtrans*exp(fabs(x)/g_rtrans);
  return fabs(x);
}
static double dr_dx(double x)
{
  if (g_rcoord == RC_SINH) return cosh(fabs(x)/g_rtrans);
  if (g_rcoord == RC_SINH_MODIFIED) {
    double e = exp(-(fabs(x)-g_factb)/g_factc);
    return cosh(fabs(x)/g_rtrans) - g_facta*e/g_factc/(1+e)/(1+e);
  }
  if (g_rcoord == RC_LOG) return exp(fabs(x)/g_rtrans);
  return 1.0;
}
static double d2r_dx2(double x)
{
  if (g_rcoord == RC_SINH) return sinh(fabs(x)/g_rtrans)/g_rtrans;
  if (g_rcoord == RC_SINH_MODIFIED) {
    double e = exp(-(fabs(x)-g_factb)/g_factc);
    return sinh(fabs(x)/g_rtrans)/g_rtrans
           - g_facta/g_factc/g_factc*(2*e*e/(1+e)/(1+e)/(1+e) - e/(1+e)/(1+e));
  }
  if (g_rcoord == RC_LOG) return exp(fabs(x)/g_rtrans)/g_rtrans;
  return 0.0;
}
/* theta maps, reflected about the polar axis */
static double th_of_x(double x)
{
  if (x < -1.0) x = -2.0 - x;
  if (x >  1.0) x =  2.0 - x;
  if (g_thcoord == TH_POLYTH)
    return g_poly_norm*x*(1.0 + pow(x/g_poly_xt,g_poly_alpha)/(g_poly_alpha+1.0)) + 0.5*M_PI;
  return 0.5*M_PI*(x+1.0);
}
static double dth_dx(double x)
{
  if (x < -1.0) x = -2.0 - x;
  if (x >  1.0) x =  2.0 - x;
  if (g_thcoord == TH_POLYTH) return g_poly_norm*(1.0 + pow(x/g_poly_xt,g_poly_alpha));
  return 0.5*M_PI;
}
static double d2th_dx2(double x)
{
  if (x < -1.0) x = -2.0 - x;
  if (x >  1.0) x =  2.0 - x;
  if (g_thcoord == TH_POLYTH)
    return g_poly_norm*g_poly_alpha*pow(x/g_poly_xt,g_poly_alpha-1.0)/g_poly_xt;
  return 0.0;
}
static double f_r2dr_dx(double x) { return pow(r_of_x(x),2)*dr_dx(x); }
static double f_xr1g(double x) { return x*pow(r_of_x(x),2)*dr_dx(x); }
static double f_xr2g(double x) { return x*x*pow(r_of_x(x),2)*dr_dx(x); }
static double f_r2d2r_dx2(double x) { return pow(r_of_x(x),2)*d2r_dx2(x); }
static double f_r3(double x) { return pow(r_of_x(x),3); }
static double f_r2dr_dx3(double x) { return pow(r_of_x(x),2)*pow(dr_dx(x),3); }
static double f_rdr_dx2(double x) { return r_of_x(x)*pow(dr_dx(x),2); }
static double f_sthdth_dx(double x) { return sin(th_of_x(x))*dth_dx(x); }
static double f_sthdth_dx3(double x) { return sin(th_of_x(x))*pow(dth_dx(x),3); }
static double f_sth3dth_dx(double x) { return pow(sin(th_of_x(x)),3)*dth_dx(x); }
static double f_sthd2th_dx2(double x) { return sin(th_of_x(x))*d2th_dx2(x); }
static double f_cthdth_dx2(double x) { return cos(th_of_x(x))*pow(dth_dx(x),2); }

/* make o's radial map the one the maps above evaluate */
static void use_map(const orc_t *o)
{
  g_rcoord = o->prm.rcoord;
  g_rtrans = o->prm.rtrans;
  g_facta = o->prm.rfact[0];
  g_factb = o->prm.rfact[1];
  g_factc = o->prm.rfact[2];
  g_thcoord = o->prm.thcoord;
  g_poly_xt = o->prm.poly_xt;
  g_poly_alpha = o->prm.poly_alpha;
  if (g_thcoord == TH_POLYTH)
    g_poly_norm = 0.5*M_PI*1.0/(1.0 + 1.0/(g_poly_alpha+1.0) * 1.0/pow(g_poly_xt,g_poly_alpha));
}

static void init_geometry(orc_t *o)
{
  const orc_params *P = &o->prm;
  int i, j, l, m, loc, d;
  if (o->geom == 0) {
    /* metric_cartesian.c:47-55 and the per-zone loops 127-295 */
    for (i=-NG; i<o->n1+NG; i++) {
      double x0 = P->startx[0] + i*P->dx[0], x1 = x0 + P->dx[0];
      o->alpha0[i+NG] = (CUBE(x1) - CUBE(x0))/3.0;
      o->beta0[i+NG] = (SQR(x1) - SQR(x0))/2.0;
      o->Gamma0[i+NG] = P->dx[0];
    }
    if (o->ndim > 1) {
      for (j=-NG; j<o->n2+NG; j++) {
        double x0 = P->startx[1] + j*P->dx[1], x1 = x0 + P->dx[1];
        o->alpha1[j+NG] = (CUBE(x1) - CUBE(x0))/3.0;
        o->beta1[j+NG] = (SQR(x1) - SQR(x0))/2.0;
        o->Gamma1[j+NG] = P->dx[1];
      }
    }
    for (int c=0; c<o->ncell; c++) {
      orc_geom *g = &o->g[c];
      memset(g, 0, sizeof *g);
      g->volume = 1.0;
      for (d=0; d<o->ndim; d++) g->volume *= P->dx[d];
      for (loc=0; loc<o->ndim; loc++) {
        g->area[loc] = 1.0;
        for (d=0; d<o->ndim; d++) g->area[loc] *= P->dx[d];
        g->area[loc] /= P->dx[loc];
      }
      for (loc=0; loc<=o->ndim; loc++) for (l=0; l<3; l++) { g->gcov[loc][l] = 1.0; g->scale[loc][l] = 1.0; }
      for (l=0; l<3; l++) g->gcon[l] = 1.0;
    }
    return;
  }
  /* spherical, 1-D, uniform radius: metric_spherical_general.c:558-568 (moments),
   * 708-740 (volume), 745-779 (area), 820-930 (conn), 941-1051 (gcov, gcon, scale) */
  for (i=-NG; i<o->n1+NG; i++) {
    double x0 = P->startx[0] + i*P->dx[0], x1 = P->startx[0] + (i+1)*P->dx[0];
    o->Gamma0[i+NG] = romb(x0,x1,f_r2dr_dx);
    o->beta0[i+NG] = romb(x0,x1,f_xr1g);
    o->alpha0[i+NG] = romb(x0,x1,f_xr2g);
  }
  {
    const double x1lo = -1.0, x1hi = 1.0, dph = 2.0*M_PI;  /* dx[1]=2, dx[2]=2pi for NDIM=1 (init_coords) */
    double vthf = romb(x1lo,x1hi,f_sthdth_dx);
    double th_sthdth_dx3 = romb(x1lo,x1hi,f_sthdth_dx3);
    double th_sth3dth_dx = romb(x1lo,x1hi,f_sth3dth_dx);
    double th_sthd2th_dx2 = romb(x1lo,x1hi,f_sthd2th_dx2);
    double th_cthdth_dx2 = romb(x1lo,x1hi,f_cthdth_dx2);
    for (i=-NG; i<o->n1+NG; i++) {
      orc_geom *g = &o->g[C(o,i,0)];
      double x0lo = P->startx[0] + i*P->dx[0], x0hi = P->startx[0] + (i+1)*P->dx[0];
      double r2dr_int = romb(x0lo,x0hi,f_r2dr_dx);
      double vrf = r2dr_int;
      double rint_r2dr_dx3 = romb(x0lo,x0hi,f_r2dr_dx3);
      memset(g, 0, sizeof *g);
      g->volume = r2dr_int*vthf*1*dph;
      if (i >= 0 && i <= o->n1) g->area[0] = f_r2dr_dx(x0lo)*vthf*(1*dph);
      for (loc=0; loc<=1; loc++) for (m=0; m<3; m++) g->gcov[loc][m] = 0.0;
      g->gcov[0][0] = rint_r2dr_dx3/vrf;
      g->gcov[0][1] = fabs(0.2*(pow(r_of_x(x0hi),5) - pow(r_of_x(x0lo),5))/vrf * th_sthdth_dx3/vthf);
      g->gcov[0][2] = fabs(0.2*(pow(r_of_x(x0hi),5) - pow(r_of_x(x0lo),5))/vrf * th_sth3dth_dx/vthf);
      g->gcov[1][0] = pow(dr_dx(x0lo),2);
      g->gcov[1][1] = pow(r_of_x(x0lo),2)*th_sthdth_dx3/vthf;
      g->gcov[1][2] = pow(r_of_x(x0lo),2)*th_sth3dth_dx/vthf;
      for (m=0; m<3; m++) g->gcon[m] = (fabs(g->gcov[0][m]) > 1.0e-50) ? 1.0/g->gcov[0][m] : 0.0;
      for (loc=0; loc<=1; loc++) for (m=0; m<3; m++) g->scale[loc][m] = sqrt(g->gcov[loc][m]);
      if (i >= 0 && i < o->n1) {
        double rint_r2d2r_dx2 = romb(x0lo,x0hi,f_r2d2r_dx2);
        double rint_r3 = romb(x0lo,x0hi,f_r3);
        double rint_rdr_dx2 = romb(x0lo,x0hi,f_rdr_dx2);
        double vr = romb(x0lo,x0lo+P->dx[0],f_r2dr_dx);
        g->conn[0][0][0] = rint_r2d2r_dx2/vr;
        g->conn[0][1][1] = -(rint_r3/vr)*(th_sthdth_dx3/vthf);
        g->conn[1][0][1] = rint_rdr_dx2/vr;
        g->conn[1][1][0] = g->conn[1][0][1];
        g->conn[2][0][2] = g->conn[1][0][1];
        g->conn[2][2][0] = g->conn[2][0][2];
        g->conn[2][1][2] = th_cthdth_dx2/vthf;
        g->conn[2][2][1] = g->conn[2][1][2];
        g->conn[0][2][2] = -g->conn[2][2][0] * g->gcov[0][2]/g->gcov[0][0];
        g->conn[1][2][2] = -g->conn[2][2][1] * g->gcov[0][2]/g->gcov[0][1];
        g->conn[1][1][1] = th_sthd2th_dx2/vthf;
      }
    }
  }
}

/* ------------------------------------------------------------------ EOS */
static void eos_cell(const orc_t *o, double *const *p, int c)
{
  const double gam = o->prm.gam;
  double press, cs, tp;
  if (o->prm.eos_kind == 0) {
    press = (gam-1.0)*p[UU][c];
    cs = sqrt(gam*press/p[RHO][c]);
    tp = press/(2.0*p[RHO][c]*KBOLTZ)*(MP+ME);
  } else {
    press = o->prm.Kpoly*pow(p[RHO][c],gam);
    cs = sqrt(gam*press/p[RHO][c]);
    tp = press/(p[RHO][c]*KBOLTZ)*MP;
  }
  o->eos[PRESS][c] = press;
  o->eos[CS][c] = cs;
  o->eos[TEMP][c] = tp;
  o->eos[GAMMA][c] = gam;
}

static int is_interior(const orc_t *o, int i, int j)
{
  return i >= 0 && i < o->n1 && (o->ndim == 1 || (j >= 0 && j < o->n2));
}

static void update_eos(orc_t *o, double *const *p, int ghosts)
{
  for (int i=-NG; i<o->n1+NG; i++) {
    int jlo = (o->ndim > 1) ? -NG : 0, jhi = (o->ndim > 1) ? o->n2+NG : 1;
    for (int j=jlo; j<jhi; j++) {
      if (is_interior(o,i,j) != !ghosts) continue;
      eos_cell(o, p, C(o,i,j));
    }
  }
}

/* ------------------------------------------------------------------ BCs */
/* problems/init_spherical_noh.c:63-79 with ijk_to_r of metric_spherical_general.c:483-496 */
static void prob_bounds(const orc_t *o, int i, double *pv)
{
  if (o->prm.prob_kind != 1) return;
  double gam = o->prm.gam;
  double x = o->beta0[i+NG]/o->Gamma0[i+NG];
  double r = r_of_x(x), rhat0 = dr_dx(x);
  pv[RHO] = 1.;
  pv[UU] = 1.e-6/(gam-1.);
  pv[U1] = -1./rhat0;
  pv[U2] = 0.;
  pv[U3] = 0.;
  pv[RHO] += o->t/r;
  pv[RHO] *= pv[RHO];
}

/* bc.c:705-1422, the kinds used by 1-D/2-D non-dendritic grids */
static void reset_boundaries(orc_t *o, double **p, int half_step)
{
  const int n1 = o->n1, n2 = o->n2;
  int i, j, v;
  if (half_step) o->t += o->dt;
  int jl = 0, jh = (o->ndim > 1) ? n2 : 1;
  for (v=0; v<NPRIM; v++) {
    int kind = o->prm.bc_lo[0];
    for (i=-NG; i<0; i++) for (j=jl; j<jh; j++) {
      int c = C(o,i,j);
      switch (kind) {
        case OUTFLOW: p[v][c] = p[v][C(o,0,j)]; break;
        case REFLECT: p[v][c] = p[v][C(o,-1-i,j)]; if (v==U1) p[v][c] *= -1.0; break;
        case SPHERICAL_ORIGIN:
          if (o->geom == 1) {
            int jp = (o->ndim > 1) ? (n2 - 1 - j) : j;
            p[v][c] = p[v][C(o,-1-i,jp)];
            if (v==U1 || v==U3) p[v][c] *= -1.0;
          }
          break;
        case EXTRAP: p[v][c] = p[v][C(o,0,j)] + (i-0)*(p[v][C(o,1,j)]-p[v][C(o,0,j)]); break;
        case PROB: { double pv[NPRIM]; int w; for (w=0;w<NPRIM;w++) pv[w]=p[w][c]; prob_bounds(o,i,pv); for (w=0;w<NPRIM;w++) p[w][c]=pv[w]; } break;
        case PERIODIC: p[v][c] = p[v][C(o,i+n1,j)]; break;
      }
    }
  }
  for (v=0; v<NPRIM; v++) {
    int kind = o->prm.bc_hi[0];
    for (i=n1; i<n1+NG; i++) for (j=jl; j<jh; j++) {
      int c = C(o,i,j);
      switch (kind) {
        case OUTFLOW: p[v][c] = p[v][C(o,n1-1,j)]; break;
        case REFLECT: p[v][c] = p[v][C(o,2*n1-i-1,j)]; if (v==U1) p[v][c] *= -1.0; break;
        case EXTRAP: p[v][c] = p[v][C(o,n1-1,j)] + (i-n1+1)*(p[v][C(o,n1-1,j)]-p[v][C(o,n1-2,j)]); break;
        case PROB: { double pv[NPRIM]; int w; for (w=0;w<NPRIM;w++) pv[w]=p[w][c]; prob_bounds(o,i,pv); for (w=0;w<NPRIM;w++) p[w][c]=pv[w]; } break;
        case PERIODIC: p[v][c] = p[v][C(o,i-n1,j)]; break;
      }
    }
  }
  if (o->ndim > 1) {
    for (v=0; v<NPRIM; v++) {
      int kind = o->prm.bc_lo[1];
      for (i=0; i<n1; i++) for (j=-NG; j<0; j++) {
        int c = C(o,i,j);
        switch (kind) {
          case OUTFLOW: p[v][c] = p[v][C(o,i,0)]; break;
          case REFLECT: p[v][c] = p[v][C(o,i,-1-j)]; if (v==U2) p[v][c] *= -1.0; break;
          case PERIODIC: p[v][c] = p[v][C(o,i,j+n2)]; break;
          case PROB: { double pv[NPRIM]; int w; for (w=0;w<NPRIM;w++) pv[w]=p[w][c]; prob_bounds(o,i,pv); for (w=0;w<NPRIM;w++) p[w][c]=pv[w]; } break;
        }
      }
    }
    for (v=0; v<NPRIM; v++) {
      int kind = o->prm.bc_hi[1];
      for (i=0; i<n1; i++) for (j=n2; j<n2+NG; j++) {
        int c = C(o,i,j);
        switch (kind) {
          case OUTFLOW: p[v][c] = p[v][C(o,i,n2-1)]; break;
          case REFLECT: p[v][c] = p[v][C(o,i,2*n2-1-j)]; if (v==U2) p[v][c] *= -1.0; break;
          case PERIODIC: p[v][c] = p[v][C(o,i,j-n2)]; break;
          case PROB: { double pv[NPRIM]; int w; for (w=0;w<NPRIM;w++) pv[w]=p[w][c]; prob_bounds(o,i,pv); for (w=0;w<NPRIM;w++) p[w][c]=pv[w]; } break;
        }
      }
    }
  }
  if (half_step) o->t -= o->dt;
}

/* ------------------------------------------------------------------ reconstruction */
/* reconstruct.c:127-213 for the single zone i of a 4-point stencil (indices 1 or 2) */
static void para_recon_zone(const double *a, double *al, double *ar, const double *alpha,
                            const double *beta, const double *Gamma, const double *x, int i)
{
  double dqm, dqp, dqc, den, A, B, Cc, xzero, xmid, xlo, xhi, mask_sign, mean;
  double a0b1g2, a0b2g1, a1b0g2, a1b2g0, a2b0g1, a2b1g0;
  dqm = a[i  ] - a[i-1];
  dqp = a[i+1] - a[i  ];
  if (dqm*dqp <= 0.0) { al[i] = ar[i] = a[i]; return; }
  dqc = a[i+1] - a[i-1];
  a0b1g2 = alpha[i-1]*beta[i  ]*Gamma[i+1];
  a0b2g1 = alpha[i-1]*beta[i+1]*Gamma[i  ];
  a1b0g2 = alpha[i  ]*beta[i-1]*Gamma[i+1];
  a1b2g0 = alpha[i  ]*beta[i+1]*Gamma[i-1];
  a2b0g1 = alpha[i+1]*beta[i-1]*Gamma[i  ];
  a2b1g0 = alpha[i+1]*beta[i  ]*Gamma[i-1];
  den = 1.0/(a0b1g2 + a1b2g0 + a2b0g1 - a0b2g1 - a1b0g2 - a2b1g0);
  A =  (dqm* beta[i+1]*Gamma[i-1]*Gamma[i] + Gamma[i+1]*(dqp* beta[i-1]*Gamma[i] - dqc* beta[i]*Gamma[i-1]))*den;
  B = -(dqm*alpha[i+1]*Gamma[i-1]*Gamma[i] + Gamma[i+1]*(dqp*alpha[i-1]*Gamma[i] - dqc*alpha[i]*Gamma[i-1]))*den;
  Cc = a[i] - (alpha[i]*A + beta[i]*B)/Gamma[i];
  al[i] = x[i  ]*(A*x[i  ] + B) + Cc;
  ar[i] = x[i+1]*(A*x[i+1] + B) + Cc;
  mean = 0.75*a[i-1] + 0.25*a[i];
  mask_sign = (a[i] - al[i])*(al[i] - mean);
  al[i] = (mask_sign < 0.0) ? mean : al[i];
  mean = 0.75*a[i+1] + 0.25*a[i];
  mask_sign = (mean - ar[i])*(ar[i] - a[i]);
  ar[i] = (mask_sign < 0.0) ? mean : ar[i];
  den = (x[i] - x[i+1])*(alpha[i] + Gamma[i]*x[i]*x[i+1] - beta[i]*(x[i]+x[i+1]));
  den = 1.0/den;
  A = ( beta[i]*(ar[i] - al[i]) + Gamma[i]*( a[i]*(x[i] - x[i+1]) - ar[i]*x[i] + al[i]*x[i+1]))*den;
  B = (alpha[i]*(al[i] - ar[i]) + Gamma[i]*(ar[i] - a[i])*SQR(x[i]) + Gamma[i]*(a[i]-al[i])*SQR(x[i+1]))*den;
  Cc = a[i] - (alpha[i]*A + beta[i]*B)/Gamma[i];
  xzero = -B/(2*A+1.0e-16);
  if (isinf(xzero) || isnan(xzero)) xzero = -1.0e-200;
  xlo = x[i];
  xhi = x[i+1];
  xmid = 0.5*(x[i]+x[i+1]);
  if (xzero > xlo && xzero < xhi) {
    if (xzero > xmid) {
      A = Gamma[i]*(a[i] - ar[i])/(alpha[i] + xhi*(Gamma[i]*xhi - 2.0*beta[i]));
      B = -2.0*A*xhi;
      Cc = a[i] - (alpha[i]*A + beta[i]*B)/Gamma[i];
      al[i] = x[i]*(A*x[i] + B) + Cc;
    } else {
      A = Gamma[i]*(a[i] - al[i])/(alpha[i] + xlo*(Gamma[i]*xlo - 2.0*beta[i]));
      B = -2.0*A*xlo;
      Cc = a[i] - (alpha[i]*A + beta[i]*B)/Gamma[i];
      ar[i] = x[i+1]*(A*x[i+1] + B) + Cc;
    }
  }
}

/* reconstruct.c:89-124 */
static void lin_recon_zone(const double *a, double *al, double *ar, const double *beta,
                           const double *Gamma, const double *x, int i)
{
  double sp, sc, sm, A, B, xm, xp, x0;
  xm = beta[i-1]/Gamma[i-1];
  xp = beta[i+1]/Gamma[i+1];
  x0 = beta[i  ]/Gamma[i  ];
  sm = (a[i  ] - a[i-1])/(x0-0.5*(x[i]+xm));
  sp = (a[i+1] - a[i  ])/(0.5*(x[i+1]+xp)-x0);
  if (sm*sp <= 0.0) { al[i] = ar[i] = a[i]; return; }
  sc = (a[i+1]-a[i-1])/(xp-xm);
  A = SIGN(sc)*MIN(MIN(fabs(sm),fabs(sp)),fabs(sc));
  B = a[i] - A*beta[i]/Gamma[i];
  al[i] = A*x[i  ] + B;
  ar[i] = A*x[i+1] + B;
}

/* interp() of reconstruct.c:225-279 on a 4-zone pencil; returns pl (right state of
 * zone 1) and pr (left state of zone 2) as prim_to_fluxesN does (step.c:539-547). */
static void interp_face(const orc_t *o, double pencil[NINT][4], const double *alpha,
                        const double *beta, const double *Gamma, const double *x,
                        double *pl, double *pr)
{
  double al[4], ar[4];
  for (int v=0; v<NINT; v++) {
    for (int i=1; i<=2; i++) {
      if (o->interp_order == 3) para_recon_zone(pencil[v], al, ar, alpha, beta, Gamma, x, i);
      else if (o->interp_order == 2) lin_recon_zone(pencil[v], al, ar, beta, Gamma, x, i);
      else { al[i] = ar[i] = pencil[v][i]; }
    }
    pl[v] = ar[1];
    pr[v] = al[2];
  }
}

/* ------------------------------------------------------------------ Riemann */
typedef struct { double area, scale_dd, gcov[3]; } face_geom;

/* riemann.c:4-37 */
static void p_uflux(const double *p, const face_geom *g, double press, int dir, double *u, double *f)
{
  double vcov[3], vsq, etot, v = p[U1+dir];
  int dd;
  for (dd=0; dd<3; dd++) vcov[dd] = g->gcov[dd]*p[U1+dd];
  u[RHO] = p[RHO];
  vsq = 0.0;
  for (dd=0; dd<3; dd++) vsq += p[U1+dd]*vcov[dd];
  etot = 0.5*u[RHO]*vsq + p[UU];
  u[UU] = etot;
  for (dd=0; dd<3; dd++) u[U1+dd] = u[RHO]*vcov[dd];
  f[RHO] = u[RHO]*v;
  f[UU] = v*(etot + press);
  for (dd=0; dd<3; dd++) f[U1+dd] = f[RHO]*vcov[dd];
  f[U1+dir] += press;
}

/* riemann.c:39-62 */
static void pflux(const double *p, double press, const face_geom *g, int dir, double *f)
{
  double vcov[3], vsq, etot, v = p[U1+dir], area = g->area;
  int dd;
  for (dd=0; dd<3; dd++) vcov[dd] = g->gcov[dd]*p[U1+dd];
  f[RHO] = area*p[RHO]*v;
  for (dd=0; dd<3; dd++) f[U1+dd] = f[RHO]*vcov[dd];
  f[U1+dir] += area*press;
  vsq = 0.0;
  for (dd=0; dd<3; dd++) vsq += p[U1+dd]*vcov[dd];
  etot = 0.5*p[RHO]*vsq + p[UU];
  f[UU] = area*v*(etot + press);
}

/* wave-speed estimate shared by HLLC and HLLE: riemann.c:368-429 (= 210-303) */
static void wave_speeds(const double *pl, const double *pr, double u_l, double u_r, int hlle,
                        double *sl_o, double *sr_o, double *ss_o, double *ps_o, int *isshock)
{
  double p_l = pl[5], p_r = pr[5], Gamma_l = pl[6], Gamma_r = pr[6];
  double cs_l, cs_r, p_max, p_min, pratio, p_s, q_l, q_r, sl, sr, ss;
  cs_l = sqrt(Gamma_l*p_l/pl[RHO]);
  cs_r = sqrt(Gamma_r*p_r/pr[RHO]);
  if (p_l > p_r) { p_max = p_l; p_min = p_r; } else { p_max = p_r; p_min = p_l; }
  pratio = p_max/p_min;
  *isshock = ((p_max-p_min)/p_min > 0.5) ? 1 : 0;
  p_s = 0.5*(p_l + p_r) - 0.125*(u_r-u_l)*(pl[RHO]+pr[RHO])*(cs_l+cs_r);
  /* HLLC clamps with MAX(0,p_s) (riemann.c:386), HLLE with MAX(p_s,0.0) (riemann.c:226):
   * they differ only for a NaN p_s */
  if (hlle) p_s = MAX(p_s, 0.0); else p_s = MAX(0,p_s);
  if (pratio < 2.0 && p_s >= p_min && p_s <= p_max) {
    /* PVRS estimate kept */
  } else if (p_s < p_min) {
    double Gamma_avg = 0.5*(Gamma_l + Gamma_r);
    double plr = pow(p_l/p_r, (Gamma_avg-1.0)/(2.0*Gamma_avg));
    ss = (plr*u_l/cs_l + u_r/cs_r + 2.0*(plr - 1.0)/(Gamma_avg - 1.0))/(plr/cs_l + 1.0/cs_r);
    p_s = 0.5*(p_l*pow(1.0 + (Gamma_l-1.0)/(2.0*cs_l)*(u_l - ss),2.0*Gamma_l/(Gamma_l-1.0)) + p_r*pow(1.0 + (Gamma_r-1.0)/(2.0*cs_r)*(ss - u_r),2.0*Gamma_r/(Gamma_r-1.0)));
    p_s = MAX(p_s, 0.0);
  } else {
    double a_l = 2.0/((Gamma_l+1.0)*pl[RHO]);
    double a_r = 2.0/((Gamma_r+1.0)*pr[RHO]);
    double b_l = (Gamma_l-1.0)/(Gamma_l+1.0)*p_l;
    double b_r = (Gamma_r-1.0)/(Gamma_r+1.0)*p_r;
    double g_l = sqrt(a_l/(p_s + b_l));
    double g_r = sqrt(a_r/(p_s + b_r));
    p_s = (g_l*p_l + g_r*p_r - (u_r-u_l))/(g_l + g_r);
    p_s = MAX(p_s, 0.0);
  }
  q_l = (p_s <= p_l) ? 1.0 : sqrt(1.0 + (Gamma_l+1.0)/(2.0*Gamma_l)*(p_s/p_l - 1.0));
  q_r = (p_s <= p_r) ? 1.0 : sqrt(1.0 + (Gamma_r+1.0)/(2.0*Gamma_r)*(p_s/p_r - 1.0));
  sl = u_l - cs_l*q_l;
  sr = u_r + cs_r*q_r;
  ss = (p_r - p_l + pl[RHO]*u_l*(sl - u_l) - pr[RHO]*u_r*(sr - u_r))/(pl[RHO]*(sl - u_l) - pr[RHO]*(sr - u_r));
  *sl_o = sl; *sr_o = sr; *ss_o = ss; *ps_o = p_s;
}

/* riemann.c:328-499 */
static int riemann_hllc(const double *pl, const double *pr, const face_geom *g, int dir,
                        double *flux, double *sig_speed)
{
  double u_l, u_r, sl, sr, ss, p_s, slr, vcov[3], vsq, u[NPRIM], fx[NPRIM], Us[NPRIM];
  double p_l = pl[5], p_r = pr[5], area = g->area, sc = g->scale_dd;
  int isshock = 0, dd, vv;
  if (area < 1.0e-16) {
    *sig_speed = 1.0e-200;
    for (vv=0; vv<NPRIM; vv++) flux[vv] = 0.0;
    return isshock;
  }
  u_l = pl[U1+dir]*sc;
  u_r = pr[U1+dir]*sc;
  wave_speeds(pl, pr, u_l, u_r, 0, &sl, &sr, &ss, &p_s, &isshock);
  if (ss > sr) sr = 1.001*ss;
  if (ss < sl) sl = 1.001*ss;
  *sig_speed = MAX(fabs(sl),fabs(sr))/sc;
  if (sl > 0.0) { pflux(pl, p_l, g, dir, flux); return isshock; }
  else if (sr < 0.0) { pflux(pr, p_r, g, dir, flux); return isshock; }
  if (ss > 0.0) {
    p_uflux(pl, g, p_l, dir, u, fx);
    Us[0] = pl[RHO]*(sl - u_l)/(sl - ss);
    Us[UU] = (u[UU]*(sl - u_l) - p_l*u_l + p_s*ss)/(sl - ss);
    for (dd=0; dd<3; dd++) Us[U1+dd] = pl[U1+dd];
    Us[U1+dir] = ss/sc;
    slr = sl/sc;
  } else {
    p_uflux(pr, g, p_r, dir, u, fx);
    Us[0] = pr[RHO]*(sr - u_r)/(sr - ss);
    Us[UU] = (u[UU]*(u_r - sr) + p_r*u_r - p_s*ss)/(ss - sr);
    for (dd=0; dd<3; dd++) Us[U1+dd] = pr[U1+dd];
    Us[U1+dir] = ss/sc;
    slr = sr/sc;
  }
  for (dd=0; dd<3; dd++) vcov[dd] = g->gcov[dd]*Us[U1+dd];
  vsq = 0.0;
  for (dd=0; dd<3; dd++) { vsq += Us[U1+dd]*vcov[dd]; Us[U1+dd] = vcov[dd]*Us[0]; }
  for (vv=0; vv<NPRIM; vv++) flux[vv] = area*(fx[vv] + slr*(Us[vv] - u[vv]));
  return isshock;
}

/* riemann.c:178-325 */
static void riemann_hlle(const double *pl, const double *pr, const face_geom *g, int dir,
                         double *flux, double *sig_speed)
{
  double u_l, u_r, sl, sr, ss, p_s, ul[NPRIM], ur[NPRIM], fl[NPRIM], fr[NPRIM];
  double cmax, cmin, area = g->area, sc = g->scale_dd;
  int isshock, vv;
  if (area < 1.0e-16) {
    *sig_speed = 1.0e-200;
    for (vv=0; vv<NPRIM; vv++) flux[vv] = 0.0;
    return;
  }
  u_l = pl[U1+dir]*sc;
  u_r = pr[U1+dir]*sc;
  wave_speeds(pl, pr, u_l, u_r, 1, &sl, &sr, &ss, &p_s, &isshock);
  p_uflux(pl, g, pl[5], dir, ul, fl);
  p_uflux(pr, g, pr[5], dir, ur, fr);
  cmax = MAX(sr/sc, 0.0);
  cmin = fabs(MIN(sl/sc, 0.0));
  *sig_speed = MAX(cmax,cmin);
  for (vv=0; vv<NPRIM; vv++)
    flux[vv] = area*(cmin*fr[vv] + cmax*fl[vv] - cmax*cmin*(ur[vv]-ul[vv]))/(cmax+cmin);
}

static void face_geom_at(const orc_t *o, int c, int dir, face_geom *fg)
{
  const orc_geom *g = &o->g[c];
  fg->area = g->area[dir];
  fg->scale_dd = g->scale[1+dir][dir];
  for (int d=0; d<3; d++) fg->gcov[d] = g->gcov[1+dir][d];
}

/* ------------------------------------------------------------------ fluxes */
static void gather_cell(const orc_t *o, double *const *p, int c, double *out)
{
  for (int v=0; v<NPRIM; v++) out[v] = p[v][c];
  out[5] = o->eos[PRESS][c];
  out[6] = o->eos[GAMMA][c];
}

/* 2-D prolongate0 (step.c:579-628) for a Cartesian grid: the level-0 coordinate of the
 * prolongation point coincides with the coarse zone centre, so this returns
 * p + sg*(x1p-x11) with x1p-x11 == 0 exactly. */
static void prolongate0_2d(const orc_t *o, double *const *p, int ii, int jj, double *pp)
{
  double x1p = o->beta1[jj+NG]/o->Gamma1[jj+NG];
  double x10 = o->beta1[jj-1+NG]/o->Gamma1[jj-1+NG];
  double x11 = o->beta1[jj+NG]/o->Gamma1[jj+NG];
  double x12 = o->beta1[jj+1+NG]/o->Gamma1[jj+1+NG];
  double idx1m = 1.0/(x11-x10), idx1p = 1.0/(x12-x11), idx1c = 1.0/(x12-x10);
  double a0[NINT], a1[NINT], a2[NINT];
  gather_cell(o, p, C(o,ii,jj-1), a0);
  gather_cell(o, p, C(o,ii,jj), a1);
  gather_cell(o, p, C(o,ii,jj+1), a2);
  for (int v=0; v<NINT; v++) {
    double sm = (a1[v] - a0[v])*idx1m;
    double sp = (a2[v] - a1[v])*idx1p;
    double sc = (a2[v] - a0[v])*idx1c;
    double sg = MINMOD(2.0*MINMOD(sm,sp),sc);
    pp[v] = a1[v] + sg*(x1p-x11);
  }
}

static void compute_fluxes(orc_t *o, double *const *p, int stage, unsigned char *mark0)
{
  const orc_params *P = &o->prm;
  double pencil[NINT][4], al[4], be[4], Ga[4], xx[4], pl[NINT], pr[NINT], flux[NPRIM], ss;
  face_geom fg;
  int i, j, v, k;
  if (o->ndim == 1) {
    /* step.c:501-562 */
    for (i=0; i<=o->n1; i++) {
      for (k=0; k<4; k++) {
        int ii = i-NG+k;
        al[k] = o->alpha0[ii+NG]; be[k] = o->beta0[ii+NG]; Ga[k] = o->Gamma0[ii+NG];
        xx[k] = P->startx[0] + ii*P->dx[0];
        double cv[NINT]; gather_cell(o, p, C(o,ii,0), cv);
        for (v=0; v<NINT; v++) pencil[v][k] = cv[v];
      }
      interp_face(o, pencil, al, be, Ga, xx, pl, pr);
      face_geom_at(o, C(o,i,0), 0, &fg);
      riemann_hllc(pl, pr, &fg, 0, flux, &ss);
      for (v=0; v<NPRIM; v++) o->f0[v][C(o,i,0)] = flux[v];
      o->min_dt = MIN(o->min_dt, P->dx[0]/fabs(ss));
    }
    return;
  }
  /* 2-D, step.c:676-760: cells in the reference's collapsed order (interior i-major,
   * then ghosts i-major); each cell does its 0-face and then its 1-face. */
  for (int pass=0; pass<2; pass++) {
    for (i=-NG; i<o->n1+NG; i++) {
      for (j=-NG; j<o->n2+NG; j++) {
        if (is_interior(o,i,j) != (pass == 0)) continue;
        int c = C(o,i,j);
        if (i >= 0 && i <= o->n1 && j >= 0 && j < o->n2) {
          for (k=0; k<4; k++) {
            int ii = i-NG+k;
            al[k] = o->alpha0[ii+NG]; be[k] = o->beta0[ii+NG]; Ga[k] = o->Gamma0[ii+NG];
            xx[k] = P->startx[0] + ii*P->dx[0];
            double pp[NINT]; prolongate0_2d(o, p, ii, j, pp);
            for (v=0; v<NINT; v++) pencil[v][k] = pp[v];
          }
          interp_face(o, pencil, al, be, Ga, xx, pl, pr);
          face_geom_at(o, c, 0, &fg);
          int isshock = riemann_hllc(pl, pr, &fg, 0, flux, &ss);
          for (v=0; v<NPRIM; v++) o->f0[v][c] = flux[v];
          if (isshock) {
            o->flag[c] = 0;
            o->flag[C(o,i-1,j)] = 0;
            o->flag[C(o,i-2,j)] = 0;
            if (mark0) mark0[c] = 1;
          }
          o->min_dt = MIN(o->min_dt, P->dx[0]/fabs(ss));
        }
        if (i >= 0 && i < o->n1 && j >= 0 && j <= o->n2) {
          for (k=0; k<4; k++) {
            int jj = j-NG+k;
            al[k] = o->alpha1[jj+NG]; be[k] = o->beta1[jj+NG]; Ga[k] = o->Gamma1[jj+NG];
            xx[k] = P->startx[1] + jj*1*P->dx[1];
            double cv[NINT]; gather_cell(o, p, C(o,i,jj), cv);
            for (v=0; v<NINT; v++) pencil[v][k] = cv[v];
          }
          interp_face(o, pencil, al, be, Ga, xx, pl, pr);
          face_geom_at(o, c, 1, &fg);
          /* transverse_shock, fluid.c:189-210 (dir 1, no k refinement) */
          int ts = (o->flag[c] == 0) || (o->flag[C(o,i,j-1)] == 0);
          if (ts) riemann_hlle(pl, pr, &fg, 1, flux, &ss);
          else riemann_hllc(pl, pr, &fg, 1, flux, &ss);
          for (v=0; v<NPRIM; v++) o->f1[v][c] = flux[v];
          o->min_dt = MIN(o->min_dt, 1*P->dx[1]/fabs(ss));
        }
      }
    }
  }
  (void)stage;
}

/* ------------------------------------------------------------------ sources, push */
/* fluid.c:56-73 + rad_fluid.c:164-192 */
static void geom_src(const orc_t *o, double *const *p)
{
  for (int i=0; i<o->n1; i++) {
    int jh = (o->ndim > 1) ? o->n2 : 1;
    for (int j=0; j<jh; j++) {
      int c = C(o,i,j), v, l, m, n;
      for (v=0; v<NPRIM; v++) o->src[v][c] = 0;
      const orc_geom *g = &o->g[c];
      if (o->geom == 1) {
        double T[3][3], vcov[3];
        for (l=0; l<3; l++) vcov[l] = g->gcov[0][l]*p[U1+l][c];
        for (l=0; l<3; l++) {
          for (m=0; m<3; m++) T[l][m] = p[RHO][c]*p[U1+m][c]*vcov[l];
          T[l][l] += o->eos[PRESS][c];
        }
        for (l=0; l<3; l++) for (m=0; m<3; m++) for (n=0; n<3; n++)
          o->src[U1+m][c] += T[l][n]*g->conn[l][m][n];
      }
      if (o->grav_on) {
        /* fixed_gravity (gravity.c:38-64): g0 is contravariant; geom_dot (geometry.c:65-73) */
        double vsq = 0.0;
        for (l=0; l<3; l++) vsq += p[U1+l][c]*o->prm.grav[l]*g->gcov[0][l];
        o->src[UU][c] += p[RHO][c]*vsq;
        for (l=0; l<o->ndim; l++) o->src[U1+l][c] += p[RHO][c]*o->prm.grav[l]*g->gcov[0][l];
      }
    }
  }
}

/* fluid.c:4-24 */
static void p_to_u(const double *pv, double *u, const double *gcov)
{
  double vcov[3], vsq = 0.0;
  int dd;
  for (dd=0; dd<3; dd++) vcov[dd] = gcov[dd]*pv[U1+dd];
  u[RHO] = pv[RHO];
  for (dd=0; dd<3; dd++) { vsq += pv[dd+U1]*vcov[dd]; u[dd+U1] = u[RHO]*vcov[dd]; }
  u[UU] = 0.5*u[RHO]*vsq + pv[UU];
}

/* fluid.c:27-53; the floors of fluid.c:43-46 when the ENFORCE_FLOORS switch is on */
static void u_to_p(double *u, double *pv, const double *gcon, const orc_params *P)
{
  double vsq = 0.0;
  int dd;
  pv[RHO] = u[RHO];
  for (dd=U1; dd<U1+3; dd++) u[dd] /= u[RHO];
  for (dd=0; dd<3; dd++) pv[U1+dd] = gcon[dd]*u[U1+dd];
  for (dd=0; dd<3; dd++) vsq += u[U1+dd]*pv[U1+dd];
  pv[UU] = u[UU] - 0.5*pv[RHO]*vsq;
  if (P->enforce_floors) {
    pv[RHO] = MAX(pv[RHO], P->rho_floor);
    pv[UU] = MAX(pv[UU], P->e_floor);
  }
}

/* step.c:205-223 */
static double dt_source_control(const double *pv, const double *u, const double *s)
{
  const double alpha = 0.02;
  double local_dt, momterm = 0.0, mdt = 1.0e100;
  local_dt = alpha*u[0]/(fabs(s[0])+1.0e-16);
  mdt = MIN(mdt,local_dt);
  local_dt = alpha*u[1]/(fabs(s[1])+1.0e-16);
  mdt = MIN(mdt,local_dt);
  for (int dd=0; dd<3; dd++) momterm += pv[U1+dd]*s[U1+dd];
  local_dt = 100*alpha*pv[UU]/(fabs(fabs(s[1])-fabs(momterm)) + 1.0e-16);
  mdt = MIN(mdt,local_dt);
  return mdt;
}

/* step.c:327-478 */
static void push(orc_t *o, double dtpush, double *const *p, double *const *ph, double **pf, int stage)
{
  double pfact = (stage == 0) ? 1 : 0.5, phfact = (stage == 0) ? 0 : 0.5, ffact = (stage == 0) ? 1 : 0.5;
  double min_dt_src = 1.0e100;
  for (int i=0; i<o->n1; i++) {
    int jh = (o->ndim > 1) ? o->n2 : 1;
    for (int j=0; j<jh; j++) {
      int c = C(o,i,j), v;
      const orc_geom *g = &o->g[c];
      double pv[NPRIM], phv[NPRIM], u[NPRIM], uh[NPRIM], s[NPRIM], divF[NPRIM], out[NPRIM];
      for (v=0; v<NPRIM; v++) { pv[v] = p[v][c]; phv[v] = ph[v][c]; s[v] = o->src[v][c]; }
      p_to_u(pv, u, g->gcov[0]);
      p_to_u(phv, uh, g->gcov[0]);
      double local_dt = dt_source_control(pv, u, s);
      min_dt_src = MIN(min_dt_src, local_dt);
      for (v=0; v<NPRIM; v++) divF[v] = 0.0;
      for (v=0; v<NPRIM; v++) divF[v] += o->f0[v][C(o,i+1,j)];
      for (v=0; v<NPRIM; v++) divF[v] -= o->f0[v][c];
      if (o->ndim > 1) {
        for (v=0; v<NPRIM; v++) divF[v] += o->f1[v][C(o,i,j+1)];
        for (v=0; v<NPRIM; v++) divF[v] -= o->f1[v][c];
      }
      for (v=0; v<NPRIM; v++) {
        double ddt = divF[v]/g->volume - s[v];
        u[v] = pfact*u[v] + phfact*uh[v] - ffact*dtpush * ddt;
      }
      u_to_p(u, out, g->gcon, &o->prm);
      for (v=0; v<NPRIM; v++) pf[v][c] = out[v];
    }
  }
  o->min_dt = MIN(o->min_dt, min_dt_src);
}

/* ------------------------------------------------------------------ step, dt */
static void set_shock_flag0(orc_t *o)
{
  for (int i=0; i<o->n1; i++) {
    int jh = (o->ndim > 1) ? o->n2 : 1;
    for (int j=0; j<jh; j++) o->flag[C(o,i,j)] = -1;
  }
}

/* step.c:28-129 */
void orc_step(orc_t *o, double dtin)
{
  use_map(o);
  o->dt = dtin;
  o->min_dt = 1.0e100;
  set_shock_flag0(o);
  reset_boundaries(o, o->p, 0);
  update_eos(o, o->p, 0);
  geom_src(o, o->p);
  update_eos(o, o->p, 1);
  compute_fluxes(o, o->p, 0, NULL);
  push(o, o->dt, o->p, o->p, o->ph, 0);
  reset_boundaries(o, o->ph, 1);
  update_eos(o, o->ph, 0);
  geom_src(o, o->ph);
  update_eos(o, o->ph, 1);
  compute_fluxes(o, o->ph, 1, NULL);
  push(o, o->dt, o->p, o->ph, o->p, 1);
  o->t += o->dt;
  o->istep++;
}

/* step.c:163-203 */
double orc_estimate_dt(orc_t *o)
{
  use_map(o);
  const orc_params *P = &o->prm;
  if (o->est_first) { o->min_dt = 1.0e100; o->est_first = 0; }
  for (int i=0; i<o->n1; i++) {
    int jh = (o->ndim > 1) ? o->n2 : 1;
    for (int j=0; j<jh; j++) {
      int c = C(o,i,j);
      double local_dt = 0.0;
      for (int dd=0; dd<o->ndim; dd++) {
        double local_dx = P->dx[dd];
        if (dd==1) local_dx *= 1;
        local_dt += (fabs(o->p[U1+dd][c]) + o->eos[CS][c]/o->g[c].scale[0][dd])/local_dx;
        o->min_dt = MIN(o->min_dt, 1.0/local_dt);
      }
    }
  }
  if (o->istep == 0) o->min_dt = MIN(o->min_dt, P->initial_dt);
  o->min_dt = MIN(o->min_dt, P->dtmax);
  o->min_dt *= P->cfl;
  o->dt = o->min_dt;
  return o->dt;
}

/* main.c:226-264 */
double orc_advance_one(orc_t *o)
{
  const orc_params *P = &o->prm;
  double dt = orc_estimate_dt(o);
  if (o->istep == 0) dt *= P->dt_init_safety;
  else dt = MIN(o->dtold*P->dt_grow_safety, dt);
  o->dtold = dt;
  if (o->t + 1*dt > P->tmax) dt = 1.000000001*(P->tmax - o->t)/1;
  if (dt < P->dtmin) dt = P->dtmin;
  orc_step(o, dt);
  return dt;
}

/* ------------------------------------------------------------------ lifecycle */
orc_t *orc_create(const orc_params *prm, int ndim, int geom, const double *ic)
{
  /* maps the oracle does not restate are refused, not approximated */
  if (prm->rcoord < RC_UNIFORM || prm->rcoord > RC_LOG || prm->thcoord < TH_UNIFORM || prm->thcoord > TH_POLYTH)
    return NULL;
  if (geom == 0 && (prm->rcoord != RC_UNIFORM || prm->thcoord != TH_UNIFORM)) return NULL;
  orc_t *o = calloc(1, sizeof *o);
  int v;
  o->prm = *prm;
  o->ndim = ndim;
  o->geom = geom;
  o->n1 = prm->n1;
  o->n2 = (ndim > 1) ? prm->n2 : 1;
  o->s1 = o->n1 + 2*NG;
  o->s2 = (ndim > 1) ? o->n2 + 2*NG : 1;
  o->ncell = o->s1*o->s2;
  for (v=0; v<NPRIM; v++) {
    o->p[v] = calloc(o->ncell, sizeof(double));
    o->ph[v] = calloc(o->ncell, sizeof(double));
    o->src[v] = calloc(o->ncell, sizeof(double));
    o->f0[v] = calloc(o->ncell, sizeof(double));
    o->f1[v] = calloc(o->ncell, sizeof(double));
  }
  for (v=0; v<5; v++) o->eos[v] = calloc(o->ncell, sizeof(double));
  o->flag = calloc(o->ncell, sizeof(int));
  o->g = calloc(o->ncell, sizeof(orc_geom));
  o->alpha0 = calloc(o->s1, sizeof(double));
  o->beta0 = calloc(o->s1, sizeof(double));
  o->Gamma0 = calloc(o->s1, sizeof(double));
  o->alpha1 = calloc(o->n2 + 2*NG, sizeof(double));
  o->beta1 = calloc(o->n2 + 2*NG, sizeof(double));
  o->Gamma1 = calloc(o->n2 + 2*NG, sizeof(double));
  o->interp_order = prm->hydro_interp_order;
  o->grav_on = (prm->grav[0] != 0.0 || prm->grav[1] != 0.0 || prm->grav[2] != 0.0);
  o->est_first = 1;
  o->dtold = 1.0e100;
  use_map(o);
  init_geometry(o);
  int cidx = 0;
  for (int i=0; i<o->n1; i++) for (int j=0; j<o->n2; j++) {
    for (v=0; v<NPRIM; v++) o->p[v][C(o,i,j)] = ic[NPRIM*cidx+v];
    cidx++;
  }
  update_eos(o, o->p, 0);   /* main.c:180-182 */
  return o;
}

void orc_destroy(orc_t *o)
{
  if (!o) return;
  for (int v=0; v<NPRIM; v++) { free(o->p[v]); free(o->ph[v]); free(o->src[v]); free(o->f0[v]); free(o->f1[v]); }
  for (int v=0; v<5; v++) free(o->eos[v]);
  free(o->flag); free(o->g); free(o->alpha0); free(o->beta0); free(o->Gamma0);
  free(o->alpha1); free(o->beta1); free(o->Gamma1);
  free(o);
}

double orc_get_t(const orc_t *o) { return o->t; }
double orc_get_min_dt(const orc_t *o) { return o->min_dt; }
int orc_get_istep(const orc_t *o) { return o->istep; }
int orc_cell_count(const orc_t *o) { return o->n1*o->n2; }

void orc_get_interior(const orc_t *o, double *prim, double *eos)
{
  int cidx = 0;
  for (int i=0; i<o->n1; i++) for (int j=0; j<o->n2; j++) {
    int c = C(o,i,j);
    for (int v=0; v<NPRIM; v++) prim[NPRIM*cidx+v] = o->p[v][c];
    if (eos) for (int v=0; v<5; v++) eos[5*cidx+v] = o->eos[v][c];
    cidx++;
  }
}

void orc_set_interior(orc_t *o, const double *prim)
{
  int cidx = 0;
  for (int i=0; i<o->n1; i++) for (int j=0; j<o->n2; j++) {
    for (int v=0; v<NPRIM; v++) o->p[v][C(o,i,j)] = prim[NPRIM*cidx+v];
    cidx++;
  }
}

/* A run resumed from a restart file (io.c restart_read_v2: the state, Time and Step) in a
 * new process: the EOS records of the state (main.c:180-182), dtold = 1e100 (main.c:194)
 * and estimate_dt's first-call reset of min_dt (step.c:171-174). */
void orc_restart(orc_t *o, const double *prim, double t, int istep)
{
  orc_set_interior(o, prim);
  update_eos(o, o->p, 0);
  o->t = t;
  o->istep = istep;
  o->dtold = 1.0e100;
  o->est_first = 1;
}

void orc_get_moments0(const orc_t *o, double *a, double *b, double *g)
{
  for (int i=0; i<o->s1; i++) { a[i] = o->alpha0[i]; b[i] = o->beta0[i]; g[i] = o->Gamma0[i]; }
}

/* volume, area[ndim], gcov[0..ndim][3], gcon[3], scale[0..ndim][3], conn[27] of cell (i,j) */
int orc_get_geom(const orc_t *o, int i, int j, double *out)
{
  const orc_geom *g = &o->g[C(o,i,j)];
  int c = 0, d, l, m, n;
  out[c++] = g->volume;
  for (d=0; d<o->ndim; d++) out[c++] = g->area[d];
  for (l=0; l<=o->ndim; l++) for (m=0; m<3; m++) out[c++] = g->gcov[l][m];
  for (m=0; m<3; m++) out[c++] = g->gcon[m];
  for (l=0; l<=o->ndim; l++) for (m=0; m<3; m++) out[c++] = g->scale[l][m];
  for (l=0; l<3; l++) for (m=0; m<3; m++) for (n=0; n<3; n++) out[c++] = g->conn[l][m][n];
  return c;
}
