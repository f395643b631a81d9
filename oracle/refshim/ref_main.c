/*
 * TEST INFRASTRUCTURE ONLY.
 *
 * Command-line driver around ref_harness.c.  One process runs one problem, because
 * the reference keeps its whole state in globals and function-local statics
 * (estimate_dt's firstc, step.c:165).
 *
 *   ref_<cfg> run   <input.bin> <output.bin> <nsteps> <snap_every>
 *       input : ref_params (raw struct) followed by the interior primitives
 *       output: for the initial state and every snap_every-th step:
 *               [istep, t, dt_used, min_dt] + interior prims [ncell][5] (all double)
 *   ref_<cfg> time  <input.bin> <warmup> <steps>
 *       prints one line: "zone_updates_per_s=<v> seconds=<s> steps=<n> cells=<c>"; a
 *       DO_TIMING=TRUE build (reftime_<cfg>) also writes the reference's timers of the
 *       timed steps to timing.csv in the working directory
 *   ref_<cfg> grid  <input.bin> <output.bin>
 *       output: int32 nj[n1+2NG], then int32 nk for every row (i, j) of ref_get_grid
 *   ref_<cfg> geom  <input.bin> <output.bin>
 *       output: for every row (i, j) of ref_get_grid, the ref_get_geom record of zone
 *       (i, j, 0), 64 doubles each (unused tail zero)
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

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
  int rcoord;
  double rfact[3];
  int thcoord;
  double poly_xt, poly_alpha;
} ref_params;

int ref_init(const ref_params *prm, const double *ic);
double ref_advance_one(void);
double ref_get_t(void);
double ref_get_min_dt(void);
void ref_timers_reset(void);
void ref_timers_write(void);
int ref_get_istep(void);
int ref_cell_count(void);
void ref_get_interior(double *prim, double *eos);
int ref_get_grid(int *nj, int *nk);
int ref_get_geom(int i, int j, int k, double *out);

static void *read_all(const char *path, size_t *len)
{
  FILE *f = fopen(path, "rb");
  if (!f) { perror(path); exit(2); }
  fseek(f, 0, SEEK_END);
  long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  void *buf = malloc((size_t)n);
  if (fread(buf, 1, (size_t)n, f) != (size_t)n) { fprintf(stderr, "short read\n"); exit(2); }
  fclose(f);
  *len = (size_t)n;
  return buf;
}

static double now_s(void)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9*ts.tv_nsec;
}

int main(int argc, char **argv)
{
  if (argc < 3) { fprintf(stderr, "usage: %s run|time ...\n", argv[0]); return 2; }
  size_t len;
  char *buf = read_all(argv[2], &len);
  ref_params prm;
  memcpy(&prm, buf, sizeof prm);
  const double *ic = (const double *)(buf + sizeof prm);

  if (ref_init(&prm, ic) < 0) return 2;
  int ncell = ref_cell_count();
  double *prim = malloc(sizeof(double)*5*ncell);
  double *eos = malloc(sizeof(double)*5*ncell);

  if (strcmp(argv[1], "run") == 0) {
    if (argc < 6) return 2;
    FILE *out = fopen(argv[3], "wb");
    int nsteps = atoi(argv[4]);
    int every = atoi(argv[5]);
    double hdr[4];
    hdr[0] = 0; hdr[1] = ref_get_t(); hdr[2] = 0; hdr[3] = 0;
    ref_get_interior(prim, eos);
    fwrite(hdr, sizeof(double), 4, out);
    fwrite(prim, sizeof(double), 5*(size_t)ncell, out);
    for (int s=1; s<=nsteps; s++) {
      double dtu = ref_advance_one();
      if (s % every == 0 || s == nsteps) {
        hdr[0] = ref_get_istep(); hdr[1] = ref_get_t(); hdr[2] = dtu; hdr[3] = ref_get_min_dt();
        ref_get_interior(prim, eos);
        fwrite(hdr, sizeof(double), 4, out);
        fwrite(prim, sizeof(double), 5*(size_t)ncell, out);
      }
    }
    fclose(out);
  } else if (strcmp(argv[1], "time") == 0) {
    if (argc < 5) return 2;
    int warm = atoi(argv[3]);
    int steps = atoi(argv[4]);
    for (int s=0; s<warm; s++) ref_advance_one();
    ref_timers_reset();
    double t0 = now_s();
    for (int s=0; s<steps; s++) ref_advance_one();
    double el = now_s() - t0;
    ref_timers_write();
    printf("zone_updates_per_s=%.6e seconds=%.6f steps=%d cells=%d\n",
           (double)ncell*steps/el, el, steps, ncell);
  } else if (strcmp(argv[1], "grid") == 0 || strcmp(argv[1], "geom") == 0) {
    if (argc < 4) return 2;
    int n1 = prm.n1;
    int nrow = ref_get_grid(NULL, NULL);
    int *nj = malloc(sizeof(int)*(n1+4));
    int *nk = malloc(sizeof(int)*(size_t)nrow);
    ref_get_grid(nj, nk);
    FILE *out = fopen(argv[3], "wb");
    if (argv[1][1] == 'r') {
      fwrite(nj, sizeof(int), (size_t)(n1+4), out);
      fwrite(nk, sizeof(int), (size_t)nrow, out);
    } else {
      double rec[64];
      for (int i=-2; i<n1+2; i++) {
        for (int j=-2; j<nj[i+2]+2; j++) {
          memset(rec, 0, sizeof rec);
          ref_get_geom(i, j, 0, rec);
          fwrite(rec, sizeof(double), 64, out);
        }
      }
    }
    fclose(out);
  } else {
    return 2;
  }
  return 0;
}
