/*
 * TEST INFRASTRUCTURE ONLY -- never linked into, called by, or shipped with the
 * medusa_b200 product path.
 *
 * Runs the UNMODIFIED reference zone update of the tabulated EOS,
 * eos_given_rex_per_zone (eos/burrows/eos_stuff.c:768-902, compiled from the reference
 * tree by oracle/build_ref.py), on a table and zones read from files:
 *
 *   refeos <table.bin> <zones.bin> <out.bin>
 *     table.bin: 16 x 50 x 300 x 300 doubles (TAB_ELEM's layout and the sizes of
 *                DEFINE_EOSCONST_1, eos_stuff.c:7-21)
 *     zones.bin: int64 n, then n x (rho, u, Ye, temperature guess) doubles
 *     out.bin  : n x (pressure, sound speed, temperature, entropy, Gamma_1) doubles
 *   prints "seconds=<s> zones=<n>": the time of the zone loop alone (one core)
 *
 * The state and EOS records of a zone are passed as the reference's own arrays would
 * hold them (p[RHO], p[UU], p[YE]; eos[TEMP] the guess).  The globals that the rest of
 * eos_stuff.c references come from defs.h.
 */
#include "decs.h"
#include "defs.h"
#include "eos/burrows/eos_stuff.h"
#include <time.h>

#define TABLE_SIZE (16L * 50L * 300L * 300L)
#define NVAR_MAX_HARNESS 16   /* room for every primitive index the zone update reads (RHO, UU, YE) */

static void *read_file(const char *path, long *len)
{
  FILE *f = fopen(path, "rb");
  if (!f) { perror(path); exit(2); }
  fseek(f, 0, SEEK_END);
  long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  void *buf = malloc((size_t)n);
  if (fread(buf, 1, (size_t)n, f) != (size_t)n) { fprintf(stderr, "short read %s\n", path); exit(2); }
  fclose(f);
  *len = n;
  return buf;
}

int main(int argc, char **argv)
{
  if (argc < 4) { fprintf(stderr, "usage: %s table.bin zones.bin out.bin\n", argv[0]); return 2; }
  long tlen = 0, zlen = 0;
  double *table = read_file(argv[1], &tlen);
  if (tlen != TABLE_SIZE * (long)sizeof(double)) { fprintf(stderr, "table size %ld\n", tlen); return 2; }
  char *zb = read_file(argv[2], &zlen);
  long n = *(long *)zb;
  const double *z = (const double *)(zb + sizeof(long));
  double *out = malloc(sizeof(double) * 5 * (size_t)n);
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (long i = 0; i < n; i++) {
    double p[NVAR_MAX_HARNESS], eos[NEOS];
    memset(p, 0, sizeof p);
    memset(eos, 0, sizeof eos);
    p[RHO] = z[4 * i + 0];
    p[UU] = z[4 * i + 1];
    p[YE] = z[4 * i + 2];
    eos[TEMP] = z[4 * i + 3];
    eos_given_rex_per_zone(table, p, eos);
    out[5 * i + 0] = eos[PRESS];
    out[5 * i + 1] = eos[CS];
    out[5 * i + 2] = eos[TEMP];
    out[5 * i + 3] = eos[ENT];
    out[5 * i + 4] = eos[GAMMA];
  }
  clock_gettime(CLOCK_MONOTONIC, &t1);
  printf("seconds=%.6f zones=%ld\n", (t1.tv_sec - t0.tv_sec) + 1e-9 * (t1.tv_nsec - t0.tv_nsec), n);
  FILE *f = fopen(argv[3], "wb");
  if (!f || fwrite(out, sizeof(double), 5 * (size_t)n, f) != 5 * (size_t)n) { perror(argv[3]); return 2; }
  fclose(f);
  return 0;
}
