/*
 * TEST INFRASTRUCTURE ONLY -- never linked into, called by, or shipped with the
 * medusa_b200 product path.
 *
 * CPU restatement of the tabulated (nuclear) EOS update of one zone,
 * eos_given_rex_per_zone (eos/burrows/eos_stuff.c:768-902): given density, internal
 * energy density, Ye and a temperature guess, find the temperature at which the table's
 * energy matches (scan down from the guess's row, eos_stuff.c:813-825, then up,
 * :830-842), then interpolate log pressure, entropy and Gamma_1 bilinearly in (log rho,
 * Ye) and linearly in the temperature fraction (:858-894).  The table has the layout of
 * TAB_ELEM (eos_stuff.c:7): nrec records of ny x nr x nt doubles, jt fastest; records 1
 * (energy), 2 (log pressure), 3 (entropy) and 12 (Gamma_1) are read.  The grid bounds
 * and sizes are arguments (the reference fixes them in DEFINE_EOSCONST_1,
 * eos_stuff.c:8-21), as is const_hack (0 there).  Compiled with -fno-fast-math
 * -ffp-contract=off, the operations round as in the reference's build of the same file;
 * tests/test_eos_table.py pins it against that build.
 *
 * Indices the reference would take outside the table (inputs outside its range, or a
 * temperature guess on its top row) are clamped here: jr to [1, nr], jy to [1, ny], the
 * starting jt to [1, nt - 1]; inside the table nothing differs.
 */
#include <math.h>

#define ORC_API __attribute__((visibility("default")))

typedef struct {
  int nrec, ny, nr, nt;
  double r1, r2, t1, t2, y1, y2;   /* log10 rho, log10 T (MeV) and Ye ranges */
  double const_hack;
} orc_eos_grid;

static inline double tab(const double *a, const orc_eos_grid *g, int irec, int jy, int jr, int jt)
{
  return a[(long)(irec - 1) * g->ny * g->nr * g->nt + (long)(jy - 1) * g->nr * g->nt + (long)(jr - 1) * g->nt +
           (jt - 1)];
}

/* out[0..4] = pressure, sound speed, temperature, entropy, Gamma_1 (the PRESS, CS, TEMP,
 * ENT, GAMMA slots of sim_eos); temp_guess is eos[TEMP] before the call */
ORC_API void orc_eos_given_rex(const double *table, const orc_eos_grid *g, double rho, double u, double ye,
                               double temp_guess, double *out)
{
  const int nr = g->nr, nt = g->nt, ny = g->ny;
  const double r1 = g->r1, r2 = g->r2, t1 = g->t1, t2 = g->t2, y1c = g->y1, y2c = g->y2;
  double temp_eos = temp_guess;
  const double den_eos = rho;
  double e_eos = u / den_eos;
  const double ye_eos = ye;
  if (temp_eos < 1.0e-10) temp_eos = 1.0;

  e_eos = e_eos / 0.95655684e18 - g->const_hack;
  const double rl = log10(den_eos);
  const double tl = log10(temp_eos);
  const double dr = (r2 - r1) / (nr - 1);
  const double dt = (t2 - t1) / (nt - 1);
  const double dy = (y2c - y1c) / (ny - 1);
  int jr = 1 + (int)((rl - r1) / dr);
  int jt = 1 + (int)((tl - t1) / dt);
  int jy = 1 + (int)((ye_eos - y1c) / dy);
  if (jr < 1) jr = 1;
  if (jr > nr) jr = nr;
  if (jy < 1) jy = 1;
  if (jy > ny) jy = ny;
  if (jt < 1) jt = 1;
  if (jt > nt - 1) jt = nt - 1;
  int jyp = jy + 1;
  int jrp = jr + 1;
  double drho = (rl - (r1 + (jr - 1) * dr)) / dr;
  double dye = (ye_eos - (y1c + (jy - 1) * dy)) / dy;
  if (jy == ny) {
    jyp = jy;
    dye = 0.0;
  }
  if (jr == nr) {
    jrp = jr;
    drho = 0.0;
  }
  const double coeff0 = (1.0 - drho) * (1.0 - dye);
  const double coeff1 = dye * (1.0 - drho);
  const double coeff2 = (1.0 - dye) * drho;
  const double coeff3 = dye * drho;

  /* bracket e_eos between rows jt and jt+1 of the energy record */
  double elo, ehi = -1e99;
  while (1) {
    elo = coeff0 * tab(table, g, 1, jy, jr, jt);
    elo = elo + coeff1 * tab(table, g, 1, jyp, jr, jt);
    elo = elo + coeff2 * tab(table, g, 1, jy, jrp, jt);
    elo = elo + coeff3 * tab(table, g, 1, jyp, jrp, jt);
    if (elo < e_eos || jt == 1) break;
    ehi = elo;
    jt = jt - 1;
  }
  if (ehi < -1e98) {
    while (1) {
      ehi = coeff0 * tab(table, g, 1, jy, jr, jt + 1);
      ehi = ehi + coeff1 * tab(table, g, 1, jyp, jr, jt + 1);
      ehi = ehi + coeff2 * tab(table, g, 1, jy, jrp, jt + 1);
      ehi = ehi + coeff3 * tab(table, g, 1, jyp, jrp, jt + 1);
      if (ehi > e_eos || jt == nt - 1) break;
      elo = ehi;
      jt = jt + 1;
    }
  }

  const double tlo = t1 + (jt - 1) * dt;
  const double thi = tlo + dt;
  const double dtemp = (e_eos - elo) / (ehi - elo);
  temp_eos = tlo + (thi - tlo) * dtemp;
  const int jtp = jt + 1;

  double f[3];
  const int recs[3] = {2, 3, 12};
  for (int k = 0; k < 3; k++) {
    const int irec = recs[k];
    double v = coeff0 * (1 - dtemp) * tab(table, g, irec, jy, jr, jt);
    v += coeff1 * (1 - dtemp) * tab(table, g, irec, jyp, jr, jt);
    v += coeff2 * (1 - dtemp) * tab(table, g, irec, jy, jrp, jt);
    v += coeff3 * (1 - dtemp) * tab(table, g, irec, jyp, jrp, jt);
    v += coeff0 * dtemp * tab(table, g, irec, jy, jr, jtp);
    v += coeff1 * dtemp * tab(table, g, irec, jyp, jr, jtp);
    v += coeff2 * dtemp * tab(table, g, irec, jy, jrp, jtp);
    v += coeff3 * dtemp * tab(table, g, irec, jyp, jrp, jtp);
    f[k] = v;
  }
  const double p_eos = exp(f[0]) * 1.60217733e33;   /* MeV/fm^3 -> dyn/cm^2 */
  const double s_eos = f[1];
  const double gam1_eos = f[2];
  temp_eos = pow(10, temp_eos);
  const double cs_eos = sqrt((gam1_eos) * (p_eos) / (den_eos));
  out[0] = p_eos;
  out[1] = cs_eos;
  out[2] = temp_eos;
  out[3] = s_eos;
  out[4] = gam1_eos;
}

ORC_API void orc_eos_given_rex_n(const double *table, const orc_eos_grid *g, int n, const double *rho,
                                 const double *u, const double *ye, const double *temp_guess, double *out)
{
  for (int i = 0; i < n; i++) orc_eos_given_rex(table, g, rho[i], u[i], ye[i], temp_guess[i], out + 5 * i);
}
