// Tabulated (nuclear) EOS zone update on the device: eos_given_rex_per_zone of the
// reference's production EOS (eos/burrows/eos_stuff.c:768-902), one thread per zone.
//
// Per zone: the temperature whose tabulated energy matches the zone's specific internal
// energy -- the energy record bilinear in (log10 rho, Ye), scanned down from the row of the
// zone's temperature guess and then up (eos_stuff.c:811-842), linear between the bracketing
// rows -- then log pressure, entropy and Gamma_1 interpolated with the same weights
// (:858-894), p = exp(log p) in dyn/cm^2, cs = sqrt(Gamma_1 p / rho), T = 10^log T.  The
// expressions keep the reference's operation order (this file is compiled without
// multiply-add contraction); log10, exp and pow are CUDA's, so results agree with the
// reference's to a few ulps rather than bit for bit.
//
// Table layout in HBM (built from the reference layout by mdg_eos_table_create): the four
// records the update reads interleaved per grid point as {e, log p, s, Gamma_1} (32 bytes,
// one DRAM sector), jt fastest.  The temperature scan touches one sector per corner and
// row, and the interpolation then reads the same sectors of rows jt and jt+1 again (L1/L2
// hits): with a warm temperature guess a zone moves about 8 sectors of table.  With the
// energy record stored apart and the other three records interleaved, each energy read
// took a sector of its own and the interpolation 4 more 64-byte runs: 632 B of DRAM
// traffic per zone against 72 B streamed (ncu), the kernel at 70 % of DRAM peak.
#include "mdg_hydro.cuh"
#include "mdg_kernels.cuh"

namespace mdg {

__global__ void __launch_bounds__(256)
eos_rex_kernel(EosTableDev d, long long n, const double *__restrict__ rho, const double *__restrict__ u,
               const double *__restrict__ ye, double *__restrict__ temp, double *__restrict__ press,
               double *__restrict__ cs, double *__restrict__ ent, double *__restrict__ gam1)
{
  const int nr = d.nr, nt = d.nt, ny = d.ny;
  const double r1 = d.r1, r2 = d.r2, t1 = d.t1, t2 = d.t2, y1c = d.y1, y2c = d.y2;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    double temp_eos = temp[i];
    const double den_eos = rho[i];
    double e_eos = u[i] / den_eos;
    const double ye_eos = ye[i];
    if (temp_eos < 1.0e-10) temp_eos = 1.0;

    e_eos = e_eos / 0.95655684e18 - d.const_hack;
    const double rl = log10(den_eos);
    const double tl = log10(temp_eos);
    const double dr = (r2 - r1) / (nr - 1);
    const double dt = (t2 - t1) / (nt - 1);
    const double dy = (y2c - y1c) / (ny - 1);
    int jr = 1 + (int)((rl - r1) / dr);
    int jt = 1 + (int)((tl - t1) / dt);
    int jy = 1 + (int)((ye_eos - y1c) / dy);
    // indices the reference would take outside the table are clamped (inside it nothing
    // changes: a guess on the top row brackets the same rows from one row lower)
    jr = jr < 1 ? 1 : (jr > nr ? nr : jr);
    jy = jy < 1 ? 1 : (jy > ny ? ny : jy);
    jt = jt < 1 ? 1 : (jt > nt - 1 ? nt - 1 : jt);
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
    // row offsets (jt = 1 at offset 0) of the four (Ye, rho) corners
    const long long c00 = ((long long)(jy - 1) * nr + (jr - 1)) * nt;
    const long long c10 = ((long long)(jyp - 1) * nr + (jr - 1)) * nt;
    const long long c01 = ((long long)(jy - 1) * nr + (jrp - 1)) * nt;
    const long long c11 = ((long long)(jyp - 1) * nr + (jrp - 1)) * nt;
    const double2 *f = d.f;   // grid point p: f[2p] = (e, log p), f[2p+1] = (s, Gamma_1)
    auto energy = [&](int k) {
      double e = coeff0 * __ldg(f + 2 * (c00 + k - 1)).x;
      e = e + coeff1 * __ldg(f + 2 * (c10 + k - 1)).x;
      e = e + coeff2 * __ldg(f + 2 * (c01 + k - 1)).x;
      e = e + coeff3 * __ldg(f + 2 * (c11 + k - 1)).x;
      return e;
    };

    double elo, ehi = -1e99;
    while (true) {
      elo = energy(jt);
      if (elo < e_eos || jt == 1) break;
      ehi = elo;
      jt = jt - 1;
    }
    if (ehi < -1e98) {
      while (true) {
        ehi = energy(jt + 1);
        if (ehi > e_eos || jt == nt - 1) break;
        elo = ehi;
        jt = jt + 1;
      }
    }
    const double tlo = t1 + (jt - 1) * dt;
    const double thi = tlo + dt;
    const double dtemp = (e_eos - elo) / (ehi - elo);
    temp_eos = tlo + (thi - tlo) * dtemp;

    // the interpolated records at rows jt and jt+1 of each corner
    const long long q[4] = {c00, c10, c01, c11};
    double2 a[4][2], b[4][2];   // a: (e, log p), b: (s, Gamma_1); [corner][row]
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const long long k = 2 * (q[c] + jt - 1);
      a[c][0] = __ldg(f + k);
      b[c][0] = __ldg(f + k + 1);
      a[c][1] = __ldg(f + k + 2);
      b[c][1] = __ldg(f + k + 3);
    }
    const double w[4] = {coeff0, coeff1, coeff2, coeff3};
    double lp = w[0] * (1 - dtemp) * a[0][0].y, s = w[0] * (1 - dtemp) * b[0][0].x,
           g1 = w[0] * (1 - dtemp) * b[0][0].y;
#pragma unroll
    for (int c = 1; c < 4; c++) {
      lp += w[c] * (1 - dtemp) * a[c][0].y;
      s += w[c] * (1 - dtemp) * b[c][0].x;
      g1 += w[c] * (1 - dtemp) * b[c][0].y;
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
      lp += w[c] * dtemp * a[c][1].y;
      s += w[c] * dtemp * b[c][1].x;
      g1 += w[c] * dtemp * b[c][1].y;
    }
    const double p_eos = exp(lp) * 1.60217733e33;   // MeV/fm^3 -> dyn/cm^2
    temp[i] = pow(10.0, temp_eos);
    press[i] = p_eos;
    cs[i] = sqrt((g1) * (p_eos) / (den_eos));
    ent[i] = s;
    gam1[i] = g1;
  }
}

void launch_eos_rex(const EosTableDev &d, long long n, const double *rho, const double *u, const double *ye,
                    double *temp, double *press, double *cs, double *ent, double *gam1, int num_sms,
                    cudaStream_t st)
{
  if (n <= 0) return;
  const long long blocks = (n + 255) / 256;
  const long long cap = (long long)(num_sms > 0 ? num_sms : 148) * 8;
  const int grid = (int)(blocks < cap ? blocks : cap);
  eos_rex_kernel<<<grid, 256, 0, st>>>(d, n, rho, u, ye, temp, press, cs, ent, gam1);
}

}  // namespace mdg
