// FP32 parts of the mixed-precision sweeps, shared by the 1-D batched sweep and the 3-D
// sweep: para_recon in difference form with FP64-computed FP32 weights, and the HLLC
// solver with FP32 wave speeds and star-state increments around an FP64 upwind flux.
#pragma once
#include "mdg_hydro.cuh"

namespace mdg {

// FP32 reconstruction weights of one zone
struct MixW { float wlm, wlp, wrm, wrp, eal, ear, ebl, ebr, dxz, mr, ml; };

__device__ __forceinline__ MixW load_mixw(const float *__restrict__ w, int64_t st)
{
  MixW m;
  m.wlm = __ldg(w + MX_WLM * st); m.wlp = __ldg(w + MX_WLP * st);
  m.wrm = __ldg(w + MX_WRM * st); m.wrp = __ldg(w + MX_WRP * st);
  m.eal = __ldg(w + MX_EAL * st); m.ear = __ldg(w + MX_EAR * st);
  m.ebl = __ldg(w + MX_EBL * st); m.ebr = __ldg(w + MX_EBR * st);
  m.dxz = __ldg(w + MX_DXZ * st); m.mr = __ldg(w + MX_MR * st); m.ml = __ldg(w + MX_ML * st);
  return m;
}

// The same from any address space (shared-memory copies of the weights): plain loads.
__device__ __forceinline__ MixW load_mixw_any(const float *w, int64_t st)
{
  MixW m;
  m.wlm = w[MX_WLM * st]; m.wlp = w[MX_WLP * st];
  m.wrm = w[MX_WRM * st]; m.wrp = w[MX_WRP * st];
  m.eal = w[MX_EAL * st]; m.ear = w[MX_EAR * st];
  m.ebl = w[MX_EBL * st]; m.ebr = w[MX_EBR * st];
  m.dxz = w[MX_DXZ * st]; m.mr = w[MX_MR * st]; m.ml = w[MX_ML * st];
  return m;
}

// para_recon of one variable in difference form (reconstruct.c:142-201): returns the face
// offsets dl = al - a and dr = ar - a.
__device__ __forceinline__ void mixed_recon(float dqm, float dqp, const MixW &w, float &dl, float &dr)
{
  if (dqm * dqp <= 0.0f) { dl = 0.0f; dr = 0.0f; return; }
  float l = w.wlm * dqm + w.wlp * dqp;
  float r = w.wrm * dqm + w.wrp * dqp;
  // face values limited to the range of the neighbouring means (reconstruct.c:165-171)
  if ((-l) * (l + 0.75f * dqm) < 0.0f) l = -0.75f * dqm;
  if ((0.75f * dqp - r) * r < 0.0f) r = 0.75f * dqp;
  // re-fit and move an interior extremum to the nearer edge (reconstruct.c:174-200)
  const float A2 = w.eal * l + w.ear * r;
  const float B2 = w.ebl * l + w.ebr * r;
  const float s = -B2 / (2.0f * A2);
  if (s > 0.0f && s < w.dxz) {
    if (s > 0.5f * w.dxz) l = r * w.mr;
    else r = l * w.ml;
  }
  dl = l;
  dr = r;
}

// A subsonic face is ill-conditioned in FP32 when max(rho u^2 + p) over its two states
// exceeds MIX_COND_MAX times the smaller pressure.  FP32 face states and star-state
// increments carry absolute errors of about 6e-8 (rho u^2 + p) (times the jump, for the
// face states); where the colder side's internal energy is a tiny fraction of that
// (strong shocks into cold or hypersonic gas) the error would swamp it -- it can drive the
// internal energy negative, and through dt_source_control's internal-energy term it
// steers dt.  Such faces are recomputed in FP64: both face states and the Riemann solve.
// Supersonic faces take the upwind FP64 flux of the FP32-reconstructed face state, whose
// error leaves the upwind zone's internal energy unchanged to first order.
#ifndef MDG_MIX_COND_MAX
#define MDG_MIX_COND_MAX 1000.0f
#endif
constexpr float MIX_COND_MAX = MDG_MIX_COND_MAX;

// HLLC (riemann.c:328-499) in direction DIR with FP32 wave speeds and star-state
// increments and an FP64 upwind flux; pl/pr: FP64 face states (rho, u, v1, v2, v3, p).  Returns false, with no
// flux written, for an ill-conditioned subsonic face (see MIX_COND_MAX).
template <int DIR>
__device__ __forceinline__ bool riemann_hllc_mixed(const double *pl, const double *pr, const FaceGeom<double> &g,
                                                   const GamConst<float> &gc, double *flux, float &sig, int &isshock)
{
  isshock = 0;
  if (g.area < 1.0e-16) {
    sig = 1.0e-30f;
#pragma unroll
    for (int v = 0; v < NPRIM; v++) flux[v] = 0.0;
    return true;
  }
  const float sc = (float)g.scale;
  float plf[6], prf[6];
#pragma unroll
  for (int v = 0; v < 6; v++) { plf[v] = (float)pl[v]; prf[v] = (float)pr[v]; }
  const float u_l = plf[U1 + DIR] * sc, u_r = prf[U1 + DIR] * sc;
  float sl, sr, ss, p_s;
  wave_speeds<float>(plf, prf, u_l, u_r, false, gc, sl, sr, ss, p_s, isshock);
  if (ss > sr) sr = 1.001f * ss;
  if (ss < sl) sl = 1.001f * ss;
  sig = fmaxf(fabsf(sl), fabsf(sr)) / sc;
  if (sl > 0.0f) { pflux<DIR, false, double>(pl, pl[5], g, flux); return true; }
  if (sr < 0.0f) { pflux<DIR, false, double>(pr, pr[5], g, flux); return true; }
  const float emax = fmaxf(plf[RHO] * u_l * u_l + plf[5], prf[RHO] * u_r * u_r + prf[5]);
  if (!(emax <= MIX_COND_MAX * fminf(plf[5], prf[5]))) return false;
  const bool left = ss > 0.0f;
  double pk[6];
#pragma unroll
  for (int v = 0; v < 6; v++) pk[v] = left ? pl[v] : pr[v];
  const float sk = left ? sl : sr, uk = left ? u_l : u_r;
  double u[NPRIM], fx[NPRIM];
  p_uflux<DIR, false, double>(pk, g, pk[5], u, fx);
  // U* - U of the upwind side in a form where nothing cancels in FP32:
  //   rho* - rho = rho (ss-uk)/(sk-ss),  E* - E = (E (ss-uk) + p* ss - p uk)/(sk-ss)
  const float rk = left ? plf[RHO] : prf[RHO];
  const float pkf = left ? plf[5] : prf[5];
  const float inv = 1.0f / (sk - ss);
  const float dU0 = rk * (ss - uk) * inv;
  const float dUE = ((float)u[UU] * (ss - uk) + p_s * ss - pkf * uk) * inv;
  double dU[NPRIM];
  dU[RHO] = (double)dU0;
  dU[UU] = (double)dUE;
  const double gd[3] = {g.g0, g.g1, g.g2};
#pragma unroll
  for (int m = 0; m < 3; m++)   // normal component: (ss-uk) rho + ss (rho*-rho), over the scale
    dU[U1 + m] = (m == DIR) ? gd[m] * (double)(((ss - uk) * rk + ss * dU0) / sc) : gd[m] * pk[U1 + m] * (double)dU0;
  const double slr = (double)(sk / sc);
#pragma unroll
  for (int v = 0; v < NPRIM; v++) flux[v] = g.area * (fx[v] + slr * dU[v]);
  return true;
}

}  // namespace mdg
