// The per-problem time bookkeeping of one step, as device functions: the dt rules that
// open a step and the time update that closes it.  The small kernels of mdg_misc.cu run
// them one thread per problem; the resident 1-D stepper (mdg_sweep1d.cu) runs them
// inside its time loop.  Both translation units are compiled without multiply-add
// contraction, so the two paths produce the same dt and t bit for bit.
#pragma once
#include "mdg_hydro.cuh"

namespace mdg {

// estimate_dt() (step.c:192-198) applied to the accumulated minimum, then the safety,
// growth and end-time rules of main.c:239-251, for problem P with time record *Tp.
__device__ __forceinline__ void dt_finalize_one(const ProbDev &P, ProbTime *Tp, int *err)
{
  ProbTime T = *Tp;
  if (T.dt_ready) return;
  // the reference's time loop runs while t < tmax (main.c:206); past it nothing changes
  // (an empty slot of a solve server has tmax = 0 and is done from the start)
  if (!(T.t < P.tmax)) {
    T.done = 1;
    T.dt_ready = 1;
    *Tp = T;
    return;
  }
  double min_dt = ord_to_dbl(T.minacc);
  if (T.istep == 0) min_dt = tmin(min_dt, P.initial_dt);
  min_dt = tmin(min_dt, P.dtmax);
  min_dt *= P.cfl;
  // main.c:229-238 aborts the run when the estimate drops below dtmin; here the
  // condition is recorded for the host (mdg_synchronize returns MDG_ERR_NONFINITE)
  if (!(min_dt >= P.dtmin)) {
    atomicExch(err, MDG_ERR_NONFINITE);
    T.err = MDG_ERR_NONFINITE;
  }
  double dt = min_dt;
  if (T.istep == 0) dt *= P.dt_init_safety;
  else dt = tmin(T.dtold * P.dt_grow_safety, dt);
  T.dtold = dt;
  if (T.t + 1 * dt > P.tmax) dt = 1.000000001 * (P.tmax - T.t) / 1;
  if (dt < P.dtmin) dt = P.dtmin;
  T.dt = dt;
  T.t_bc1 = T.t + dt;                  // reset_boundaries_gpu: t += dt (bc.c:721)
  T.t_next = (T.t_bc1 - dt) + dt;      // ... t -= dt (bc.c:1418), then main.c:263 t += dt
  T.minacc = dbl_to_ord(1.0e100);      // step.c:49
  T.dt_ready = 1;
  *Tp = T;
}

// main.c:262-264: t += dt, istep++ (nothing once the loop has ended); the next step's dt
// is finalized afresh.
__device__ __forceinline__ void finish_one(ProbTime *T)
{
  if (!T->done) {
    T->t = T->t_next;
    T->istep += 1;
  }
  T->dt_ready = 0;
}

}  // namespace mdg
