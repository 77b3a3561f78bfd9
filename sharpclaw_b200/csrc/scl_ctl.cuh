// scl_ctl.cuh -- the time-step controller of src/sharpclaw.f90:118-221 on the
// device, shared by the step graphs (one grid), the batched solver (one
// controller per instance) and the cluster-resident run.  ctl_begin opens a
// controller iteration (dt clipped to tend, t advanced); ctl_end judges the
// step by its last stage's CFL number (accept: q <- the final role; reject:
// t = told and, with variable dt, a retake) and updates dt.
#pragma once
#include "scl_common.cuh"

namespace scl {

__device__ __forceinline__ void ctl_begin(Ctl* c) {
  if (c->done) return;
  if (c->n_iter >= c->maxn) { c->done = 1; return; }   // do n=1,maxn exhausted
  c->n_iter += 1;
  c->fresh = !c->retake;                                             // b4step runs on new steps only
  if (!c->retake) {
    c->told = c->t;                                                  // :120
    if (c->told + c->dt > c->tend && c->tstart < c->tend) c->dt = c->tend - c->told;  // :124
    // b4step: default no-op (src/b4step.f90); qold = q is the Q role (:132-135)
  }
  c->retake = 0;
  c->t = c->told + c->dt;                                            // :139
  for (int s = 0; s < MAXSTAGES; ++s) c->stage_cfl[s] = 0.0;
}

__device__ __forceinline__ void ctl_end(Ctl* c, int last_stage, int final_role) {
  if (c->done) return;
  // A bounded wait of a stage kernel ran out (its staged data may be
  // incomplete): discard the step and stop, q = qold; the host reports it.
  if (c->status & SCL_STATUS_TIMEOUT) {
    c->t = c->told;
    c->done = 1;
    return;
  }
  const double cfl = c->stage_cfl[last_stage];   // the last stage's CFL (:184, A2)
  c->cfl_last = cfl;
  // A NaN CFL number cannot drive dt control (the reference would reject and
  // retake with a NaN or dt_max step forever): stop with q = qold.
  if (cfl != cfl) {
    c->status |= SCL_STATUS_NONFINITE;
    c->info = SCL_INFO_NONFINITE;
    c->t = c->told;
    c->done = 1;
    return;
  }
  // Non-finite stage outputs matter only if the step is accepted; a rejected
  // step's stages are discarded (q = qold) as in the reference.
  if (cfl <= c->cfl_max && (c->status & SCL_STATUS_NONFINITE)) {
    c->info = SCL_INFO_NONFINITE;
    c->t = c->told;
    c->done = 1;
    return;
  }
  c->status &= ~SCL_STATUS_NONFINITE;
  if (c->dt_variable == 1) {                                        // :184-192
    if (cfl > 0.0) {
      c->dt = fmin(c->dt_max, c->dt * c->cfl_desired / cfl);
      c->dtmin = fmin(c->dt, c->dtmin);
      c->dtmax = fmax(c->dt, c->dtmax);
    } else {
      c->dt = c->dt_max;
    }
  }
  if (cfl <= c->cfl_max) {                                          // :195-197 accept
    c->cflmax = fmax(cfl, c->cflmax);
    const int tmp = c->role[ROLE_Q];
    c->role[ROLE_Q] = c->role[final_role];
    c->role[final_role] = tmp;
    if (c->totals) {                  // the accepted state's totals (scl_totals.cuh)
      for (int m = 0; m < MAXEQ; ++m) {
        c->tot[m] = c->tot_cand[m];
        c->drift[m] = fmax(c->drift[m], fabs(c->tot[m] - c->tot0[m]));
      }
    }
  } else {                                                          // :198-216 reject
    c->t = c->told;
    c->rejected += 1;
    if (c->dt_variable == 1) {
      c->retake = 1;
    } else {
      c->cflmax = fmax(cfl, c->cflmax);
      c->done = 1;
      return;
    }
  }
  c->steps_taken += 1;                                              // :219
  if (c->t >= c->tend) c->done = 1;                                 // :220
}

}  // namespace scl
