// scl_resident.cuh -- the whole time loop of a small 1-D grid in one launch.
//
// A grid of a few thousand cells leaves the step graphs launch-bound: every
// stage kernel and controller kernel costs microseconds of launch latency
// while its arithmetic takes less.  Here one thread-block cluster (at most
// RES_CLUSTER CTAs, co-scheduled by the cluster launch) stays resident for up
// to max_iters controller iterations of src/sharpclaw.f90:118-221:
//   * CTA r computes tiles r, r + nc, ... of every stage with the tile code of
//     the stage kernels (stage1d_tile), so the arithmetic, and therefore every
//     result, is the step graphs';
//   * a cluster barrier (arrive.release / wait.acquire at cluster scope)
//     separates the stages, which orders each stage's global-memory output,
//     ghost images included, before the next stage reads its halo;
//   * the controller lives in CTA 0's shared memory for the whole launch
//     (copied from and back to global memory at its ends): thread 0 of CTA 0
//     runs it (ctl_end of the previous step, ctl_begin of the next) between
//     steps, and every CTA reads its roles, dt and done flag through
//     distributed shared memory, so no controller access waits on L2;
//   * each CTA accumulates its stage CFL numbers and status in its own shared
//     memory (the tile code's atomics stay CTA-local); the controller thread
//     combines the CTAs' values of the last stage (maximum of the bit
//     patterns, as the global atomic max does, and OR) before ctl_end.
// The loop ends after max_iters iterations at most; the host relaunches while
// the controller is not done.
#pragma once
#include <cooperative_groups.h>

#include "scl_ctl.cuh"
#include "scl_kernels.cuh"

namespace scl {

template <class P, int CD, int TF, int PREC, int NT>
__global__ void __launch_bounds__(NT) k_run1d(RunArgs a) {
  namespace cg = cooperative_groups;
  using S = typename Prec<PREC>::S;
  __shared__ Tile1DSmem<P, PREC, NT> sm;
  // this step's stage lines (roles and dt are fixed within a step); raw
  // storage, as shared variables take no constructors
  __shared__ __align__(16) unsigned char lines_raw[sizeof(Line<S>) * MAXSTAGES];
  Line<S>* lines = reinterpret_cast<Line<S>*>(lines_raw);
  __shared__ Ctl sctl;    // CTA 0's copy is the cluster's controller
  __shared__ Ctl spart;   // this CTA's stage CFL maxima and status (only those fields)
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank(), nc = (int)cl.num_blocks();
  const bool leader = rank == 0 && threadIdx.x == 0;
  Ctl* gctl = a.st.ctl;
  if (leader) sctl = *gctl;
  cl.sync();
  Ctl* ctl = cl.map_shared_rank(&sctl, 0);
  const int ntiles = (a.st.mx + NT - 2) / (NT - 1);
  const int last = a.nstages - 1;
  for (int it = 0;; ++it) {
    if (leader) {
      if (it > 0) {
        unsigned long long m = 0;
        int st = 0;
        for (int r = 0; r < nc; ++r) {
          const Ctl* pr = cl.map_shared_rank(&spart, r);
          const unsigned long long b = __double_as_longlong(pr->stage_cfl[last]);
          m = b > m ? b : m;
          st |= pr->status;
        }
        sctl.stage_cfl[last] = __longlong_as_double(m);
        sctl.status |= st;
        ctl_end(&sctl, last, a.final_role);
      }
      if (it < a.max_iters) ctl_begin(&sctl);
    }
    cl.sync();
    // The same value in every thread: the controller writes ctl only before
    // the barrier that follows the last stage of this iteration.
    if (it == a.max_iters || ctl->done) break;
    // one read of the controller's roles and dt per step, all stages at once
    if (threadIdx.x < a.nstages) {
      Line<S> L = line1d<S>(a.st, a.sd[threadIdx.x], threadIdx.x, ctl);
      L.ctl = &spart;
      lines[threadIdx.x] = L;
      spart.stage_cfl[threadIdx.x] = 0.0;
    }
    if (threadIdx.x == 0) spart.status = 0;
    __syncthreads();
    for (int s = 0; s < a.nstages; ++s) {
      const Line<S> L = lines[s];
      for (int t = rank; t < ntiles; t += nc)
        stage1d_tile<P, CD, TF, PREC, NT>(L, a.st.ph, 1 + t * (NT - 1), sm);
      cl.sync();
    }
  }
  // every CTA has left the loop (no more reads of CTA 0's shared memory)
  // before the controller goes back to global memory and CTA 0 exits
  cl.sync();
  if (leader) *gctl = sctl;
}

}  // namespace scl
