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
//   * thread 0 of CTA 0 runs the controller (ctl_end of the previous step,
//     ctl_begin of the next) between steps, and every thread reads the done
//     flag after the following barrier.
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
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank(), nc = (int)cl.num_blocks();
  const bool leader = rank == 0 && threadIdx.x == 0;
  Ctl* ctl = a.st.ctl;
  const int ntiles = (a.st.mx + NT - 2) / (NT - 1);
  for (int it = 0;; ++it) {
    if (leader) {
      if (it > 0) ctl_end(ctl, a.nstages - 1, a.final_role);
      if (it < a.max_iters) ctl_begin(ctl);
    }
    cl.sync();
    // The same value in every thread: the controller writes ctl only before
    // the barrier that follows the last stage of this iteration.
    if (it == a.max_iters || ctl->done) break;
    // one read of the controller's roles and dt per step, all stages at once
    if (threadIdx.x < a.nstages) lines[threadIdx.x] = line1d<S>(a.st, a.sd[threadIdx.x], threadIdx.x);
    __syncthreads();
    for (int s = 0; s < a.nstages; ++s) {
      const Line<S> L = lines[s];
      for (int t = rank; t < ntiles; t += nc)
        stage1d_tile<P, CD, TF, PREC, NT>(L, a.st.ph, 1 + t * (NT - 1), sm);
      cl.sync();
    }
  }
}

}  // namespace scl
