// scl_batch.cuh -- many independent 1-D problems of uneven size in one
// persistent launch per stage.
//
// Every instance k keeps its own controller (t, dt, CFL, roles, status: the
// scalars of src/sharpclaw.f90) in ctl[k], so instances take their own
// adaptive steps, rejections and final times.  A step of the batch is
//   begin (one CTA: ctl_begin for every instance, then the list of active
//   instances and the prefix sum of their tiles),
//   one persistent stage kernel per RK stage (a fixed grid of CTAs walks the
//   active tiles of all instances: tile -> instance by binary search),
//   end (one thread per instance: ctl_end).
// The host captures K such steps in a CUDA graph and replays it until no
// instance is active; inside the graph the end of step k runs in the begin
// kernel of step k+1 (same thread per instance, end logic first).
#pragma once
#include "scl_ctl.cuh"
#include "scl_kernels.cuh"

namespace scl {

struct BatchArgs {
  Ctl* ctl;                 // [ninst]
  const long* off;          // [ninst] element offset of instance k in a state arena
  const long* aoff;         // [ninst] element offset of instance k in the aux arena
  const long* plane;        // [ninst] component stride of instance k
  const int* mx;            // [ninst]
  const double* dx;         // [ninst]
  const int* active;        // [ninst] ids of the active instances (first nact entries)
  const int* prefix;        // [ninst+1] tile prefix over the active list
  const int* nact;          // number of active instances (device scalar)
  void* arena[NROLES];      // state arenas, one per register role
  const void* aux;          // aux arena or nullptr
  StageDesc sd;
  int stage;
  int mthbc[2];
  int mcapa;
  Phys ph;
};

// Begin of a batch step on one CTA of 1024 threads: controller begin for every
// instance (after the end of the previous step when end_stage >= 0: its last
// stage index), then the ordered list of active instances with the exclusive
// prefix sum of their tile counts (a block-wide scan in chunks of 1024).
// Tile j of an instance updates the STRIDE cells from FIRST + j*STRIDE, so
// an instance of mx cells has (mx - FIRST)/STRIDE + 1 tiles.
template <int STRIDE, int FIRST>
__global__ void __launch_bounds__(1024) k_batch_begin(Ctl* ctl, const int* mx, int ninst, int* active,
                                                      int* prefix, int* nact, int end_stage, int final_role) {
  __shared__ int wact[32], wtiles[32];
  __shared__ int base_tiles, base_act;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) { base_tiles = 0; base_act = 0; }
  __syncthreads();
  for (int k0 = 0; k0 < ninst; k0 += 1024) {
    const int k = k0 + tid;
    int act = 0, tiles = 0;
    if (k < ninst) {
      if (end_stage >= 0) ctl_end(&ctl[k], end_stage, final_role);
      ctl_begin(&ctl[k]);
      act = ctl[k].done ? 0 : 1;
      tiles = act ? (mx[k] - FIRST) / STRIDE + 1 : 0;
    }
    // inclusive warp scans of (act, tiles)
    int a = act, t = tiles;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int ya = __shfl_up_sync(0xffffffffu, a, o), yt = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) { a += ya; t += yt; }
    }
    if (lane == 31) { wact[wid] = a; wtiles[wid] = t; }
    __syncthreads();
    if (wid == 0) {   // inclusive scan of the 32 warp totals
      int wa = wact[lane], wt = wtiles[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int ya = __shfl_up_sync(0xffffffffu, wa, o), yt = __shfl_up_sync(0xffffffffu, wt, o);
        if (lane >= o) { wa += ya; wt += yt; }
      }
      wact[lane] = wa;
      wtiles[lane] = wt;
    }
    __syncthreads();
    const int wa_ex = wid ? wact[wid - 1] : 0, wt_ex = wid ? wtiles[wid - 1] : 0;
    if (act) {
      const int pos = base_act + wa_ex + a - 1;
      active[pos] = k;
      prefix[pos] = base_tiles + wt_ex + t - tiles;
    }
    __syncthreads();
    if (tid == 0) { base_act += wact[31]; base_tiles += wtiles[31]; }
    __syncthreads();
  }
  if (tid == 0) {
    prefix[base_act] = base_tiles;
    *nact = base_act;
  }
}

static __global__ void k_batch_end(Ctl* ctl, int ninst, int last_stage, int final_role) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < ninst) ctl_end(&ctl[k], last_stage, final_role);
}

// Persistent stage kernel: a fixed grid walks the active tiles.
template <class P, int CD, int TF, int PREC, int NT>
__global__ void __launch_bounds__(NT) k_batch_stage(BatchArgs a) {
  using S = typename Prec<PREC>::S;
  __shared__ Tile1DSmem<P, PREC, NT> sm;
  const int na = *a.nact;
  if (na == 0) return;
  const int ntiles = a.prefix[na];
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    // find the active slot j with prefix[j] <= t < prefix[j+1]
    int lo = 0, hi = na - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (a.prefix[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const int k = a.active[lo];
    Ctl* ctl = &a.ctl[k];
    const long off = a.off[k];
    Line<S> L;
    L.ctl = ctl;
    L.qin = static_cast<const S*>(a.arena[ctl->role[a.sd.in]]) + off;
    L.qo = a.sd.aux_in >= 0 ? static_cast<const S*>(a.arena[ctl->role[a.sd.aux_in]]) + off : nullptr;
    L.out = static_cast<S*>(a.arena[ctl->role[a.sd.out]]) + off;
    L.out2 = a.sd.out2 >= 0 ? static_cast<S*>(a.arena[ctl->role[a.sd.out2]]) + off : nullptr;
    L.dq_out = nullptr;
    L.aux = a.aux ? static_cast<const void*>(static_cast<const S*>(a.aux) + a.aoff[k]) : nullptr;
    L.mx = a.mx[k];
    L.plane = a.plane[k];
    L.dx = a.dx[k];
    L.bl = a.mthbc[0];
    L.br = a.mthbc[1];
    L.mcapa = a.mcapa;
    L.kind = a.sd.kind;
    L.stage = a.stage;
    L.ixy = 1;
    L.dt = ctl->dt;
    stage1d_tile<P, CD, TF, PREC, NT>(L, a.ph, 1 + (t - a.prefix[lo]) * (NT - 1), sm);
  }
}

}  // namespace scl
