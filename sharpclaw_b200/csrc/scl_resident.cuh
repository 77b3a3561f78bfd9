// scl_resident.cuh -- the whole time loop of a small 1-D grid in one launch.
//
// A grid of a few thousand cells leaves the step graphs launch-bound: every
// stage kernel and controller kernel costs microseconds of launch latency
// while its arithmetic takes less.  Here one thread-block cluster (at most
// RES_CLUSTER CTAs, co-scheduled by the cluster launch) stays resident for up
// to max_iters controller iterations of src/sharpclaw.f90:118-221, and the
// run's registers stay in shared memory:
//   * CTA r owns the chunk of T consecutive tiles r*T .. r*T+T-1 and keeps,
//     for every physical buffer, the chunk's cells plus three halo cells on
//     each side in shared memory (ResView, scl_kernels.cuh), loaded from
//     global memory when the launch starts and written back when it ends;
//   * each stage runs stage1d_res on those rows: the interface, cell and
//     combination code of the stage kernels' tiles, so the arithmetic, and
//     therefore every result, is the step graphs'; a thread solves both
//     interfaces of its cell, so a tile has no barrier; a stage stores the
//     cells next to a chunk edge, and the ghost images, straight into the
//     neighbouring CTAs' rows through distributed shared memory;
//   * one cluster barrier (arrive.release / wait.acquire) per stage orders
//     those stores before the next stage reads its window, and is the only
//     wait between CTAs;
//   * every CTA keeps its own copy of the controller in shared memory and
//     runs it (ctl_end of the previous step, ctl_begin of the next) on the
//     same inputs: the CTAs' last-stage CFL maxima and status (and, with
//     conserved totals on, their compensated (sum, error) pairs in rank
//     order), read from every CTA through distributed shared memory.  These
//     per-CTA values are double-buffered by step parity, so no barrier
//     beyond the stages' is needed between the reads and the next step's
//     writes.  CTA 0's copy goes back to global memory at the end.
// The loop ends after max_iters iterations at most; the host relaunches while
// the controller is not done.
#pragma once
#include <cooperative_groups.h>

#include "scl_ctl.cuh"
#include "scl_kernels.cuh"
#include "scl_launch.h"

namespace scl {

// Dynamic shared memory of a resident run with T tiles per CTA: the rows
// of every physical buffer.
template <class S>
inline size_t run1d_rows_bytes(int meqn, int T, int nt) {
  return sizeof(S) * (size_t)NROLES * (size_t)meqn * (size_t)(T * (nt - 1) + 6);
}

// Threads of a resident CTA: NT tile threads (warps 0 .. NT/32-1) and one
// controller warp.
template <int NT>
constexpr int run1d_threads() { return NT + 32; }

// Conserved totals of this CTA's cells in row buffer v.bout (the step's last
// stage output): per tile and warp a compensated (sum, error) pair, then
// thread 0 combines them in tile-then-warp order into tp[m].  Called by every
// thread of the CTA (it contains a CTA barrier); out of line, so that runs
// without totals carry none of its code.
template <class P, int PREC, int NT>
__device__ __noinline__ void res_totals_cta(const Line<typename Prec<PREC>::S>& L, const ResView& v, int t0, int t1,
                                            double (*tsum)[NT / 32][MAXEQ][2], double (*tp)[2]) {
  using S = typename Prec<PREC>::S;
  constexpr int M = P::MEQN;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tid = threadIdx.x, lane = tid & 31;
  if (tid < NT) {
    for (int t = t0; t < t1; ++t) {
      const int c = 1 + t * (NT - 1) + tid;
      const bool own = tid < NT - 1 && c <= L.mx;
#pragma unroll
      for (int m = 0; m < M; ++m) {
        CSum acc{0.0, 0.0};
        if (own) {
          const S* row = reinterpret_cast<const S*>(smem_raw) + ((long)v.bout * M + m) * v.rw;
          const double x = (double)row[(t - t0) * (NT - 1) + tid + 3];
          if (L.mcapa > 0)
            acc.add(x * (double)static_cast<const S*>(L.aux)[(long)(L.mcapa - 1) * L.plane + c + 2]);
          else
            acc.add(x);
        }
        acc = warp_csum(acc);
        if (lane == 0) { tsum[t - t0][tid >> 5][m][0] = acc.s; tsum[t - t0][tid >> 5][m][1] = acc.c; }
      }
    }
  }
  __syncthreads();
  if (tid == 0) {
    for (int m = 0; m < M; ++m) {
      CSum tt{0.0, 0.0};
      for (int t = 0; t < t1 - t0; ++t)
        for (int w = 0; w < NT / 32; ++w) tt.add(tsum[t][w][m][0], tsum[t][w][m][1]);
      tp[m][0] = tt.s;
      tp[m][1] = tt.c;
    }
  }
}

// The step's candidate totals from every CTA's (sum, error) pairs tp (this
// CTA's copy, read in each rank through distributed shared memory), combined
// in rank order; called by the 32 lanes of the controller warp, the result
// in lane 0's cand[].  Out of line for the same reason.
static __device__ __noinline__ void res_totals_gather(const double (*tp)[2], int nc, int meqn, double dx, double* cand) {
  cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
  const int lane = threadIdx.x & 31;
  double ts[MAXEQ], tc[MAXEQ];
#pragma unroll
  for (int q = 0; q < MAXEQ; ++q) { ts[q] = 0.0; tc[q] = 0.0; }
  if (lane < nc) {
    const double(*pt)[2] = cl.map_shared_rank(&tp[0], lane);
#pragma unroll
    for (int q = 0; q < MAXEQ; ++q) { ts[q] = pt[q][0]; tc[q] = pt[q][1]; }
  }
#pragma unroll
  for (int q = 0; q < MAXEQ; ++q) {
    if (q >= meqn) {
      if (lane == 0) cand[q] = 0.0;
      continue;
    }
    CSum t{0.0, 0.0};
    for (int r = 0; r < nc; ++r) t.add(__shfl_sync(0xffffffffu, ts[q], r), __shfl_sync(0xffffffffu, tc[q], r));
    if (lane == 0) cand[q] = (t.s + t.c) * dx;
  }
}

// GEN: the run may have a capacity field, conserved totals or a stage with a
// second output; the launcher picks GEN = false when it has none of them,
// and that kernel carries none of their code (measured at 1000 cells, where
// a step takes about 5 us: 4.57 against 5.22 us per step in the mixed form,
// 4.96 against 5.47 in FP64).
template <class P, int CD, int TF, int PREC, int NT, bool GEN>
__global__ void __launch_bounds__(run1d_threads<NT>(), 1) k_run1d(RunArgs a) {
  namespace cg = cooperative_groups;
  using S = typename Prec<PREC>::S;
  using R = typename Prec<PREC>::R;
  constexpr int M = P::MEQN;
  constexpr int NTH = run1d_threads<NT>();
  // per step parity: the step's stage lines and row views (roles and dt
  // are fixed within a step); raw storage, as shared variables take no
  // constructors
  __shared__ __align__(16) unsigned char lines_raw[2][sizeof(Line<S>) * MAXSTAGES];
  __shared__ ResView views[2][MAXSTAGES];
  __shared__ StageDesc sds[MAXSTAGES];
  __shared__ Ctl sctl;                    // this CTA's copy of the controller
  __shared__ Ctl spart[2];                // per step parity: this CTA's stage CFL maxima and status
  __shared__ double tpart[2][MAXEQ][2];   // per step parity: this CTA's totals of the last stage
  __shared__ double tsum[RES_TILES_PER_CTA][NT / 32][MAXEQ][2];   // per tile and warp (sum, error)
  __shared__ int sdone;                   // the loop ends (set by the controller warp)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S* rows = reinterpret_cast<S*>(smem_raw);
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank(), nc = (int)cl.num_blocks();
  const int tid = threadIdx.x;
  const bool cw = tid >= NT;              // the controller warp
  const int mx = a.st.mx;
  const int ntiles = (mx + NT - 2) / (NT - 1);
  const int T = (ntiles + nc - 1) / nc;   // the host launches nc = ceil(ntiles / T) CTAs
  const int cspan = T * (NT - 1);
  const int rw = cspan + 6;
  const int t0 = rank * T, t1 = t0 + T < ntiles ? t0 + T : ntiles;
  const int last = a.nstages - 1;
  const long e0 = (long)rank * cspan;     // element offset of row element 0
  // the rows from global memory (elements past the buffer's ghost cells read
  // 1, as the stage kernels' staging does)
#pragma unroll
  for (int b = 0; b < NROLES; ++b) {
    const S* g = static_cast<const S*>(a.st.buf[b]);
    if (!g) continue;
    for (int m = 0; m < M; ++m)
      for (int k = tid; k < rw; k += NTH)
        rows[((long)b * M + m) * rw + k] = e0 + k < (long)mx + 6 ? g[(long)m * a.st.plane + e0 + k] : (S)1;
  }
  // the stage descriptors (constant indices: a runtime index into a kernel
  // parameter array copies the whole argument struct to local memory)
#pragma unroll
  for (int s = 0; s < MAXSTAGES; ++s)
    if (tid == s) sds[s] = a.sd[s];
  {
    const int* src = reinterpret_cast<const int*>(a.st.ctl);
    int* dst = reinterpret_cast<int*>(&sctl);
    for (int k = tid; k < (int)(sizeof(Ctl) / sizeof(int)); k += NTH) dst[k] = src[k];
  }
  // every CTA's rows are loaded before any stage stores into them
  cl.sync();
  // Speculation: while the controller warp judges step n, the tile threads
  // solve the interfaces of step n+1's first stage (first tile) as if step n
  // were accepted (its input is then the last stage's output); a rejected
  // step or a one-stage integrator solves them after the controller.
  const bool spec_ok = a.nstages > 1;
  for (int it = 0;; ++it) {
    const int p = it & 1;
    Line<S>* lines = reinterpret_cast<Line<S>*>(lines_raw[p]);
    ResIface<R, M> pre;
    int spec_buf = -1;
    if (cw) {
      const int lane = tid - NT;
      if (it > 0) {
        const int pp = p ^ 1;
        unsigned long long bits = 0;
        int st = 0;
        if (lane < nc) {
          const Ctl* pr = cl.map_shared_rank(&spart[pp], lane);
          bits = (unsigned long long)__double_as_longlong(pr->stage_cfl[last]);
          st = pr->status;
        }
        // maximum of the bit patterns (as the global atomic max), OR of status
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const unsigned long long ob = __shfl_xor_sync(0xffffffffu, bits, o);
          bits = ob > bits ? ob : bits;
          st |= __shfl_xor_sync(0xffffffffu, st, o);
        }
        if (GEN && sctl.totals) res_totals_gather(tpart[pp], nc, M, a.st.dx, sctl.tot_cand);
        if (lane == 0) {
          sctl.stage_cfl[last] = __longlong_as_double((long long)bits);
          sctl.status |= st;
          ctl_end(&sctl, last, a.final_role);
        }
      }
      if (lane == 0) {
        if (it < a.max_iters) ctl_begin(&sctl);
        // the same value in every CTA: the copies run on the same inputs
        sdone = it == a.max_iters || sctl.done;
      }
      __syncwarp();
      if (lane < a.nstages) {
        const StageDesc sd = sds[lane];
        Line<S> L = line1d<S>(a.st, sd, lane, &sctl);
        L.ctl = &spart[p];
        L.dtdx = L.dt / L.dx;
        lines[lane] = L;
        ResView v;
        v.rw = rw;
        v.rsh = 0;
        v.cspan = cspan;
        v.rank = rank;
        v.rlast = nc - 1;
        v.bin = sctl.role[sd.in];
        v.bqo = sd.aux_in >= 0 ? sctl.role[sd.aux_in] : -1;
        v.bout = sd.kind == SK_DQ ? -1 : sctl.role[sd.out];
        v.bout2 = sd.out2 >= 0 ? sctl.role[sd.out2] : -1;
        views[p][lane] = v;
        spart[p].stage_cfl[lane] = 0.0;
      }
      if (lane == 0) spart[p].status = 0;
      if (lane < MAXEQ * 2) tpart[p][lane / 2][lane % 2] = 0.0;
    } else if (spec_ok && it > 0) {
      // step it-1's lines and views (the other parity) stay unchanged here
      spec_buf = views[p ^ 1][last].bout;
      const int c = 1 + t0 * (NT - 1) + tid;
      if (tid < NT - 1 && c <= mx) {
        const Line<S>& Lp = reinterpret_cast<const Line<S>*>(lines_raw[p ^ 1])[0];
        ResView v = views[p ^ 1][0];
        CflMax<R> unused;
        res_ifaces<P, CD, PREC, GEN>(Lp, a.st.ph, c, v, spec_buf, false, unused, pre);
      }
    }
    __syncthreads();
    if (sdone) break;
    const bool tot = GEN && sctl.totals;
    for (int s = 0; s < a.nstages; ++s) {
      const bool lst = s == last;
      if (!cw) {
        const Line<S> L = lines[s];
        ResView v = views[p][s];
        for (int t = t0; t < t1; ++t) {
          v.rsh = (t - t0) * (NT - 1);
          const int c0 = 1 + t * (NT - 1);
          const bool use_pre = s == 0 && t == t0 && spec_buf >= 0 && spec_buf == v.bin;
          stage1d_res<P, CD, TF, PREC, NT, GEN>(L, a.st.ph, c0, v, lst, &spart[p], pre, use_pre);
        }
      }
      // this CTA's totals of the step's output (its own cells: no wait
      // beyond the CTA barrier inside)
      if (tot && lst) res_totals_cta<P, PREC, NT>(lines[s], views[p][s], t0, t1, tsum, tpart[p]);
      cl.sync();
    }
  }
  // the rows back to global memory: the chunk's cells, and the ghost cells
  // of the two ends
  const int klo = rank == 0 ? 0 : 3;
  const int khi = (int)((rank == nc - 1 ? (long)mx + 6 : e0 + cspan + 3) - e0);   // exclusive
#pragma unroll
  for (int b = 0; b < NROLES; ++b) {
    S* g = static_cast<S*>(a.st.buf[b]);
    if (!g) continue;
    for (int m = 0; m < M; ++m)
      for (int k = klo + tid; k < khi; k += NTH) g[(long)m * a.st.plane + e0 + k] = rows[((long)b * M + m) * rw + k];
  }
  if (rank == 0) {
    const int* src = reinterpret_cast<const int*>(&sctl);
    int* dst = reinterpret_cast<int*>(a.st.ctl);
    for (int k = tid; k < (int)(sizeof(Ctl) / sizeof(int)); k += NTH) dst[k] = src[k];
  }
  // no CTA exits while another may still read its shared memory
  cl.sync();
}

}  // namespace scl
