// scl_totals.cuh -- conserved totals of the state in FP64 with compensated
// summation, whatever the arithmetic form of the stages.
//
// T_m = (sum over interior cells of kappa * q(., m)) * dx [* dy], kappa the
// capacity aux(., mcapa) (1 without one).  Every thread accumulates its cells
// with Knuth's error-free TwoSum (s + e == a + b exactly), the pairs (sum,
// error) are combined the same way across the warp, the CTA and, in the last
// CTA to finish (a self-resetting ticket in the controller), across CTAs in a
// fixed order, so the result is deterministic and carries the error of one
// final rounding plus a few ulps of the error terms.  No counterpart in the
// reference, which keeps no totals.
#pragma once
#include "scl_common.cuh"

namespace scl {

// s + e == a + b exactly (round-to-nearest, no reassociation)
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double z = s - a;
  e = (a - (s - z)) + (b - z);
}

struct CSum {
  double s, c;
  __device__ __forceinline__ void add(double x) {
    double t, e;
    two_sum(s, x, t, e);
    s = t;
    c += e;
  }
  __device__ __forceinline__ void add(double os, double oc) {
    double t, e;
    two_sum(s, os, t, e);
    s = t;
    c += e + oc;
  }
};

struct TotalsArgs {
  Ctl* ctl;
  const void* buf[NROLES];
  int role;            // role whose state is summed
  int mode;            // 0: the step's final stage output -> tot_cand; 1: the run's start -> tot0, tot
  int mx, my, ndim, meqn;
  long pitch, plane;
  const void* capa;    // capacity plane (storage type), or nullptr
  double area;         // dx (1-D) or dx*dy (2-D)
  double* partials;    // [gridDim.x][MAXEQ][2]
};

constexpr int TOT_NT = 256;
constexpr int TOT_U = 4;   // cells in flight per thread and plane
constexpr int TOT_BLOCKS_MAX = 148 * 4;   // CTAs of one launch at most (the partials' rows)

// (sum, error) pairs of a warp combined into lane 0 (a fixed shuffle tree)
__device__ __forceinline__ CSum warp_csum(CSum t) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double os = __shfl_down_sync(0xffffffffu, t.s, o);
    const double oc = __shfl_down_sync(0xffffffffu, t.c, o);
    t.add(os, oc);
  }
  return t;
}

// TOT_U cells at element offsets off + u * stride (u < n <= TOT_U) added
// to acc: the loads of all of them are issued before their sums.
template <class S, int M, bool CAP>
__device__ __forceinline__ void totals_take(CSum (&acc)[M], const S* __restrict__ q, const S* __restrict__ kap,
                                            long plane, long off, long stride, int n) {
  S v[TOT_U][M], w[TOT_U];
#pragma unroll
  for (int u = 0; u < TOT_U; ++u) {
    if (u < n) {
#pragma unroll
      for (int m = 0; m < M; ++m) v[u][m] = q[(long)m * plane + off + u * stride];
      if constexpr (CAP) w[u] = kap[off + u * stride];
    }
  }
#pragma unroll
  for (int u = 0; u < TOT_U; ++u) {
    if (u < n) {
#pragma unroll
      for (int m = 0; m < M; ++m) acc[m].add(CAP ? (double)v[u][m] * (double)w[u] : (double)v[u][m]);
    }
  }
}

// M components, CAP: weighted by the capacity plane  Every thread keeps
// TOT_U * M (+ TOT_U) loads in flight.
template <class S, int M, bool CAP>
__global__ void __launch_bounds__(TOT_NT) k_totals(TotalsArgs a) {
  Ctl* ctl = a.ctl;
  if (a.mode == 0 && (ctl->done || !ctl->totals)) return;
  const S* __restrict__ q = static_cast<const S*>(pick_buf(a.buf, ctl->role[a.role]));
  const S* __restrict__ kap = static_cast<const S*>(a.capa);
  CSum acc[M];
#pragma unroll
  for (int m = 0; m < M; ++m) acc[m] = CSum{0.0, 0.0};
  // 1-D: a grid-stride walk over the cells; 2-D: CTAs take rows, threads
  // walk the row (no division per cell)
  if (a.ndim == 1) {
    const long step = (long)gridDim.x * blockDim.x;
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + (TOT_U - 1) * step < a.mx; i += TOT_U * step) totals_take<S, M, CAP>(acc, q, kap, a.plane, i + 3, step, TOT_U);
    if (i < a.mx) totals_take<S, M, CAP>(acc, q, kap, a.plane, i + 3, step, (int)((a.mx - 1 - i) / step) + 1);
  } else {
    for (long j = blockIdx.x; j < a.my; j += gridDim.x) {
      const long row = (j + 3) * a.pitch + 3;
      long i = threadIdx.x;
      for (; i + (TOT_U - 1) * TOT_NT < a.mx; i += TOT_U * TOT_NT) totals_take<S, M, CAP>(acc, q, kap, a.plane, row + i, TOT_NT, TOT_U);
      if (i < a.mx) totals_take<S, M, CAP>(acc, q, kap, a.plane, row + i, TOT_NT, (int)((a.mx - 1 - i) / TOT_NT) + 1);
    }
  }
  // warp, then CTA (warp 0 combines the warps' pairs)
  constexpr int NW = TOT_NT / 32;
  __shared__ double ss[NW][M][2];
  __shared__ int last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const CSum t = warp_csum(acc[m]);
    if (lane == 0) { ss[wid][m][0] = t.s; ss[wid][m][1] = t.c; }
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const CSum t = warp_csum(lane < NW ? CSum{ss[lane][m][0], ss[lane][m][1]} : CSum{0.0, 0.0});
      if (lane == 0) {
        a.partials[((long)blockIdx.x * MAXEQ + m) * 2] = t.s;
        a.partials[((long)blockIdx.x * MAXEQ + m) * 2 + 1] = t.c;
      }
    }
    if (lane == 0) {
      __threadfence();   // the partials are visible before the ticket is taken
      last = atomicAdd(&ctl->tot_ticket, 1u) == gridDim.x - 1;
    }
  }
  __syncthreads();
  if (!last) return;
  // the last CTA combines the partials of every CTA in a fixed order; a
  // thread loads all of its CTAs' pairs (L2-coherent loads, at most
  // TOT_PB CTAs per thread) before it adds them
  __threadfence();
  constexpr int TOT_PB = (TOT_BLOCKS_MAX + TOT_NT - 1) / TOT_NT;
  double pv[TOT_PB][M][2];
#pragma unroll
  for (int j = 0; j < TOT_PB; ++j) {
    const int b = threadIdx.x + j * TOT_NT;
#pragma unroll
    for (int m = 0; m < M; ++m) {
      pv[j][m][0] = b < (int)gridDim.x ? __ldcg(&a.partials[((long)b * MAXEQ + m) * 2]) : 0.0;
      pv[j][m][1] = b < (int)gridDim.x ? __ldcg(&a.partials[((long)b * MAXEQ + m) * 2 + 1]) : 0.0;
    }
  }
#pragma unroll
  for (int m = 0; m < M; ++m) {
    CSum t{0.0, 0.0};
#pragma unroll
    for (int j = 0; j < TOT_PB; ++j) t.add(pv[j][m][0], pv[j][m][1]);
    t = warp_csum(t);
    if (lane == 0) { ss[wid][m][0] = t.s; ss[wid][m][1] = t.c; }
  }
  __syncthreads();
  if (wid == 0) {
    double v[MAXEQ] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const CSum t = warp_csum(lane < NW ? CSum{ss[lane][m][0], ss[lane][m][1]} : CSum{0.0, 0.0});
      v[m] = (t.s + t.c) * a.area;
    }
    if (lane == 0) {
#pragma unroll
      for (int m = 0; m < MAXEQ; ++m) {
        if (a.mode == 0) {
          ctl->tot_cand[m] = v[m];
        } else {
          ctl->tot0[m] = v[m];
          ctl->tot[m] = v[m];
          ctl->drift[m] = 0.0;
        }
      }
      ctl->tot_ticket = 0u;   // ready for the next launch
    }
  }
}

}  // namespace scl
