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

template <class S>
__global__ void __launch_bounds__(TOT_NT) k_totals(TotalsArgs a) {
  Ctl* ctl = a.ctl;
  if (a.mode == 0 && (ctl->done || !ctl->totals)) return;
  const S* q = static_cast<const S*>(a.buf[ctl->role[a.role]]);
  const S* kap = static_cast<const S*>(a.capa);
  CSum acc[MAXEQ];
#pragma unroll
  for (int m = 0; m < MAXEQ; ++m) acc[m] = CSum{0.0, 0.0};
  const long n = (long)a.mx * a.my;
  const long step = (long)gridDim.x * blockDim.x;
  for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += step) {
    const long i = k % a.mx, j = k / a.mx;
    const long off = (a.ndim == 2 ? (j + 3) * a.pitch : 0) + i + 3;   // interior cell (i+1[, j+1])
    const double w = kap ? (double)kap[off] : 1.0;
#pragma unroll
    for (int m = 0; m < MAXEQ; ++m)
      if (m < a.meqn) acc[m].add(kap ? (double)q[(long)m * a.plane + off] * w : (double)q[(long)m * a.plane + off]);
  }
  // warp, then CTA
  __shared__ double ss[TOT_NT / 32][MAXEQ][2];
  __shared__ int last;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int m = 0; m < MAXEQ; ++m) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double os = __shfl_down_sync(0xffffffffu, acc[m].s, o);
      const double oc = __shfl_down_sync(0xffffffffu, acc[m].c, o);
      acc[m].add(os, oc);
    }
    if (lane == 0) { ss[wid][m][0] = acc[m].s; ss[wid][m][1] = acc[m].c; }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int m = 0; m < MAXEQ; ++m) {
      CSum t{0.0, 0.0};
      for (int w = 0; w < TOT_NT / 32; ++w) t.add(ss[w][m][0], ss[w][m][1]);
      a.partials[((long)blockIdx.x * MAXEQ + m) * 2] = t.s;
      a.partials[((long)blockIdx.x * MAXEQ + m) * 2 + 1] = t.c;
    }
    __threadfence();   // the partials are visible before the ticket is taken
    last = atomicAdd(&ctl->tot_ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  // the last CTA combines the partials of every CTA in a fixed order
  __threadfence();
  const volatile double* P = a.partials;
#pragma unroll
  for (int m = 0; m < MAXEQ; ++m) {
    CSum t{0.0, 0.0};
    for (int b = threadIdx.x; b < (int)gridDim.x; b += TOT_NT) t.add(P[((long)b * MAXEQ + m) * 2], P[((long)b * MAXEQ + m) * 2 + 1]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double os = __shfl_down_sync(0xffffffffu, t.s, o);
      const double oc = __shfl_down_sync(0xffffffffu, t.c, o);
      t.add(os, oc);
    }
    if (lane == 0) { ss[wid][m][0] = t.s; ss[wid][m][1] = t.c; }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int m = 0; m < MAXEQ; ++m) {
      CSum t{0.0, 0.0};
      for (int w = 0; w < TOT_NT / 32; ++w) t.add(ss[w][m][0], ss[w][m][1]);
      const double v = m < a.meqn ? (t.s + t.c) * a.area : 0.0;
      if (a.mode == 0) {
        ctl->tot_cand[m] = v;
      } else {
        ctl->tot0[m] = v;
        ctl->tot[m] = v;
        ctl->drift[m] = 0.0;
      }
    }
    ctl->tot_ticket = 0u;   // ready for the next launch
  }
}

}  // namespace scl
