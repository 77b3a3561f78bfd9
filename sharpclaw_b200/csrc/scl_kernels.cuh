// scl_kernels.cuh -- fused SSP-RK stage kernels for the SharpClaw WENO step.
//
// One launch = one Runge-Kutta stage over the whole grid: bc (as ghost
// images written with the stage output), src (dq starts at zero), the
// reconstruction + Riemann solves of flux1/flux2, the CFL maximum, the total
// fluctuation and the Shu-Osher stage combination of src/sharpclaw.f90.  No
// intermediate array (ql, qr, amdq, apdq, wave, s, dq) touches HBM: a CTA
// stages its cells plus ghosts in shared memory, solves one interface per
// thread into shared memory, then updates one cell per thread.
#pragma once
#include <cooperative_groups.h>
#include <type_traits>

#include "scl_common.cuh"
#include "scl_plugins.cuh"
#include "scl_tma.cuh"
#include "scl_totals.cuh"
#include "scl_weno.cuh"

namespace scl {

// Arithmetic forms (template parameter PREC): SCL_FP64 / SCL_FP64_STRICT
// (double throughout; strict is the same source compiled without FMA
// contraction), SCL_MIXED (float reconstruction and Riemann solves on
// double state), SCL_FP32 (float state).
template <int PREC> struct Prec;
// FD: the FP64 form divides through reciprocals (within a few ulp of the
// reference's divisions); the strict form keeps the reference's operations.
template <> struct Prec<SCL_FP64> { using R = double; using S = double; using A = double; static constexpr bool EXACT = true, FD = true; };
template <> struct Prec<SCL_FP64_STRICT> { using R = double; using S = double; using A = double; static constexpr bool EXACT = true, FD = false; };
template <> struct Prec<SCL_MIXED> { using R = float; using S = double; using A = double; static constexpr bool EXACT = false, FD = false; };
template <> struct Prec<SCL_FP32> { using R = float; using S = float; using A = float; static constexpr bool EXACT = false, FD = false; };



// ---------------------------------------------------------------------------
// Shu-Osher stage combinations (src/sharpclaw.f90), evaluated in A precision.
// DIV3: divide by 3 as the reference does (strict form); otherwise multiply
// by 1/3 (within an ulp).
// ---------------------------------------------------------------------------
template <class A, bool DIV3 = true>
__device__ __forceinline__ void combine(int kind, A q, A qo, A dq, A& out, A& out2) {
  switch (kind) {
    case SK_ADD: out = q + dq; break;                                            // :264,:356
    case SK_SSP33_2: out = (A)0.75 * qo + (A)0.25 * (q + dq); break;             // :365
    case SK_SSP33_3:                                                             // :374
      if constexpr (DIV3) out = (qo + (A)2.0 * (q + dq)) / (A)3.0;
      else out = (qo + (A)2.0 * (q + dq)) * (A)(1.0 / 3.0);
      break;
    case SK_ADD_SIXTH: out = q + (A)(1.0 / 6.0) * dq; break;                     // :396..455
    case SK_SSP104_5: {                                                          // :424-426
      A r2 = q + (A)(1.0 / 6.0) * dq;
      out2 = (A)0.04 * qo + (A)0.36 * r2;
      out = (A)0.6 * qo + (A)0.4 * r2;
      break;
    }
    case SK_SSP104_10: out = (qo + (A)0.6 * q) + (A)0.1 * dq; break;             // :462 (qo = r1)
    case SK_SSP22_2: out = (A)0.5 * ((qo + q) + dq); break;                      // :274
    case SK_ADD_THIRD: out = q + (A)(1.0 / 3.0) * dq; break;                     // :304,313,322
    case SK_SSP42_4: out = ((A)0.25 * qo + (A)0.75 * q) + (A)0.25 * dq; break;   // :331
    default: out = dq; break;                                                    // SK_DQ
  }
}

// ---------------------------------------------------------------------------
// Ghost images.  bc1.f90/bc2.f90 fill ghost cells from interior cells before
// every stage; here the thread that writes interior cell i also writes every
// ghost cell whose bc source is i.  The map ghost -> source is a function, so
// each ghost is written exactly once, and in 2-D the corners come out as the
// reference's x-then-y sweep leaves them.
// ---------------------------------------------------------------------------
struct Images {
  int n;
  int idx[6];
  bool neg[6];
};

// images along one direction of cell c (1-based) for normal component `mnorm`
// (0-based) of the wall condition.
__device__ __forceinline__ Images images_1d(int c, int n, int bl, int br) {
  Images im;
  im.n = 1; im.idx[0] = c; im.neg[0] = false;
  if (bl == 1 && c == 1) { for (int g = -2; g <= 0; ++g) { im.idx[im.n] = g; im.neg[im.n++] = false; } }
  if (bl == 2 && c >= n - 2) { im.idx[im.n] = c - n; im.neg[im.n++] = false; }
  if (bl == 3 && c <= 3) { im.idx[im.n] = 1 - c; im.neg[im.n++] = true; }
  if (br == 1 && c == n) { for (int g = n + 1; g <= n + 3; ++g) { im.idx[im.n] = g; im.neg[im.n++] = false; } }
  if (br == 2 && c <= 3) { im.idx[im.n] = c + n; im.neg[im.n++] = false; }
  if (br == 3 && c >= n - 2) { im.idx[im.n] = 2 * n + 1 - c; im.neg[im.n++] = true; }
  return im;
}

// Store the value of cell c (1..n) of component m and its ghost images (the
// images of images_1d, in its order, negated for component 1 at a wall),
// written directly: no indexed array, so no local memory.
template <class S, class A>
__device__ __forceinline__ void put_1d_img(S* base, long plane, int m, int c, int n, int bl, int br, A v) {
  S* p = base + (long)m * plane;
  p[c + 2] = (S)v;
  auto g = [&](int gi, bool neg) { p[gi + 2] = (S)((m == 1 && neg) ? -v : v); };
  if (bl == 1 && c == 1) { g(-2, false); g(-1, false); g(0, false); }
  if (bl == 2 && c >= n - 2) g(c - n, false);
  if (bl == 3 && c <= 3) g(1 - c, true);
  if (br == 1 && c == n) { g(n + 1, false); g(n + 2, false); g(n + 3, false); }
  if (br == 2 && c <= 3) g(c + n, false);
  if (br == 3 && c >= n - 2) g(2 * n + 1 - c, true);
}

template <class S, class A>
__device__ __forceinline__ void put_2d(S* base, long plane, long pitch, int m, int i, int j,
                                       const Images& ix, const Images& iy, A v) {
  S* p = base + (long)m * plane;
  for (int a = 0; a < ix.n; ++a) {
    A vx = (m == 1 && ix.neg[a]) ? -v : v;
    for (int b = 0; b < iy.n; ++b) {
      A vy = (m == 2 && iy.neg[b]) ? -vx : vx;
      p[(long)(iy.idx[b] + 2) * pitch + (ix.idx[a] + 2)] = (S)vy;
    }
  }
}

// Out-of-line entry points of the plugins for the FP32 forms (see SCL_FP32_FN).
template <class P>
__device__ SCL_FP32_FN void rp_f32(const Phys& ph, int ixy, const float* L, const float* Rt, const float* dl,
                                    const float* al, const float* ar, float* s, float* am, float* ap) {
  P::template rp<float>(ph, ixy, L, Rt, dl, al, ar, s, am, ap);
}
template <class P>
__device__ SCL_FP32_FN void tfluct_f32(const Phys& ph, int ixy, const float* L, const float* Rt,
                                        const float* dl, const float* aux, float* adq) {
  P::template tfluct<float>(ph, ixy, L, Rt, dl, aux, adq);
}
template <class P>
__device__ SCL_FP32_FN void evec_f32(const Phys& ph, int ixy, const float* qm, const float* q0,
                                      const float* am, const float* a0, float (*evl)[P::MEQN],
                                      float (*evr)[P::MEQN]) {
  P::template evec<float>(ph, ixy, qm, q0, am, a0, evl, evr);
}

// ---------------------------------------------------------------------------
// One interface c-1/2 (between cells c-1 and c) of a line: reconstruction,
// Riemann solve and the CFL contribution.  `qs(k, m)` returns cell c-3+k,
// `as(k, j)` aux field j of that cell (read only by the wave-based form).
// Results: xl = qr(c-1), xr = ql(c) (states in the exact form, offsets from
// q(c-1)/q(c) in the offset form), fluctuations amdq(c), apdq(c).
// ---------------------------------------------------------------------------
template <class P, int CD, int PREC, class QS, class AS>
__device__ __forceinline__ void solve_interface(const Phys& ph, int ixy, QS qs, AS as,
                                                const typename Prec<PREC>::R* auxm,
                                                const typename Prec<PREC>::R* aux0,
                                                typename Prec<PREC>::R xl[P::MEQN],
                                                typename Prec<PREC>::R xr[P::MEQN],
                                                typename Prec<PREC>::R amdq[P::MEQN],
                                                typename Prec<PREC>::R apdq[P::MEQN],
                                                typename Prec<PREC>::R s[P::MWAVES]) {
  using R = typename Prec<PREC>::R;
  constexpr int M = P::MEQN, MW = P::MWAVES, MA = P::MAUX;
  constexpr bool FD = Prec<PREC>::FD;
  if constexpr (Prec<PREC>::EXACT) {
    double q[6][M];
#pragma unroll
    for (int k = 0; k < 6; ++k)
#pragma unroll
      for (int m = 0; m < M; ++m) q[k][m] = (double)qs(k, m);
    if constexpr (CD == 2) {
      double evl[M][M], evr[M][M];
      P::template evec<double, FD>(ph, ixy, q[2], q[3], auxm, aux0, evl, evr);
      weno5_char_exact<M, FD>(q, evl, evr, xl, xr);
    } else if constexpr (CD == 1) {
      // waves of the cell-average Riemann problems at c-2 .. c+2 (flux1.f90:99-100)
      double w[5][MW][M], ak[6][MA > 0 ? MA : 1];
#pragma unroll
      for (int k = 0; k < 6; ++k)
#pragma unroll
        for (int j = 0; j < MA; ++j) ak[k][j] = (double)as(k, j);
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        double dk[M];
#pragma unroll
        for (int m = 0; m < M; ++m) dk[m] = q[k + 1][m] - q[k][m];
        P::template waves<double, FD>(ph, ixy, q[k], q[k + 1], dk, ak[k], ak[k + 1], w[k]);
      }
      weno5_wave_exact<M, MW, FD>(q, w, xl, xr);
    } else if constexpr (CD == 3) {
      // eigenvectors of the five interfaces c-2 .. c+2 (flux1.f90:108-110)
      double evlc[M][M], evrc[M][M], h[5][M];
      auto axk = [&](int k, double* out) {
#pragma unroll
        for (int j = 0; j < MA; ++j) out[j] = (double)as(k, j);
      };
      double a2[MA > 0 ? MA : 1], a3[MA > 0 ? MA : 1];
      axk(2, a2);
      axk(3, a3);
      P::template evec<double, FD>(ph, ixy, q[2], q[3], a2, a3, evlc, evrc);
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        double dk[M];
#pragma unroll
        for (int m = 0; m < M; ++m) dk[m] = q[k + 1][m] - q[k][m];
        if (k == 2) {
          trans_project<double, M>(evlc, evrc, dk, evlc, h[k]);
        } else {
          double evl[M][M], evr[M][M], ak0[MA > 0 ? MA : 1], ak1[MA > 0 ? MA : 1];
          axk(k, ak0);
          axk(k + 1, ak1);
          P::template evec<double, FD>(ph, ixy, q[k], q[k + 1], ak0, ak1, evl, evr);
          trans_project<double, M>(evl, evr, dk, evlc, h[k]);
        }
      }
      weno5_trans_exact<M, FD>(q, h, evrc, xl, xr);
    } else if constexpr (CD == 10) {                      // lim_type 1: tvd2
      tvd2_exact<M>(q, ph.mthlim, xl, xr);
    } else if constexpr (CD == 11) {                      // lim_type 1: tvd2_wave
      double w[3][MW][M], sc[MW], ak[4][MA > 0 ? MA : 1];
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int i = 0; i < MA; ++i) ak[j][i] = (double)as(j + 1, i);
#pragma unroll
      for (int j = 0; j < 3; ++j) {                       // interfaces c-1, c, c+1
        double dk[M];
#pragma unroll
        for (int m = 0; m < M; ++m) dk[m] = q[j + 2][m] - q[j + 1][m];
        P::template waves<double, FD>(ph, ixy, q[j + 1], q[j + 2], dk, ak[j], ak[j + 1], w[j],
                                      j == 1 ? sc : (double*)nullptr);
      }
      tvd2_wave_core<double, M, MW>(w, sc, ph.mthlim, q[2], q[3], xl, xr);
    } else if constexpr (CD == 12) {                      // lim_type 1: tvd2_char
      double evl[M][M], evr[M][M], d3[3][M];
      P::template evec<double, FD>(ph, ixy, q[2], q[3], auxm, aux0, evl, evr);
#pragma unroll
      for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int m = 0; m < M; ++m) d3[j][m] = q[j + 2][m] - q[j + 1][m];
      tvd2_char_core<double, M>(d3, evl, evr, ph.mthlim, q[2], q[3], xl, xr);
    } else if constexpr (CD == 20) {                      // lim_type 0: q2qlqr_poly
      poly3_exact<M>(q, xl, xr);
    } else if constexpr (CD == 21) {                      // lim_type 0: q2qlqr_poly_wave
      double w[3][MW][M], ak[4][MA > 0 ? MA : 1];
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int i = 0; i < MA; ++i) ak[j][i] = (double)as(j + 1, i);
#pragma unroll
      for (int j = 0; j < 3; ++j) {                       // interfaces c-1, c, c+1 (flux1.f90:73-75)
        double dk[M];
#pragma unroll
        for (int m = 0; m < M; ++m) dk[m] = q[j + 2][m] - q[j + 1][m];
        P::template waves<double, FD>(ph, ixy, q[j + 1], q[j + 2], dk, ak[j], ak[j + 1], w[j]);
      }
      poly3_wave_core<double, M, MW>(w, q[2], q[3], xl, xr);
    } else {
      weno5_exact<M, FD>(q, xl, xr);
    }
    double dl[M];
#pragma unroll
    for (int m = 0; m < M; ++m) dl[m] = xr[m] - xl[m];   // delta = ql(i) - qr(i-1)
    P::template rp<double, FD>(ph, ixy, xl, xr, dl, auxm, aux0, s, amdq, apdq);
  } else {
    float d[5][M];
#pragma unroll
    for (int k = 0; k < 5; ++k)
#pragma unroll
      for (int m = 0; m < M; ++m) d[k][m] = (float)(qs(k + 1, m) - qs(k, m));
    if constexpr (CD == 2) {
      float qm[M], q0[M], evl[M][M], evr[M][M];
#pragma unroll
      for (int m = 0; m < M; ++m) { qm[m] = (float)qs(2, m); q0[m] = (float)qs(3, m); }
      evec_f32<P>(ph, ixy, qm, q0, auxm, aux0, evl, evr);
      weno5_char_offset<M>(d, evl, evr, xl, xr);
    } else if constexpr (CD == 1) {
      float qf[6][M], w[5][MW][M], ak[6][MA > 0 ? MA : 1];
#pragma unroll
      for (int k = 0; k < 6; ++k) {
#pragma unroll
        for (int m = 0; m < M; ++m) qf[k][m] = (float)qs(k, m);
#pragma unroll
        for (int j = 0; j < MA; ++j) ak[k][j] = (float)as(k, j);
      }
#pragma unroll
      for (int k = 0; k < 5; ++k) P::template waves<float>(ph, ixy, qf[k], qf[k + 1], d[k], ak[k], ak[k + 1], w[k]);
      weno5_wave_offset<M, MW>(d, w, xl, xr);
    } else if constexpr (CD == 3) {
      float qf[6][M], ak[6][MA > 0 ? MA : 1], evlc[M][M], evrc[M][M], h[5][M];
#pragma unroll
      for (int k = 0; k < 6; ++k) {
#pragma unroll
        for (int m = 0; m < M; ++m) qf[k][m] = (float)qs(k, m);
#pragma unroll
        for (int j = 0; j < MA; ++j) ak[k][j] = (float)as(k, j);
      }
      evec_f32<P>(ph, ixy, qf[2], qf[3], ak[2], ak[3], evlc, evrc);
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        if (k == 2) {
          trans_project<float, M>(evlc, evrc, d[k], evlc, h[k]);
        } else {
          float evl[M][M], evr[M][M];
          evec_f32<P>(ph, ixy, qf[k], qf[k + 1], ak[k], ak[k + 1], evl, evr);
          trans_project<float, M>(evl, evr, d[k], evlc, h[k]);
        }
      }
      weno5_trans_offset<M>(d, h, evrc, xl, xr);
    } else if constexpr (CD == 10) {
      tvd2_offset<M>(d, ph.mthlim, xl, xr);
    } else if constexpr (CD == 11) {
      float qf[4][M], ak[4][MA > 0 ? MA : 1], w[3][MW][M], sc[MW], z[M];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int m = 0; m < M; ++m) qf[j][m] = (float)qs(j + 1, m);
#pragma unroll
        for (int i = 0; i < MA; ++i) ak[j][i] = (float)as(j + 1, i);
      }
#pragma unroll
      for (int m = 0; m < M; ++m) z[m] = 0.0f;
#pragma unroll
      for (int j = 0; j < 3; ++j)
        P::template waves<float>(ph, ixy, qf[j], qf[j + 1], d[j + 1], ak[j], ak[j + 1], w[j],
                                 j == 1 ? sc : (float*)nullptr);
      tvd2_wave_core<float, M, MW>(w, sc, ph.mthlim, z, z, xl, xr);
    } else if constexpr (CD == 12) {
      float qm[M], q0[M], evl[M][M], evr[M][M], d3[3][M], z[M];
#pragma unroll
      for (int m = 0; m < M; ++m) {
        qm[m] = (float)qs(2, m);
        q0[m] = (float)qs(3, m);
        z[m] = 0.0f;
#pragma unroll
        for (int j = 0; j < 3; ++j) d3[j][m] = d[j + 1][m];
      }
      evec_f32<P>(ph, ixy, qm, q0, auxm, aux0, evl, evr);
      tvd2_char_core<float, M>(d3, evl, evr, ph.mthlim, z, z, xl, xr);
    } else if constexpr (CD == 20) {
      poly3_offset<M>(d, xl, xr);
    } else if constexpr (CD == 21) {
      float qf[4][M], ak[4][MA > 0 ? MA : 1], w[3][MW][M], z[M];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int m = 0; m < M; ++m) qf[j][m] = (float)qs(j + 1, m);
#pragma unroll
        for (int i = 0; i < MA; ++i) ak[j][i] = (float)as(j + 1, i);
      }
#pragma unroll
      for (int m = 0; m < M; ++m) z[m] = 0.0f;
#pragma unroll
      for (int j = 0; j < 3; ++j) P::template waves<float>(ph, ixy, qf[j], qf[j + 1], d[j + 1], ak[j], ak[j + 1], w[j]);
      poly3_wave_core<float, M, MW>(w, z, z, xl, xr);
    } else {
      weno5_offset<M>(d, xl, xr);
    }
    float L[M], Rt[M], dl[M];
#pragma unroll
    for (int m = 0; m < M; ++m) {
      L[m] = (float)qs(2, m) + xl[m];
      Rt[m] = (float)qs(3, m) + xr[m];
      dl[m] = d[2][m] + (xr[m] - xl[m]);   // (q(c)-q(c-1)) + (el - er)
    }
    rp_f32<P>(ph, ixy, L, Rt, dl, auxm, aux0, s, amdq, apdq);
  }
}

// Total fluctuation of cell c from its edge values (flux1.f90:136-188):
// returns the bracket that multiplies -dtdx, in the reference's order.
template <class P, int TF, int PREC>
__device__ __forceinline__ void cell_bracket(const Phys& ph, int ixy, const typename Prec<PREC>::R* qc,
                                             const typename Prec<PREC>::R* auxc,
                                             const typename Prec<PREC>::R* qlc,   // ql(c)
                                             const typename Prec<PREC>::R* qrc,   // qr(c)
                                             const typename Prec<PREC>::R* apdq_c,
                                             const typename Prec<PREC>::R* amdq_c1,
                                             typename Prec<PREC>::R* br) {
  using R = typename Prec<PREC>::R;
  constexpr int M = P::MEQN;
  R L[M], Rt[M], dl[M];
#pragma unroll
  for (int m = 0; m < M; ++m) {
    if constexpr (Prec<PREC>::EXACT) {
      L[m] = qlc[m]; Rt[m] = qrc[m]; dl[m] = qrc[m] - qlc[m];
    } else {
      L[m] = qc[m] + qlc[m]; Rt[m] = qc[m] + qrc[m]; dl[m] = qrc[m] - qlc[m];
    }
  }
  if constexpr (TF == 1) {
    R adq[M];
    if constexpr (Prec<PREC>::EXACT) P::template tfluct<R, Prec<PREC>::FD>(ph, ixy, L, Rt, dl, auxc, adq);
    else tfluct_f32<P>(ph, ixy, L, Rt, dl, auxc, adq);
#pragma unroll
    for (int m = 0; m < M; ++m) br[m] = (apdq_c[m] + adq[m]) + amdq_c1[m];       // :151-152
  } else {
    R s2[P::MWAVES], am2[M], ap2[M];
    const R* a0 = auxc + (tfluct_nb<P>::value ? P::MAUX : 0);   // the cell's own aux
    if constexpr (Prec<PREC>::EXACT) P::template rp<R, Prec<PREC>::FD>(ph, ixy, L, Rt, dl, a0, a0, s2, am2, ap2);  // :181-182
    else rp_f32<P>(ph, ixy, L, Rt, dl, a0, a0, s2, am2, ap2);
#pragma unroll
    for (int m = 0; m < M; ++m) br[m] = ((amdq_c1[m] + apdq_c[m]) + am2[m]) + ap2[m];  // :185-186
  }
}

template <class R>
__device__ __forceinline__ R load_aux(const void* aux, long off) {
  return (R)static_cast<const R*>(aux)[off];
}

// Running CFL maximum of flux1.f90:126-133 (max over waves of
// max(dtdx(i)*s, -dtdx(i-1)*s)) and flux2.f90:47,80.  The exact forms form
// the reference's products in double.  The FP32 forms keep the largest |s|
// per direction (an exact FP32 maximum) and reduce it across the CTA in
// FP32; one thread multiplies it by dt/dx (dt/dy) in double: with one dtdx
// per direction max(dtdx s, -dtdx s) = dtdx |s|, and since rounding is
// monotonic that product equals the maximum of the per-interface FP64
// products, so the CFL number is FP64.  Capacity grids (a dtdx per cell)
// form each product in FP64 and keep it rounded up to FP32 (an upper bound
// within an FP32 ulp).  NaN propagates.
template <class R>
struct CflMax {
  double v = 0.0;          // exact forms
  float sx = 0.f, sy = 0.f;  // FP32 forms: max |s| (or capacity products) along x / y
  template <int MW>
  __device__ __forceinline__ void add(const R* s, double d_c, double d_m, bool per_cell, bool isx) {
    if constexpr (std::is_same_v<R, double>) {
#pragma unroll
      for (int w = 0; w < MW; ++w) v = nanmax(v, nanmax(d_c * s[w], -d_m * s[w]));
    } else {
      float m = isx ? sx : sy;
      if (per_cell) {
#pragma unroll
        for (int w = 0; w < MW; ++w) {
          const double sw = (double)s[w];
          m = nanmax(m, __double2float_ru(nanmax(d_c * sw, -d_m * sw)));
        }
      } else {
#pragma unroll
        for (int w = 0; w < MW; ++w) m = nanmax(m, fabsf(s[w]));
      }
      if (isx) sx = m; else sy = m;
    }
  }
};

// CTA maximum of the threads' CflMax into one double, in thread 0 (the
// other threads' return value is unused).  sred: NT/32 doubles, fred: 2 x
// NT/32 floats of shared memory.  Contains the CTA barrier bar.sync and
// returns the OR of `bad` over the CTA in *anybad.  Y: the y direction is
// used (2-D).
template <class R, int NT, bool Y = true>
__device__ __forceinline__ double cfl_cta_max(const CflMax<R>& c, double dtdx, double dtdy, bool per_cell,
                                              double* sred, float (*fred)[NT / 32], int bad, int* anybad) {
  const int tid = threadIdx.x;
  if constexpr (std::is_same_v<R, double>) {
    const double w = warp_max(c.v);
    if ((tid & 31) == 0) sred[tid >> 5] = w;
    *anybad = __syncthreads_or(bad);
    double v = 0.0;
    if (tid < 32) v = warp_max((tid < NT / 32) ? sred[tid] : 0.0);
    return v;
  } else {
    const float wx = warp_max(c.sx);
    float wy = 0.f;
    if constexpr (Y) wy = warp_max(c.sy);
    if ((tid & 31) == 0) { fred[0][tid >> 5] = wx; fred[1][tid >> 5] = wy; }
    *anybad = __syncthreads_or(bad);
    float mx = 0.f, my = 0.f;
    if (tid < 32) {
      mx = warp_max((tid < NT / 32) ? fred[0][tid] : 0.f);
      if constexpr (Y) my = warp_max((tid < NT / 32) ? fred[1][tid] : 0.f);
    }
    return per_cell ? nanmax((double)mx, (double)my) : nanmax(dtdx * (double)mx, dtdy * (double)my);
  }
}

// ---------------------------------------------------------------------------
// One line (a 1-D grid, a batched instance, or a line of a 2-D plugin) as a
// stage sees it: buffers already resolved through the controller's roles.
// ---------------------------------------------------------------------------
template <class S>
struct Line {
  Ctl* ctl;            // controller of this line (dt, stage CFL slots, status)
  const S* qin;        // stage input (read with halo)
  const S* qo;         // pointwise extra input (qold or r1), or nullptr
  S* out;              // stage output (with ghost images), unused for SK_DQ
  S* out2;             // second output (SSP104 stage 5), or nullptr
  double* dq_out;      // SK_DQ output
  const void* aux;     // aux planes, or nullptr
  int mx;
  long plane;          // component stride (elements)
  double dx;
  int bl, br;          // mthbc of the two ends
  int mcapa, kind, stage, ixy;
  int src = SCL_SRC_NONE;  // source-term hook and the grid's lower edge (radial hook)
  double xlower = 0.0;
  double dt = 0.0;         // the controller's dt for this step (read with the roles)
  unsigned long long wait_ns = MBAR_LIMIT_NS;   // bound of a bulk-copy wait
  unsigned int tx_extra = 0;                    // test hook (StageArgs::tx_extra)
  double dtdx = 0.0;       // dt/dx of the step (shared-memory resident runs)
};

// A tile of a cluster-resident run whose registers live in shared memory
// (k_run1d).  The CTA of cluster rank r keeps, for each of the NROLES
// physical buffers and each component, a row of rw = cspan + 6 elements:
// the cspan cells of its chunk (cells 1 + r*cspan .. (r+1)*cspan, the tiles
// r*T .. r*T + T - 1) and three halo cells on each side.  Row element k
// holds element offset r*cspan + k of the buffer (cell r*cspan + k - 2), so
// every row element equals the element of the buffer in global memory that
// the step graphs would hold at that point of the run: a stage stores each
// cell it updates in its own row and in every neighbour row that holds the
// cell as a halo, and each ghost image in every row that holds the ghost
// cell.  The row base of (buffer b, component m) is element (b*MEQN + m)*rw
// of the dynamic shared memory.
struct ResView {
  int rw;             // elements per row
  int rsh;            // row element of this tile's first window element (tile index in the chunk x (NT-1))
  int cspan;          // cells per chunk
  int rank, rlast;    // this CTA's cluster rank; the rank of the last chunk
  int bin, bqo, bout, bout2;   // physical buffers of the stage input, pointwise input, outputs (-1: none)
};

// Store the value of cell c (1..mx) of component m in the row `row` (this
// CTA's row of the output buffer) and in every other CTA's row of that
// buffer that holds the cell: the neighbours' halos, and, when `edge`, the
// rows that hold its ghost images (the images of images_1d, negated as
// put_1d_img negates).  No division and no indexed local array: only the
// chunk-edge threads do more than the first store.  (An out-of-line image
// store measured slower: the few threads that call it are on the critical
// path of the stage's cluster barrier.)
template <class S, class A>
__device__ __forceinline__ void res_put(const ResView& v, S* row, int m, int c, int mx, int bl, int br, bool edge,
                                        A val) {
  const int cf = v.rank * v.cspan;   // the chunk's cells are cf+1 .. cf+cspan
  const S x = (S)val;
  row[c + 2 - cf] = x;
  const bool lo = v.rank > 0 && c <= cf + 3;                   // in the left neighbour's right halo
  const bool hi = v.rank < v.rlast && c > cf + v.cspan - 3;    // in the right neighbour's left halo
  if (!lo && !hi && !edge) return;
  cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
  if (lo) *cl.map_shared_rank(row + (c + 2 - cf + v.cspan), v.rank - 1) = x;
  if (hi) *cl.map_shared_rank(row + (c + 2 - cf - v.cspan), v.rank + 1) = x;
  if (edge) {
    // ghost cell g: the first chunk's row (g <= 0), or the last chunk's row
    // and the row before it when g lies in that row's right halo
    auto ghost = [&](int g, bool neg) {
      const S y = (S)((m == 1 && neg) ? -val : val);
      if (g <= 0) {
        *cl.map_shared_rank(row + (g + 2), 0) = y;
        return;
      }
      const int r1 = v.rlast;
      *cl.map_shared_rank(row + (g + 2 - r1 * v.cspan), r1) = y;
      if (r1 > 0 && g + 2 - (r1 - 1) * v.cspan < v.rw) *cl.map_shared_rank(row + (g + 2 - (r1 - 1) * v.cspan), r1 - 1) = y;
    };
    if (bl == 1 && c == 1) { ghost(-2, false); ghost(-1, false); ghost(0, false); }
    if (bl == 2 && c >= mx - 2) ghost(c - mx, false);
    if (bl == 3 && c <= 3) ghost(1 - c, true);
    if (br == 1 && c == mx) { ghost(mx + 1, false); ghost(mx + 2, false); ghost(mx + 3, false); }
    if (br == 2 && c <= 3) ghost(c + mx, false);
    if (br == 3 && c >= mx - 2) ghost(2 * mx + 1 - c, true);
  }
}

// The source-term hooks, src(q,dq,aux,t,dt) of the app (src/1d/step1d.f90:23):
// dq of cell c (1-based) from the stage input (h, hu) and the step's dt, in
// the written evaluation order.
//   SCL_SRC_RADIAL_SW      1dRadialSymm-qwave/src1.f90:24-28
//   SCL_SRC_BATHYMETRY_SW  1dPerturbSteady/src1.f90:31-34, b = aux(:,1)
template <class A, class S>
__device__ __forceinline__ void source_1d(int kind, const Phys& ph, double xlower, double dx, double dt,
                                          int c, A h, A hu, const void* aux, A* out) {
  if (kind == SCL_SRC_RADIAL_SW) {
    const A rad = (A)(xlower + ((double)c - 0.5) * dx);
    out[0] = -(((A)dt * hu) / rad);
    out[1] = -((((A)dt * (hu * hu)) / h) / rad);
  } else {
    const S* b = static_cast<const S*>(aux);
    const A db = (A)b[c + 2] - (A)b[c + 1];
    out[0] = (A)0;
    out[1] = -(((((A)ph.grav * h) * db) / (A)dx) * (A)dt);
  }
}

template <class P, int PREC, int NT>
struct Tile1DSmem {
  using S = typename Prec<PREC>::S;
  static constexpr int AL = 16 / (int)sizeof(S);                  // elements per 16 bytes
  static constexpr int SQW = (NT + 5 + AL - 1 + AL - 1) / AL * AL;  // staged window incl. alignment slack
  __align__(16) S sq[P::MEQN][SQW];
  typename Prec<PREC>::R rec[4][P::MEQN][NT];   // 0: qr(c-1)  1: ql(c)  2: amdq(c)  3: apdq(c)
  double sred[NT / 32];
  float fred[2][NT / 32];
  double dtdx;   // dt/dx, one division per tile
  uint64_t bar;  // completion of the tile's bulk copies (TMA staging)
  double tsum[NT / 32][MAXEQ][2];   // per-warp (sum, error) of the tile's outputs (TOT)
};

// One tile of a 1-D stage: the CTA solves interfaces c = c0 .. c0+NT-1 and
// updates cells c0 .. c0+NT-2; neighbouring tiles both solve the interface on
// their common edge (1/NT redundant work).  Ends with a CTA-wide barrier, so
// a CTA may run tiles back to back.
//
// Staging: the cells c0-3 .. c0+NT+1 of every component (offsets c0-1 ..
// c0+NT+3).  TMA: thread 0 copies the window from the 16-byte boundary at or
// below offset c0-1 with one bulk copy per plane, completed on sm.bar (phase
// `parity`; the caller initialised the barrier), and the stencil reads are
// shifted by sh = (c0-1) - that boundary.  Otherwise the threads load it.
// A thread whose bounded wait for the copies runs out raises
// SCL_STATUS_TIMEOUT (the controller then stops the run and discards the
// step), waits once more, bounded, for copies still in flight, and goes on.
//
// TOT: also add the conserved totals of the tile's outputs (sum over its
// cells of the stored value, times the capacity when mcapa > 0) to the CTA's
// running (sum, error) pairs tot2[m] with compensated sums (scl_totals.cuh).
template <class P, int CD, int TF, int PREC, int NT, bool TMA = false, bool TOT = false>
__device__ __forceinline__ void stage1d_tile(const Line<typename Prec<PREC>::S>& L, const Phys& ph,
                                             int c0, Tile1DSmem<P, PREC, NT>& sm, uint32_t parity = 0,
                                             double (*tot2)[2] = nullptr) {
  using R = typename Prec<PREC>::R;
  using S = typename Prec<PREC>::S;
  using Ac = typename Prec<PREC>::A;
  using Sm = Tile1DSmem<P, PREC, NT>;
  constexpr int M = P::MEQN, MW = P::MWAVES, MA = P::MAUX;
  const int tid = threadIdx.x;
  const int mx = L.mx;
  const double dt = L.dt;
  int sh = 0;
  // the window element j (0 .. NT+4) of component m of the stage input
  auto qwin = [&](int m, int j) -> S { return sm.sq[m][sh + j]; };
  if constexpr (TMA) {
    const int a0 = (c0 - 1) / Sm::AL * Sm::AL;   // c0 >= 1
    sh = c0 - 1 - a0;
    if (tid == 0) {
      const int hend = (mx + 6 + Sm::AL - 1) / Sm::AL * Sm::AL;   // <= plane (host-checked)
      const int hi = a0 + Sm::SQW < hend ? a0 + Sm::SQW : hend;
      const uint32_t bytes = (uint32_t)(hi - a0) * (uint32_t)sizeof(S);
      sm.dtdx = dt / L.dx;
      fence_proxy_async_smem();   // earlier reads of the window come before the copies' writes
      mbar_arrive_expect_tx(&sm.bar, bytes * M + L.tx_extra);
#pragma unroll
      for (int m = 0; m < M; ++m) bulk_g2s(&sm.sq[m][0], L.qin + (long)m * L.plane + a0, bytes, &sm.bar);
    }
    if (!mbar_wait_bounded(&sm.bar, parity, L.wait_ns)) {
      atomicOr(&L.ctl->status, SCL_STATUS_TIMEOUT);
      mbar_wait_bounded(&sm.bar, parity, L.wait_ns);   // let copies still in flight land
    }
  } else {
    if (tid == 0) sm.dtdx = dt / L.dx;
    for (int k = tid; k < NT + 5; k += NT) {
      const long g = (long)c0 - 1 + k;
      const bool ok = g < (long)mx + 6;
#pragma unroll
      for (int m = 0; m < M; ++m) sm.sq[m][k] = ok ? L.qin[(long)m * L.plane + g] : (S)1;
    }
    __syncthreads();
  }
  const double dtdx0 = sm.dtdx;

  // ---- interface phase ----
  CflMax<R> cfl;
  int bad = 0;   // a non-finite stage output (reported through ctl->status)
  [[maybe_unused]] CSum tacc[M];
  if constexpr (TOT) {
#pragma unroll
    for (int m = 0; m < M; ++m) tacc[m] = CSum{0.0, 0.0};
  }
  {
    const int c = c0 + tid;
    if (c <= mx + 1) {
      R auxm[MA > 0 ? MA : 1], aux0[MA > 0 ? MA : 1];
#pragma unroll
      for (int k = 0; k < MA; ++k) {
        auxm[k] = load_aux<S>(L.aux, (long)k * L.plane + c + 1);
        aux0[k] = load_aux<S>(L.aux, (long)k * L.plane + c + 2);
      }
      auto qs = [&](int k, int m) -> S { return qwin(m, tid + k); };
      auto as = [&](int k, int j) -> R { return load_aux<S>(L.aux, (long)j * L.plane + c - 1 + k); };
      R xl[M], xr[M], am[M], ap[M], s[MW];
      solve_interface<P, CD, PREC>(ph, L.ixy, qs, as, auxm, aux0, xl, xr, am, ap, s);
#pragma unroll
      for (int m = 0; m < M; ++m) {
        sm.rec[0][m][tid] = xl[m]; sm.rec[1][m][tid] = xr[m];
        sm.rec[2][m][tid] = am[m]; sm.rec[3][m][tid] = ap[m];
      }
      // flux1.f90:126-133: max(dtdx(i)*s, -dtdx(i-1)*s)
      double dtdx_c = dtdx0, dtdx_m = dtdx0;
      if (L.mcapa > 0) {
        const S* cap = static_cast<const S*>(L.aux) + (long)(L.mcapa - 1) * L.plane;
        dtdx_c = dt / (L.dx * (double)cap[c + 2]);
        dtdx_m = dt / (L.dx * (double)cap[c + 1]);
      }
      cfl.template add<MW>(s, dtdx_c, dtdx_m, L.mcapa > 0, true);
    }
  }
  __syncthreads();

  // ---- cell phase ----
  {
    const int c = c0 + tid;
    if (tid < NT - 1 && c <= mx) {
      R qc[M], qlc[M], qrc[M], apc[M], amc1[M], br[M];
#pragma unroll
      for (int m = 0; m < M; ++m) {
        qc[m] = (R)qwin(m, tid + 3);
        qlc[m] = sm.rec[1][m][tid];
        apc[m] = sm.rec[3][m][tid];
        qrc[m] = sm.rec[0][m][tid + 1];
        amc1[m] = sm.rec[2][m][tid + 1];
      }
      // the cell's aux (and, for TFLUCT_NB plugins, its neighbours' on both sides)
      constexpr int NB = tfluct_nb<P>::value ? 3 : 1;
      R auxc[NB * (MA > 0 ? MA : 1)];
#pragma unroll
      for (int j = 0; j < NB; ++j)
#pragma unroll
        for (int k = 0; k < MA; ++k)
          auxc[j * MA + k] = load_aux<S>(L.aux, (long)k * L.plane + c + 2 + j - (NB - 1) / 2);
      cell_bracket<P, TF, PREC>(ph, L.ixy, qc, auxc, qlc, qrc, apc, amc1, br);
      double dtdx_c = dtdx0;
      if (L.mcapa > 0) {
        const S* cap = static_cast<const S*>(L.aux) + (long)(L.mcapa - 1) * L.plane;
        dtdx_c = dt / (L.dx * (double)cap[c + 2]);
      }
      // dq starts from the source term (zero without one) and loses the
      // fluctuations, flux1.f90:150-152 / 184-187
      Ac srcv[M];
      const bool has_src = L.src != SCL_SRC_NONE;
      if constexpr (M == 2) {
        if (has_src)
          source_1d<Ac, S>(L.src, ph, L.xlower, L.dx, dt, c, (Ac)qwin(0, tid + 3), (Ac)qwin(1, tid + 3),
                           L.aux, srcv);
      }
      auto dq_of = [&](int m) -> Ac {
        if constexpr (M == 2) {
          if (has_src) {
            if constexpr (std::is_same_v<R, Ac>) return srcv[m] - (R)dtdx_c * br[m];
            else return srcv[m] + (Ac)((R)0 - (R)dtdx_c * br[m]);
          }
        }
        return (Ac)((R)0 - (R)dtdx_c * br[m]);
      };
      const int kind = L.kind;
      if (kind == SK_DQ) {
#pragma unroll
        for (int m = 0; m < M; ++m) L.dq_out[(long)m * L.plane + c + 2] = (double)dq_of(m);
      } else {
        const bool edge = c <= 3 || c >= mx - 2;   // only these cells have ghost images
#pragma unroll
        for (int m = 0; m < M; ++m) {
          Ac dqv = dq_of(m);
          Ac qv = (Ac)qwin(m, tid + 3);
          Ac qov = L.qo ? (Ac)L.qo[(long)m * L.plane + c + 2] : (Ac)0;
          Ac o1, o2 = (Ac)0;
          combine<Ac, PREC == SCL_FP64_STRICT>(kind, qv, qov, dqv, o1, o2);
          bad |= !isfinite(o1);
          if constexpr (TOT) {
            const double v = (double)(S)o1;
            if (L.mcapa > 0)
              tacc[m].add(v * (double)static_cast<const S*>(L.aux)[(long)(L.mcapa - 1) * L.plane + c + 2]);
            else
              tacc[m].add(v);
          }
          if (edge) put_1d_img<S, Ac>(L.out, L.plane, m, c, mx, L.bl, L.br, o1);
          else L.out[(long)m * L.plane + c + 2] = (S)o1;
          if (L.out2) L.out2[(long)m * L.plane + c + 2] = (S)o2;
        }
      }
    }
  }

  // ---- CFL reduction: warp max, block max, one atomic per tile ----
  if constexpr (TOT) {
#pragma unroll
    for (int m = 0; m < M; ++m) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double os = __shfl_down_sync(0xffffffffu, tacc[m].s, o);
        const double oc = __shfl_down_sync(0xffffffffu, tacc[m].c, o);
        tacc[m].add(os, oc);
      }
      if ((tid & 31) == 0) { sm.tsum[tid >> 5][m][0] = tacc[m].s; sm.tsum[tid >> 5][m][1] = tacc[m].c; }
    }
  }
  int anybad = 0;
  const double v = cfl_cta_max<R, NT, false>(cfl, dtdx0, dtdx0, L.mcapa > 0, sm.sred, sm.fred, bad, &anybad);
  if (tid < 32) {
    if (tid == 0) {
      atomic_max_nonneg(&L.ctl->stage_cfl[L.stage], v);
      if (anybad) atomicOr(&L.ctl->status, SCL_STATUS_NONFINITE);
      if constexpr (TOT) {
#pragma unroll
        for (int m = 0; m < M; ++m) {
          CSum t{tot2[m][0], tot2[m][1]};
          for (int w = 0; w < NT / 32; ++w) t.add(sm.tsum[w][m][0], sm.tsum[w][m][1]);
          tot2[m][0] = t.s;
          tot2[m][1] = t.c;
        }
      }
    }
  }
}

// A value the compiler must treat as opaque: no multiply-add contraction
// across it.  The step graphs pass the interface results through shared
// memory between the interface and the cell phase, which keeps the cell
// phase's additions from fusing with the interface phase's products; a
// resident tile that keeps them in registers passes them through this (an
// empty volatile asm with a register operand: no instruction, but the
// compiler can neither see that the result equals the operand nor move the
// point where the value is fixed; a non-volatile one let the FP64 form
// differ from the graphs in the last bit again).
__device__ __forceinline__ float opaque(float x) {
  asm volatile("" : "+f"(x));
  return x;
}
__device__ __forceinline__ double opaque(double x) {
  asm volatile("" : "+d"(x));
  return x;
}

// The interface results one thread of a resident tile needs for its cell c:
// ql(c), apdq(c) from interface c and qr(c), amdq(c+1) from interface c+1.
template <class R, int M>
struct ResIface {
  R qlc[M], apc[M], qrc[M], amc1[M];
};

// Both interfaces of cell c = c0 + tid from the rows of buffer `bin`
// (window element rsh + tid + j + k is cell c - 3 + j + k), with their CFL
// contributions added to cfl when CFL.  GEN: the grid may have a capacity
// field (false: the caller checked that it has none).
template <class P, int CD, int PREC, bool GEN>
__device__ __forceinline__ void res_ifaces(const Line<typename Prec<PREC>::S>& L, const Phys& ph, int c,
                                           const ResView& rv, int bin, bool CFL,
                                           CflMax<typename Prec<PREC>::R>& cfl,
                                           ResIface<typename Prec<PREC>::R, P::MEQN>& f) {
  using R = typename Prec<PREC>::R;
  using S = typename Prec<PREC>::S;
  constexpr int M = P::MEQN, MW = P::MWAVES, MA = P::MAUX;
  const int tid = threadIdx.x;
  const double dt = L.dt;
  const double dtdx0 = L.dtdx;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const S* qin = reinterpret_cast<const S*>(smem_raw) + (long)bin * M * rv.rw;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const int ci = c + j;   // interface ci-1/2
    R auxm[MA > 0 ? MA : 1], aux0[MA > 0 ? MA : 1];
#pragma unroll
    for (int k = 0; k < MA; ++k) {
      auxm[k] = load_aux<S>(L.aux, (long)k * L.plane + ci + 1);
      aux0[k] = load_aux<S>(L.aux, (long)k * L.plane + ci + 2);
    }
    auto qs = [&](int k, int m) -> S { return qin[(long)m * rv.rw + rv.rsh + tid + j + k]; };
    auto as = [&](int k, int jj) -> R { return load_aux<S>(L.aux, (long)jj * L.plane + ci - 1 + k); };
    R xl[M], xr[M], am[M], ap[M], s[MW];
    solve_interface<P, CD, PREC>(ph, L.ixy, qs, as, auxm, aux0, xl, xr, am, ap, s);
#pragma unroll
    for (int m = 0; m < M; ++m) {
      if (j == 0) { f.qlc[m] = opaque(xr[m]); f.apc[m] = opaque(ap[m]); }
      else { f.qrc[m] = opaque(xl[m]); f.amc1[m] = opaque(am[m]); }
    }
    if (CFL) {
      // flux1.f90:126-133: max(dtdx(i)*s, -dtdx(i-1)*s); capacity grids are
      // the rare case (kept off the common path's registers)
      if (GEN && __builtin_expect(L.mcapa > 0, 0)) {
        const S* cap = static_cast<const S*>(L.aux) + (long)(L.mcapa - 1) * L.plane;
        const double dtdx_c = dt / (L.dx * (double)cap[ci + 2]);
        const double dtdx_m = dt / (L.dx * (double)cap[ci + 1]);
        cfl.template add<MW>(s, dtdx_c, dtdx_m, true, true);
      } else {
        cfl.template add<MW>(s, dtdx0, dtdx0, false, true);
      }
    }
  }
}

// One tile of a stage of a shared-memory resident run (k_run1d): the cells
// c0 .. c0+NT-2 (<= mx) of the rows of `rv`.  Thread tid owns cell
// c = c0 + tid and solves both of its interfaces, c and c+1 (the next thread
// solves c+1 again as its left interface), so the tile needs no record in
// shared memory and no barrier: its input rows are complete once the cluster
// barrier that ended the previous stage has passed, and its outputs go to
// the rows (res_put: halos and ghost images included).  Every interface,
// cell bracket, source term and combination is the code and the operands of
// stage1d_tile, so the outputs are those of the step graphs bit for bit.
// use_pre: take the thread's interface results from pre, already solved
// from the stage input (res_ifaces).  GEN: the run may have a capacity field
// or a stage with a second output (false: the caller checked that it has
// neither, and their code is left out).
//
// CFL: the stage's CFL number and non-finite flag are reduced over each
// warp and combined into part->stage_cfl[stage] / part->status by one atomic
// per warp (the maximum is exact: dt/dx times a float and the conversions
// are monotonic).  A resident run asks for them in the last stage only (CFL;
// never with pre): the controller judges a step by its last stage, and a
// non-finite output of an earlier stage reaches the last stage's output in
// the same cell through the pointwise combinations.
template <class P, int CD, int TF, int PREC, int NT, bool GEN>
__device__ __forceinline__ void stage1d_res(const Line<typename Prec<PREC>::S>& L, const Phys& ph, int c0,
                                            const ResView& rv, bool CFL, Ctl* part,
                                            const ResIface<typename Prec<PREC>::R, P::MEQN>& pre, bool use_pre) {
  using R = typename Prec<PREC>::R;
  using S = typename Prec<PREC>::S;
  using Ac = typename Prec<PREC>::A;
  constexpr int M = P::MEQN, MA = P::MAUX;
  const int tid = threadIdx.x;
  const int mx = L.mx;
  const double dt = L.dt;
  const double dtdx0 = L.dtdx;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto rrow = [&](int b, int m) -> S* { return reinterpret_cast<S*>(smem_raw) + ((long)b * M + m) * rv.rw; };
  const S* qin = rrow(rv.bin, 0);
  // window element j (0 .. NT+4) of component m of the stage input
  auto qwin = [&](int m, int j) -> S { return qin[(long)m * rv.rw + rv.rsh + j]; };
  const int c = c0 + tid;
  const bool own = tid < NT - 1 && c <= mx;
  CflMax<R> cfl;
  int bad = 0;
  if (own) {
    ResIface<R, M> f;
    if (use_pre) f = pre;
    else res_ifaces<P, CD, PREC, GEN>(L, ph, c, rv, rv.bin, CFL, cfl, f);
    // ---- the cell ----
    R qc[M], br[M];
#pragma unroll
    for (int m = 0; m < M; ++m) qc[m] = (R)qwin(m, tid + 3);
    constexpr int NB = tfluct_nb<P>::value ? 3 : 1;
    R auxc[NB * (MA > 0 ? MA : 1)];
#pragma unroll
    for (int j = 0; j < NB; ++j)
#pragma unroll
      for (int k = 0; k < MA; ++k)
        auxc[j * MA + k] = load_aux<S>(L.aux, (long)k * L.plane + c + 2 + j - (NB - 1) / 2);
    cell_bracket<P, TF, PREC>(ph, L.ixy, qc, auxc, f.qlc, f.qrc, f.apc, f.amc1, br);
    double dtdx_c = dtdx0;
    if (GEN && __builtin_expect(L.mcapa > 0, 0)) {
      const S* cap = static_cast<const S*>(L.aux) + (long)(L.mcapa - 1) * L.plane;
      dtdx_c = dt / (L.dx * (double)cap[c + 2]);
    }
    Ac srcv[M];
    const bool has_src = L.src != SCL_SRC_NONE;
    if constexpr (M == 2) {
      if (has_src)
        source_1d<Ac, S>(L.src, ph, L.xlower, L.dx, dt, c, (Ac)qwin(0, tid + 3), (Ac)qwin(1, tid + 3), L.aux, srcv);
    }
    auto dq_of = [&](int m) -> Ac {
      if constexpr (M == 2) {
        if (has_src) {
          if constexpr (std::is_same_v<R, Ac>) return srcv[m] - (R)dtdx_c * br[m];
          else return srcv[m] + (Ac)((R)0 - (R)dtdx_c * br[m]);
        }
      }
      return (Ac)((R)0 - (R)dtdx_c * br[m]);
    };
    const bool edge = c <= 3 || c >= mx - 2;   // only these cells have ghost images
#pragma unroll
    for (int m = 0; m < M; ++m) {
      Ac dqv = dq_of(m);
      Ac qv = (Ac)qwin(m, tid + 3);
      Ac qov = rv.bqo >= 0 ? (Ac)rrow(rv.bqo, m)[rv.rsh + tid + 3] : (Ac)0;
      Ac o1, o2 = (Ac)0;
      combine<Ac, PREC == SCL_FP64_STRICT>(L.kind, qv, qov, dqv, o1, o2);
      bad |= !isfinite(o1);
      res_put<S, Ac>(rv, rrow(rv.bout, m), m, c, mx, L.bl, L.br, edge, o1);
      if (GEN && __builtin_expect(rv.bout2 >= 0, 0)) res_put<S, Ac>(rv, rrow(rv.bout2, m), m, c, mx, 0, 0, false, o2);
    }
  }
  const int lane = tid & 31;
  if (CFL) {
    double v;
    if constexpr (std::is_same_v<R, double>) {
      v = warp_max(cfl.v);
    } else {
      const float w = warp_max(cfl.sx);
      v = (GEN && L.mcapa > 0) ? nanmax((double)w, 0.0) : nanmax(dtdx0 * (double)w, dtdx0 * 0.0);
    }
    const int anybad = __any_sync(0xffffffffu, bad);
    if (lane == 0) {
      atomic_max_nonneg(&part->stage_cfl[L.stage], v);
      if (anybad) atomicOr(&part->status, SCL_STATUS_NONFINITE);
    }
  }
}

// ---------------------------------------------------------------------------
// 1-D stage kernel: one tile per CTA over a single grid.
// ---------------------------------------------------------------------------
// The line of stage `stage` (descriptor sd) of a single 1-D grid: its
// buffers resolved through the controller's current roles.
template <class S>
__device__ __forceinline__ Line<S> line1d(const StageArgs& a, const StageDesc& sd, int stage,
                                          Ctl* ctl_override = nullptr) {
  Ctl* ctl = ctl_override ? ctl_override : a.ctl;
  Line<S> L;
  L.ctl = ctl;
  L.qin = static_cast<const S*>(pick_buf(a.buf, ctl->role[sd.in]));
  L.qo = sd.aux_in >= 0 ? static_cast<const S*>(pick_buf(a.buf, ctl->role[sd.aux_in])) : nullptr;
  L.out = sd.kind == SK_DQ ? nullptr : static_cast<S*>(pick_buf(a.buf, ctl->role[sd.out]));
  L.out2 = sd.out2 >= 0 ? static_cast<S*>(pick_buf(a.buf, ctl->role[sd.out2])) : nullptr;
  L.dq_out = a.dq_out;
  L.aux = a.aux;
  L.mx = a.mx;
  L.plane = a.plane;
  L.dx = a.dx;
  L.bl = a.mthbc[0];
  L.br = a.mthbc[1];
  L.mcapa = a.mcapa;
  L.kind = sd.kind;
  L.stage = stage;
  L.ixy = a.ixy;
  L.src = a.src_term;
  L.xlower = a.xlower;
  L.dt = ctl->dt;
  L.wait_ns = a.wait_ns ? a.wait_ns : MBAR_LIMIT_NS;   // 0: the default bound
  L.tx_extra = a.tx_extra;
  return L;
}

// TMA: the tile is staged by bulk copies (the launcher checked that every
// role buffer starts on 16 bytes and the component stride keeps the planes
// there).  MINB: CTAs per SM the registers are budgeted for (0: no bound).
template <class P, int CD, int TF, int PREC, int NT, bool TMA = false, int MINB = 0>
__global__ void __launch_bounds__(NT, MINB) k_stage1d(StageArgs a) {
  using S = typename Prec<PREC>::S;
  __shared__ Tile1DSmem<P, PREC, NT> sm;
  if (a.ctl->done) return;
  if constexpr (TMA) {
    if (threadIdx.x == 0) {
      mbar_init(&sm.bar, 1);
      fence_mbar_init();
    }
    __syncthreads();   // the barrier is initialised before any thread waits on it
  }
  stage1d_tile<P, CD, TF, PREC, NT, TMA>(line1d<S>(a, a.sd, a.stage), a.ph, 1 + blockIdx.x * (NT - 1), sm);
}

// ---------------------------------------------------------------------------
// 2-D stage kernel (flux2.f90 dimension by dimension).  A CTA owns a TX x TY
// block of cells; it stages the block plus three ghost layers, solves the
// (TX+1)*TY x-interfaces and TX*(TY+1) y-interfaces into shared memory, then
// updates each cell with dq = (0 + dq_x) + dq_y as flux2.f90:52-53,84-85
// accumulate it.
// ---------------------------------------------------------------------------
template <int TX, int TY>
struct Tile2D {
  static constexpr int WX = TX + 6, WY = TY + 6;
  static constexpr int NXI = (TX + 1) * TY, NYI = TX * (TY + 1);
};

// The block is staged by the threads (coalesced loads of every row):
// measured faster than one bulk copy per staged row, which issues dozens of
// small (176-byte) copies per CTA.  MINB: CTAs per SM the registers are
// budgeted for (0: no bound).
template <class P, int CD, int TF, int PREC, int TX, int TY, int NT, int MINB = 0>
__global__ void __launch_bounds__(NT, MINB) k_stage2d(StageArgs a) {
  using R = typename Prec<PREC>::R;
  using S = typename Prec<PREC>::S;
  using Ac = typename Prec<PREC>::A;
  using T = Tile2D<TX, TY>;
  constexpr int M = P::MEQN, MW = P::MWAVES, MA = P::MAUX;
  constexpr int WXS = T::WX;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S* sq = reinterpret_cast<S*>(smem_raw);                                  // [M][WY][WX]
  R* recx = reinterpret_cast<R*>(sq + M * WXS * T::WY);                    // [4][M][NXI]
  R* recy = recx + 4 * M * T::NXI;                                         // [4][M][NYI]
  __shared__ double sred[NT / 32];
  __shared__ float fred[2][NT / 32];

  const Ctl* ctl = a.ctl;
  if (ctl->done) return;
  const int tid = threadIdx.x;
  const int nx = a.mx, ny = a.my;
  const int i0 = 1 + blockIdx.x * TX, j0 = 1 + blockIdx.y * TY;
  const S* qin = static_cast<const S*>(pick_buf(a.buf, ctl->role[a.sd.in]));
  const double dt = ctl->dt;
  __shared__ double s_dtd[2];   // dt/dx, dt/dy: two divisions per CTA
  if (tid == 0) { s_dtd[0] = dt / a.dx; s_dtd[1] = dt / a.dy; }

  // stage the block: cells (i0-3 .. i0+TX+2, j0-3 .. j0+TY+2)
  {
    for (int k = tid; k < T::WX * T::WY; k += NT) {
      const int kx = k % T::WX, ky = k / T::WX;
      const int gi = i0 - 3 + kx, gj = j0 - 3 + ky;  // 1-based cell indices
      const bool ok = gi <= nx + 3 && gj <= ny + 3;
      const long off = (long)(gj + 2) * a.pitch + (gi + 2);
#pragma unroll
      for (int m = 0; m < M; ++m) sq[(m * T::WY + ky) * WXS + kx] = ok ? qin[(long)m * a.plane + off] : (S)1;
    }
    __syncthreads();
  }
  const double dtdx0 = s_dtd[0], dtdy0 = s_dtd[1];

  CflMax<R> cfl;
  int bad = 0;
  for (int w = tid; w < T::NXI + T::NYI; w += NT) {
    const bool isx = w < T::NXI;
    int li, lj, gi, gj;  // interface between (gi-1,gj) and (gi,gj) [x] or (gi,gj-1) and (gi,gj) [y]
    // x-interfaces: columns 0..TX-1 row by row (a half-warp reads 16
    // consecutive cells of one smem row), then column TX of every row
    if (isx) {
      if (w < TX * TY) { li = w % TX; lj = w / TX; }
      else { li = TX; lj = w - TX * TY; }
    } else { li = (w - T::NXI) % TX; lj = (w - T::NXI) / TX; }
    gi = i0 + li; gj = j0 + lj;
    const bool valid = isx ? (gi <= nx + 1 && gj <= ny) : (gi <= nx && gj <= ny + 1);
    if (!valid) continue;
    const int ixy = isx ? 1 : 2;
    R auxm[MA > 0 ? MA : 1], aux0[MA > 0 ? MA : 1];
    const long o0 = (long)(gj + 2) * a.pitch + (gi + 2);
    const long om = isx ? o0 - 1 : o0 - a.pitch;
#pragma unroll
    for (int k = 0; k < MA; ++k) {
      auxm[k] = load_aux<S>(a.aux, (long)k * a.plane + om);
      aux0[k] = load_aux<S>(a.aux, (long)k * a.plane + o0);
    }
    // local smem coordinates of cell (gi, gj): (li+3, lj+3)
    const int bx = li + 3, by = lj + 3;
    auto qs = [&](int k, int m) -> S {
      return isx ? sq[(m * T::WY + by) * WXS + (bx - 3 + k)]
                 : sq[(m * T::WY + (by - 3 + k)) * WXS + bx];
    };
    const long st = isx ? 1 : a.pitch;
    auto as = [&](int k, int j) -> R { return load_aux<S>(a.aux, (long)j * a.plane + o0 + (long)(k - 3) * st); };
    R xl[M], xr[M], am[M], ap[M], s[MW];
    solve_interface<P, CD, PREC>(a.ph, ixy, qs, as, auxm, aux0, xl, xr, am, ap, s);
    R* rec = isx ? recx : recy;
    const int n = isx ? T::NXI : T::NYI;
    const int slot = isx ? w : w - T::NXI;
#pragma unroll
    for (int m = 0; m < M; ++m) {
      rec[(0 * M + m) * n + slot] = xl[m];
      rec[(1 * M + m) * n + slot] = xr[m];
      rec[(2 * M + m) * n + slot] = am[m];
      rec[(3 * M + m) * n + slot] = ap[m];
    }
    double d_c = isx ? dtdx0 : dtdy0, d_m = d_c;
    if (a.mcapa > 0) {
      const S* cap = static_cast<const S*>(a.aux) + (long)(a.mcapa - 1) * a.plane;
      const double h = isx ? a.dx : a.dy;
      d_c = dt / (h * (double)cap[o0]);
      d_m = dt / (h * (double)cap[om]);
    }
    // interior lines only; flux2.f90 also scans the ghost lines j=0,ny+1 /
    // i=0,nx+1, which the ghost-line kernel covers.
    cfl.template add<MW>(s, d_c, d_m, a.mcapa > 0, isx);
  }
  __syncthreads();

  const int kind = a.sd.kind;
  for (int w = tid; w < TX * TY; w += NT) {
    const int li = w % TX, lj = w / TX;
    const int gi = i0 + li, gj = j0 + lj;
    if (gi > nx || gj > ny) continue;
    const long o0 = (long)(gj + 2) * a.pitch + (gi + 2);
    R auxc[MA > 0 ? MA : 1];
#pragma unroll
    for (int k = 0; k < MA; ++k) auxc[k] = load_aux<S>(a.aux, (long)k * a.plane + o0);
    R qc[M];
#pragma unroll
    for (int m = 0; m < M; ++m) qc[m] = (R)sq[(m * T::WY + lj + 3) * WXS + li + 3];
    double dx_c = dtdx0, dy_c = dtdy0;
    if (a.mcapa > 0) {
      const S* cap = static_cast<const S*>(a.aux) + (long)(a.mcapa - 1) * a.plane;
      dx_c = dt / (a.dx * (double)cap[o0]);
      dy_c = dt / (a.dy * (double)cap[o0]);
    }
    R dqs[M];
    {
      // x records follow the interface order above: (li, lj) at li + lj*TX
      // for li < TX, column TX at TX*TY + lj
      const int sa = li + lj * TX, sb = li + 1 < TX ? sa + 1 : TX * TY + lj;
      R qlc[M], qrc[M], apc[M], amc1[M], br[M];
#pragma unroll
      for (int m = 0; m < M; ++m) {
        qlc[m] = recx[(1 * M + m) * T::NXI + sa];
        apc[m] = recx[(3 * M + m) * T::NXI + sa];
        qrc[m] = recx[(0 * M + m) * T::NXI + sb];
        amc1[m] = recx[(2 * M + m) * T::NXI + sb];
      }
      cell_bracket<P, TF, PREC>(a.ph, 1, qc, auxc, qlc, qrc, apc, amc1, br);
#pragma unroll
      for (int m = 0; m < M; ++m) dqs[m] = (R)0 + ((R)0 - (R)dx_c * br[m]);
    }
    {
      const int sa = li + lj * TX, sb = sa + TX;
      R qlc[M], qrc[M], apc[M], amc1[M], br[M];
#pragma unroll
      for (int m = 0; m < M; ++m) {
        qlc[m] = recy[(1 * M + m) * T::NYI + sa];
        apc[m] = recy[(3 * M + m) * T::NYI + sa];
        qrc[m] = recy[(0 * M + m) * T::NYI + sb];
        amc1[m] = recy[(2 * M + m) * T::NYI + sb];
      }
      cell_bracket<P, TF, PREC>(a.ph, 2, qc, auxc, qlc, qrc, apc, amc1, br);
#pragma unroll
      for (int m = 0; m < M; ++m) dqs[m] = dqs[m] + ((R)0 - (R)dy_c * br[m]);
    }
    if (kind == SK_DQ) {
#pragma unroll
      for (int m = 0; m < M; ++m) a.dq_out[(long)m * a.plane + o0] = (double)dqs[m];
    } else {
      S* out = static_cast<S*>(pick_buf(a.buf, ctl->role[a.sd.out]));
      S* out2 = a.sd.out2 >= 0 ? static_cast<S*>(pick_buf(a.buf, ctl->role[a.sd.out2])) : nullptr;
      const S* qo = a.sd.aux_in >= 0 ? static_cast<const S*>(pick_buf(a.buf, ctl->role[a.sd.aux_in])) : nullptr;
      const bool edge = gi <= 3 || gi >= nx - 2 || gj <= 3 || gj >= ny - 2;
#pragma unroll
      for (int m = 0; m < M; ++m) {
        Ac qv = (Ac)sq[(m * T::WY + lj + 3) * WXS + li + 3];
        Ac qov = qo ? (Ac)qo[(long)m * a.plane + o0] : (Ac)0;
        Ac o1, o2 = (Ac)0;
        combine<Ac, PREC == SCL_FP64_STRICT>(kind, qv, qov, (Ac)dqs[m], o1, o2);
        bad |= !isfinite(o1);
        if (edge)
          put_2d<S, Ac>(out, a.plane, a.pitch, m, gi, gj, images_1d(gi, nx, a.mthbc[0], a.mthbc[1]),
                        images_1d(gj, ny, a.mthbc[2], a.mthbc[3]), o1);
        else
          out[(long)m * a.plane + o0] = (S)o1;
        if (out2) out2[(long)m * a.plane + o0] = (S)o2;
      }
    }
  }

  int anybad = 0;
  const double v = cfl_cta_max<R, NT>(cfl, dtdx0, dtdy0, a.mcapa > 0, sred, fred, bad, &anybad);
  if (tid < 32) {
    if (tid == 0) {
      atomic_max_nonneg(&a.ctl->stage_cfl[a.stage], v);
      if (anybad) atomicOr(&a.ctl->status, SCL_STATUS_NONFINITE);
    }
  }
}

// CFL contribution of the ghost lines that flux2.f90 also sweeps: x-lines
// j = 0 and ny+1 (interfaces i = 1..nx+1) and y-lines i = 0 and nx+1
// (interfaces j = 1..ny+1).  One thread per interface, global loads.
template <class P, int CD, int PREC>
__global__ void __launch_bounds__(128) k_ghost_cfl2d(StageArgs a) {
  using R = typename Prec<PREC>::R;
  using S = typename Prec<PREC>::S;
  constexpr int M = P::MEQN, MW = P::MWAVES, MA = P::MAUX;
  __shared__ double sred[4];
  __shared__ float fred[2][4];
  const Ctl* ctl = a.ctl;
  if (ctl->done) return;
  const int nx = a.mx, ny = a.my;
  const int nxl = nx + 1, nyl = ny + 1;
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  const S* qin = static_cast<const S*>(pick_buf(a.buf, ctl->role[a.sd.in]));
  const double dt = ctl->dt;
  CflMax<R> cfl;
  if (w < 2 * nxl + 2 * nyl) {
    int ixy, gi, gj;
    if (w < 2 * nxl) { ixy = 1; gi = 1 + (w % nxl); gj = (w < nxl) ? 0 : ny + 1; }
    else { const int v = w - 2 * nxl; ixy = 2; gj = 1 + (v % nyl); gi = (v < nyl) ? 0 : nx + 1; }
    const long o0 = (long)(gj + 2) * a.pitch + (gi + 2);
    const long st = (ixy == 1) ? 1 : a.pitch;
    const long om = o0 - st;
    R auxm[MA > 0 ? MA : 1], aux0[MA > 0 ? MA : 1];
#pragma unroll
    for (int k = 0; k < MA; ++k) {
      auxm[k] = load_aux<S>(a.aux, (long)k * a.plane + om);
      aux0[k] = load_aux<S>(a.aux, (long)k * a.plane + o0);
    }
    auto qs = [&](int k, int m) -> S { return qin[(long)m * a.plane + o0 + (long)(k - 3) * st]; };
    auto as = [&](int k, int j) -> R { return load_aux<S>(a.aux, (long)j * a.plane + o0 + (long)(k - 3) * st); };
    R xl[M], xr[M], am[M], ap[M], s[MW];
    solve_interface<P, CD, PREC>(a.ph, ixy, qs, as, auxm, aux0, xl, xr, am, ap, s);
    double d_c = dt / (ixy == 1 ? a.dx : a.dy), d_m = d_c;
    if (a.mcapa > 0) {
      const S* cap = static_cast<const S*>(a.aux) + (long)(a.mcapa - 1) * a.plane;
      const double h = ixy == 1 ? a.dx : a.dy;
      d_c = dt / (h * (double)cap[o0]);
      d_m = dt / (h * (double)cap[om]);
    }
    cfl.template add<MW>(s, d_c, d_m, a.mcapa > 0, ixy == 1);
  }
  int anybad = 0;
  const double v = cfl_cta_max<R, 128>(cfl, dt / a.dx, dt / a.dy, a.mcapa > 0, sred, fred, 0, &anybad);
  if (threadIdx.x == 0) atomic_max_nonneg(&a.ctl->stage_cfl[a.stage], v);
}

}  // namespace scl
