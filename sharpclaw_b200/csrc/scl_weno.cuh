// scl_weno.cuh -- WENO5 reconstruction at one interface (src/reconstruct.f90).
//
// Interface c-1/2 sits between cells c-1 and c.  The five cell-average jumps
// d[k] = q(c-3+k+1) - q(c-3+k), k = 0..4, are dq(c-2) .. dq(c+2) of the
// reference (reconstruct.f90:96-99, 166-169).  Side 1 (m1=1) builds qr(c-1)
// from dq(c-2..c+1); side 2 (m1=2) builds ql(c) from dq(c+2..c-1) with
// im = -1 (reconstruct.f90:108-132, 196-229).
//
// Two arithmetic forms:
//  * exact (double): the reference's operations in the reference's order;
//  * scaled (float): the same algebra on jumps divided by their largest
//    magnitude, with epsilon set in the scaled range.  The reference's product
//    form s1 = tt2*tt3 of fourth powers under- and overflows in FP32; scaling
//    keeps every product within float range while leaving the weights
//    unchanged (they are homogeneous of degree 0 in the jumps).
#pragma once
#include "scl_common.cuh"

namespace scl {

// reconstruct.f90:6 `double precision :: epweno = 1.e-36` (a REAL(4) literal)
__device__ __forceinline__ double epweno() { return (double)1.0e-36f; }
// epsilon of the scaled FP32 form: the squared smoothness indicators then lie
// in [1e-16, 1e4], so every weight product stays between 1e-32 and 1e9.
constexpr float EPS_SCALED = 1.0e-8f;

// One side of the WENO5 correction, reference order (reconstruct.f90:113-132);
// FD (fast division) multiplies by 1/3 instead of dividing by 3.
template <bool FD = false>
__device__ __forceinline__ double weno_side(double dm2, double dm1, double d0, double dp1,
                                            double im) {
  double t1 = im * (dm2 - dm1);
  double t2 = im * (dm1 - d0);
  double t3 = im * (d0 - dp1);
  double x1 = dm2 - 3.0 * dm1;
  double x2 = dm1 + d0;
  double x3 = 3.0 * d0 - dp1;
  double tt1 = 13.0 * (t1 * t1) + 3.0 * (x1 * x1);
  double tt2 = 13.0 * (t2 * t2) + 3.0 * (x2 * x2);
  double tt3 = 13.0 * (t3 * t3) + 3.0 * (x3 * x3);
  const double ep = epweno();
  tt1 = (ep + tt1) * (ep + tt1);
  tt2 = (ep + tt2) * (ep + tt2);
  tt3 = (ep + tt3) * (ep + tt3);
  double s1 = tt2 * tt3;
  double s2 = (6.0 * tt1) * tt3;
  double s3 = (3.0 * tt1) * tt2;
  double t0 = 1.0 / ((s1 + s2) + s3);
  s1 = s1 * t0;
  s3 = s3 * t0;
  if constexpr (FD) return ((s1 * (t2 - t1)) + ((0.5 * s3 - 0.25) * (t3 - t2))) * (1.0 / 3.0);
  return ((s1 * (t2 - t1)) + ((0.5 * s3 - 0.25) * (t3 - t2))) / 3.0;
}

// c/12 of the central stencil (reconstruct.f90:131-132)
template <bool FD>
__device__ __forceinline__ double twelfth(double c) {
  if constexpr (FD) return c * (1.0 / 12.0);
  return c / 12.0;
}

// Scaled FP32 form of weno_side on jumps already divided by `scale`.
__device__ __forceinline__ float weno_side_scaled(float dm2, float dm1, float d0, float dp1,
                                                  float im) {
  float t1 = im * (dm2 - dm1);
  float t2 = im * (dm1 - d0);
  float t3 = im * (d0 - dp1);
  float x1 = dm2 - 3.0f * dm1;
  float x2 = dm1 + d0;
  float x3 = 3.0f * d0 - dp1;
  float tt1 = 13.0f * (t1 * t1) + 3.0f * (x1 * x1);
  float tt2 = 13.0f * (t2 * t2) + 3.0f * (x2 * x2);
  float tt3 = 13.0f * (t3 * t3) + 3.0f * (x3 * x3);
  tt1 = (EPS_SCALED + tt1) * (EPS_SCALED + tt1);
  tt2 = (EPS_SCALED + tt2) * (EPS_SCALED + tt2);
  tt3 = (EPS_SCALED + tt3) * (EPS_SCALED + tt3);
  float s1 = tt2 * tt3;
  float s2 = (6.0f * tt1) * tt3;
  float s3 = (3.0f * tt1) * tt2;
  float t0 = rcp32((s1 + s2) + s3);
  s1 = s1 * t0;
  s3 = s3 * t0;
  return ((s1 * (t2 - t1)) + ((0.5f * s3 - 0.25f) * (t3 - t2))) * (1.0f / 3.0f);
}

// The FP32 forms can call their large device functions out of line:
// one shared copy shrinks the kernel's instruction footprint, but the call
// overhead made the char-wise Euler stage kernel 1.85x slower on B200, so it
// is off by default.
#ifndef SCL_OUTLINE_FP32
#define SCL_OUTLINE_FP32 0
#endif
#if SCL_OUTLINE_FP32
#define SCL_FP32_FN __noinline__
#else
#define SCL_FP32_FN __forceinline__
#endif

// Packed FP32 (sm_100 f32x2 arithmetic): one instruction computes both lanes,
// each lane rounded exactly as its scalar operation would be.
#ifndef SCL_WENO_PACKED
#define SCL_WENO_PACKED 1
#endif
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
  return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);  // a + (-1)b: one rounding, = a - b
}
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 pk2(float s) { return make_float2(s, s); }

// weno_side_scaled for both sides at once: lane x is side 1 on
// (dm2, dm1, d0, dp1) = (n0, n1, n2, n3), lane y side 2 on (n4, n3, n2, n1).
// Side 2's im = -1 negates t1, t2, t3 exactly, hence the result exactly; the
// squares do not see it, so it is applied to the result only (`post` holds
// the scale factor with the sign of each side).
__device__ __forceinline__ float2 weno_sides_packed(float2 dm2, float2 dm1, float2 d0, float2 dp1,
                                                    float2 post) {
  const float2 t1 = psub(dm2, dm1), t2 = psub(dm1, d0), t3 = psub(d0, dp1);
  const float2 x1 = pfma(dm1, pk2(-3.0f), dm2);
  const float2 x2 = padd(dm1, d0);
  const float2 x3 = pfma(d0, pk2(-3.0f), dp1);  // -(3 d0 - dp1): only its square is used
  float2 tt1 = pfma(pmul(t1, t1), pk2(13.0f), pmul(pmul(x1, x1), pk2(3.0f)));
  float2 tt2 = pfma(pmul(t2, t2), pk2(13.0f), pmul(pmul(x2, x2), pk2(3.0f)));
  float2 tt3 = pfma(pmul(t3, t3), pk2(13.0f), pmul(pmul(x3, x3), pk2(3.0f)));
  tt1 = padd(pk2(EPS_SCALED), tt1);
  tt2 = padd(pk2(EPS_SCALED), tt2);
  tt3 = padd(pk2(EPS_SCALED), tt3);
  tt1 = pmul(tt1, tt1);
  tt2 = pmul(tt2, tt2);
  tt3 = pmul(tt3, tt3);
  float2 s1 = pmul(tt2, tt3);
  const float2 s2 = pmul(pmul(pk2(6.0f), tt1), tt3);
  float2 s3 = pmul(pmul(pk2(3.0f), tt1), tt2);
  const float2 den = padd(padd(s1, s2), s3);
  const float2 t0 = make_float2(rcp32(den.x), rcp32(den.y));
  s1 = pmul(s1, t0);
  s3 = pmul(s3, t0);
  const float2 r = pfma(s1, psub(t2, t1), pmul(pfma(s3, pk2(0.5f), pk2(-0.25f)), psub(t3, t2)));
  return pmul(pmul(r, pk2(1.0f / 3.0f)), post);
}

// Both sides of the scaled correction for one set of five jumps h[0..4].
static __device__ SCL_FP32_FN void weno_pair_scaled(const float h[5], float& u1, float& u2) {
  float sc = fmaxf(fmaxf(fmaxf(fabsf(h[0]), fabsf(h[1])), fmaxf(fabsf(h[2]), fabsf(h[3]))),
                   fabsf(h[4]));
  // all-zero stencil, or non-finite / beyond 8e37 (where the reciprocal
  // would be subnormal; FP32 states cannot carry such jumps: their squares overflow)
  if (!(sc > 0.0f) || !(sc < 8.0e37f)) {
    u1 = (sc == 0.0f) ? 0.0f : sc;
    u2 = u1;
    return;
  }
  float inv = rcp32(sc);
#if SCL_WENO_PACKED
  const float2 iv = pk2(inv);
  const float2 n04 = pmul(make_float2(h[0], h[4]), iv);
  const float2 n13 = pmul(make_float2(h[1], h[3]), iv);
  const float n2 = h[2] * inv;
  const float2 u = weno_sides_packed(n04, n13, pk2(n2), make_float2(n13.y, n13.x), make_float2(sc, -sc));
  u1 = u.x;
  u2 = u.y;
#else
  float n0 = h[0] * inv, n1 = h[1] * inv, n2 = h[2] * inv, n3 = h[3] * inv, n4 = h[4] * inv;
  u1 = weno_side_scaled(n0, n1, n2, n3, 1.0f) * sc;
  u2 = weno_side_scaled(n4, n3, n2, n1, -1.0f) * sc;
#endif
}

// ---------------------------------------------------------------------------
// Exact form (FP64): returns the reconstructed states qr(c-1) (qrl) and ql(c)
// (qlr).  q[k][m] holds cells c-3+k, k = 0..5.
// ---------------------------------------------------------------------------
template <int M, bool FD = false>
__device__ __forceinline__ void weno5_exact(const double q[6][M], double qrl[M], double qlr[M]) {
#pragma unroll
  for (int m = 0; m < M; ++m) {
    double d[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) d[k] = q[k + 1][m] - q[k][m];
    double c = ((-q[1][m]) + 7.0 * (q[2][m] + q[3][m])) - q[4][m];
    qrl[m] = weno_side<FD>(d[0], d[1], d[2], d[3], 1.0) + twelfth<FD>(c);
    qlr[m] = weno_side<FD>(d[4], d[3], d[2], d[1], -1.0) + twelfth<FD>(c);
  }
}

// reconstruct.f90:146-241 for one interface; evl[p][m] = evl(i,p,m),
// evr[m][p] = evr(i,m,p).
template <int M, bool FD = false>
__device__ __forceinline__ void weno5_char_exact(const double q[6][M], const double evl[M][M],
                                                 const double evr[M][M], double qrl[M],
                                                 double qlr[M]) {
  double d[5][M];
#pragma unroll
  for (int k = 0; k < 5; ++k)
#pragma unroll
    for (int m = 0; m < M; ++m) d[k][m] = q[k + 1][m] - q[k][m];
#pragma unroll
  for (int m = 0; m < M; ++m) {
    double c = ((-q[1][m]) + 7.0 * (q[2][m] + q[3][m])) - q[4][m];
    qrl[m] = twelfth<FD>(c);
    qlr[m] = qrl[m];
  }
#pragma unroll
  for (int p = 0; p < M; ++p) {
    double h[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      double s = 0.0;
#pragma unroll
      for (int m = 0; m < M; ++m) s = s + evl[p][m] * d[k][m];
      h[k] = s;
    }
    double u1 = weno_side<FD>(h[0], h[1], h[2], h[3], 1.0);
    double u2 = weno_side<FD>(h[4], h[3], h[2], h[1], -1.0);
#pragma unroll
    for (int m = 0; m < M; ++m) {
      qrl[m] = qrl[m] + evr[m][p] * u1;
      qlr[m] = qlr[m] + evr[m][p] * u2;
    }
  }
}

// ---------------------------------------------------------------------------
// Offset form (FP32): from the jumps d[k][m] (formed in the storage precision)
// return er = qr(c-1) - q(c-1) and el = ql(c) - q(c).  The linear part is the
// reference's central stencil (-q(c-2)+7q(c-1)+7q(c)-q(c+1))/12 rewritten in
// jumps: minus q(c-1) it is (d(c-1)+6d(c)-d(c+1))/12, minus q(c) it is
// (d(c-1)-6d(c)-d(c+1))/12.
// ---------------------------------------------------------------------------
template <int M>
__device__ __forceinline__ void weno5_offset(const float d[5][M], float er[M], float el[M]) {
#pragma unroll
  for (int m = 0; m < M; ++m) {
    float h[5] = {d[0][m], d[1][m], d[2][m], d[3][m], d[4][m]};
    float u1, u2;
    weno_pair_scaled(h, u1, u2);
    er[m] = (d[1][m] + 6.0f * d[2][m] - d[3][m]) * (1.0f / 12.0f) + u1;
    el[m] = (d[1][m] - 6.0f * d[2][m] - d[3][m]) * (1.0f / 12.0f) + u2;
  }
}

template <int M>
__device__ __forceinline__ void weno5_char_offset(const float d[5][M], const float evl[M][M],
                                                  const float evr[M][M], float er[M],
                                                  float el[M]) {
#pragma unroll
  for (int m = 0; m < M; ++m) {
    er[m] = (d[1][m] + 6.0f * d[2][m] - d[3][m]) * (1.0f / 12.0f);
    el[m] = (d[1][m] - 6.0f * d[2][m] - d[3][m]) * (1.0f / 12.0f);
  }
#pragma unroll
  for (int p = 0; p < M; ++p) {
    float h[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      float s = 0.0f;
#pragma unroll
      for (int m = 0; m < M; ++m) s = s + evl[p][m] * d[k][m];
      h[k] = s;
    }
    float u1, u2;
    weno_pair_scaled(h, u1, u2);
#pragma unroll
    for (int m = 0; m < M; ++m) {
      er[m] = er[m] + evr[m][p] * u1;
      el[m] = el[m] + evr[m][p] * u2;
    }
  }
}

// ---------------------------------------------------------------------------
// Wave-based form (char_decomp = 1, reconstruct.f90:350-428).  The waves W of
// the cell-average Riemann problems at the five interfaces c-2 .. c+2 around
// interface c-1/2 are projected on the wave of the same family at c-1/2:
// theta_k = W(c-2+k) . W(c), theta_2 = |W(c)|^2.  The WENO algebra runs on the
// thetas (side 1 on theta_0..3, side 2 on theta_4..1 with im = -1, exactly the
// weno_side arguments), and the correction is u * W(c) / |W(c)|^2, dropped
// when |W(c)|^2 <= 1e-14.  w[k][mw][m] = component m of wave mw at c-2+k.
// ---------------------------------------------------------------------------
// reconstruct.f90:413 `if (wnorm2.gt.1.e-14)` (a REAL(4) literal)
__device__ __forceinline__ double wave_floor() { return (double)1.0e-14f; }

template <int M, int MW, bool FD = false>
__device__ __forceinline__ void weno5_wave_exact(const double q[6][M], const double w[5][MW][M],
                                                 double qrl[M], double qlr[M]) {
#pragma unroll
  for (int m = 0; m < M; ++m) {
    double c = ((-q[1][m]) + 7.0 * (q[2][m] + q[3][m])) - q[4][m];   // :371-372
    qrl[m] = twelfth<FD>(c);
    qlr[m] = qrl[m];
  }
#pragma unroll
  for (int mw = 0; mw < MW; ++mw) {
    double th[5];                                                     // :383-392
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      th[k] = w[k][mw][0] * w[2][mw][0];
#pragma unroll
      for (int m = 1; m < M; ++m) th[k] = th[k] + w[k][mw][m] * w[2][mw][m];
    }
    double u1 = 0.0, u2 = 0.0, winv = 0.0;                            // :413-419
    if (th[2] > wave_floor()) {
      u1 = weno_side<FD>(th[0], th[1], th[2], th[3], 1.0);
      u2 = weno_side<FD>(th[4], th[3], th[2], th[1], -1.0);
      winv = 1.0 / th[2];
    }
#pragma unroll
    for (int m = 0; m < M; ++m) {                                     // :421-424
      qrl[m] = qrl[m] + (u1 * w[2][mw][m]) * winv;
      qlr[m] = qlr[m] + (u2 * w[2][mw][m]) * winv;
    }
  }
}

// FP32 offset form of weno5_wave_exact: jumps d (as weno5_offset), waves from
// FP32 cell values and jumps; the thetas go through the scaled pair.
template <int M, int MW>
__device__ __forceinline__ void weno5_wave_offset(const float d[5][M], const float w[5][MW][M], float er[M],
                                                  float el[M]) {
#pragma unroll
  for (int m = 0; m < M; ++m) {
    er[m] = (d[1][m] + 6.0f * d[2][m] - d[3][m]) * (1.0f / 12.0f);
    el[m] = (d[1][m] - 6.0f * d[2][m] - d[3][m]) * (1.0f / 12.0f);
  }
#pragma unroll
  for (int mw = 0; mw < MW; ++mw) {
    float th[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      th[k] = w[k][mw][0] * w[2][mw][0];
#pragma unroll
      for (int m = 1; m < M; ++m) th[k] = th[k] + w[k][mw][m] * w[2][mw][m];
    }
    if (th[2] > 1.0e-14f) {
      float u1, u2;
      weno_pair_scaled(th, u1, u2);
      const float winv = rcp32(th[2]);
#pragma unroll
      for (int m = 0; m < M; ++m) {
        er[m] = er[m] + (u1 * w[2][mw][m]) * winv;
        el[m] = el[m] + (u2 * w[2][mw][m]) * winv;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Transmission-based form (char_decomp = 3, reconstruct.f90:244-347).  Each of
// the five interfaces c-2+k (k = 0..4) around c-1/2 has its own eigenvectors;
// its wave strengths gg = evl_k . dq_k, carried to physical space by evr_k,
// are projected on the left eigenvectors of c-1/2 (h_k), the WENO algebra runs
// on h per field, and the result returns through evr of c-1/2.
// ---------------------------------------------------------------------------
// h_k of one neighbour interface (reconstruct.f90:273-294 for one i+m1).
template <class T, int M>
__device__ __forceinline__ void trans_project(const T evlk[M][M], const T evrk[M][M], const T dk[M],
                                              const T evlc[M][M], T hk[M]) {
  T gg[M];
#pragma unroll
  for (int mw = 0; mw < M; ++mw) {
    T g = (T)0;
#pragma unroll
    for (int m = 0; m < M; ++m) g = g + evlk[mw][m] * dk[m];
    gg[mw] = g;
  }
#pragma unroll
  for (int mw = 0; mw < M; ++mw) {
    T h = (T)0;
#pragma unroll
    for (int m = 0; m < M; ++m) h = h + (evlc[mw][m] * gg[mw]) * evrk[m][mw];
    hk[mw] = h;
  }
}

// reconstruct.f90:298-345 from h[k][mw]; evrc = evr of c-1/2.
template <int M, bool FD = false>
__device__ __forceinline__ void weno5_trans_exact(const double q[6][M], const double h[5][M],
                                                  const double evrc[M][M], double qrl[M], double qlr[M]) {
  double u1[M], u2[M];
#pragma unroll
  for (int mw = 0; mw < M; ++mw) {
    u1[mw] = weno_side<FD>(h[0][mw], h[1][mw], h[2][mw], h[3][mw], 1.0);
    u2[mw] = weno_side<FD>(h[4][mw], h[3][mw], h[2][mw], h[1][mw], -1.0);
  }
#pragma unroll
  for (int m = 0; m < M; ++m) {
    double c = ((-q[1][m]) + 7.0 * (q[2][m] + q[3][m])) - q[4][m];
    double a = twelfth<FD>(c), b = twelfth<FD>(c);
#pragma unroll
    for (int mw = 0; mw < M; ++mw) {
      a = a + evrc[m][mw] * u1[mw];
      b = b + evrc[m][mw] * u2[mw];
    }
    qrl[m] = a;
    qlr[m] = b;
  }
}

template <int M>
__device__ __forceinline__ void weno5_trans_offset(const float d[5][M], const float h[5][M],
                                                   const float evrc[M][M], float er[M], float el[M]) {
#pragma unroll
  for (int m = 0; m < M; ++m) {
    er[m] = (d[1][m] + 6.0f * d[2][m] - d[3][m]) * (1.0f / 12.0f);
    el[m] = (d[1][m] - 6.0f * d[2][m] - d[3][m]) * (1.0f / 12.0f);
  }
#pragma unroll
  for (int mw = 0; mw < M; ++mw) {
    const float hh[5] = {h[0][mw], h[1][mw], h[2][mw], h[3][mw], h[4][mw]};
    float u1, u2;
    weno_pair_scaled(hh, u1, u2);
#pragma unroll
    for (int m = 0; m < M; ++m) {
      er[m] = er[m] + evrc[m][mw] * u1;
      el[m] = el[m] + evrc[m][mw] * u2;
    }
  }
}

// ---------------------------------------------------------------------------
// Second-order TVD reconstructions (lim_type = 1, reconstruct.f90:525-761).
// q[k][m] holds cells c-3+k (only c-2 .. c+1 are read).
// ---------------------------------------------------------------------------
// reconstruct.f90:551-571: limiter mthlim = 1 minmod, 2 superbee, 3 van Leer,
// 4 monotonized centered, 5 Cada & Torrilhon
template <class T>
__device__ __forceinline__ T tvd_limiter(int t, T r) {
  auto mn = [](T a, T b) { return a < b ? a : b; };
  auto mx = [](T a, T b) { return a > b ? a : b; };
  switch (t) {
    case 1: return mx((T)0, mn((T)1, r));
    case 2: return mx(mx((T)0, mn((T)1, (T)2 * r)), mn((T)2, r));
    case 3: return (r + fabs(r)) / ((T)1 + fabs(r));
    case 4: {
      const T c = ((T)1 + r) / (T)2;
      return mx((T)0, mn(mn(c, (T)2), (T)2 * r));
    }
    case 5: {
      const T beta = (T)2, xgamma = (T)2, alpha = (T)(1.0 / 3.0);
      const T pp = ((T)2 + r) / (T)3;
      const T amax = mx(mx(-alpha * r, (T)0), mn(mn(beta * r, pp), xgamma));
      return mx((T)0, mn(pp, amax));
    }
  }
  return (T)0;
}

// tvd2, componentwise (reconstruct.f90:543-574): qr(c-1) from cell c-1,
// ql(c) from cell c; a cell whose backward jump is 0 gets no slope.
template <int M>
__device__ __forceinline__ void tvd2_exact(const double q[6][M], const int* mthlim, double qrl[M], double qlr[M]) {
#pragma unroll
  for (int m = 0; m < M; ++m) {
    double dqm = q[2][m] - q[1][m], dqp = q[3][m] - q[2][m];
    double phi = dqm != 0.0 ? tvd_limiter(mthlim[m], dqp / dqm) : 0.0;
    qrl[m] = q[2][m] + (0.5 * phi) * dqm;
    dqm = q[3][m] - q[2][m];
    dqp = q[4][m] - q[3][m];
    phi = dqm != 0.0 ? tvd_limiter(mthlim[m], dqp / dqm) : 0.0;
    qlr[m] = q[3][m] - (0.5 * phi) * dqm;
  }
}

// offsets er = qr(c-1)-q(c-1), el = ql(c)-q(c) from the jumps d[k] (FP32 forms)
template <int M>
__device__ __forceinline__ void tvd2_offset(const float d[5][M], const int* mthlim, float er[M], float el[M]) {
#pragma unroll
  for (int m = 0; m < M; ++m) {
    float phi = d[1][m] != 0.0f ? tvd_limiter(mthlim[m], d[2][m] / d[1][m]) : 0.0f;
    er[m] = (0.5f * phi) * d[1][m];
    phi = d[2][m] != 0.0f ? tvd_limiter(mthlim[m], d[3][m] / d[2][m]) : 0.0f;
    el[m] = -((0.5f * phi) * d[2][m]);
  }
}

// tvd2_char (reconstruct.f90:580-651): jumps at interfaces c-1, c, c+1
// (d[0..2]) projected on the left eigenvectors of c-1/2; with base = the
// cell values (exact form) or 0 (offset form).
template <class T, int M>
__device__ __forceinline__ void tvd2_char_core(const T d[3][M], const T evl[M][M], const T evr[M][M],
                                               const int* mthlim, const T* base_r, const T* base_l, T xr[M],
                                               T xl[M]) {
  const T floor14 = (T)(double)1.0e-14f;                       // :609, a REAL(4) literal
  T u1[M], u2[M];
#pragma unroll
  for (int p = 0; p < M; ++p) {
    T h[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      T t = (T)0;
#pragma unroll
      for (int m = 0; m < M; ++m) t = t + evl[p][m] * d[k][m];
      h[k] = t;
    }
    T r = fabs(h[0]) > floor14 ? h[1] / h[0] : (T)0;
    u1[p] = ((T)0.5 * tvd_limiter(mthlim[p], r)) * h[0];
    r = fabs(h[1]) > floor14 ? h[2] / h[1] : (T)0;
    u2[p] = ((T)(-0.5) * tvd_limiter(mthlim[p], r)) * h[1];
  }
#pragma unroll
  for (int m = 0; m < M; ++m) {
    T a = base_r[m], b = base_l[m];
#pragma unroll
    for (int p = 0; p < M; ++p) {
      a = a + evr[m][p] * u1[p];
      b = b + evr[m][p] * u2[p];
    }
    xr[m] = a;
    xl[m] = b;
  }
}

// tvd2_wave (reconstruct.f90:654-761): waves w[k] at interfaces c-1, c, c+1,
// speeds s of c-1/2; the same base convention as tvd2_char_core.
template <class T, int M, int MW>
__device__ __forceinline__ void tvd2_wave_core(const T w[3][MW][M], const T s[MW], const int* mthlim,
                                               const T* base_r, const T* base_l, T xr[M], T xl[M]) {
#pragma unroll
  for (int m = 0; m < M; ++m) { xr[m] = base_r[m]; xl[m] = base_l[m]; }
#pragma unroll
  for (int mw = 0; mw < MW; ++mw) {
    T wnorm2 = (T)0, dotl = (T)0, dotr = (T)0;
#pragma unroll
    for (int m = 0; m < M; ++m) {
      wnorm2 = wnorm2 + w[1][mw][m] * w[1][mw][m];
      dotl = dotl + w[0][mw][m] * w[1][mw][m];
      dotr = dotr + w[1][mw][m] * w[2][mw][m];
    }
    if (wnorm2 == (T)0) continue;
    const T r = s[mw] > (T)0 ? dotl / wnorm2 : dotr / wnorm2;
    const T uu = (T)0.5 * tvd_limiter(mthlim[mw], r);
#pragma unroll
    for (int m = 0; m < M; ++m) {
      xr[m] = xr[m] + w[1][mw][m] * uu;
      xl[m] = xl[m] - w[1][mw][m] * uu;
    }
  }
}

// ---------------------------------------------------------------------------
// Unlimited polynomial reconstruction of order 3 (lim_type 0, polyrecon.f90):
// c(-1) = 1/6, c(0) = 2/6 (:27-29); ur and ul accumulate from 0 in the
// reference's order (:66-69); qr(c-1) = q(c-1) + ur, ql(c) = q(c) - ul.
// ---------------------------------------------------------------------------
template <int M>
__device__ __forceinline__ void poly3_exact(const double q[6][M], double qrl[M], double qlr[M]) {
  const double cm1 = 1.0 / 6.0, c0 = 2.0 / 6.0;
#pragma unroll
  for (int m = 0; m < M; ++m) {
    const double tm1 = q[2][m] - q[1][m], t0 = q[3][m] - q[2][m], tp1 = q[4][m] - q[3][m];
    const double ur = (0.0 + cm1 * tm1) + c0 * t0;
    const double ul = (0.0 + cm1 * tp1) + c0 * t0;
    qrl[m] = q[2][m] + ur;
    qlr[m] = q[3][m] - ul;
  }
}

// offsets er = qr(c-1)-q(c-1), el = ql(c)-q(c) from the jumps d[k] (FP32 forms)
template <int M>
__device__ __forceinline__ void poly3_offset(const float d[5][M], float er[M], float el[M]) {
  const float cm1 = (float)(1.0 / 6.0), c0 = (float)(2.0 / 6.0);
#pragma unroll
  for (int m = 0; m < M; ++m) {
    er[m] = (0.0f + cm1 * d[1][m]) + c0 * d[2][m];
    el[m] = -((0.0f + cm1 * d[3][m]) + c0 * d[2][m]);
  }
}

// q2qlqr_poly_wave (polyrecon.f90:214-251), order 3: per wave family the
// projections theta(j) = wave(c+j).wave(c), j = -1..1 (w[0..2] = waves of
// interfaces c-1, c, c+1), skipped when theta(0) <= 1e-14 (a REAL(4) literal);
// base = the cell values (exact form) or 0 (offset form).
template <class T, int M, int MW>
__device__ __forceinline__ void poly3_wave_core(const T w[3][MW][M], const T* base_r, const T* base_l, T xr[M],
                                                T xl[M]) {
  const T floor14 = (T)(double)1.0e-14f;
  const T cm1 = (T)(1.0 / 6.0), c0 = (T)(2.0 / 6.0);
#pragma unroll
  for (int m = 0; m < M; ++m) {
    xr[m] = base_r[m];
    xl[m] = base_l[m];
  }
#pragma unroll
  for (int mw = 0; mw < MW; ++mw) {
    T th[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      T t = w[j][mw][0] * w[1][mw][0];
#pragma unroll
      for (int m = 1; m < M; ++m) t = t + w[j][mw][m] * w[1][mw][m];
      th[j] = t;
    }
    if (th[1] > floor14) {
      const T wn = (T)1 / th[1];
      const T ur = ((T)0 + cm1 * th[0]) + c0 * th[1];
      const T ul = ((T)0 + cm1 * th[2]) + c0 * th[1];
#pragma unroll
      for (int m = 0; m < M; ++m) {
        xr[m] = xr[m] + (ur * wn) * w[1][mw][m];
        xl[m] = xl[m] - (ul * wn) * w[1][mw][m];
      }
    }
  }
}

}  // namespace scl
