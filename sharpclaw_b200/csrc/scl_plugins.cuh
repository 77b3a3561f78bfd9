// scl_plugins.cuh -- device Riemann solvers, total-fluctuation solvers and
// eigenvector routines, selected by plugin id.
//
// Every reference plugin loops `do i = 2-mbc, mx+mbc` over independent
// interfaces, so each is restated here as a pointwise function of one
// interface (rp, evec) or one cell (tfluct), keeping the arithmetic order of
// the loop body.  States are passed as (left, right) of the Riemann problem:
// for rp at interface i-1/2 left = qr(i-1), right = ql(i); for tfluct of cell i
// left = ql(i), right = qr(i).  `dl` is right - left, formed by the caller:
// in FP64 it is the same subtraction the reference does; in the FP32 forms it
// is computed from FP64 cell-average jumps, so it keeps the precision of the
// jump rather than of the states.
#pragma once
#include <type_traits>
#include "scl_common.cuh"

namespace scl {

// FP32 Euler plugins use reciprocal-square-root forms of the Roe averages and
// the entropy-fix sound speeds (algebraically the reference's, not its
// operation order).  The FP64 forms keep the reference's order unless the
// template flag FD (fast division) is set: then divisions become reciprocal
// multiplies and square roots reciprocal square roots, as in FP32, within a
// few ulp of the reference's values (the SCL_FP64 form; SCL_FP64_STRICT and
// the adjoint keep FD = false).
#ifndef SCL_FAST_ROE
#define SCL_FAST_ROE 1
#endif

template <class R>
__device__ __forceinline__ R rmin(R a, R b) { return a < b ? a : b; }
template <class R>
__device__ __forceinline__ R rmax(R a, R b) { return a > b ? a : b; }

// ------------------------------------------------------------------------
// Linear advection, apps/advection/1d/rp1.f:35-43, tfluct1.f:78-87, evec.f:118-121
// ------------------------------------------------------------------------
struct PAdvection {
  static constexpr int MEQN = 1, MWAVES = 1, MAUX = 0, NDIM = 1;
  static constexpr bool HAS_TFLUCT = true;
  template <class R, bool FD = false>
  __device__ static void rp(const Phys& ph, int, const R*, const R*, const R* dl, const R*,
                            const R*, R* s, R* amdq, R* apdq) {
    const R u = (R)ph.u;
    s[0] = u;
    amdq[0] = rmin(u, (R)0) * dl[0];
    apdq[0] = rmax(u, (R)0) * dl[0];
  }
  // waves of rp1.f:35 (the jump itself), for the wave-based reconstruction
  template <class R, bool FD = false>
  __device__ static void waves(const Phys& ph, int, const R*, const R*, const R* dl, const R*, const R*,
                               R w[1][1], R* s = nullptr) {
    w[0][0] = dl[0];
    if (s) s[0] = (R)ph.u;
  }
  template <class R, bool FD = false>
  __device__ static void tfluct(const Phys& ph, int, const R*, const R*, const R* dl, const R*,
                                R* adq) {
    const R u = (R)ph.u;
    R am = rmin(u, (R)0) * dl[0];
    R ap = rmax(u, (R)0) * dl[0];
    adq[0] = am + ap;
  }
  template <class R, bool FD = false>
  __device__ static void evec(const Phys&, int, const R*, const R*, const R*, const R*,
                              R evl[1][1], R evr[1][1]) {
    evl[0][0] = (R)1;
    evr[0][0] = (R)1;
  }
};

// ------------------------------------------------------------------------
// 1-D Euler, Roe solver with Harten-Hyman entropy fix,
// apps/euler/shockentropy/rp1eu.f:44-213.  No tfluct exists for this family
// (the app runs with tfluct_solver = 0, the swap path of flux1.f90:155-188).
// ------------------------------------------------------------------------
struct PEuler {
  static constexpr int MEQN = 3, MWAVES = 3, MAUX = 0, NDIM = 1;
  static constexpr bool HAS_TFLUCT = false;

  // `ia` (FP32 form only) receives 1/a.
  template <class R, bool FD = false>
  __device__ static void roe(const Phys& ph, const R* L, const R* Rt, R& u, R& enth, R& a,
                             R* ia = nullptr) {
#if SCL_FAST_ROE
    if constexpr (sizeof(R) == 4) {
      // FP32 form: the same Roe averages with reciprocal square roots,
      // sqrt(rho) = rho*w and m/sqrt(rho) = m*w for w = 1/sqrt(rho)
      const float g1 = (float)ph.gamma1;
      const float wl = rsqrtf(L[0]), wr = rsqrtf(Rt[0]);
      const float pl = g1 * (L[2] - 0.5f * (L[1] * L[1]) * (wl * wl));
      const float pr = g1 * (Rt[2] - 0.5f * (Rt[1] * Rt[1]) * (wr * wr));
      const float inv = rcp32(L[0] * wl + Rt[0] * wr);
      u = (L[1] * wl + Rt[1] * wr) * inv;
      enth = ((L[2] + pl) * wl + (Rt[2] + pr) * wr) * inv;
      const float a2 = g1 * (enth - 0.5f * (u * u));
      const float ra = rsqrtf(a2);
      a = a2 * ra;
      if (ia) *ia = ra;
      return;
    }
#endif
    if constexpr (FD && sizeof(R) == 8) {
      const double g1 = ph.gamma1;
      const double wl = rsqrt(L[0]), wr = rsqrt(Rt[0]);
      const double pl = g1 * (L[2] - 0.5 * (L[1] * L[1]) * (wl * wl));
      const double pr = g1 * (Rt[2] - 0.5 * (Rt[1] * Rt[1]) * (wr * wr));
      const double inv = 1.0 / (L[0] * wl + Rt[0] * wr);
      u = (L[1] * wl + Rt[1] * wr) * inv;
      enth = ((L[2] + pl) * wl + (Rt[2] + pr) * wr) * inv;
      const double a2 = g1 * (enth - 0.5 * (u * u));
      const double ra = rsqrt(a2);
      a = a2 * ra;
      if (ia) *ia = ra;
      return;
    }
    const R g1 = (R)ph.gamma1;
    R rhsqrtl = sqrt(L[0]);
    R rhsqrtr = sqrt(Rt[0]);
    R pl = g1 * (L[2] - ((R)0.5 * (L[1] * L[1])) / L[0]);
    R pr = g1 * (Rt[2] - ((R)0.5 * (Rt[1] * Rt[1])) / Rt[0]);
    R rhsq2 = rhsqrtl + rhsqrtr;
    u = (L[1] / rhsqrtl + Rt[1] / rhsqrtr) / rhsq2;
    enth = ((L[2] + pl) / rhsqrtl + (Rt[2] + pr) / rhsqrtr) / rhsq2;
    R a2 = g1 * (enth - (R)0.5 * (u * u));
    a = sqrt(a2);
  }

  // u - c (PLUS false) or u + c (PLUS true) of one state, the four
  // characteristic speeds of the entropy fix (rp1eu.f:132-134, 150-152,
  // 170-172, 180-182).
  template <bool PLUS, class R, bool FD = false>
  __device__ static R efix_speed(const Phys& ph, R rho, R m, R en) {
#if SCL_FAST_ROE
    if constexpr (sizeof(R) == 4) {  // one reciprocal, one square root
      const float ir = rcp32(rho), u = m * ir;
      const float p = (float)ph.gamma1 * (en - 0.5f * (m * u));
      const float c = sqrtf(((float)ph.gamma * p) * ir);
      return PLUS ? u + c : u - c;
    }
#endif
    if constexpr (FD && sizeof(R) == 8) {
      const double ir = 1.0 / rho, u = m * ir;
      const double p = ph.gamma1 * (en - 0.5 * (m * u));
      const double c = sqrt((ph.gamma * p) * ir);
      return PLUS ? u + c : u - c;
    }
    const R g1 = (R)ph.gamma1, gamma = (R)ph.gamma;
    R p = g1 * (en - ((R)0.5 * (m * m)) / rho);
    R c = sqrt((gamma * p) / rho);
    return PLUS ? m / rho + c : m / rho - c;
  }

  // Roe averages and the three waves of rp1eu.f:44-86, w[wave][component].
  template <class R, bool FD = false>
  __device__ static void wave_set(const Phys& ph, const R* L, const R* Rt, const R* dl, R& u, R& enth,
                                  R& a, R w[3][3]) {
    const R g1 = (R)ph.gamma1;
    R ia = (R)0;
    roe<R, FD>(ph, L, Rt, u, enth, a, &ia);                       // rp1eu.f:44-55
    R a2, a3;
    if constexpr ((sizeof(R) == 4 && SCL_FAST_ROE) || FD) {
      a2 = (g1 * (ia * ia)) * (((enth - u * u) * dl[0] + u * dl[1]) - dl[2]);
      a3 = ((dl[1] + (a - u) * dl[0]) - a * a2) * ((R)0.5 * ia);
    } else {
      a2 = (g1 / (a * a)) * (((enth - u * u) * dl[0] + u * dl[1]) - dl[2]);   // :65-66
      a3 = ((dl[1] + (a - u) * dl[0]) - a * a2) / ((R)2 * a);                   // :67
    }
    R a1 = (dl[0] - a2) - a3;                                                   // :68
    w[0][0] = a1; w[0][1] = a1 * (u - a); w[0][2] = a1 * (enth - u * a);
    w[1][0] = a2; w[1][1] = a2 * u;       w[1][2] = (a2 * (R)0.5) * (u * u);
    w[2][0] = a3; w[2][1] = a3 * (u + a); w[2][2] = a3 * (enth + u * a);
  }

  template <class R, bool FD = false>
  __device__ static void waves(const Phys& ph, int, const R* L, const R* Rt, const R* dl, const R*,
                               const R*, R w[3][3], R* s = nullptr) {
    R u, enth, a;
    wave_set<R, FD>(ph, L, Rt, dl, u, enth, a, w);
    if (s) { s[0] = u - a; s[1] = u; s[2] = u + a; }
  }

  template <class R, bool FD = false>
  __device__ static void rp(const Phys& ph, int, const R* L, const R* Rt, const R* dl, const R*,
                            const R*, R* s, R* amdq, R* apdq) {
    R u, enth, a, w[3][3];  // w[wave][component]
    wave_set<R, FD>(ph, L, Rt, dl, u, enth, a, w);
    s[0] = u - a; s[1] = u; s[2] = u + a;
    if (!ph.efix) {                                                            // :100-111
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        R am = (R)0, ap = (R)0;
#pragma unroll
        for (int mw = 0; mw < 3; ++mw) {
          if (s[mw] < (R)0) am = am + s[mw] * w[mw][m];
          else ap = ap + s[mw] * w[mw][m];
        }
        amdq[m] = am; apdq[m] = ap;
      }
      return;
    }
    // entropy fix, rp1eu.f:126-201
    do {
      R s0 = efix_speed<false, R, FD>(ph, L[0], L[1], L[2]);
      if (s0 >= (R)0 && s[0] > (R)0) {
        amdq[0] = amdq[1] = amdq[2] = (R)0;
        break;
      }
      R rho1 = L[0] + w[0][0];
      R rhou1 = L[1] + w[0][1];
      R en1 = L[2] + w[0][2];
      R s1 = efix_speed<false, R, FD>(ph, rho1, rhou1, en1);
      R sfract;
      if (s0 < (R)0 && s1 > (R)0) sfract = (s0 * (s1 - s[0])) / (s1 - s0);
      else if (s[0] < (R)0) sfract = s[0];
      else sfract = (R)0;
#pragma unroll
      for (int m = 0; m < 3; ++m) amdq[m] = sfract * w[0][m];
      if (s[1] >= (R)0) break;
#pragma unroll
      for (int m = 0; m < 3; ++m) amdq[m] = amdq[m] + s[1] * w[1][m];
      R s3 = efix_speed<true, R, FD>(ph, Rt[0], Rt[1], Rt[2]);
      R rho2 = Rt[0] - w[2][0];
      R rhou2 = Rt[1] - w[2][1];
      R en2 = Rt[2] - w[2][2];
      R s2 = efix_speed<true, R, FD>(ph, rho2, rhou2, en2);
      if (s2 < (R)0 && s3 > (R)0) sfract = (s2 * (s3 - s[2])) / (s3 - s2);
      else if (s[2] < (R)0) sfract = s[2];
      else break;
#pragma unroll
      for (int m = 0; m < 3; ++m) amdq[m] = amdq[m] + sfract * w[2][m];
    } while (0);
#pragma unroll
    for (int m = 0; m < 3; ++m) {                                                // :206-213
      R df = (R)0;
#pragma unroll
      for (int mw = 0; mw < 3; ++mw) df = df + s[mw] * w[mw][m];
      apdq[m] = df - amdq[m];
    }
  }

  template <class R, bool FD = false>
  __device__ static void tfluct(const Phys&, int, const R*, const R*, const R*, const R*, R*) {}

  // Roe eigenvectors (new; the reference's evec1eu.f is incomplete).  Averages
  // as rp1eu.f:44-55 from the cell averages q(i-1), q(i).
  template <class R, bool FD = false>
  __device__ static void evec(const Phys& ph, int, const R* qm, const R* q0, const R*, const R*,
                              R evl[3][3], R evr[3][3]) {
    if constexpr ((sizeof(R) == 4 && SCL_FAST_ROE) || FD) {
      R u, h, a, ia;
      roe<R, FD>(ph, qm, q0, u, h, a, &ia);
      const R g1 = (R)ph.gamma1, h5 = (R)0.5;
      evr[0][0] = (R)1;      evr[0][1] = (R)1;             evr[0][2] = (R)1;
      evr[1][0] = u - a;     evr[1][1] = u;                evr[1][2] = u + a;
      evr[2][0] = h - u * a; evr[2][1] = h5 * (u * u);     evr[2][2] = h + u * a;
      const R b1 = g1 * (ia * ia), b2 = h5 * (b1 * (u * u)), ua = u * ia, b1u = b1 * u;
      evl[0][0] = h5 * (b2 + ua); evl[0][1] = -h5 * (b1u + ia); evl[0][2] = h5 * b1;
      evl[1][0] = (R)1 - b2;      evl[1][1] = b1u;              evl[1][2] = -b1;
      evl[2][0] = h5 * (b2 - ua); evl[2][1] = -h5 * (b1u - ia); evl[2][2] = h5 * b1;
      return;
    }
    const R g1 = (R)ph.gamma1;
    R rhsqrtl = sqrt(qm[0]);
    R rhsqrtr = sqrt(q0[0]);
    R pl = g1 * (qm[2] - ((R)0.5 * (qm[1] * qm[1])) / qm[0]);
    R pr = g1 * (q0[2] - ((R)0.5 * (q0[1] * q0[1])) / q0[0]);
    R rhsq2 = rhsqrtl + rhsqrtr;
    R u = (qm[1] / rhsqrtl + q0[1] / rhsqrtr) / rhsq2;
    R h = ((qm[2] + pl) / rhsqrtl + (q0[2] + pr) / rhsqrtr) / rhsq2;
    R a2 = g1 * (h - (R)0.5 * (u * u));
    R a = sqrt(a2);
    // evr[m][p] = evr(i,m,p): component m of right eigenvector p
    evr[0][0] = (R)1;        evr[0][1] = (R)1;               evr[0][2] = (R)1;
    evr[1][0] = u - a;       evr[1][1] = u;                  evr[1][2] = u + a;
    evr[2][0] = h - u * a;   evr[2][1] = (R)0.5 * (u * u);   evr[2][2] = h + u * a;
    R b1 = g1 / a2;
    R b2 = (R)0.5 * (b1 * (u * u));
    R ua = u / a;
    R ra = (R)1 / a;
    R b1u = b1 * u;
    // evl[p][m] = evl(i,p,m): component m of left eigenvector p
    evl[0][0] = (R)0.5 * (b2 + ua); evl[0][1] = (R)(-0.5) * (b1u + ra); evl[0][2] = (R)0.5 * b1;
    evl[1][0] = (R)1 - b2;          evl[1][1] = b1u;                    evl[1][2] = -b1;
    evl[2][0] = (R)0.5 * (b2 - ua); evl[2][1] = (R)(-0.5) * (b1u - ra); evl[2][2] = (R)0.5 * b1;
  }
};

// ------------------------------------------------------------------------
// 2-D shallow water Roe solver along a slice,
// apps/shallowWater/2dRadialDam/rpn2sw.f:60-228 and tfluct1sw.f:297-467.
// ------------------------------------------------------------------------
struct PShallow2D {
  static constexpr int MEQN = 3, MWAVES = 3, MAUX = 0, NDIM = 2;
  static constexpr bool HAS_TFLUCT = true;

  // Roe averages of rpn2sw.f:80-88: normal and tangential velocity u, v (mu,
  // mv the normal / tangential momentum), celerity a, and ha = 0.5/a.
  template <class R, bool FD = false>
  __device__ static void roe(const Phys& ph, int mu, int mv, const R* L, const R* Rt, R& u, R& v, R& a,
                             R& ha) {
#if SCL_FAST_ROE
    if constexpr (sizeof(R) == 4) {
      // FP32 form with reciprocal square roots: sqrt(h) = h*w, m/sqrt(h) = m*w
      // for w = 1/sqrt(h), and 0.5/a = 0.5/sqrt(g*hbar)
      const float wl = rsqrtf(L[0]), wr = rsqrtf(Rt[0]);
      const float inv = rcp32(L[0] * wl + Rt[0] * wr);
      u = (L[mu] * wl + Rt[mu] * wr) * inv;
      v = (L[mv] * wl + Rt[mv] * wr) * inv;
      const float gh = (float)ph.grav * ((L[0] + Rt[0]) * 0.50f);
      const float ia = rsqrtf(gh);
      a = gh * ia;
      ha = 0.50f * ia;
      return;
    }
#endif
    if constexpr (FD && sizeof(R) == 8) {
      const double wl = rsqrt(L[0]), wr = rsqrt(Rt[0]);
      const double inv = 1.0 / (L[0] * wl + Rt[0] * wr);
      u = (L[mu] * wl + Rt[mu] * wr) * inv;
      v = (L[mv] * wl + Rt[mv] * wr) * inv;
      const double gh = ph.grav * ((L[0] + Rt[0]) * 0.50);
      const double ia = rsqrt(gh);
      a = gh * ia;
      ha = 0.50 * ia;
      return;
    }
    const R g = (R)ph.grav;
    R h = (L[0] + Rt[0]) * (R)0.50;
    R hsqrtl = sqrt(L[0]);
    R hsqrtr = sqrt(Rt[0]);
    R hsq2 = hsqrtl + hsqrtr;
    u = (L[mu] / hsqrtl + Rt[mu] / hsqrtr) / hsq2;
    v = (L[mv] / hsqrtl + Rt[mv] / hsqrtr) / hsq2;
    a = sqrt(g * h);
    ha = (R)0.50 / a;
  }

  // Roe averages and the three waves of rpn2sw.f:80-118 along ixy.
  template <class R, bool FD = false>
  __device__ static void wave_set(const Phys& ph, int ixy, const R* L, const R* Rt, const R* dl, R& u,
                                  R& a, R w[3][3]) {
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    R v, ha;
    roe<R, FD>(ph, mu, mv, L, Rt, u, v, a, ha);                             // rpn2sw.f:80-88
    R a1 = ((u + a) * dl[0] - dl[mu]) * ha;                                 // :98-100
    R a2 = -(v * dl[0]) + dl[mv];
    R a3 = (-((u - a) * dl[0]) + dl[mu]) * ha;
    w[0][0] = a1; w[0][mu] = a1 * (u - a); w[0][mv] = a1 * v;
    w[1][0] = (R)0; w[1][mu] = (R)0;       w[1][mv] = a2;
    w[2][0] = a3; w[2][mu] = a3 * (u + a); w[2][mv] = a3 * v;
  }

  template <class R, bool FD = false>
  __device__ static void waves(const Phys& ph, int ixy, const R* L, const R* Rt, const R* dl, const R*,
                               const R*, R w[3][3], R* s = nullptr) {
    R u, a;
    wave_set<R, FD>(ph, ixy, L, Rt, dl, u, a, w);
    if (s) { s[0] = u - a; s[1] = u; s[2] = u + a; }
  }

  template <class R, bool FD = false>
  __device__ static void solve(const Phys& ph, int ixy, const R* L, const R* Rt, const R* dl,
                               R* s, R* amdq, R* apdq) {
    const R g = (R)ph.grav;
    const int mu = (ixy == 1) ? 1 : 2;
    R u, a, w[3][3];
    wave_set<R, FD>(ph, ixy, L, Rt, dl, u, a, w);
    s[0] = u - a; s[1] = u; s[2] = u + a;
    if (!ph.efix) {                                                         // :132-143
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        R am = (R)0, ap = (R)0;
#pragma unroll
        for (int mw = 0; mw < 3; ++mw) {
          if (s[mw] < (R)0) am = am + s[mw] * w[mw][m];
          else ap = ap + s[mw] * w[mw][m];
        }
        amdq[m] = am; apdq[m] = ap;
      }
      return;
    }
    do {                                                                    // :158-217
      R him1 = L[0];
      R s0 = L[mu] / him1 - sqrt(g * him1);
      if (s0 > (R)0 && s[0] > (R)0) {
        amdq[0] = amdq[1] = amdq[2] = (R)0;
        break;
      }
      R h1 = L[0] + w[0][0];
      R hu1 = L[mu] + w[0][mu];
      R s1 = hu1 / h1 - sqrt(g * h1);
      R sfract;
      if (s0 < (R)0 && s1 > (R)0) sfract = s0 * ((s1 - s[0]) / (s1 - s0));
      else if (s[0] < (R)0) sfract = s[0];
      else sfract = (R)0;
#pragma unroll
      for (int m = 0; m < 3; ++m) amdq[m] = sfract * w[0][m];
      if (s[1] > (R)0) break;
#pragma unroll
      for (int m = 0; m < 3; ++m) amdq[m] = amdq[m] + s[1] * w[1][m];
      R hi = Rt[0];
      R s03 = Rt[mu] / hi + sqrt(g * hi);
      R h3 = Rt[0] - w[2][0];
      R hu3 = Rt[mu] - w[2][mu];
      R s3 = hu3 / h3 + sqrt(g * h3);
      if (s3 < (R)0 && s03 > (R)0) sfract = s3 * ((s03 - s[2]) / (s03 - s3));
      else if (s[2] < (R)0) sfract = s[2];
      else break;
#pragma unroll
      for (int m = 0; m < 3; ++m) amdq[m] = amdq[m] + sfract * w[2][m];
    } while (0);
#pragma unroll
    for (int m = 0; m < 3; ++m) {                                           // :221-228
      R df = (R)0;
#pragma unroll
      for (int mw = 0; mw < 3; ++mw) df = df + s[mw] * w[mw][m];
      apdq[m] = df - amdq[m];
    }
  }

  template <class R, bool FD = false>
  __device__ static void rp(const Phys& ph, int ixy, const R* L, const R* Rt, const R* dl, const R*,
                            const R*, R* s, R* amdq, R* apdq) {
    solve<R, FD>(ph, ixy, L, Rt, dl, s, amdq, apdq);
  }
  // tfluct1sw.f: the same Roe solve with left ql(i), right qr(i); adq = amdq+apdq
  template <class R, bool FD = false>
  __device__ static void tfluct(const Phys& ph, int ixy, const R* L, const R* Rt, const R* dl,
                                const R*, R* adq) {
    R s[3], am[3], ap[3];
    solve<R, FD>(ph, ixy, L, Rt, dl, s, am, ap);
#pragma unroll
    for (int m = 0; m < 3; ++m) adq[m] = am[m] + ap[m];
  }
  // Shallow-water Roe eigenvectors along ixy (new; the reference has none).
  // Averages as rpn2sw.f:80-88; left eigenvectors are the rows rpn2sw.f:98-100
  // uses for a1..a3.
  template <class R, bool FD = false>
  __device__ static void evec(const Phys& ph, int ixy, const R* qm, const R* q0, const R*,
                              const R*, R evl[3][3], R evr[3][3]) {
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
    R u, v, a, ha;
    roe<R, FD>(ph, mu, mv, qm, q0, u, v, a, ha);
    evr[0][0] = (R)1;  evr[mu][0] = u - a; evr[mv][0] = v;
    evr[0][1] = (R)0;  evr[mu][1] = (R)0;  evr[mv][1] = (R)1;
    evr[0][2] = (R)1;  evr[mu][2] = u + a; evr[mv][2] = v;
    evl[0][0] = (u + a) * ha;    evl[0][mu] = -ha;    evl[0][mv] = (R)0;
    evl[1][0] = -v;              evl[1][mu] = (R)0;   evl[1][mv] = (R)1;
    evl[2][0] = -((u - a) * ha); evl[2][mu] = ha;     evl[2][mv] = (R)0;
  }
};

// ------------------------------------------------------------------------
// 1-D shallow water: apps/shallowWater/2dRadialDam/1dRadialSymm-qwave/
// rp1sw.f:43-185 (Roe solver, Harten-Hyman entropy fix when ph.efix, the
// app's data efix /.true./) and tfluct1sw.f:44-186 of the same app (the same
// solve with left ql(i), right qr(i); adq = amdq + apdq).
// ------------------------------------------------------------------------
struct PShallow1D {
  static constexpr int MEQN = 2, MWAVES = 2, MAUX = 0, NDIM = 1;
  static constexpr bool HAS_TFLUCT = true;

  // Roe averages of rp1sw.f:47-49: velocity u, celerity c, ha = 0.5/c (ha
  // only in the forms that multiply by it).
  template <class R, bool FD = false>
  __device__ static void roe(const Phys& ph, const R* L, const R* Rt, R& u, R& c, R& ha) {
#if SCL_FAST_ROE
    if constexpr (sizeof(R) == 4) {
      const float wl = rsqrtf(L[0]), wr = rsqrtf(Rt[0]);
      u = (L[1] * wl + Rt[1] * wr) * rcp32(L[0] * wl + Rt[0] * wr);
      const float gh = (0.5f * (float)ph.grav) * (L[0] + Rt[0]);
      const float ia = rsqrtf(gh);
      c = gh * ia;
      ha = 0.5f * ia;
      return;
    }
#endif
    if constexpr (FD && sizeof(R) == 8) {
      const double wl = rsqrt(L[0]), wr = rsqrt(Rt[0]);
      u = (L[1] * wl + Rt[1] * wr) * (1.0 / (L[0] * wl + Rt[0] * wr));
      const double gh = (0.5 * ph.grav) * (L[0] + Rt[0]);
      const double ia = rsqrt(gh);
      c = gh * ia;
      ha = 0.5 * ia;
      return;
    }
    u = (L[1] / sqrt(L[0]) + Rt[1] / sqrt(Rt[0])) / (sqrt(L[0]) + sqrt(Rt[0]));
    c = sqrt(((R)0.5 * (R)ph.grav) * (L[0] + Rt[0]));
    ha = (R)0.5 / c;
  }

  // The two waves and speeds of rp1sw.f:52-66 (dl = right - left state).
  template <class R, bool FD = false>
  __device__ static void wave_set(const Phys& ph, const R* L, const R* Rt, const R* dl, R w[2][2], R* s) {
    R u, c, ha;
    roe<R, FD>(ph, L, Rt, u, c, ha);
    R a1, a2;
    if constexpr (sizeof(R) == 4 || FD) {
      a1 = ((u + c) * dl[0] - dl[1]) * ha;
      a2 = (dl[1] - (u - c) * dl[0]) * ha;
    } else {
      a1 = ((R)0.5 * ((u + c) * dl[0] - dl[1])) / c;    // :56, -d2 + x == x - d2
      a2 = ((R)0.5 * (dl[1] - (u - c) * dl[0])) / c;    // :57
    }
    w[0][0] = a1; w[0][1] = a1 * (u - c); s[0] = u - c;
    w[1][0] = a2; w[1][1] = a2 * (u + c); s[1] = u + c;
  }

  template <class R, bool FD = false>
  __device__ static void waves(const Phys& ph, int, const R* L, const R* Rt, const R* dl, const R*,
                               const R*, R w[2][2], R* s = nullptr) {
    R sp[2];
    wave_set<R, FD>(ph, L, Rt, dl, w, sp);
    if (s) { s[0] = sp[0]; s[1] = sp[1]; }
  }

  template <class R, bool FD = false>
  __device__ static void solve(const Phys& ph, const R* L, const R* Rt, const R* dl, R* s, R* amdq,
                               R* apdq) {
    R w[2][2];
    wave_set<R, FD>(ph, L, Rt, dl, w, s);
    if (!ph.efix) {                                                         // :80-92
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        R am = (R)0, ap = (R)0;
#pragma unroll
        for (int mw = 0; mw < 2; ++mw) {
          if (s[mw] < (R)0) am = am + s[mw] * w[mw][m];
          else ap = ap + s[mw] * w[mw][m];
        }
        amdq[m] = am; apdq[m] = ap;
      }
      return;
    }
    const R g = (R)ph.grav;
    do {                                                                    // :113-173
      R s0 = L[1] / L[0] - sqrt(g * L[0]);
      if (s0 >= (R)0 && s[0] > (R)0) {
        amdq[0] = amdq[1] = (R)0;
        break;
      }
      R hr1 = L[0] + w[0][0];
      R uhr1 = L[1] + w[0][1];
      R s1 = uhr1 / hr1 - sqrt(g * hr1);
      R sfract;
      if (s0 < (R)0 && s1 > (R)0) sfract = (s0 * (s1 - s[0])) / (s1 - s0);
      else if (s[0] < (R)0) sfract = s[0];
      else sfract = (R)0;
      amdq[0] = sfract * w[0][0];
      amdq[1] = sfract * w[0][1];
      R s3 = Rt[1] / Rt[0] + sqrt(g * Rt[0]);
      R hl2 = Rt[0] - w[1][0];
      R uhl2 = Rt[1] - w[1][1];
      R s2 = uhl2 / hl2 + sqrt(g * hl2);
      if (s2 < (R)0 && s3 > (R)0) sfract = (s2 * (s3 - s[1])) / (s3 - s2);
      else if (s[1] < (R)0) sfract = s[1];
      else break;
      amdq[0] = amdq[0] + sfract * w[1][0];
      amdq[1] = amdq[1] + sfract * w[1][1];
    } while (0);
#pragma unroll
    for (int m = 0; m < 2; ++m) {                                           // :176-183
      R df = (R)0;
#pragma unroll
      for (int mw = 0; mw < 2; ++mw) df = df + s[mw] * w[mw][m];
      apdq[m] = df - amdq[m];
    }
  }

  template <class R, bool FD = false>
  __device__ static void rp(const Phys& ph, int, const R* L, const R* Rt, const R* dl, const R*,
                            const R*, R* s, R* amdq, R* apdq) {
    solve<R, FD>(ph, L, Rt, dl, s, amdq, apdq);
  }
  template <class R, bool FD = false>
  __device__ static void tfluct(const Phys& ph, int, const R* L, const R* Rt, const R* dl, const R*,
                                R* adq) {
    R s[2], am[2], ap[2];
    solve<R, FD>(ph, L, Rt, dl, s, am, ap);
    adq[0] = am[0] + ap[0];
    adq[1] = am[1] + ap[1];
  }
  // Roe eigenvectors (new; the reference has none): averages of rp1sw.f:47-49,
  // left eigenvectors the rows rp1sw.f:56-57 uses for a1, a2.
  template <class R, bool FD = false>
  __device__ static void evec(const Phys& ph, int, const R* qm, const R* q0, const R*, const R*,
                              R evl[2][2], R evr[2][2]) {
    R u, c, ha;
    roe<R, FD>(ph, qm, q0, u, c, ha);
    evr[0][0] = (R)1;  evr[0][1] = (R)1;
    evr[1][0] = u - c; evr[1][1] = u + c;
    evl[0][0] = (u + c) * ha;    evl[0][1] = -ha;
    evl[1][0] = -((u - c) * ha); evl[1][1] = ha;
  }
};

// ------------------------------------------------------------------------
// f-wave shallow water, the solvers of three apps (rpf-wave.f90:55-122 and
// tfluctf-wave.f90:55-126 of each): Roe averages, the app's flux difference
// split on the Roe eigenvectors into two f-waves, amdq / apdq by the sign of
// the speeds (half each for a NaN speed).  V selects the app:
//   0  apps/shallowWater/1dPerturbSteady: bathymetry b = aux(:,1); its source
//      g hbar (b(i+1) - b(i-1))/2 enters the cell's total fluctuation, which
//      therefore reads the aux of both neighbours (TFLUCT_NB)
//   1  2dRadialDam/1dRadialSymm-fwave: aux = (r, dx); the geometric source
//      hbar (uhat, uhat^2) dx / r enters the interface flux difference
//   2  2dRadialDam/1dRadialSymm-fwave-kappa: aux = (r(i-1/2), r, r, dx),
//      area-weighted fluxes (capacity aux(:,2)).
// ------------------------------------------------------------------------
template <int V>
struct PShallowF1D {
  static constexpr int MEQN = 2, MWAVES = 2, MAUX = V == 0 ? 1 : (V == 1 ? 2 : 4), NDIM = 1;
  static constexpr bool HAS_TFLUCT = true;
  static constexpr bool TFLUCT_NB = V == 0;

  // states, velocities and Roe averages (rpf-wave.f90:55-65)
  template <class R, bool FD>
  __device__ static void roe(const Phys& ph, const R* L, const R* Rt, R& ul, R& ur, R& hbar, R& uhat, R& chat) {
    const R hl = L[0], hr = Rt[0];
    if constexpr (sizeof(R) == 4 || FD) {
      // sqrt(h) u = m / sqrt(h) = m w for w = 1/sqrt(h)
      R wl, wr, inv;
      if constexpr (sizeof(R) == 4) {
        wl = rsqrtf(hl); wr = rsqrtf(hr);
        inv = rcp32(hl * wl + hr * wr);
      } else {
        wl = rsqrt(hl); wr = rsqrt(hr);
        inv = (R)1 / (hl * wl + hr * wr);
      }
      ul = L[1] * (wl * wl);
      ur = Rt[1] * (wr * wr);
      uhat = (L[1] * wl + Rt[1] * wr) * inv;
    } else {
      ul = L[1] / hl;
      ur = Rt[1] / hr;
      uhat = (sqrt(hl) * ul + sqrt(hr) * ur) / (sqrt(hl) + sqrt(hr));
    }
    hbar = (R)0.5 * (hr + hl);
    chat = sqrt((R)ph.grav * hbar);
  }

  // the app's flux difference at an interface (CELL false: left qr(i-1),
  // right ql(i), am = aux(i-1), a0 = aux(i)) or inside a cell (CELL true:
  // left ql(i), right qr(i); a0 = aux(i), for V = 0 a0 points at aux(i-1..i+1))
  template <bool CELL, class R>
  __device__ static void flux_diff(const Phys& ph, const R* L, const R* Rt, R ul, R ur, R hbar, R uhat,
                                   const R* am, const R* a0, R& f1, R& f2) {
    const R hl = L[0], hr = Rt[0], g = (R)ph.grav, hg = (R)0.5 * g;
    if constexpr (V == 0 && !CELL) {                           // 1dPerturbSteady/rpf-wave.f90:67-68
      f1 = (hr * ur) - (hl * ul);
      f2 = ((hr * ur) * ur + hg * (hr * hr)) - ((hl * ul) * ul + hg * (hl * hl));
    } else if constexpr (V == 0) {                             // tfluctf-wave.f90:56-70
      const R bl = a0[0], br = a0[2];
      f1 = (hr * ur) - (hl * ul);
      f2 = (((hr * ur) * ur + (hg * hr) * hr) - ((hl * ul) * ul + (hg * hl) * hl)) + ((g * hbar) * (br - bl)) / (R)2;
    } else if constexpr (V == 1 && !CELL) {                    // 1dRadialSymm-fwave/rpf-wave.f90:69-70
      f1 = ((hr * ur) - (hl * ul)) + ((hbar * uhat) / a0[0]) * a0[1];
      f2 = (((hr * ur) * ur + hg * (hr * hr)) - ((hl * ul) * ul + hg * (hl * hl))) +
           ((hbar * (uhat * uhat)) / a0[0]) * a0[1];
    } else if constexpr (V == 1) {                             // tfluctf-wave.f90:68-69
      f1 = (hr * ur) - (hl * ul);
      f2 = ((hr * ur) * ur + (hg * hr) * hr) - ((hl * ul) * ul + (hg * hl) * hl);
    } else if constexpr (!CELL) {                              // -kappa/rpf-wave.f90:69-70
      f1 = a0[0] * (hr * ur) - am[0] * (hl * ul);
      f2 = (a0[0] * ((hr * ur) * ur + (hg * hr) * hr) - am[0] * ((hl * ul) * ul + (hg * hl) * hl)) -
           ((hg * hbar) * hbar) * a0[3];
    } else {                                                   // -kappa/tfluctf-wave.f90:68-69
      f1 = a0[1] * (hr * ur) - a0[1] * (hl * ul);
      f2 = a0[1] * ((hr * ur) * ur + (hg * hr) * hr) - a0[2] * ((hl * ul) * ul + (hg * hl) * hl);
    }
  }

  // f-waves fw[k][j] and speeds (rpf-wave.f90:72-103)
  template <bool CELL, class R, bool FD>
  __device__ static void fwaves(const Phys& ph, const R* L, const R* Rt, const R* am, const R* a0, R fw[2][2],
                                R* s) {
    R ul, ur, hbar, uhat, chat, f1, f2;
    roe<R, FD>(ph, L, Rt, ul, ur, hbar, uhat, chat);
    flux_diff<CELL, R>(ph, L, Rt, ul, ur, hbar, uhat, am, a0, f1, f2);
    s[0] = uhat - chat;
    s[1] = uhat + chat;
    R l11, l12, l21, l22;
    if constexpr (sizeof(R) == 4 || FD) {
      R i2c;
      if constexpr (sizeof(R) == 4) i2c = rcp32((R)2 * chat);
      else i2c = (R)1 / ((R)2 * chat);
      l11 = (chat + uhat) * i2c; l12 = -i2c;
      l21 = (chat - uhat) * i2c; l22 = i2c;
    } else {
      l11 = (chat + uhat) / ((R)2 * chat); l12 = -((R)1 / ((R)2 * chat));
      l21 = (chat - uhat) / ((R)2 * chat); l22 = (R)1 / ((R)2 * chat);
    }
    const R b1 = ((R)0 + l11 * f1) + l12 * f2;
    const R b2 = ((R)0 + l21 * f1) + l22 * f2;
    fw[0][0] = b1 * (R)1; fw[0][1] = b1 * s[0];
    fw[1][0] = b2 * (R)1; fw[1][1] = b2 * s[1];
  }

  template <class R>
  __device__ static void split(const R fw[2][2], const R* s, R* amdq, R* apdq) {   // rpf-wave.f90:106-119
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      R am = (R)0, ap = (R)0;
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        if (s[k] < (R)0) am = am + fw[k][j];
        else if (s[k] >= (R)0) ap = ap + fw[k][j];
        else { am = am + (R)0.5 * fw[k][j]; ap = ap + (R)0.5 * fw[k][j]; }
      }
      amdq[j] = am; apdq[j] = ap;
    }
  }

  template <class R, bool FD = false>
  __device__ static void rp(const Phys& ph, int, const R* L, const R* Rt, const R*, const R* auxm,
                            const R* aux0, R* s, R* amdq, R* apdq) {
    R fw[2][2];
    fwaves<false, R, FD>(ph, L, Rt, auxm, aux0, fw, s);
    split<R>(fw, s, amdq, apdq);
  }
  template <class R, bool FD = false>
  __device__ static void waves(const Phys& ph, int, const R* L, const R* Rt, const R*, const R* auxm,
                               const R* aux0, R w[2][2], R* s = nullptr) {
    R sp[2];
    fwaves<false, R, FD>(ph, L, Rt, auxm, aux0, w, sp);
    if (s) { s[0] = sp[0]; s[1] = sp[1]; }
  }
  template <class R, bool FD = false>
  __device__ static void tfluct(const Phys& ph, int, const R* L, const R* Rt, const R*, const R* aux,
                                R* adq) {
    R fw[2][2], s[2], am[2], ap[2];
    fwaves<true, R, FD>(ph, L, Rt, aux, aux, fw, s);
    split<R>(fw, s, am, ap);
    adq[0] = am[0] + ap[0];                                  // tfluctf-wave.f90:121-123
    adq[1] = am[1] + ap[1];
  }
  // Roe eigenvectors R and L of rpf-wave.f90:71-88 from q(i-1), q(i)
  template <class R, bool FD = false>
  __device__ static void evec(const Phys& ph, int, const R* qm, const R* q0, const R*, const R*,
                              R evl[2][2], R evr[2][2]) {
    R ul, ur, hbar, uhat, chat;
    roe<R, FD>(ph, qm, q0, ul, ur, hbar, uhat, chat);
    evr[0][0] = (R)1; evr[0][1] = (R)1;
    evr[1][0] = uhat - chat; evr[1][1] = uhat + chat;
    if constexpr (sizeof(R) == 4 || FD) {
      R i2c;
      if constexpr (sizeof(R) == 4) i2c = rcp32((R)2 * chat);
      else i2c = (R)1 / ((R)2 * chat);
      evl[0][0] = (chat + uhat) * i2c; evl[0][1] = -i2c;
      evl[1][0] = (chat - uhat) * i2c; evl[1][1] = i2c;
    } else {
      evl[0][0] = (chat + uhat) / ((R)2 * chat); evl[0][1] = -((R)1 / ((R)2 * chat));
      evl[1][0] = (chat - uhat) / ((R)2 * chat); evl[1][1] = (R)1 / ((R)2 * chat);
    }
  }
};

// ------------------------------------------------------------------------
// Constant-coefficient acoustics, apps/acoustics/1d/homogeneous (rp1.f:50-76,
// tfluct.f, evec.f): cc = sqrt(bulk/rho), zz = cc*rho (setprob.f), passed in
// Phys as cc, zz.
// ------------------------------------------------------------------------
struct PAcousticsConst {
  static constexpr int MEQN = 2, MWAVES = 2, MAUX = 0, NDIM = 1;
  static constexpr bool HAS_TFLUCT = true;

  template <class R, bool FD = false>
  __device__ static void waves(const Phys& ph, int, const R*, const R*, const R* dl, const R*, const R*,
                               R w[2][2], R* s = nullptr) {
    const R zz = (R)ph.zz, cc = (R)ph.cc;
    R a1, a2;
    if constexpr (sizeof(R) == 4 || FD) {
      const R i2z = (R)1 / ((R)2 * zz);
      a1 = ((-dl[0]) + zz * dl[1]) * i2z;
      a2 = (dl[0] + zz * dl[1]) * i2z;
    } else {
      a1 = ((-dl[0]) + zz * dl[1]) / ((R)2 * zz);
      a2 = (dl[0] + zz * dl[1]) / ((R)2 * zz);
    }
    w[0][0] = -(a1 * zz); w[0][1] = a1;
    w[1][0] = a2 * zz;    w[1][1] = a2;
    if (s) { s[0] = -cc; s[1] = cc; }
  }
  template <class R, bool FD = false>
  __device__ static void rp(const Phys& ph, int ixy, const R* L, const R* Rt, const R* dl, const R* am,
                            const R* a0, R* s, R* amdq, R* apdq) {
    R w[2][2];
    waves<R, FD>(ph, ixy, L, Rt, dl, am, a0, w, s);
#pragma unroll
    for (int m = 0; m < 2; ++m) {
      amdq[m] = s[0] * w[0][m];
      apdq[m] = s[1] * w[1][m];
    }
  }
  template <class R, bool FD = false>
  __device__ static void tfluct(const Phys& ph, int ixy, const R* L, const R* Rt, const R* dl, const R* aux,
                                R* adq) {
    R w[2][2], s[2];
    waves<R, FD>(ph, ixy, L, Rt, dl, aux, aux, w, s);
#pragma unroll
    for (int m = 0; m < 2; ++m) adq[m] = s[0] * w[0][m] + s[1] * w[1][m];
  }
  template <class R, bool FD = false>
  __device__ static void evec(const Phys& ph, int, const R*, const R*, const R*, const R*, R evl[2][2],
                              R evr[2][2]) {
    const R zz = (R)ph.zz;
    evr[0][0] = -zz;   evr[0][1] = zz;
    evr[1][0] = (R)1;  evr[1][1] = (R)1;
    const R z = (R)1 / (zz + zz);
    evl[0][0] = -z;        evl[0][1] = zz * z;
    evl[1][0] = (R)1 * z;  evl[1][1] = zz * z;
  }
};

// ------------------------------------------------------------------------
// Elasticity in strain / momentum form with f-waves, q = (eps, rho u):
//   NL = 0  apps/acoustics/1d/fwave (rp1acfw.f:53-109, tfluct1.f, evec.f):
//           linear stress sigma = bulk*eps (rp1acfw.f:116-140), aux = (rho, bulk)
//   NL = 1  apps/elasticity/stegoton (rp1nel.f:53-175, tfluct1.f): sigma =
//           exp(A eps) - 1 where A > 0, else B eps; aux = (rho, A, B)
// The acoustics app's evec puts the rows (1, 1) and (zim, -zi) in evl and
// their inverse in evr; kept as written, and used with the stegoton's
// stress law too (that app builds no evec; new).
// ------------------------------------------------------------------------
template <int NL>
struct PElasticFwave {
  static constexpr int MEQN = 2, MWAVES = 2, MAUX = NL ? 3 : 2, NDIM = 1;
  static constexpr bool HAS_TFLUCT = true;

  // stress and its derivative of the material a at strain eps.  In FP32,
  // exp(A eps) - 1 cancels at small strain (1.0004f - 1 keeps ~3 digits), so
  // the FP32 forms evaluate the same function as expm1f; FP64 keeps the
  // written form of rp1nel.f:124.
  template <class R>
  __device__ static R sigma(R eps, const R* a) {
    if constexpr (NL) {
      if constexpr (sizeof(R) == 4) {
        if (a[1] > (R)0) return expm1f(a[1] * eps);
      } else {
        if (a[1] > (R)0) return exp(a[1] * eps) - (R)1;
      }
      return a[2] * eps;
    } else {
      return a[1] * eps;
    }
  }
  template <class R>
  __device__ static R sigmap(R eps, const R* a) {
    if constexpr (NL) {
      if (a[1] > (R)0) return a[1] * exp(a[1] * eps);
      return a[2];
    } else {
      return a[1];
    }
  }

  // f-waves between the left state L (material am) and the right state Rt
  // (material a0)
  template <class R, bool FD = false>
  __device__ static void fwaves(const R* L, const R* Rt, const R* am, const R* a0, R w[2][2], R* s) {
    const R rhoi = a0[0], rhoim = am[0], ki = sigmap<R>(Rt[0], a0), kim = sigmap<R>(L[0], am);
    R ci, cim, du, inv;
    if constexpr (sizeof(R) == 4 || FD) {
      const R iri = (R)1 / rhoi, irim = (R)1 / rhoim;
      ci = sqrt(ki * iri);
      cim = sqrt(kim * irim);
      du = Rt[1] * iri - L[1] * irim;
    } else {
      ci = sqrt(ki / rhoi);
      cim = sqrt(kim / rhoim);
      du = Rt[1] / rhoi - L[1] / rhoim;
    }
    const R zi = ci * rhoi, zim = cim * rhoim;
    const R dsig = sigma<R>(Rt[0], a0) - sigma<R>(L[0], am);
    R b1, b2;
    if constexpr (sizeof(R) == 4 || FD) {
      inv = (R)1 / (zim + zi);
      b1 = -((zi * du + dsig) * inv);
      b2 = -((zim * du - dsig) * inv);
    } else {
      b1 = -((zi * du + dsig) / (zim + zi));
      b2 = -((zim * du - dsig) / (zim + zi));
    }
    w[0][0] = b1; w[0][1] = b1 * zim;    s[0] = -cim;
    w[1][0] = b2; w[1][1] = b2 * (-zi);  s[1] = ci;
  }
  template <class R, bool FD = false>
  __device__ static void waves(const Phys&, int, const R* L, const R* Rt, const R*, const R* am,
                               const R* a0, R w[2][2], R* s = nullptr) {
    R sp[2];
    fwaves<R, FD>(L, Rt, am, a0, w, sp);
    if (s) { s[0] = sp[0]; s[1] = sp[1]; }
  }
  template <class R, bool FD = false>
  __device__ static void rp(const Phys&, int, const R* L, const R* Rt, const R*, const R* am, const R* a0,
                            R* s, R* amdq, R* apdq) {
    R w[2][2];
    fwaves<R, FD>(L, Rt, am, a0, w, s);
#pragma unroll
    for (int m = 0; m < 2; ++m) { amdq[m] = w[0][m]; apdq[m] = w[1][m]; }
  }
  template <class R, bool FD = false>
  __device__ static void tfluct(const Phys&, int, const R* L, const R* Rt, const R*, const R* aux, R* adq) {
    R w[2][2], s[2];
    fwaves<R, FD>(L, Rt, aux, aux, w, s);
#pragma unroll
    for (int m = 0; m < 2; ++m) adq[m] = w[0][m] + w[1][m];
  }
  template <class R, bool FD = false>
  __device__ static void evec(const Phys&, int, const R* qm, const R* q0, const R* am, const R* a0, R evl[2][2],
                              R evr[2][2]) {
    const R ki = sigmap<R>(q0[0], a0), kim = sigmap<R>(qm[0], am);
    R ci, cim;
    if constexpr (sizeof(R) == 4 || FD) {
      ci = sqrt(ki * ((R)1 / a0[0]));
      cim = sqrt(kim * ((R)1 / am[0]));
    } else {
      ci = sqrt(ki / a0[0]);
      cim = sqrt(kim / am[0]);
    }
    const R zi = ci * a0[0], zim = cim * am[0];
    evl[0][0] = (R)1; evl[0][1] = (R)1;
    evl[1][0] = zim;  evl[1][1] = -zi;
    const R zh = (R)1 / (zim + zi);
    evr[0][0] = zi * zh;  evr[0][1] = zh;
    evr[1][0] = zim * zh; evr[1][1] = -zh;
  }
};

// ------------------------------------------------------------------------
// Traffic flow with a variable speed limit, apps/traffic/congTraffic
// (rpf-wave.f90:42-90, tfluct1.f90:39-49): flux umax(x) q (1-q), aux = umax;
// the f-wave goes left, right, or (transonic rarefaction) splits at the
// sonic flux min(umax) / 4.
// ------------------------------------------------------------------------
struct PTraffic {
  static constexpr int MEQN = 1, MWAVES = 1, MAUX = 1, NDIM = 1;
  static constexpr bool HAS_TFLUCT = true;
  template <class R, bool FD = false>
  __device__ static void rp(const Phys&, int, const R* L, const R* Rt, const R*, const R* am, const R* a0,
                            R* s, R* amdq, R* apdq) {
    const R fim1 = (am[0] * L[0]) * ((R)1 - L[0]);
    const R fi = (a0[0] * Rt[0]) * ((R)1 - Rt[0]);
    const R fw = fi - fim1;
    const R sim1 = am[0] * ((R)1 - (R)2 * L[0]);
    const R si = a0[0] * ((R)1 - (R)2 * Rt[0]);
    if (sim1 < (R)0 && si <= (R)0) {
      s[0] = sim1; amdq[0] = fw; apdq[0] = (R)0;
    } else if (sim1 >= (R)0 && si > (R)0) {
      s[0] = si; amdq[0] = (R)0; apdq[0] = fw;
    } else if (sim1 < (R)0 && si > (R)0) {
      s[0] = (R)0.5 * (sim1 + si);
      const R f0 = rmin(am[0], a0[0]) * (R)0.25;
      amdq[0] = f0 - fim1;
      apdq[0] = fi - f0;
    } else {
      s[0] = (R)0.5 * (sim1 + si);
      if (s[0] < (R)0) { amdq[0] = fw; apdq[0] = (R)0; }
      else if (s[0] > (R)0) { amdq[0] = (R)0; apdq[0] = fw; }
      else { amdq[0] = (R)0.5 * fw; apdq[0] = (R)0.5 * fw; }
    }
  }
  template <class R, bool FD = false>
  __device__ static void waves(const Phys& ph, int ixy, const R* L, const R* Rt, const R* dl, const R* am,
                               const R* a0, R w[1][1], R* s = nullptr) {
    w[0][0] = (a0[0] * Rt[0]) * ((R)1 - Rt[0]) - (am[0] * L[0]) * ((R)1 - L[0]);
    if (s) {
      R sp[1], m1[1], p1[1];
      rp<R, FD>(ph, ixy, L, Rt, dl, am, a0, sp, m1, p1);
      s[0] = sp[0];
    }
  }
  template <class R, bool FD = false>
  __device__ static void tfluct(const Phys&, int, const R* L, const R* Rt, const R*, const R* aux, R* adq) {
    adq[0] = (aux[0] * Rt[0]) * ((R)1 - Rt[0]) - (aux[0] * L[0]) * ((R)1 - L[0]);
  }
  template <class R, bool FD = false>
  __device__ static void evec(const Phys&, int, const R*, const R*, const R*, const R*, R evl[1][1],
                              R evr[1][1]) {
    evl[0][0] = (R)1;
    evr[0][0] = (R)1;
  }
};

// ------------------------------------------------------------------------
// Conservative advection with cell velocities, apps/traffic/flux-uq
// (rpf-wave.f90:43-64): f-wave u(i) q(i) - u(i-1) q(i-1), to the right when
// u(i) > 0, aux = u.  The app has no tfluct (tfluct_solver 0).
// ------------------------------------------------------------------------
struct PAdvCons {
  static constexpr int MEQN = 1, MWAVES = 1, MAUX = 1, NDIM = 1;
  static constexpr bool HAS_TFLUCT = false;
  template <class R, bool FD = false>
  __device__ static void rp(const Phys&, int, const R* L, const R* Rt, const R*, const R* am, const R* a0,
                            R* s, R* amdq, R* apdq) {
    const R fw = a0[0] * Rt[0] - am[0] * L[0];
    if (a0[0] > (R)0) { s[0] = a0[0]; amdq[0] = (R)0; apdq[0] = fw; }
    else { s[0] = am[0]; amdq[0] = fw; apdq[0] = (R)0; }
  }
  template <class R, bool FD = false>
  __device__ static void waves(const Phys&, int, const R* L, const R* Rt, const R*, const R* am, const R* a0,
                               R w[1][1], R* s = nullptr) {
    w[0][0] = a0[0] * Rt[0] - am[0] * L[0];
    if (s) s[0] = a0[0] > (R)0 ? a0[0] : am[0];
  }
  template <class R, bool FD = false>
  __device__ static void tfluct(const Phys&, int, const R*, const R*, const R*, const R*, R*) {}
  template <class R, bool FD = false>
  __device__ static void evec(const Phys&, int, const R*, const R*, const R*, const R*, R evl[1][1],
                              R evr[1][1]) {
    evl[0][0] = (R)1;
    evr[0][0] = (R)1;
  }
};

// Plugins whose total fluctuation reads the aux of cells c-1, c, c+1 (three
// MAUX groups, centre in the middle) declare TFLUCT_NB = true.
template <class P, class = void>
struct tfluct_nb : std::false_type {};
template <class P>
struct tfluct_nb<P, std::void_t<decltype(P::TFLUCT_NB)>> : std::bool_constant<P::TFLUCT_NB> {};

// ------------------------------------------------------------------------
// 2-D advection with edge velocities (apps/advection/2d/swirl/rpn2ad1.f:
// 39-45): aux(i,j,1) = u on the left edge, aux(i,j,2) = v on the bottom edge
// of cell (i,j); the speed at interface i-1/2 along ixy is aux(i,ixy) of the
// right cell.  No tfluct exists (the app runs the swapped second solve).
// ------------------------------------------------------------------------
struct PAdvEdge2D {
  static constexpr int MEQN = 1, MWAVES = 1, MAUX = 2, NDIM = 2;
  static constexpr bool HAS_TFLUCT = false;
  template <class R, bool FD = false>
  __device__ static void rp(const Phys&, int ixy, const R*, const R*, const R* dl, const R*,
                            const R* auxr, R* s, R* amdq, R* apdq) {
    const R u = auxr[ixy - 1];
    s[0] = u;
    amdq[0] = rmin(u, (R)0) * dl[0];
    apdq[0] = rmax(u, (R)0) * dl[0];
  }
  template <class R, bool FD = false>
  __device__ static void waves(const Phys&, int ixy, const R*, const R*, const R* dl, const R*,
                               const R* auxr, R w[1][1], R* s = nullptr) {
    w[0][0] = dl[0];
    if (s) s[0] = auxr[ixy - 1];
  }
  template <class R, bool FD = false>
  __device__ static void tfluct(const Phys&, int, const R*, const R*, const R*, const R*, R*) {}
  template <class R, bool FD = false>
  __device__ static void evec(const Phys&, int, const R*, const R*, const R*, const R*,
                              R evl[1][1], R evr[1][1]) {
    evl[0][0] = (R)1;
    evr[0][0] = (R)1;
  }
};

// ------------------------------------------------------------------------
// Variable-coefficient acoustics, aux(:,1) = impedance Z, aux(:,2) = c.
// 1-D: apps/acoustics/1d/interface/rp1acv.f:49-80, tfluct1acv.f:134-166,
// evec.f90:196-206.  2-D (new): the same solve normal to the slice
// (mu = normal velocity), the tangential velocity carries no wave.
// ------------------------------------------------------------------------
template <int NEQ>
struct PAcoustics {
  static constexpr int MEQN = NEQ, MWAVES = 2, MAUX = 2, NDIM = (NEQ == 2 ? 1 : 2);
  static constexpr bool HAS_TFLUCT = true;
  template <class R, bool FD = false>
  __device__ static void rp(const Phys& ph, int ixy, const R* L, const R* Rt, const R* dl, const R* auxl,
                            const R* auxr, R* s, R* amdq, R* apdq) {
    // auxl = aux of the left cell (auxr(i-1,:)), auxr = aux of the right cell (auxl(i,:))
    R w[2][NEQ];
    waves<R, FD>(ph, ixy, L, Rt, dl, auxl, auxr, w);
    s[0] = -auxl[1];
    s[1] = auxr[1];
#pragma unroll
    for (int m = 0; m < NEQ; ++m) {
      amdq[m] = s[0] * w[0][m];
      apdq[m] = s[1] * w[1][m];
    }
  }
  // the two waves of rp1acv.f:49-60 (zero tangential component in 2-D)
  template <class R, bool FD = false>
  __device__ static void waves(const Phys&, int ixy, const R*, const R*, const R* dl, const R* auxl,
                               const R* auxr, R w[2][NEQ], R* s = nullptr) {
    const int mu = (ixy == 1) ? 1 : 2;
    if (s) { s[0] = -auxl[1]; s[1] = auxr[1]; }
    R zi = auxr[0];
    R zim = auxl[0];
    R a1, a2;
    if constexpr (FD) {
      const R iz = (R)1 / (zim + zi);
      a1 = ((-dl[0]) + zi * dl[mu]) * iz;
      a2 = (dl[0] + zim * dl[mu]) * iz;
    } else {
      a1 = ((-dl[0]) + zi * dl[mu]) / (zim + zi);
      a2 = (dl[0] + zim * dl[mu]) / (zim + zi);
    }
#pragma unroll
    for (int m = 0; m < NEQ; ++m) { w[0][m] = (R)0; w[1][m] = (R)0; }
    w[0][0] = -(a1 * zim); w[0][mu] = a1;
    w[1][0] = a2 * zi;     w[1][mu] = a2;
  }
  template <class R, bool FD = false>
  __device__ static void tfluct(const Phys&, int ixy, const R*, const R*, const R* dl,
                                const R* aux, R* adq) {
    const int mu = (ixy == 1) ? 1 : 2;
    R zi = aux[0];
    R zim = aux[0];
    R a1, a2;
    if constexpr (FD) {
      const R iz = (R)1 / (zim + zi);
      a1 = ((-dl[0]) + zi * dl[mu]) * iz;
      a2 = (dl[0] + zim * dl[mu]) * iz;
    } else {
      a1 = ((-dl[0]) + zi * dl[mu]) / (zim + zi);
      a2 = (dl[0] + zim * dl[mu]) / (zim + zi);
    }
    R s1 = -aux[1], s2 = aux[1];
    R w1[NEQ], w2[NEQ];
#pragma unroll
    for (int m = 0; m < NEQ; ++m) { w1[m] = (R)0; w2[m] = (R)0; }
    w1[0] = -(a1 * zim); w1[mu] = a1;
    w2[0] = a2 * zi;     w2[mu] = a2;
#pragma unroll
    for (int m = 0; m < NEQ; ++m) {
      R am = s1 * w1[m];
      R ap = s2 * w2[m];
      adq[m] = am + ap;
    }
  }
  template <class R, bool FD = false>
  __device__ static void evec(const Phys&, int ixy, const R*, const R*, const R* auxm,
                              const R* aux0, R evl[NEQ][NEQ], R evr[NEQ][NEQ]) {
    const int mu = (ixy == 1) ? 1 : 2, mv = (ixy == 1) ? 2 : 1;
#pragma unroll
    for (int a = 0; a < NEQ; ++a)
#pragma unroll
      for (int b = 0; b < NEQ; ++b) { evl[a][b] = (R)0; evr[a][b] = (R)0; }
    evr[0][0] = -auxm[0];
    evr[0][1] = aux0[0];
    evr[mu][0] = (R)1;
    evr[mu][1] = (R)1;
    R z = (R)1 / (auxm[0] + aux0[0]);
    evl[0][0] = (R)(-1) * z;
    evl[0][mu] = aux0[0] * z;
    evl[1][0] = (R)1 * z;
    evl[1][mu] = auxm[0] * z;
    if (NEQ == 3) {
      evr[mv][2] = (R)1;
      evl[2][mv] = (R)1;
    }
  }
};

}  // namespace scl
