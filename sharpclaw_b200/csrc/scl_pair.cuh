// scl_pair.cuh -- the 1-D Euler stage with two interfaces (and two cells) per
// thread in packed FP32 arithmetic (sm_100 f32x2: one instruction computes
// both lanes).  Lane x is interface/cell c, lane y interface/cell c+1; every
// operation of the FP32 forms of k_stage1d (char-wise WENO5 on offsets, Roe
// eigenvectors, Roe solver with Harten-Hyman entropy fix, the swapped second
// solve of flux1.f90:155-188) runs once for both.  Data-dependent branches of
// the entropy fix become per-lane selects, entered when either lane needs
// them.  Used for PEuler, char_decomp 0 or 2, tfluct_solver 0, mixed / FP32.
#pragma once
#include "scl_batch.cuh"
#include "scl_kernels.cuh"
#include "scl_tma.cuh"

namespace scl {

// ---- packed FP32 helpers ------------------------------------------------
using f2 = float2;
struct m2 { bool x, y; };

__device__ __forceinline__ f2 F2(float a) { return make_float2(a, a); }
__device__ __forceinline__ f2 F2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ f2 add(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 sub(f2 a, f2 b) { return __ffma2_rn(b, F2(-1.0f), a); }
__device__ __forceinline__ f2 mul(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ f2 rsq2(f2 a) { return F2(rsqrtf(a.x), rsqrtf(a.y)); }
__device__ __forceinline__ f2 rcp2(f2 a) { return F2(rcp32(a.x), rcp32(a.y)); }
__device__ __forceinline__ f2 sqrt2(f2 a) { return F2(sqrtf(a.x), sqrtf(a.y)); }
__device__ __forceinline__ f2 sel(m2 m, f2 a, f2 b) { return F2(m.x ? a.x : b.x, m.y ? a.y : b.y); }
__device__ __forceinline__ m2 lt0(f2 a) { return {a.x < 0.0f, a.y < 0.0f}; }
__device__ __forceinline__ m2 gt0(f2 a) { return {a.x > 0.0f, a.y > 0.0f}; }
__device__ __forceinline__ m2 ge0(f2 a) { return {a.x >= 0.0f, a.y >= 0.0f}; }
__device__ __forceinline__ m2 operator&(m2 a, m2 b) { return {a.x && b.x, a.y && b.y}; }
__device__ __forceinline__ m2 operator|(m2 a, m2 b) { return {a.x || b.x, a.y || b.y}; }
__device__ __forceinline__ m2 operator!(m2 a) { return {!a.x, !a.y}; }
__device__ __forceinline__ bool any(m2 a) { return a.x || a.y; }
__device__ __forceinline__ bool all(m2 a) { return a.x && a.y; }

// ---- Euler, FP32 forms of the PEuler plugin on two lanes ----------------
struct EulerPair {
  // Roe averages (rp1eu.f:44-55 in the reciprocal-square-root form)
  __device__ static void roe(const Phys& ph, const f2* L, const f2* R, f2& u, f2& enth, f2& a, f2& ia) {
    const f2 g1 = F2((float)ph.gamma1);
    const f2 wl = rsq2(L[0]), wr = rsq2(R[0]);
    const f2 pl = mul(g1, fma2(mul(F2(-0.5f), mul(L[1], L[1])), mul(wl, wl), L[2]));
    const f2 pr = mul(g1, fma2(mul(F2(-0.5f), mul(R[1], R[1])), mul(wr, wr), R[2]));
    const f2 inv = rcp2(fma2(L[0], wl, mul(R[0], wr)));
    u = mul(fma2(L[1], wl, mul(R[1], wr)), inv);
    enth = mul(fma2(add(L[2], pl), wl, mul(add(R[2], pr), wr)), inv);
    const f2 a2 = mul(g1, fma2(F2(-0.5f), mul(u, u), enth));
    ia = rsq2(a2);
    a = mul(a2, ia);
  }

  // Roe eigenvectors from the cell averages (PEuler::evec)
  __device__ static void evec(const Phys& ph, const f2* qm, const f2* q0, f2 evl[3][3], f2 evr[3][3]) {
    f2 u, h, a, ia;
    roe(ph, qm, q0, u, h, a, ia);
    const f2 g1 = F2((float)ph.gamma1), h5 = F2(0.5f), ua = mul(u, a), uu = mul(u, u);
    evr[0][0] = F2(1.0f); evr[0][1] = F2(1.0f); evr[0][2] = F2(1.0f);
    evr[1][0] = sub(u, a); evr[1][1] = u; evr[1][2] = add(u, a);
    evr[2][0] = sub(h, ua); evr[2][1] = mul(h5, uu); evr[2][2] = add(h, ua);
    const f2 b1 = mul(g1, mul(ia, ia));
    const f2 b2 = mul(h5, mul(b1, uu));
    const f2 uia = mul(u, ia), b1u = mul(b1, u);
    evl[0][0] = mul(h5, add(b2, uia)); evl[0][1] = mul(F2(-0.5f), add(b1u, ia)); evl[0][2] = mul(h5, b1);
    evl[1][0] = sub(F2(1.0f), b2);     evl[1][1] = b1u;                           evl[1][2] = F2(-b1.x, -b1.y);
    evl[2][0] = mul(h5, sub(b2, uia)); evl[2][1] = mul(F2(-0.5f), sub(b1u, ia)); evl[2][2] = mul(h5, b1);
  }

  // u -/+ c of one state (the entropy fix speeds, one reciprocal and one root)
  template <bool PLUS>
  __device__ static f2 speed(const Phys& ph, f2 rho, f2 m, f2 en) {
    const f2 ir = rcp2(rho), u = mul(m, ir);
    const f2 p = mul(F2((float)ph.gamma1), fma2(F2(-0.5f), mul(m, u), en));
    const f2 c = sqrt2(mul(mul(F2((float)ph.gamma), p), ir));
    return PLUS ? add(u, c) : sub(u, c);
  }

  // rp1eu.f:44-213: fluctuations of two Riemann problems (L | R, jump dl)
  __device__ static void rp(const Phys& ph, const f2* L, const f2* R, const f2* dl, f2* s, f2* am, f2* ap) {
    f2 u, enth, a, ia;
    roe(ph, L, R, u, enth, a, ia);
    const f2 g1 = F2((float)ph.gamma1);
    const f2 a2 = mul(mul(g1, mul(ia, ia)), sub(fma2(u, dl[1], mul(fma2(F2(-1.0f), mul(u, u), enth), dl[0])), dl[2]));
    const f2 a3 = mul(sub(fma2(sub(a, u), dl[0], dl[1]), mul(a, a2)), mul(F2(0.5f), ia));
    const f2 a1 = sub(sub(dl[0], a2), a3);
    const f2 ua = mul(u, a);
    f2 w[3][3];
    w[0][0] = a1; w[0][1] = mul(a1, sub(u, a)); w[0][2] = mul(a1, sub(enth, ua));
    w[1][0] = a2; w[1][1] = mul(a2, u);         w[1][2] = mul(mul(a2, F2(0.5f)), mul(u, u));
    w[2][0] = a3; w[2][1] = mul(a3, add(u, a)); w[2][2] = mul(a3, add(enth, ua));
    s[0] = sub(u, a); s[1] = u; s[2] = add(u, a);
    if (!ph.efix) {
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        f2 sa = F2(0.0f), sb = F2(0.0f);
#pragma unroll
        for (int mw = 0; mw < 3; ++mw) {
          const f2 sw = mul(s[mw], w[mw][m]);
          const m2 neg = lt0(s[mw]);
          sa = add(sa, sel(neg, sw, F2(0.0f)));
          sb = add(sb, sel(neg, F2(0.0f), sw));
        }
        am[m] = sa;
        ap[m] = sb;
      }
      return;
    }
    // entropy fix (rp1eu.f:126-201), lane by lane through selects
#pragma unroll
    for (int m = 0; m < 3; ++m) am[m] = F2(0.0f);
    const f2 s0 = speed<false>(ph, L[0], L[1], L[2]);
    const m2 done = ge0(s0) & gt0(s[0]);          // left-going wave supersonic to the right
    if (!all(done)) {
      const f2 s1 = speed<false>(ph, add(L[0], w[0][0]), add(L[1], w[0][1]), add(L[2], w[0][2]));
      const m2 c1 = lt0(s0) & gt0(s1);             // transonic 1-rarefaction
      const f2 sfa = sel(c1, mul(mul(s0, sub(s1, s[0])), rcp2(sub(s1, s0))), sel(lt0(s[0]), s[0], F2(0.0f)));
#pragma unroll
      for (int m = 0; m < 3; ++m) am[m] = sel(done, F2(0.0f), mul(sfa, w[0][m]));
      const m2 go = (!done) & lt0(s[1]);           // contact moving left
      if (any(go)) {
#pragma unroll
        for (int m = 0; m < 3; ++m) am[m] = add(am[m], sel(go, mul(s[1], w[1][m]), F2(0.0f)));
        const f2 s3 = speed<true>(ph, R[0], R[1], R[2]);
        const f2 s2 = speed<true>(ph, sub(R[0], w[2][0]), sub(R[1], w[2][1]), sub(R[2], w[2][2]));
        const m2 c2 = lt0(s2) & gt0(s3);           // transonic 3-rarefaction
        const f2 sfb = sel(c2, mul(mul(s2, sub(s3, s[2])), rcp2(sub(s3, s2))), s[2]);
        const m2 take = go & (c2 | lt0(s[2]));
#pragma unroll
        for (int m = 0; m < 3; ++m) am[m] = add(am[m], sel(take, mul(sfb, w[2][m]), F2(0.0f)));
      }
    }
#pragma unroll
    for (int m = 0; m < 3; ++m) {                  // :206-213
      f2 df = F2(0.0f);
#pragma unroll
      for (int mw = 0; mw < 3; ++mw) df = fma2(s[mw], w[mw][m], df);
      ap[m] = sub(df, am[m]);
    }
  }
};

// ---- WENO5 on offsets, two interfaces ------------------------------------
// weno_side_scaled on two lanes of jumps already divided by their scales; IM
// is the side (+1, -1): im*(a-b) is computed as b-a for IM = -1.
template <int IM>
__device__ __forceinline__ f2 weno_side2(f2 dm2, f2 dm1, f2 d0, f2 dp1) {
  const f2 t1 = IM > 0 ? sub(dm2, dm1) : sub(dm1, dm2);
  const f2 t2 = IM > 0 ? sub(dm1, d0) : sub(d0, dm1);
  const f2 t3 = IM > 0 ? sub(d0, dp1) : sub(dp1, d0);
  const f2 x1 = fma2(dm1, F2(-3.0f), dm2);
  const f2 x2 = add(dm1, d0);
  const f2 x3 = fma2(d0, F2(-3.0f), dp1);          // -(3 d0 - dp1): only its square is used
  f2 tt1 = fma2(mul(t1, t1), F2(13.0f), mul(mul(x1, x1), F2(3.0f)));
  f2 tt2 = fma2(mul(t2, t2), F2(13.0f), mul(mul(x2, x2), F2(3.0f)));
  f2 tt3 = fma2(mul(t3, t3), F2(13.0f), mul(mul(x3, x3), F2(3.0f)));
  tt1 = add(F2(EPS_SCALED), tt1);
  tt2 = add(F2(EPS_SCALED), tt2);
  tt3 = add(F2(EPS_SCALED), tt3);
  tt1 = mul(tt1, tt1);
  tt2 = mul(tt2, tt2);
  tt3 = mul(tt3, tt3);
  f2 s1 = mul(tt2, tt3);
  const f2 s2 = mul(mul(F2(6.0f), tt1), tt3);
  f2 s3 = mul(mul(F2(3.0f), tt1), tt2);
  const f2 t0 = rcp2(add(add(s1, s2), s3));
  s1 = mul(s1, t0);
  s3 = mul(s3, t0);
  const f2 r = fma2(s1, sub(t2, t1), mul(fma2(s3, F2(0.5f), F2(-0.25f)), sub(t3, t2)));
  return mul(r, F2(1.0f / 3.0f));
}

// Both sides of the scaled correction for five jumps h[0..4] on two lanes.
__device__ __forceinline__ void weno_pair2(const f2 h[5], f2& u1, f2& u2) {
  f2 sc;
  sc.x = fmaxf(fmaxf(fmaxf(fabsf(h[0].x), fabsf(h[1].x)), fmaxf(fabsf(h[2].x), fabsf(h[3].x))), fabsf(h[4].x));
  sc.y = fmaxf(fmaxf(fmaxf(fabsf(h[0].y), fabsf(h[1].y)), fmaxf(fabsf(h[2].y), fabsf(h[3].y))), fabsf(h[4].y));
  // lanes with an all-zero stencil, a non-finite one, or jumps beyond 8e37
  const m2 odd = {!(sc.x > 0.0f) || !(sc.x < 8.0e37f), !(sc.y > 0.0f) || !(sc.y < 8.0e37f)};
  const f2 sc1 = sel(odd, F2(1.0f), sc);
  const f2 inv = rcp2(sc1);
  f2 n[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) n[k] = mul(h[k], inv);
  u1 = mul(weno_side2<1>(n[0], n[1], n[2], n[3]), sc1);
  u2 = mul(weno_side2<-1>(n[4], n[3], n[2], n[1]), sc1);
  if (any(odd)) {
    const f2 f = F2(sc.x == 0.0f ? 0.0f : sc.x, sc.y == 0.0f ? 0.0f : sc.y);
    u1 = sel(odd, f, u1);
    u2 = sel(odd, f, u2);
  }
}

// char-wise (CD = 2) or componentwise (CD = 0) offsets er = qr(c-1)-q(c-1),
// el = ql(c)-q(c) from the jumps d[k] (as weno5_char_offset / weno5_offset)
template <int CD>
__device__ __forceinline__ void weno5_offset2(const f2 d[5][3], const f2 evl[3][3], const f2 evr[3][3], f2 er[3],
                                              f2 el[3]) {
  const f2 c12 = F2(1.0f / 12.0f);
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    er[m] = mul(sub(fma2(F2(6.0f), d[2][m], d[1][m]), d[3][m]), c12);
    el[m] = mul(sub(fma2(F2(-6.0f), d[2][m], d[1][m]), d[3][m]), c12);
  }
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    f2 h[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      if constexpr (CD == 2) {
        f2 s = mul(evl[p][0], d[k][0]);
        s = fma2(evl[p][1], d[k][1], s);
        h[k] = fma2(evl[p][2], d[k][2], s);
      } else {
        h[k] = d[k][p];
      }
    }
    f2 u1, u2;
    weno_pair2(h, u1, u2);
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      if constexpr (CD == 2) {
        er[m] = fma2(evr[m][p], u1, er[m]);
        el[m] = fma2(evr[m][p], u2, el[m]);
      } else if (m == p) {
        er[m] = add(er[m], u1);
        el[m] = add(el[m], u2);
      }
    }
  }
}
// ---- the tile ---------------------------------------------------------------
#ifndef SCL_PAIR_MINB
#define SCL_PAIR_MINB 6
#endif

// Tile geometry.  Thread t owns interfaces and cells c = c0 + 2t (lane x) and
// c + 1 (lane y) with c0 = (2NT-2) b even, so a thread's two cells sit at the
// even element offset c+2 (offset = cell + 2 in the reference layout) and its
// stencil window starts at the even offset c-2: 16-byte vector accesses in
// double planes.  A tile updates the 2NT-2 cells c0 .. c0+2NT-3 (cell 0 of
// tile 0 is a ghost cell and is not written) from interfaces c0 .. c0+2NT-2;
// the last thread's second interface is not needed.
template <int PREC, int NT>
struct PairGeom {
  using S = typename Prec<PREC>::S;
  static constexpr int AL = 16 / (int)sizeof(S);                 // elements per 16 bytes
  static constexpr int STRIDE = 2 * NT - 2;                       // cells per tile
  static constexpr int SQW = (2 * NT + 8 + AL - 1) / AL * AL;     // staged offsets per component
};

// One staged window: offsets a0 .. a0+SQW-1 of the three component planes.
template <int PREC, int NT>
struct PairWin {
  __align__(16) typename Prec<PREC>::S v[3][PairGeom<PREC, NT>::SQW];
};

// Interface records of a tile: 0: qr(c-1)  1: ql(c)  2: amdq(c)  3: apdq(c).
template <int NT>
struct PairRec {
  __align__(16) float r[4][3][2 * NT + 2];
};

template <int PREC, int NT>
struct PairSmem {
  PairWin<PREC, NT> sq;    // stage input
  PairWin<PREC, NT> so;    // the stage's pointwise input (qold or r1), same window
  PairRec<NT> rec;
  float sred[NT / 32];
  double dtdx;
  uint64_t bar;            // completion of the bulk copies of the tile
};

__device__ __forceinline__ f2 ld2(const float* p) { return *reinterpret_cast<const float2*>(p); }
__device__ __forceinline__ void st2(float* p, f2 v) { *reinterpret_cast<float2*>(p) = v; }

// two consecutive elements at an even offset (one 16- or 8-byte access)
template <class S>
struct Pair2;
template <>
struct Pair2<double> {
  using V = double2;
};
template <>
struct Pair2<float> {
  using V = float2;
};
template <class S>
__device__ __forceinline__ typename Pair2<S>::V ldp(const S* p) {
  return *reinterpret_cast<const typename Pair2<S>::V*>(p);
}
template <class S>
__device__ __forceinline__ void stp(S* p, S x, S y) {
  typename Pair2<S>::V v;
  v.x = x;
  v.y = y;
  *reinterpret_cast<typename Pair2<S>::V*>(p) = v;
}

// Window of a tile: first staged offset a0 (a multiple of AL, so that the
// bulk copies start on 16 bytes) and the shift sh = (c0-2) - a0 of the
// stencil windows inside it.
template <int PREC, int NT>
__device__ __forceinline__ int pair_window(int c0, int& sh) {
  constexpr int AL = PairGeom<PREC, NT>::AL;
  const int a0 = (c0 - 2 + AL) / AL * AL - AL;   // floor to a multiple of AL (c0 - 2 >= -2)
  sh = c0 - 2 - a0;
  return a0;
}

// Issue (thread 0 only) the bulk copies of the tile at c0: the component
// planes of the stage input into wq and, when wo is given, of the pointwise
// input qo into wo, all completed on bar.  Offsets below 0 (tile 0 only) are
// filled with 1 before the arrival, so the waiting threads see them.
template <int PREC, int NT>
__device__ __forceinline__ void pair_issue(const Line<typename Prec<PREC>::S>& L, int c0, PairWin<PREC, NT>& wq,
                                           PairWin<PREC, NT>* wo, uint64_t* bar) {
  using S = typename Prec<PREC>::S;
  constexpr int AL = PairGeom<PREC, NT>::AL, SQW = PairGeom<PREC, NT>::SQW;
  int sh;
  const int a0 = pair_window<PREC, NT>(c0, sh);
  const int hend = (L.mx + 6 + AL - 1) / AL * AL;   // round_up(mx+6, AL) <= plane (host-checked)
  const int lo = a0 > 0 ? a0 : 0;
  const int hi = a0 + SQW < hend ? a0 + SQW : hend;
  for (int k = 0; k < lo - a0; ++k)
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      wq.v[m][k] = (S)1;
      if (wo) wo->v[m][k] = (S)1;
    }
  const uint32_t bytes = (uint32_t)(hi - lo) * (uint32_t)sizeof(S);
  fence_proxy_async_smem();   // earlier accesses of these buffers come before the copies' writes
  mbar_arrive_expect_tx(bar, bytes * (wo ? 6u : 3u) + L.tx_extra);
#pragma unroll
  for (int m = 0; m < 3; ++m) bulk_g2s(&wq.v[m][lo - a0], L.qin + (long)m * L.plane + lo, bytes, bar);
  if (wo)
#pragma unroll
    for (int m = 0; m < 3; ++m) bulk_g2s(&wo->v[m][lo - a0], L.qo + (long)m * L.plane + lo, bytes, bar);
}

// Every thread waits for phase `parity` of bar (an acquire: the copies' data
// and what thread 0 wrote before its arrival are visible after it, so no CTA
// barrier follows).  A thread whose bounded wait runs out raises
// SCL_STATUS_TIMEOUT (the controller then stops the run and discards the
// step), waits once more, bounded, for copies still in flight, and goes on.
__device__ __forceinline__ void pair_wait(Ctl* ctl, uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  if (!mbar_wait_bounded(bar, parity, limit_ns)) {
    atomicOr(&ctl->status, SCL_STATUS_TIMEOUT);
    mbar_wait_bounded(bar, parity, limit_ns);
  }
}

// The threads stage the window themselves (planes not on 16 bytes).
template <int PREC, int NT>
__device__ __forceinline__ void pair_load(const Line<typename Prec<PREC>::S>& L, int c0, PairWin<PREC, NT>& wq,
                                          PairWin<PREC, NT>* wo) {
  using S = typename Prec<PREC>::S;
  constexpr int SQW = PairGeom<PREC, NT>::SQW;
  int sh;
  const int a0 = pair_window<PREC, NT>(c0, sh);
  for (int k = threadIdx.x; k < SQW; k += NT) {
    const long g = (long)a0 + k;
    const bool in = g >= 0 && g < (long)L.mx + 6;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      wq.v[m][k] = in ? L.qin[(long)m * L.plane + g] : (S)1;
      if (wo) wo->v[m][k] = in ? L.qo[(long)m * L.plane + g] : (S)1;
    }
  }
}

// One staged tile: interfaces c (lane x) and c+1 (lane y) of thread t, then
// its cells c and c+1.  smax collects the largest |s| over the tile's
// interfaces of the grid (1 .. mx+1).  wo: the staged pointwise input, or
// nullptr to read it (when the stage has one) from global memory.  VEC: the
// planes' alignment allows 16-byte accesses of a thread's two cells.
template <int CD, int PREC, int NT, bool VEC>
__device__ __forceinline__ void pair_compute(const Line<typename Prec<PREC>::S>& L, const Phys& ph, int c0,
                                             const PairWin<PREC, NT>& wq, const PairWin<PREC, NT>* wo,
                                             PairRec<NT>& rec, double dtdx0, float& smax, int& bad) {
  using S = typename Prec<PREC>::S;
  using Ac = typename Prec<PREC>::A;
  const int tid = threadIdx.x;
  const int mx = L.mx;
  const float dtdx = (float)dtdx0;
  const int c = c0 + 2 * tid;
  int sh;
  pair_window<PREC, NT>(c0, sh);
  const int b = sh + 2 * tid;   // staged index of offset c-2 (cell c-4)

  // ---- interface phase: interfaces c (lane x) and c+1 (lane y) ----
  {
    f2 d[5][3], qm[3], q0[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      S e[8];   // cells c-4 .. c+3
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const auto v = ldp(&wq.v[m][b + 2 * k]);
        e[2 * k] = v.x;
        e[2 * k + 1] = v.y;
      }
      float dj[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) dj[k] = (float)(e[k + 2] - e[k + 1]);
#pragma unroll
      for (int k = 0; k < 5; ++k) d[k][m] = F2(dj[k], dj[k + 1]);
      qm[m] = F2((float)e[3], (float)e[4]);
      q0[m] = F2((float)e[4], (float)e[5]);
    }
    f2 evl[3][3], evr[3][3];
    if constexpr (CD == 2) EulerPair::evec(ph, qm, q0, evl, evr);
    f2 er[3], el[3];
    weno5_offset2<CD>(d, evl, evr, er, el);
    f2 Lq[3], Rq[3], dl[3], s[3], am[3], ap[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      Lq[m] = add(qm[m], er[m]);
      Rq[m] = add(q0[m], el[m]);
      dl[m] = add(d[2][m], sub(el[m], er[m]));
    }
    EulerPair::rp(ph, Lq, Rq, dl, s, am, ap);
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      st2(&rec.r[0][m][2 * tid], er[m]);
      st2(&rec.r[1][m][2 * tid], el[m]);
      st2(&rec.r[2][m][2 * tid], am[m]);
      st2(&rec.r[3][m][2 * tid], ap[m]);
    }
    // flux1.f90:126-133 over the interfaces 1 .. mx+1 of the grid: with one
    // dtdx, max(dtdx s, -dtdx s) = dtdx |s|, and the largest |s| is
    // multiplied by dtdx once, in FP64 (the same value as the maximum of the
    // FP64 products, since rounding is monotonic)
    const bool ix = c >= 1 && c <= mx + 1, iy = c + 1 <= mx + 1;
#pragma unroll
    for (int w = 0; w < 3; ++w) {
      if (ix) smax = nanmax(smax, fabsf(s[w].x));
      if (iy) smax = nanmax(smax, fabsf(s[w].y));
    }
  }
  __syncthreads();

  // ---- cell phase: cells c (lane x) and c+1 (lane y) ----
  if (tid < NT - 1 && c <= mx) {
    const int i = 2 * tid;
    f2 qc[3], qlc[3], qrc[3], apc[3], amc1[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const auto v = ldp(&wq.v[m][b + 4]);
      qc[m] = F2((float)v.x, (float)v.y);
      qlc[m] = ld2(&rec.r[1][m][i]);
      apc[m] = ld2(&rec.r[3][m][i]);
      qrc[m] = F2(rec.r[0][m][i + 1], rec.r[0][m][i + 2]);
      amc1[m] = F2(rec.r[2][m][i + 1], rec.r[2][m][i + 2]);
    }
    f2 Lq[3], Rq[3], dl[3], s2[3], am2[3], ap2[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      Lq[m] = add(qc[m], qlc[m]);
      Rq[m] = add(qc[m], qrc[m]);
      dl[m] = sub(qrc[m], qlc[m]);
    }
    EulerPair::rp(ph, Lq, Rq, dl, s2, am2, ap2);   // flux1.f90:181-182
    const bool vx = c >= 1;              // cell 0 of tile 0 is a ghost cell
    const bool vy = c + 1 <= mx;
    const bool edge = c <= 3 || c + 1 >= mx - 2;   // a lane has ghost images
    const int kind = L.kind;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const f2 br = add(add(add(amc1[m], apc[m]), am2[m]), ap2[m]);   // :185-186
      const f2 dq = mul(F2(-dtdx), br);
      if (kind == SK_DQ) {
        if (vx) L.dq_out[(long)m * L.plane + c + 2] = (double)dq.x;
        if (vy) L.dq_out[(long)m * L.plane + c + 3] = (double)dq.y;
        continue;
      }
      const auto qv = ldp(&wq.v[m][b + 4]);
      typename Pair2<S>::V qov;
      qov.x = (S)0;
      qov.y = (S)0;
      if (L.qo) {
        if (wo) {
          qov = ldp(&wo->v[m][b + 4]);
        } else {
          const S* pq = L.qo + (long)m * L.plane + c + 2;
          if (VEC && vx && vy) qov = ldp(pq);
          else {
            if (vx) qov.x = pq[0];
            if (vy) qov.y = pq[1];
          }
        }
      }
      Ac ox, oy, o2x = (Ac)0, o2y = (Ac)0;
      combine<Ac, false>(kind, (Ac)qv.x, (Ac)qov.x, (Ac)dq.x, ox, o2x);
      combine<Ac, false>(kind, (Ac)qv.y, (Ac)qov.y, (Ac)dq.y, oy, o2y);
      bad |= (vx && !isfinite(ox)) || (vy && !isfinite(oy));
      S* po = L.out + (long)m * L.plane + c + 2;
      if (VEC && vx && vy && !edge) {
        stp<S>(po, (S)ox, (S)oy);
        if (L.out2) stp<S>(L.out2 + (long)m * L.plane + c + 2, (S)o2x, (S)o2y);
      } else {
        if (vx) {
          if (c <= 3 || c >= mx - 2) put_1d_img<S, Ac>(L.out, L.plane, m, c, mx, L.bl, L.br, ox);
          else po[0] = (S)ox;
          if (L.out2) L.out2[(long)m * L.plane + c + 2] = (S)o2x;
        }
        if (vy) {
          if (c + 1 <= 3 || c + 1 >= mx - 2)
            put_1d_img<S, Ac>(L.out, L.plane, m, c + 1, mx, L.bl, L.br, oy);
          else po[1] = (S)oy;
          if (L.out2) L.out2[(long)m * L.plane + c + 3] = (S)o2y;
        }
      }
    }
  }
}

// CTA maximum of smax, times dtdx in FP64, into the stage's CFL slot; the
// non-finite flag into the status word.  REUSE: end with a CTA-wide barrier
// (a persistent CTA reuses sred and the staged windows for its next tile).
template <int NT, bool REUSE>
__device__ __forceinline__ void pair_reduce(Ctl* ctl, int stage, float* sred, double dtdx, float smax, int bad) {
  const int tid = threadIdx.x;
  smax = warp_max(smax);
  if ((tid & 31) == 0) sred[tid >> 5] = smax;
  const int anybad = __syncthreads_or(bad);
  if (tid < 32) {
    float v = (tid < NT / 32) ? sred[tid] : 0.0f;
    v = warp_max(v);
    if (tid == 0) {
      atomic_max_nonneg(&ctl->stage_cfl[stage], dtdx * (double)v);
      if (anybad) atomicOr(&ctl->status, SCL_STATUS_NONFINITE);
    }
  }
  if constexpr (REUSE) __syncthreads();
}

template <class S>
__device__ __forceinline__ Line<S> line_of(const StageArgs& a, Ctl* ctl) {
  Line<S> L;
  L.ctl = ctl;
  L.qin = static_cast<const S*>(pick_buf(a.buf, ctl->role[a.sd.in]));
  L.qo = a.sd.aux_in >= 0 ? static_cast<const S*>(pick_buf(a.buf, ctl->role[a.sd.aux_in])) : nullptr;
  L.out = a.sd.kind == SK_DQ ? nullptr : static_cast<S*>(pick_buf(a.buf, ctl->role[a.sd.out]));
  L.out2 = a.sd.out2 >= 0 ? static_cast<S*>(pick_buf(a.buf, ctl->role[a.sd.out2])) : nullptr;
  L.dq_out = a.dq_out;
  L.aux = a.aux;
  L.mx = a.mx;
  L.plane = a.plane;
  L.dx = a.dx;
  L.bl = a.mthbc[0];
  L.br = a.mthbc[1];
  L.mcapa = a.mcapa;
  L.kind = a.sd.kind;
  L.stage = a.stage;
  L.ixy = a.ixy;
  L.dt = ctl->dt;
  L.wait_ns = a.wait_ns ? a.wait_ns : MBAR_LIMIT_NS;   // 0: the default bound
  L.tx_extra = a.tx_extra;
  return L;
}

// One tile per CTA.  TMA: the planes are 16-byte aligned with an even (double)
// or multiple-of-4 (float) component stride, checked by the launcher, and the
// tile is staged by bulk copies; otherwise by the threads.
template <int CD, int PREC, int NT, bool TMA, int MINB = SCL_PAIR_MINB>
__global__ void __launch_bounds__(NT, MINB) k_stage1d_pair(StageArgs a) {
  using S = typename Prec<PREC>::S;
  __shared__ PairSmem<PREC, NT> sm;
  Ctl* ctl = a.ctl;
  if (ctl->done) return;
  const Line<S> L = line_of<S>(a, ctl);
  const int c0 = (int)blockIdx.x * PairGeom<PREC, NT>::STRIDE;
  PairWin<PREC, NT>* wo = L.qo ? &sm.so : nullptr;
  if constexpr (TMA) {
    if (threadIdx.x == 0) {
      mbar_init(&sm.bar, 1);
      fence_mbar_init();
      sm.dtdx = L.dt / L.dx;
      pair_issue<PREC, NT>(L, c0, sm.sq, wo, &sm.bar);
    }
    __syncthreads();   // the barrier is initialised before any thread waits on it
    pair_wait(ctl, &sm.bar, 0, L.wait_ns);
  } else {
    if (threadIdx.x == 0) sm.dtdx = L.dt / L.dx;
    pair_load<PREC, NT>(L, c0, sm.sq, wo);
    __syncthreads();
  }
  float smax = 0.0f;
  int bad = 0;
  pair_compute<CD, PREC, NT, TMA>(L, a.ph, c0, sm.sq, wo, sm.rec, sm.dtdx, smax, bad);
  pair_reduce<NT, false>(ctl, a.stage, sm.sred, sm.dtdx, smax, bad);
}

// Batched form: the persistent walk over the active instances' tiles of
// k_batch_stage with the paired tile (instances are 16-byte aligned with
// planes padded to 32 elements, so the tiles are staged by bulk copies) and
// one CFL atomic per tile into the tile's own controller.
template <int CD, int PREC, int NT>
__global__ void __launch_bounds__(NT, SCL_PAIR_MINB) k_batch_stage_pair(BatchArgs a) {
  using S = typename Prec<PREC>::S;
  __shared__ PairSmem<PREC, NT> sm;
  const int na = *a.nact;
  if (na == 0) return;
  const int ntiles = a.prefix[na];
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&sm.bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  uint32_t parity = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, parity ^= 1u) {
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
    L.aux = nullptr;
    L.mx = a.mx[k];
    L.plane = a.plane[k];
    L.dx = a.dx[k];
    L.bl = a.mthbc[0];
    L.br = a.mthbc[1];
    L.mcapa = 0;
    L.kind = a.sd.kind;
    L.stage = a.stage;
    L.ixy = 1;
    L.dt = ctl->dt;
    const int c0 = (t - a.prefix[lo]) * PairGeom<PREC, NT>::STRIDE;
    PairWin<PREC, NT>* wo = L.qo ? &sm.so : nullptr;
    if (tid == 0) {
      sm.dtdx = L.dt / L.dx;
      pair_issue<PREC, NT>(L, c0, sm.sq, wo, &sm.bar);
    }
    pair_wait(ctl, &sm.bar, parity, MBAR_LIMIT_NS);
    float smax = 0.0f;
    int bad = 0;
    pair_compute<CD, PREC, NT, true>(L, a.ph, c0, sm.sq, wo, sm.rec, sm.dtdx, smax, bad);
    pair_reduce<NT, true>(ctl, a.stage, sm.sred, sm.dtdx, smax, bad);
  }
}

}  // namespace scl
