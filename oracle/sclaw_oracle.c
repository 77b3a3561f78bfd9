/*
 * sclaw_oracle.c -- CPU oracle (test infrastructure only; see sclaw_oracle.h).
 *
 * Each routine restates one reference routine with the same loops, index
 * ranges and floating-point evaluation order (Fortran left-to-right
 * association, x**2 as x*x, REAL(4) literals widened to double, no FMA:
 * compiled with -ffp-contract=off).  File:line citations are relative to the
 * reference project root.
 *
 * Deliberate, documented differences from the reference:
 *  - workspace entries that the reference leaves uninitialised at the two
 *    outermost ghost interfaces (reconstruct.f90:113 dq1m(1), :375 hh(mbc,:))
 *    are zeroed; they never reach interior cells or the CFL number;
 *  - fixed plugin array limits (rp1eu.f:34 max2=2002, rpn2sw.f:42 maxm2=603)
 *    are lifted by allocating per call;
 *  - qold is refreshed every step, also when dt_variable == 0
 *    (sharpclaw.f90:132-135 only does so for variable dt);
 *  - plugins that the reference lacks (Euler evec, shallow-water evec, 2-D
 *    acoustics rpn2/tfluct/evec) are new and are written identically here and
 *    in the CUDA kernels.
 */
#include "sclaw_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* reconstruct.f90:6  double precision :: epweno = 1.e-36  (REAL(4) literal) */
#define EPWENO ((double)1.0e-36f)

static double dmax1(double a, double b) { return a > b ? a : b; }
static double dmin1(double a, double b) { return a < b ? a : b; }

long ocl_plane(const ocl_params *p) {
  long n = (long)p->mx + 2L * p->mbc;
  if (p->ndim == 2) n *= (long)p->my + 2L * p->mbc;
  return n;
}

/* ------------------------------------------------------------------------ */
/* Line arrays: index i in [1-mbc, mx+mbc], 1-based component m, wave w.     */
/* ------------------------------------------------------------------------ */
#define L2(a, i, m) (a)[((i) + mbc - 1) + (long)((m) - 1) * ld]
#define L3(a, i, m, w) (a)[((i) + mbc - 1) + (long)((m) - 1) * ld + (long)((w) - 1) * ld * meqn]

/* ======================================================================== */
/* Boundary conditions: src/1d/bc1.f90:1-112 and src/2d/bc2.f90:2-209.      */
/* ======================================================================== */
static int bc1(const ocl_params *p, double *q) {
  const int mbc = p->mbc, mx = p->mx, meqn = p->meqn;
  const long ld = mx + 2 * mbc;
  switch (p->mthbc[0]) {                       /* bc1.f90:198 left */
    case 1:
      for (int m = 1; m <= meqn; ++m)
        for (int ibc = 1; ibc <= mbc; ++ibc) L2(q, 1 - ibc, m) = L2(q, 1, m);
      break;
    case 2:
      for (int m = 1; m <= meqn; ++m)
        for (int ibc = 1; ibc <= mbc; ++ibc) L2(q, 1 - ibc, m) = L2(q, mx + 1 - ibc, m);
      break;
    case 3:
      for (int m = 1; m <= meqn; ++m)
        for (int ibc = 1; ibc <= mbc; ++ibc) L2(q, 1 - ibc, m) = L2(q, ibc, m);
      for (int ibc = 1; ibc <= mbc; ++ibc) L2(q, 1 - ibc, 2) = -L2(q, ibc, 2);
      break;
    default:
      return -2;
  }
  switch (p->mthbc[1]) {                       /* bc1.f90:240 right */
    case 1:
      for (int m = 1; m <= meqn; ++m)
        for (int ibc = 1; ibc <= mbc; ++ibc) L2(q, mx + ibc, m) = L2(q, mx, m);
      break;
    case 2:
      for (int m = 1; m <= meqn; ++m)
        for (int ibc = 1; ibc <= mbc; ++ibc) L2(q, mx + ibc, m) = L2(q, ibc, m);
      break;
    case 3:
      for (int m = 1; m <= meqn; ++m)
        for (int ibc = 1; ibc <= mbc; ++ibc) L2(q, mx + ibc, m) = L2(q, mx + 1 - ibc, m);
      for (int ibc = 1; ibc <= mbc; ++ibc) L2(q, mx + ibc, 2) = -L2(q, mx + 1 - ibc, 2);
      break;
    default:
      return -2;
  }
  return 0;
}

#define G3(a, i, j, m) \
  (a)[((i) + mbc - 1) + (long)((j) + mbc - 1) * ldx + (long)((m) - 1) * ldx * ldy]

static int bc2(const ocl_params *p, double *q) {
  const int mbc = p->mbc, nx = p->mx, ny = p->my, meqn = p->meqn;
  const long ldx = nx + 2 * mbc, ldy = ny + 2 * mbc;
  /* left (bc2.f90:31-69) */
  for (int m = 1; m <= meqn; ++m)
    for (int ibc = 1; ibc <= mbc; ++ibc)
      for (int j = 1 - mbc; j <= ny + mbc; ++j) {
        if (p->mthbc[0] == 1) G3(q, 1 - ibc, j, m) = G3(q, 1, j, m);
        else if (p->mthbc[0] == 2) G3(q, 1 - ibc, j, m) = G3(q, nx + 1 - ibc, j, m);
        else if (p->mthbc[0] == 3) G3(q, 1 - ibc, j, m) = G3(q, ibc, j, m);
        else return -2;
      }
  if (p->mthbc[0] == 3)
    for (int ibc = 1; ibc <= mbc; ++ibc)
      for (int j = 1 - mbc; j <= ny + mbc; ++j) G3(q, 1 - ibc, j, 2) = -G3(q, ibc, j, 2);
  /* right (bc2.f90:76-114) */
  for (int m = 1; m <= meqn; ++m)
    for (int ibc = 1; ibc <= mbc; ++ibc)
      for (int j = 1 - mbc; j <= ny + mbc; ++j) {
        if (p->mthbc[1] == 1) G3(q, nx + ibc, j, m) = G3(q, nx, j, m);
        else if (p->mthbc[1] == 2) G3(q, nx + ibc, j, m) = G3(q, ibc, j, m);
        else if (p->mthbc[1] == 3) G3(q, nx + ibc, j, m) = G3(q, nx + 1 - ibc, j, m);
        else return -2;
      }
  if (p->mthbc[1] == 3)
    for (int ibc = 1; ibc <= mbc; ++ibc)
      for (int j = 1 - mbc; j <= ny + mbc; ++j) G3(q, nx + ibc, j, 2) = -G3(q, nx + 1 - ibc, j, 2);
  /* bottom (bc2.f90:121-159) */
  for (int m = 1; m <= meqn; ++m)
    for (int jbc = 1; jbc <= mbc; ++jbc)
      for (int i = 1 - mbc; i <= nx + mbc; ++i) {
        if (p->mthbc[2] == 1) G3(q, i, 1 - jbc, m) = G3(q, i, 1, m);
        else if (p->mthbc[2] == 2) G3(q, i, 1 - jbc, m) = G3(q, i, ny + 1 - jbc, m);
        else if (p->mthbc[2] == 3) G3(q, i, 1 - jbc, m) = G3(q, i, jbc, m);
        else return -2;
      }
  if (p->mthbc[2] == 3)
    for (int jbc = 1; jbc <= mbc; ++jbc)
      for (int i = 1 - mbc; i <= nx + mbc; ++i) G3(q, i, 1 - jbc, 3) = -G3(q, i, jbc, 3);
  /* top (bc2.f90:166-204) */
  for (int m = 1; m <= meqn; ++m)
    for (int jbc = 1; jbc <= mbc; ++jbc)
      for (int i = 1 - mbc; i <= nx + mbc; ++i) {
        if (p->mthbc[3] == 1) G3(q, i, ny + jbc, m) = G3(q, i, ny, m);
        else if (p->mthbc[3] == 2) G3(q, i, ny + jbc, m) = G3(q, i, jbc, m);
        else if (p->mthbc[3] == 3) G3(q, i, ny + jbc, m) = G3(q, i, ny + 1 - jbc, m);
        else return -2;
      }
  if (p->mthbc[3] == 3)
    for (int jbc = 1; jbc <= mbc; ++jbc)
      for (int i = 1 - mbc; i <= nx + mbc; ++i) G3(q, i, ny + jbc, 3) = -G3(q, i, ny + 1 - jbc, 3);
  return 0;
}

int ocl_bc(const ocl_params *p, double *q) {
  if (p->mbc != 3) return -1;
  /* a solid wall negates component 2 (x) or 3 (y): bc1.f90:230, bc2.f90:67,157;
   * with fewer components the reference writes out of bounds */
  for (int k = 0; k < 2 * p->ndim; ++k)
    if (p->mthbc[k] == 3 && p->meqn < (k < 2 ? 2 : 3)) return -2;
  return p->ndim == 1 ? bc1(p, q) : bc2(p, q);
}

/* g0 of apps/elasticity/stegoton/bc1.f:152-166 (pi = 4 datan(1), setprob.f:20) */
static double wall_g0(double s) {
  const double pi = 4.0 * atan(1.0);
  return fabs(s) < 1.0 ? 1.0 + cos(pi * s) : 0.0;
}

/* apps/elasticity/stegoton/bc1.f:1-150 at time t, replacing bc1.f90: the
 * switch of both sides to periodic while 5 tw1 < t < 5 tw1 + 1 (:31-35; it
 * rewrites mthbc, so it stays: p->bc_switched), periodic aux ghosts of aux
 * fields 1..3 when the left side is periodic (:36-45), then each side; an
 * oscillating wall on mthbc = 0 sides (:100-106, :200-206).  bc1.f:62 reads
 * aux(i,1) with i never set; the mirror cell's aux(ibc,1) is used here, as
 * the right wall does (:206). */
static int bc1_user(ocl_params *p, double *q, double *aux, double t) {
  const int mbc = p->mbc, mx = p->mx;
  const long ld = mx + 2 * mbc;
  const double t1 = p->wall[0], a1 = p->wall[1], tw1 = p->wall[2];
  const double t2 = p->wall[3], a2 = p->wall[4], tw2 = p->wall[5];
  if (mbc != 3 || p->meqn < 2 || !aux || p->maux < 1) return -2;
  if (t > 5.0 * tw1 && t < 5.0 * tw1 + 1.0) p->bc_switched = 1;
  const int bl = p->bc_switched ? 2 : p->mthbc[0], br = p->bc_switched ? 2 : p->mthbc[1];
  if (bl == 2)
    for (int j = 1; j <= (p->maux < 3 ? p->maux : 3); ++j)
      for (int ibc = 1; ibc <= mbc; ++ibc) {
        L2(aux, 1 - ibc, j) = L2(aux, mx + 1 - ibc, j);
        L2(aux, mx + ibc, j) = L2(aux, ibc, j);
      }
  /* the standard sides as bc1.f90; a moving wall starts as a solid wall */
  ocl_params pc = *p;
  pc.mthbc[0] = bl == 0 ? 3 : bl;
  pc.mthbc[1] = br == 0 ? 3 : br;
  int rc = bc1(&pc, q);
  if (rc) return rc;
  if (bl == 0) {
    const double vwall = -(a1 * wall_g0((t - t1) / tw1));
    for (int ibc = 1; ibc <= mbc; ++ibc) L2(q, 1 - ibc, 2) = 2.0 * vwall * L2(aux, ibc, 1) - L2(q, ibc, 2);
  }
  if (br == 0) {
    const double vwall = a2 * wall_g0((t - t2) / tw2);
    for (int ibc = 1; ibc <= mbc; ++ibc)
      L2(q, mx + ibc, 2) = 2.0 * vwall * L2(aux, mx + 1 - ibc, 1) - L2(q, mx + 1 - ibc, 2);
  }
  return 0;
}

/* ======================================================================== */
/* WENO5 reconstructions, src/reconstruct.f90.  Indices are the rebased      */
/* (1-based, assumed-shape) array indices of the reference: array index k    */
/* is cell k-mbc.                                                            */
/* ======================================================================== */
#define R2(a, k, m) (a)[((k) - 1) + (long)((m) - 1) * mx2]
#define R3(a, k, p_, m) (a)[((k) - 1) + (long)((p_) - 1) * mx2 + (long)((m) - 1) * mx2 * meqn]

/* reconstruct.f90:77-143 */
int ocl_weno5(int mx2, int meqn, const double *q, double *ql, double *qr) {
  const int mbc = 3;
  double *dq1m = (double *)calloc((size_t)mx2 + 1, sizeof(double));
  double *uu = (double *)calloc(2 * ((size_t)mx2 + 1), sizeof(double));
  if (!dq1m || !uu) { free(dq1m); free(uu); return -3; }
#define D1(k) dq1m[(k) - 1]
#define UU(k, s) uu[((k) - 1) + (long)((s) - 1) * mx2]
  for (int m = 1; m <= meqn; ++m) {
    D1(1) = 0.0;  /* never assigned in the reference (ghost interface only) */
    for (int i = 2; i <= mx2; ++i) D1(i) = R2(q, i, m) - R2(q, i - 1, m);   /* :96-99 */
    for (int m1 = 1; m1 <= 2; ++m1) {
      const int im = (m1 == 1) ? 1 : -1;        /* im=(-1)**(m1+1) :108 */
      const int ione = im, inone = -im, intwo = -2 * im;
      const double dim = (double)im;
      for (int i = mbc; i <= mx2 - mbc + 1; ++i) {
        double t1 = dim * (D1(i + intwo) - D1(i + inone));
        double t2 = dim * (D1(i + inone) - D1(i));
        double t3 = dim * (D1(i) - D1(i + ione));
        double x1 = D1(i + intwo) - 3.0 * D1(i + inone);
        double x2 = D1(i + inone) + D1(i);
        double x3 = 3.0 * D1(i) - D1(i + ione);
        double tt1 = 13.0 * (t1 * t1) + 3.0 * (x1 * x1);
        double tt2 = 13.0 * (t2 * t2) + 3.0 * (x2 * x2);
        double tt3 = 13.0 * (t3 * t3) + 3.0 * (x3 * x3);
        tt1 = (EPWENO + tt1) * (EPWENO + tt1);
        tt2 = (EPWENO + tt2) * (EPWENO + tt2);
        tt3 = (EPWENO + tt3) * (EPWENO + tt3);
        double s1 = tt2 * tt3;
        double s2 = (6.0 * tt1) * tt3;
        double s3 = (3.0 * tt1) * tt2;
        double t0 = 1.0 / ((s1 + s2) + s3);
        s1 = s1 * t0;
        s3 = s3 * t0;
        double c = ((-R2(q, i - 2, m)) + 7.0 * (R2(q, i - 1, m) + R2(q, i, m))) - R2(q, i + 1, m);
        UU(i, m1) = ((s1 * (t2 - t1)) + ((0.5 * s3 - 0.25) * (t3 - t2))) / 3.0 + c / 12.0;
      }
    }
    for (int i = mbc; i <= mx2 - mbc + 1; ++i) {    /* :137-138 */
      R2(qr, i - 1, m) = UU(i, 1);
      R2(ql, i, m) = UU(i, 2);
    }
  }
#undef D1
#undef UU
  free(dq1m);
  free(uu);
  return 0;
}

/* reconstruct.f90:350-428.  wave(i,m,mw) from the rp pass on the cell
   averages.  The reference loops i = 2..mx2 (:368) and reads wave(i-2..i+2);
   those indices hold waves written by that rp pass (2..mx2) only for
   4 <= i <= mx2-2, i.e. exactly the interfaces 1..mx+1 that the update
   uses; the others (ghost interfaces, reading unset workspace there) are
   left at zero here. */
int ocl_weno5_wave(int mx2, int meqn, int mwaves, const double *q, const double *wave,
                   double *ql, double *qr) {
  const double floor14 = (double)1.0e-14f;   /* :413, a REAL(4) literal */
#define W(k, m, mw) R3(wave, k, m, mw)
  for (int i = 4; i <= mx2 - 2; ++i) {
    for (int m = 1; m <= meqn; ++m) {                                         /* :370-374 */
      R2(qr, i - 1, m) = (((-R2(q, i - 2, m)) + 7.0 * (R2(q, i - 1, m) + R2(q, i, m))) - R2(q, i + 1, m)) / 12.0;
      R2(ql, i, m) = R2(qr, i - 1, m);
    }
    for (int mw = 1; mw <= mwaves; ++mw) {
      double u[2], wnorm2 = 0.0;
      for (int m1 = 1; m1 <= 2; ++m1) {
        const int im = (m1 == 1) ? 1 : -1;
        const int ione = im, inone = -im, intwo = -2 * im;
        const double dim = (double)im;
        wnorm2 = W(i, 1, mw) * W(i, 1, mw);                                   /* :383-392 */
        double theta1 = W(i + intwo, 1, mw) * W(i, 1, mw);
        double theta2 = W(i + inone, 1, mw) * W(i, 1, mw);
        double theta3 = W(i + ione, 1, mw) * W(i, 1, mw);
        for (int m = 2; m <= meqn; ++m) {
          wnorm2 = wnorm2 + W(i, m, mw) * W(i, m, mw);
          theta1 = theta1 + W(i + intwo, m, mw) * W(i, m, mw);
          theta2 = theta2 + W(i + inone, m, mw) * W(i, m, mw);
          theta3 = theta3 + W(i + ione, m, mw) * W(i, m, mw);
        }
        double t1 = dim * (theta1 - theta2);                                  /* :394-411 */
        double t2 = dim * (theta2 - wnorm2);
        double t3 = dim * (wnorm2 - theta3);
        double x1 = theta1 - 3.0 * theta2;
        double x2 = theta2 + wnorm2;
        double x3 = 3.0 * wnorm2 - theta3;
        double tt1 = 13.0 * (t1 * t1) + 3.0 * (x1 * x1);
        double tt2 = 13.0 * (t2 * t2) + 3.0 * (x2 * x2);
        double tt3 = 13.0 * (t3 * t3) + 3.0 * (x3 * x3);
        tt1 = (EPWENO + tt1) * (EPWENO + tt1);
        tt2 = (EPWENO + tt2) * (EPWENO + tt2);
        tt3 = (EPWENO + tt3) * (EPWENO + tt3);
        double s1 = tt2 * tt3;
        double s2 = (6.0 * tt1) * tt3;
        double s3 = (3.0 * tt1) * tt2;
        double t0 = 1.0 / ((s1 + s2) + s3);
        s1 = s1 * t0;
        s3 = s3 * t0;
        if (wnorm2 > floor14) {                                               /* :413-419 */
          u[m1 - 1] = ((s1 * (t2 - t1)) + ((0.5 * s3 - 0.25) * (t3 - t2))) / 3.0;
          wnorm2 = 1.0 / wnorm2;
        } else {
          u[m1 - 1] = 0.0;
          wnorm2 = 0.0;
        }
      }
      for (int m = 1; m <= meqn; ++m) {                                       /* :421-424 */
        R2(qr, i - 1, m) = R2(qr, i - 1, m) + (u[0] * W(i, m, mw)) * wnorm2;
        R2(ql, i, m) = R2(ql, i, m) + (u[1] * W(i, m, mw)) * wnorm2;
      }
    }
  }
#undef W
  return 0;
}

/* reconstruct.f90:244-347 (transmission-based).  The reference fills hh
   only for i = mbc+1..mx2-2 (:282) but reconstructs i = mbc..mx2-mbc+1
   (:300); i = mbc reads unset workspace and feeds only the ghost interface
   2-mbc, so the loops here run over i = mbc+1..mx2-2, the interfaces 1..mx+1. */
int ocl_weno5_trans(int mx2, int meqn, const double *q, const double *evl,
                    const double *evr, double *ql, double *qr) {
  const int mbc = 3;
  double *dq = (double *)calloc((size_t)mx2 * meqn, sizeof(double));
  double *gg = (double *)calloc((size_t)mx2 * meqn, sizeof(double));
  double *hh = (double *)calloc((size_t)mx2 * 5, sizeof(double));
  double *u = (double *)calloc((size_t)mx2 * meqn * 2, sizeof(double));
  if (!dq || !gg || !hh || !u) { free(dq); free(gg); free(hh); free(u); return -3; }
#define HH(k, o) hh[((k) - 1) + (long)((o) + 2) * mx2]
#define U3(k, mw, s) u[((k) - 1) + (long)((mw) - 1) * mx2 + (long)((s) - 1) * mx2 * meqn]
  for (int m = 1; m <= meqn; ++m)
    for (int i = 2; i <= mx2; ++i) R2(dq, i, m) = R2(q, i, m) - R2(q, i - 1, m);  /* :264-269 */
  for (int mw = 1; mw <= meqn; ++mw)                                               /* :273-280 */
    for (int i = 2; i <= mx2; ++i) {
      double g = 0.0;
      for (int m = 1; m <= meqn; ++m) g = g + R3(evl, i, mw, m) * R2(dq, i, m);
      R2(gg, i, mw) = g;
    }
  for (int mw = 1; mw <= meqn; ++mw) {
    for (int m1 = -2; m1 <= 2; ++m1)                                                /* :286-294 */
      for (int i = mbc + 1; i <= mx2 - 2; ++i) {
        double h = 0.0;
        for (int m = 1; m <= meqn; ++m)
          h = h + (R3(evl, i, mw, m) * R2(gg, i + m1, mw)) * R3(evr, i + m1, m, mw);
        HH(i, m1) = h;
      }
    for (int m1 = 1; m1 <= 2; ++m1) {                                               /* :298-327 */
      const int im = (m1 == 1) ? 1 : -1;
      const int ione = im, inone = -im, intwo = -2 * im;
      const double dim = (double)im;
      for (int i = mbc + 1; i <= mx2 - 2; ++i) {
        double t1 = dim * (HH(i, intwo) - HH(i, inone));
        double t2 = dim * (HH(i, inone) - HH(i, 0));
        double t3 = dim * (HH(i, 0) - HH(i, ione));
        double x1 = HH(i, intwo) - 3.0 * HH(i, inone);
        double x2 = HH(i, inone) + HH(i, 0);
        double x3 = 3.0 * HH(i, 0) - HH(i, ione);
        double tt1 = 13.0 * (t1 * t1) + 3.0 * (x1 * x1);
        double tt2 = 13.0 * (t2 * t2) + 3.0 * (x2 * x2);
        double tt3 = 13.0 * (t3 * t3) + 3.0 * (x3 * x3);
        tt1 = (EPWENO + tt1) * (EPWENO + tt1);
        tt2 = (EPWENO + tt2) * (EPWENO + tt2);
        tt3 = (EPWENO + tt3) * (EPWENO + tt3);
        double s1 = tt2 * tt3;
        double s2 = (6.0 * tt1) * tt3;
        double s3 = (3.0 * tt1) * tt2;
        double t0 = 1.0 / ((s1 + s2) + s3);
        s1 = s1 * t0;
        s3 = s3 * t0;
        U3(i, mw, m1) = ((s1 * (t2 - t1)) + ((0.5 * s3 - 0.25) * (t3 - t2))) / 3.0;
      }
    }
  }
  for (int m1 = 1; m1 <= 2; ++m1)                                                   /* :332-342 */
    for (int m = 1; m <= meqn; ++m)
      for (int i = mbc + 1; i <= mx2 - 2; ++i) {
        double uh = (((-R2(q, i - 2, m)) + 7.0 * (R2(q, i - 1, m) + R2(q, i, m))) - R2(q, i + 1, m)) / 12.0;
        for (int mw = 1; mw <= meqn; ++mw) uh = uh + R3(evr, i, m, mw) * U3(i, mw, m1);
        if (m1 == 1) R2(qr, i - 1, m) = uh;                                        /* :344-345 */
        else R2(ql, i, m) = uh;
      }
#undef HH
#undef U3
  free(dq); free(gg); free(hh); free(u);
  return 0;
}

/* reconstruct.f90:551-571 (the same five limiters at :610-630, :699-719):
   mthlim 1 minmod, 2 superbee, 3 van Leer, 4 MC, 5 Cada-Torrilhon */
static double tvd_limiter(int t, double r) {
  switch (t) {
    case 1: return dmax1(0.0, dmin1(1.0, r));
    case 2: return dmax1(dmax1(0.0, dmin1(1.0, 2.0 * r)), dmin1(2.0, r));
    case 3: return (r + fabs(r)) / (1.0 + fabs(r));
    case 4: { double c = (1.0 + r) / 2.0; return dmax1(0.0, dmin1(dmin1(c, 2.0), 2.0 * r)); }
    case 5: {
      const double beta = 2.0, xgamma = 2.0, alpha = 1.0 / 3.0;
      double pp = (2.0 + r) / 3.0;
      double amax = dmax1(dmax1(-alpha * r, 0.0), dmin1(dmin1(beta * r, pp), xgamma));
      return dmax1(0.0, dmin1(pp, amax));
    }
  }
  return 0.0;
}

/* reconstruct.f90:525-577, componentwise.  The reference's loop starts with
   dqm left over from the previous component (unset for the first), which
   feeds the left state of interface 1; here every cell's dqm is
   q(i)-q(i-1).  A cell with dqm = 0 gets no slope (the reference's
   r = dqp/dqm is undefined there). */
int ocl_tvd2(int mx2, int meqn, const double *q, const int *mthlim, double *ql, double *qr) {
  for (int m = 1; m <= meqn; ++m)
    for (int i = 3; i <= mx2 - 2; ++i) {                      /* i = mbc+1 .. mx2-mbc, mbc = 2 */
      double dqm = R2(q, i, m) - R2(q, i - 1, m);
      double dqp = R2(q, i + 1, m) - R2(q, i, m);
      double phi = (dqm != 0.0) ? tvd_limiter(mthlim[m - 1], dqp / dqm) : 0.0;
      R2(qr, i, m) = R2(q, i, m) + (0.5 * phi) * dqm;
      R2(ql, i, m) = R2(q, i, m) - (0.5 * phi) * dqm;
    }
  return 0;
}

/* reconstruct.f90:580-651, characteristic-wise */
int ocl_tvd2_char(int mx2, int meqn, const double *q, const int *mthlim, const double *evl,
                  const double *evr, double *ql, double *qr) {
  const double floor14 = (double)1.0e-14f;                    /* :609, a REAL(4) literal */
  double *dq = (double *)calloc((size_t)mx2 * meqn, sizeof(double));
  double *u = (double *)calloc((size_t)mx2 * meqn * 2, sizeof(double));
  if (!dq || !u) { free(dq); free(u); return -3; }
#define U3(k, mw, sd) u[((k) - 1) + (long)((mw) - 1) * mx2 + (long)((sd) - 1) * mx2 * meqn]
  for (int m = 1; m <= meqn; ++m)
    for (int i = 2; i <= mx2; ++i) R2(dq, i, m) = R2(q, i, m) - R2(q, i - 1, m);
  for (int m = 1; m <= meqn; ++m)
    for (int m1 = 1; m1 <= 2; ++m1) {
      const double dim = (m1 == 1) ? 1.0 : -1.0;
      for (int i = 3; i <= mx2 - 1; ++i) {                     /* :594-603 hh(i, m1-2), hh(i, m1-1) */
        double ha = 0.0, hb = 0.0;
        for (int mm = 1; mm <= meqn; ++mm) ha = ha + R3(evl, i, m, mm) * R2(dq, i + m1 - 2, mm);
        for (int mm = 1; mm <= meqn; ++mm) hb = hb + R3(evl, i, m, mm) * R2(dq, i + m1 - 1, mm);
        double r = (fabs(ha) > floor14) ? hb / ha : 0.0;
        U3(i, m, m1) = ((dim * 0.5) * tvd_limiter(mthlim[m - 1], r)) * ha;
      }
    }
  for (int m = 1; m <= meqn; ++m)                              /* :637-646 */
    for (int i = 3; i <= mx2 - 1; ++i) {
      R2(qr, i - 1, m) = R2(q, i - 1, m);
      R2(ql, i, m) = R2(q, i, m);
      for (int mm = 1; mm <= meqn; ++mm) {
        R2(qr, i - 1, m) = R2(qr, i - 1, m) + R3(evr, i, m, mm) * U3(i, mm, 1);
        R2(ql, i, m) = R2(ql, i, m) + R3(evr, i, m, mm) * U3(i, mm, 2);
      }
    }
#undef U3
  free(dq);
  free(u);
  return 0;
}

/* reconstruct.f90:654-761, wave-based: wave and s from the rp pass on the
   cell averages (flux1.f90:84-86) */
int ocl_tvd2_wave(int mx2, int meqn, int mwaves, const double *q, const int *mthlim, const double *wave,
                  const double *s, double *ql, double *qr) {
#define W(k, m, mw) R3(wave, k, m, mw)
  for (int m = 1; m <= meqn; ++m)
    for (int i = 2; i <= mx2; ++i) {                           /* :673-676 */
      R2(qr, i - 1, m) = R2(q, i - 1, m);
      R2(ql, i, m) = R2(q, i, m);
    }
  for (int mw = 1; mw <= mwaves; ++mw) {
    double dotr = 0.0;
    for (int i = 2; i <= mx2 - 2; ++i) {                       /* i = mbc .. mx2-mbc, mbc = 2 */
      double wnorm2 = 0.0, dotl = dotr;
      dotr = 0.0;
      for (int m = 1; m <= meqn; ++m) {
        wnorm2 = wnorm2 + W(i, m, mw) * W(i, m, mw);
        dotr = dotr + W(i, m, mw) * W(i + 1, m, mw);
      }
      if (wnorm2 == 0.0) continue;
      double r = (s[(i - 1) + (long)(mw - 1) * mx2] > 0.0) ? dotl / wnorm2 : dotr / wnorm2;
      double uu = 0.5 * tvd_limiter(mthlim[mw - 1], r);
      for (int m = 1; m <= meqn; ++m) {
        R2(qr, i - 1, m) = R2(qr, i - 1, m) + W(i, m, mw) * uu;
        R2(ql, i, m) = R2(ql, i, m) - W(i, m, mw) * uu;
      }
    }
  }
#undef W
  return 0;
}

/* polyrecon.f90:5-79 (q2qlqr_poly, lim_type 0, char_decomp 0): unlimited
 * upwind-centred reconstruction of order mthlim(1) = 3 (c(-1) = 1/6,
 * c(0) = 2/6).  The reference loops over interfaces i = k+1 .. mx-k-1 only
 * and leaves ql/qr of interfaces 1, mx-1, mx, mx+1 as the workspace held them
 * (undefined); here every interface whose stencil lies in the ghost cells gets
 * the same formula, a documented deviation.  Order 7 needs four ghost cells
 * and is rejected (mbc = 3). */
int ocl_poly(int mx2, int meqn, const double *q, int order, double *ql, double *qr) {
  if (order != 3) return -5;
  const int k = (order - 1) / 2;
  const double cm1 = 1.0 / 6.0, c0 = 2.0 / 6.0;                               /* :27-29 */
  for (int m = 1; m <= meqn; ++m)
    for (int i = 1 + k + 1; i <= mx2 - k; ++i) {                               /* 1-based line index */
      double tm1 = R2(q, i - 1, m) - R2(q, i - 2, m);                          /* theta(j) = du(i+j) */
      double t0 = R2(q, i, m) - R2(q, i - 1, m);
      double tp1 = R2(q, i + 1, m) - R2(q, i, m);
      double ur = (0.0 + cm1 * tm1) + c0 * t0;                                 /* :66-69 */
      double ul = (0.0 + cm1 * tp1) + c0 * t0;
      R2(qr, i - 1, m) = R2(q, i - 1, m) + ur;                                 /* :56-57, 73-75 */
      R2(ql, i, m) = R2(q, i, m) - ul;
    }
  return 0;
}

/* polyrecon.f90:176-253 (q2qlqr_poly_wave, lim_type 0, char_decomp 1): the
 * same stencil on the projections theta(j) = wave(i+j).wave(i) of each wave
 * family, skipped when theta(0) <= 1e-14 (a REAL(4) literal), order 3. */
int ocl_poly_wave(int mx2, int meqn, int mwaves, const double *q, int order, const double *wave,
                  double *ql, double *qr) {
  if (order != 3) return -5;
  const int k = (order - 1) / 2;
  const double cm1 = 1.0 / 6.0, c0 = 2.0 / 6.0;
  const double floor14 = (double)1.0e-14f;
#define W(i, m, mw) R3(wave, i, m, mw)
  for (int i = 1 + k + 1; i <= mx2 - k; ++i) {
    for (int m = 1; m <= meqn; ++m) {                                          /* :218-222 */
      R2(qr, i - 1, m) = R2(q, i - 1, m);
      R2(ql, i, m) = R2(q, i, m);
    }
    for (int mw = 1; mw <= mwaves; ++mw) {
      double theta[3];
      for (int j = -1; j <= 1; ++j) {                                          /* :226-231 */
        double t = W(i + j, 1, mw) * W(i, 1, mw);
        for (int m = 2; m <= meqn; ++m) t = t + W(i + j, m, mw) * W(i, m, mw);
        theta[j + 1] = t;
      }
      if (theta[1] > floor14) {                                                /* :233-247 */
        double wavenormed = 1.0 / theta[1];
        double ur = (0.0 + cm1 * theta[0]) + c0 * theta[1];
        double ul = (0.0 + cm1 * theta[2]) + c0 * theta[1];
        for (int m = 1; m <= meqn; ++m) {
          R2(qr, i - 1, m) = R2(qr, i - 1, m) + (ur * wavenormed) * W(i, m, mw);
          R2(ql, i, m) = R2(ql, i, m) - (ul * wavenormed) * W(i, m, mw);
        }
      }
    }
  }
#undef W
  return 0;
}

/* reconstruct.f90:146-241 */
int ocl_weno5_char(int mx2, int meqn, const double *q, const double *evl,
                   const double *evr, double *ql, double *qr) {
  const int mbc = 3;
  double *dq = (double *)calloc((size_t)mx2 * meqn, sizeof(double));
  double *hh = (double *)calloc((size_t)mx2 * 5, sizeof(double));
  double *uu = (double *)calloc((size_t)mx2 * 2, sizeof(double));
  if (!dq || !hh || !uu) { free(dq); free(hh); free(uu); return -3; }
#define HH(k, o) hh[((k) - 1) + (long)((o) + 2) * mx2]
#define UU(k, s) uu[((k) - 1) + (long)((s) - 1) * mx2]
  for (int m = 1; m <= meqn; ++m)
    for (int i = 2; i <= mx2; ++i) R2(dq, i, m) = R2(q, i, m) - R2(q, i - 1, m);  /* :166-169 */
  for (int m = 1; m <= meqn; ++m)
    for (int i = 3; i <= mx2 - 1; ++i) {                                           /* :171-176 */
      double c = ((-R2(q, i - 2, m)) + 7.0 * (R2(q, i - 1, m) + R2(q, i, m))) - R2(q, i + 1, m);
      R2(qr, i - 1, m) = c / 12.0;
      R2(ql, i, m) = R2(qr, i - 1, m);
    }
  for (int ip = 1; ip <= meqn; ++ip) {
    for (int m2 = -2; m2 <= 2; ++m2)                                                 /* :184-191 */
      for (int i = mbc + 1; i <= mx2 - 2; ++i) {
        double h = 0.0;
        for (int m = 1; m <= meqn; ++m) h = h + R3(evl, i, ip, m) * R2(dq, i + m2, m);
        HH(i, m2) = h;
      }
    for (int m1 = 1; m1 <= 2; ++m1) {                                                /* :196-229 */
      const int im = (m1 == 1) ? 1 : -1;
      const int ione = im, inone = -im, intwo = -2 * im;
      const double dim = (double)im;
      for (int i = mbc; i <= mx2 - mbc + 1; ++i) {
        double t1 = dim * (HH(i, intwo) - HH(i, inone));
        double t2 = dim * (HH(i, inone) - HH(i, 0));
        double t3 = dim * (HH(i, 0) - HH(i, ione));
        double x1 = HH(i, intwo) - 3.0 * HH(i, inone);
        double x2 = HH(i, inone) + HH(i, 0);
        double x3 = 3.0 * HH(i, 0) - HH(i, ione);
        double tt1 = 13.0 * (t1 * t1) + 3.0 * (x1 * x1);
        double tt2 = 13.0 * (t2 * t2) + 3.0 * (x2 * x2);
        double tt3 = 13.0 * (t3 * t3) + 3.0 * (x3 * x3);
        tt1 = (EPWENO + tt1) * (EPWENO + tt1);
        tt2 = (EPWENO + tt2) * (EPWENO + tt2);
        tt3 = (EPWENO + tt3) * (EPWENO + tt3);
        double s1 = tt2 * tt3;
        double s2 = (6.0 * tt1) * tt3;
        double s3 = (3.0 * tt1) * tt2;
        double t0 = 1.0 / ((s1 + s2) + s3);
        s1 = s1 * t0;
        s3 = s3 * t0;
        UU(i, m1) = ((s1 * (t2 - t1)) + ((0.5 * s3 - 0.25) * (t3 - t2))) / 3.0;
      }
    }
    for (int m = 1; m <= meqn; ++m)                                                  /* :232-237 */
      for (int i = mbc; i <= mx2 - mbc + 1; ++i) {
        R2(qr, i - 1, m) = R2(qr, i - 1, m) + R3(evr, i, m, ip) * UU(i, 1);
        R2(ql, i, m) = R2(ql, i, m) + R3(evr, i, m, ip) * UU(i, 2);
      }
  }
#undef HH
#undef UU
  free(dq);
  free(hh);
  free(uu);
  return 0;
}

/* ======================================================================== */
/* Plugins.  Each keeps the reference loop i = 2-mbc .. mx+mbc and its      */
/* arithmetic order.  ld = mx+2*mbc for every line array.                  */
/* ======================================================================== */

/* apps/advection/1d/rp1.f:35-43 */
static void rp_advection(const ocl_params *p, int mx, const double *ql, const double *qr,
                         double *wave, double *s, double *amdq, double *apdq) {
  const int mbc = p->mbc, meqn = p->meqn;
  const long ld = mx + 2 * mbc;
  const double u = p->u;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    L3(wave, i, 1, 1) = L2(ql, i, 1) - L2(qr, i - 1, 1);
    L2(s, i, 1) = u;
    L2(amdq, i, 1) = dmin1(u, 0.0) * L3(wave, i, 1, 1);
    L2(apdq, i, 1) = dmax1(u, 0.0) * L3(wave, i, 1, 1);
  }
}

/* apps/advection/2d/swirl/rpn2ad1.f:39-45: speed auxl(i,ixy), the edge
   velocity stored with the right cell of interface i-1/2 */
static void rp_advedge(const ocl_params *p, int ixy, int mx, const double *ql, const double *qr,
                       const double *auxl, double *wave, double *s, double *amdq, double *apdq) {
  const int mbc = p->mbc, meqn = p->meqn;
  const long ld = mx + 2 * mbc;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    L3(wave, i, 1, 1) = L2(ql, i, 1) - L2(qr, i - 1, 1);
    L2(s, i, 1) = L2(auxl, i, ixy);
    L2(amdq, i, 1) = dmin1(L2(auxl, i, ixy), 0.0) * L3(wave, i, 1, 1);
    L2(apdq, i, 1) = dmax1(L2(auxl, i, ixy), 0.0) * L3(wave, i, 1, 1);
  }
}

/* apps/advection/1d/tfluct1.f:78-87 */
static void tfluct_advection(const ocl_params *p, int mx, const double *ql, const double *qr,
                             double *s, double *adq) {
  const int mbc = p->mbc;
  const long ld = mx + 2 * mbc;
  const double u = p->u;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    double w = L2(qr, i, 1) - L2(ql, i, 1);
    L2(s, i, 1) = u;
    double am = dmin1(u, 0.0) * w;
    double ap = dmax1(u, 0.0) * w;
    L2(adq, i, 1) = am + ap;
  }
}

/* apps/euler/shockentropy/rp1eu.f:44-213 (efix as p->efix, default .true.) */
static void rp_euler(const ocl_params *p, int mx, const double *ql, const double *qr,
                     double *wave, double *s, double *amdq, double *apdq) {
  const int mbc = p->mbc, meqn = p->meqn, mwaves = p->mwaves;
  const long ld = mx + 2 * mbc;
  const double gamma = p->gamma, gamma1 = p->gamma - 1.0;
  double *u = (double *)malloc(sizeof(double) * ld);
  double *enth = (double *)malloc(sizeof(double) * ld);
  double *a = (double *)malloc(sizeof(double) * ld);
#define LOC(v, i) (v)[(i) + mbc - 1]
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {                                        /* :44-55 */
    double rhsqrtl = sqrt(L2(qr, i - 1, 1));
    double rhsqrtr = sqrt(L2(ql, i, 1));
    double pl = gamma1 * (L2(qr, i - 1, 3) - (0.5 * (L2(qr, i - 1, 2) * L2(qr, i - 1, 2))) / L2(qr, i - 1, 1));
    double pr = gamma1 * (L2(ql, i, 3) - (0.5 * (L2(ql, i, 2) * L2(ql, i, 2))) / L2(ql, i, 1));
    double rhsq2 = rhsqrtl + rhsqrtr;
    LOC(u, i) = (L2(qr, i - 1, 2) / rhsqrtl + L2(ql, i, 2) / rhsqrtr) / rhsq2;
    LOC(enth, i) = ((L2(qr, i - 1, 3) + pl) / rhsqrtl + (L2(ql, i, 3) + pr) / rhsqrtr) / rhsq2;
    double a2 = gamma1 * (LOC(enth, i) - 0.5 * (LOC(u, i) * LOC(u, i)));
    LOC(a, i) = sqrt(a2);
  }
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {                                        /* :58-86 */
    double d1 = L2(ql, i, 1) - L2(qr, i - 1, 1);
    double d2 = L2(ql, i, 2) - L2(qr, i - 1, 2);
    double d3 = L2(ql, i, 3) - L2(qr, i - 1, 3);
    double ui = LOC(u, i), ai = LOC(a, i), hi = LOC(enth, i);
    double a2 = (gamma1 / (ai * ai)) * (((hi - ui * ui) * d1 + ui * d2) - d3);
    double a3 = ((d2 + (ai - ui) * d1) - ai * a2) / (2.0 * ai);
    double a1 = (d1 - a2) - a3;
    L3(wave, i, 1, 1) = a1;
    L3(wave, i, 2, 1) = a1 * (ui - ai);
    L3(wave, i, 3, 1) = a1 * (hi - ui * ai);
    L2(s, i, 1) = ui - ai;
    L3(wave, i, 1, 2) = a2;
    L3(wave, i, 2, 2) = a2 * ui;
    L3(wave, i, 3, 2) = (a2 * 0.5) * (ui * ui);
    L2(s, i, 2) = ui;
    L3(wave, i, 1, 3) = a3;
    L3(wave, i, 2, 3) = a3 * (ui + ai);
    L3(wave, i, 3, 3) = a3 * (hi + ui * ai);
    L2(s, i, 3) = ui + ai;
  }
  if (!p->efix) {                                                                    /* :100-111 */
    for (int m = 1; m <= 3; ++m)
      for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        double am = 0.0, ap = 0.0;
        for (int mw = 1; mw <= mwaves; ++mw) {
          if (L2(s, i, mw) < 0.0) am = am + L2(s, i, mw) * L3(wave, i, m, mw);
          else ap = ap + L2(s, i, mw) * L3(wave, i, m, mw);
        }
        L2(amdq, i, m) = am;
        L2(apdq, i, m) = ap;
      }
  } else {
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {                                      /* :126-201 */
      double rhoim1 = L2(qr, i - 1, 1);
      double pim1 = gamma1 * (L2(qr, i - 1, 3) - (0.5 * (L2(qr, i - 1, 2) * L2(qr, i - 1, 2))) / rhoim1);
      double cim1 = sqrt((gamma * pim1) / rhoim1);
      double s0 = L2(qr, i - 1, 2) / rhoim1 - cim1;
      if (s0 >= 0.0 && L2(s, i, 1) > 0.0) {
        for (int m = 1; m <= 3; ++m) L2(amdq, i, m) = 0.0;
        continue;
      }
      double rho1 = L2(qr, i - 1, 1) + L3(wave, i, 1, 1);
      double rhou1 = L2(qr, i - 1, 2) + L3(wave, i, 2, 1);
      double en1 = L2(qr, i - 1, 3) + L3(wave, i, 3, 1);
      double p1 = gamma1 * (en1 - (0.5 * (rhou1 * rhou1)) / rho1);
      double c1 = sqrt((gamma * p1) / rho1);
      double s1 = rhou1 / rho1 - c1;
      double sfract;
      if (s0 < 0.0 && s1 > 0.0) sfract = (s0 * (s1 - L2(s, i, 1))) / (s1 - s0);
      else if (L2(s, i, 1) < 0.0) sfract = L2(s, i, 1);
      else sfract = 0.0;
      for (int m = 1; m <= 3; ++m) L2(amdq, i, m) = sfract * L3(wave, i, m, 1);
      if (L2(s, i, 2) >= 0.0) continue;
      for (int m = 1; m <= 3; ++m) L2(amdq, i, m) = L2(amdq, i, m) + L2(s, i, 2) * L3(wave, i, m, 2);
      double rhoi = L2(ql, i, 1);
      double pi = gamma1 * (L2(ql, i, 3) - (0.5 * (L2(ql, i, 2) * L2(ql, i, 2))) / rhoi);
      double ci = sqrt((gamma * pi) / rhoi);
      double s3 = L2(ql, i, 2) / rhoi + ci;
      double rho2 = L2(ql, i, 1) - L3(wave, i, 1, 3);
      double rhou2 = L2(ql, i, 2) - L3(wave, i, 2, 3);
      double en2 = L2(ql, i, 3) - L3(wave, i, 3, 3);
      double p2 = gamma1 * (en2 - (0.5 * (rhou2 * rhou2)) / rho2);
      double c2 = sqrt((gamma * p2) / rho2);
      double s2 = rhou2 / rho2 + c2;
      if (s2 < 0.0 && s3 > 0.0) sfract = (s2 * (s3 - L2(s, i, 3))) / (s3 - s2);
      else if (L2(s, i, 3) < 0.0) sfract = L2(s, i, 3);
      else continue;
      for (int m = 1; m <= 3; ++m) L2(amdq, i, m) = L2(amdq, i, m) + sfract * L3(wave, i, m, 3);
    }
    for (int m = 1; m <= 3; ++m)                                                     /* :206-213 */
      for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        double df = 0.0;
        for (int mw = 1; mw <= mwaves; ++mw) df = df + L2(s, i, mw) * L3(wave, i, m, mw);
        L2(apdq, i, m) = df - L2(amdq, i, m);
      }
  }
#undef LOC
  free(u);
  free(enth);
  free(a);
}

/* Roe-averaged right/left eigenvectors of the 1-D Euler equations at
 * interface i-1/2 (new; the reference's evec1eu.f is incomplete).  Averages
 * are computed exactly as rp1eu.f:44-55 does, from the cell averages
 * q(i-1), q(i).  evr(i,:,p) = p-th right eigenvector, evl(i,p,:) = p-th row
 * of its inverse, the convention weno5_char uses (reconstruct.f90:188,234). */
static void evec_euler(const ocl_params *p, int mx, const double *q, double *evl, double *evr) {
  const int mbc = p->mbc, meqn = 3;
  const long ld = mx + 2 * mbc;
  const double gamma1 = p->gamma - 1.0;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    double rhsqrtl = sqrt(L2(q, i - 1, 1));
    double rhsqrtr = sqrt(L2(q, i, 1));
    double pl = gamma1 * (L2(q, i - 1, 3) - (0.5 * (L2(q, i - 1, 2) * L2(q, i - 1, 2))) / L2(q, i - 1, 1));
    double pr = gamma1 * (L2(q, i, 3) - (0.5 * (L2(q, i, 2) * L2(q, i, 2))) / L2(q, i, 1));
    double rhsq2 = rhsqrtl + rhsqrtr;
    double u = (L2(q, i - 1, 2) / rhsqrtl + L2(q, i, 2) / rhsqrtr) / rhsq2;
    double h = ((L2(q, i - 1, 3) + pl) / rhsqrtl + (L2(q, i, 3) + pr) / rhsqrtr) / rhsq2;
    double a2 = gamma1 * (h - 0.5 * (u * u));
    double a = sqrt(a2);
    L3(evr, i, 1, 1) = 1.0; L3(evr, i, 1, 2) = 1.0; L3(evr, i, 1, 3) = 1.0;
    L3(evr, i, 2, 1) = u - a; L3(evr, i, 2, 2) = u; L3(evr, i, 2, 3) = u + a;
    L3(evr, i, 3, 1) = h - u * a; L3(evr, i, 3, 2) = 0.5 * (u * u); L3(evr, i, 3, 3) = h + u * a;
    double b1 = gamma1 / a2;
    double b2 = 0.5 * (b1 * (u * u));
    double ua = u / a;
    double ra = 1.0 / a;
    double b1u = b1 * u;
    L3(evl, i, 1, 1) = 0.5 * (b2 + ua);
    L3(evl, i, 1, 2) = -0.5 * (b1u + ra);
    L3(evl, i, 1, 3) = 0.5 * b1;
    L3(evl, i, 2, 1) = 1.0 - b2;
    L3(evl, i, 2, 2) = b1u;
    L3(evl, i, 2, 3) = -b1;
    L3(evl, i, 3, 1) = 0.5 * (b2 - ua);
    L3(evl, i, 3, 2) = -0.5 * (b1u - ra);
    L3(evl, i, 3, 3) = 0.5 * b1;
  }
}

/* apps/shallowWater/2dRadialDam/rpn2sw.f:60-228 */
static void rp_sw(const ocl_params *p, int ixy, int mx, const double *ql, const double *qr,
                  double *wave, double *s, double *amdq, double *apdq, int cell_internal) {
  /* cell_internal: tfluct1sw.f:317-467 variant (left ql(i), right qr(i)) */
  const int mbc = p->mbc, meqn = p->meqn, mwaves = p->mwaves;
  const long ld = mx + 2 * mbc;
  const double g = p->grav;
  const int mu = (ixy == 1) ? 2 : 3, mv = (ixy == 1) ? 3 : 2;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    const double *L = cell_internal ? ql : qr;
    const double *R = cell_internal ? qr : ql;
    const int il = cell_internal ? i : i - 1;
#define QLT(m) L2(L, il, m)
#define QRT(m) L2(R, i, m)
    double h = (QLT(1) + QRT(1)) * 0.50;
    double hsqrtl = sqrt(QLT(1));
    double hsqrtr = sqrt(QRT(1));
    double hsq2 = hsqrtl + hsqrtr;
    double u = (QLT(mu) / hsqrtl + QRT(mu) / hsqrtr) / hsq2;
    double v = (QLT(mv) / hsqrtl + QRT(mv) / hsqrtr) / hsq2;
    double a = sqrt(g * h);
    double d1 = QRT(1) - QLT(1);
    double d2 = QRT(mu) - QLT(mu);
    double d3 = QRT(mv) - QLT(mv);
    double a1 = ((u + a) * d1 - d2) * (0.50 / a);
    double a2 = -(v * d1) + d3;
    double a3 = (-((u - a) * d1) + d2) * (0.50 / a);
    L3(wave, i, 1, 1) = a1;
    L3(wave, i, mu, 1) = a1 * (u - a);
    L3(wave, i, mv, 1) = a1 * v;
    L2(s, i, 1) = u - a;
    L3(wave, i, 1, 2) = 0.0;
    L3(wave, i, mu, 2) = 0.0;
    L3(wave, i, mv, 2) = a2;
    L2(s, i, 2) = u;
    L3(wave, i, 1, 3) = a3;
    L3(wave, i, mu, 3) = a3 * (u + a);
    L3(wave, i, mv, 3) = a3 * v;
    L2(s, i, 3) = u + a;
  }
  if (!p->efix) {
    for (int m = 1; m <= 3; ++m)
      for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        double am = 0.0, ap = 0.0;
        for (int mw = 1; mw <= mwaves; ++mw) {
          if (L2(s, i, mw) < 0.0) am = am + L2(s, i, mw) * L3(wave, i, m, mw);
          else ap = ap + L2(s, i, mw) * L3(wave, i, m, mw);
        }
        L2(amdq, i, m) = am;
        L2(apdq, i, m) = ap;
      }
    return;
  }
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    const double *L = cell_internal ? ql : qr;
    const double *R = cell_internal ? qr : ql;
    const int il = cell_internal ? i : i - 1;
    double him1 = QLT(1);
    double s0 = QLT(mu) / him1 - sqrt(g * him1);
    if (s0 > 0.0 && L2(s, i, 1) > 0.0) {
      for (int m = 1; m <= 3; ++m) L2(amdq, i, m) = 0.0;
      continue;
    }
    double h1 = QLT(1) + L3(wave, i, 1, 1);
    double hu1 = QLT(mu) + L3(wave, i, mu, 1);
    double s1 = hu1 / h1 - sqrt(g * h1);
    double sfract;
    if (s0 < 0.0 && s1 > 0.0) sfract = s0 * ((s1 - L2(s, i, 1)) / (s1 - s0));
    else if (L2(s, i, 1) < 0.0) sfract = L2(s, i, 1);
    else sfract = 0.0;
    for (int m = 1; m <= 3; ++m) L2(amdq, i, m) = sfract * L3(wave, i, m, 1);
    if (L2(s, i, 2) > 0.0) continue;
    for (int m = 1; m <= 3; ++m) L2(amdq, i, m) = L2(amdq, i, m) + L2(s, i, 2) * L3(wave, i, m, 2);
    double hi = QRT(1);
    double s03 = QRT(mu) / hi + sqrt(g * hi);
    double h3 = QRT(1) - L3(wave, i, 1, 3);
    double hu3 = QRT(mu) - L3(wave, i, mu, 3);
    double s3 = hu3 / h3 + sqrt(g * h3);
    if (s3 < 0.0 && s03 > 0.0) sfract = s3 * ((s03 - L2(s, i, 3)) / (s03 - s3));
    else if (L2(s, i, 3) < 0.0) sfract = L2(s, i, 3);
    else continue;
    for (int m = 1; m <= 3; ++m) L2(amdq, i, m) = L2(amdq, i, m) + sfract * L3(wave, i, m, 3);
  }
#undef QLT
#undef QRT
  for (int m = 1; m <= 3; ++m)
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      double df = 0.0;
      for (int mw = 1; mw <= mwaves; ++mw) df = df + L2(s, i, mw) * L3(wave, i, m, mw);
      L2(apdq, i, m) = df - L2(amdq, i, m);
    }
}

/* Shallow-water Roe eigenvectors along direction ixy at interface i-1/2 (new;
 * the reference has none).  Roe averages as rpn2sw.f:80-88 from q(i-1), q(i);
 * the left eigenvectors are the rows that rpn2sw.f:98-100 uses for a1..a3. */
static void evec_sw(const ocl_params *p, int ixy, int mx, const double *q, double *evl, double *evr) {
  const int mbc = p->mbc, meqn = 3;
  const long ld = mx + 2 * mbc;
  const double g = p->grav;
  const int mu = (ixy == 1) ? 2 : 3, mv = (ixy == 1) ? 3 : 2;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    double h = (L2(q, i - 1, 1) + L2(q, i, 1)) * 0.50;
    double hsqrtl = sqrt(L2(q, i - 1, 1));
    double hsqrtr = sqrt(L2(q, i, 1));
    double hsq2 = hsqrtl + hsqrtr;
    double u = (L2(q, i - 1, mu) / hsqrtl + L2(q, i, mu) / hsqrtr) / hsq2;
    double v = (L2(q, i - 1, mv) / hsqrtl + L2(q, i, mv) / hsqrtr) / hsq2;
    double a = sqrt(g * h);
    double ha = 0.50 / a;
    L3(evr, i, 1, 1) = 1.0;    L3(evr, i, mu, 1) = u - a; L3(evr, i, mv, 1) = v;
    L3(evr, i, 1, 2) = 0.0;    L3(evr, i, mu, 2) = 0.0;   L3(evr, i, mv, 2) = 1.0;
    L3(evr, i, 1, 3) = 1.0;    L3(evr, i, mu, 3) = u + a; L3(evr, i, mv, 3) = v;
    L3(evl, i, 1, 1) = (u + a) * ha;    L3(evl, i, 1, mu) = -ha; L3(evl, i, 1, mv) = 0.0;
    L3(evl, i, 2, 1) = -v;              L3(evl, i, 2, mu) = 0.0; L3(evl, i, 2, mv) = 1.0;
    L3(evl, i, 3, 1) = -((u - a) * ha); L3(evl, i, 3, mu) = ha;  L3(evl, i, 3, mv) = 0.0;
  }
}

/* apps/shallowWater/2dRadialDam/1dRadialSymm-qwave/rp1sw.f:43-185: 1-D
 * shallow water Roe solver, Harten-Hyman entropy fix when p->efix (the app's
 * data efix /.true./).  cell_internal: the same solve with left ql(i) and
 * right qr(i) (tfluct1sw.f of that app, which returns adq = amdq + apdq). */
static void rp_sw1d(const ocl_params *p, int mx, const double *ql, const double *qr,
                    double *wave, double *s, double *amdq, double *apdq, int cell_internal) {
  const int mbc = p->mbc, meqn = 2, mwaves = 2;
  const long ld = mx + 2 * mbc;
  const double grav = p->grav;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {                                  /* :46-67 */
    const double *L = cell_internal ? ql : qr;
    const double *R = cell_internal ? qr : ql;
    const int il = cell_internal ? i : i - 1;
#define QLT(m) L2(L, il, m)
#define QRT(m) L2(R, i, m)
    double ubar = (QLT(2) / sqrt(QLT(1)) + QRT(2) / sqrt(QRT(1))) / (sqrt(QLT(1)) + sqrt(QRT(1)));
    double cbar = sqrt((0.5 * grav) * (QLT(1) + QRT(1)));
    double d1 = QRT(1) - QLT(1);
    double d2 = QRT(2) - QLT(2);
    double a1 = (0.5 * (-d2 + (ubar + cbar) * d1)) / cbar;
    double a2 = (0.5 * (d2 - (ubar - cbar) * d1)) / cbar;
    L3(wave, i, 1, 1) = a1;
    L3(wave, i, 2, 1) = a1 * (ubar - cbar);
    L2(s, i, 1) = ubar - cbar;
    L3(wave, i, 1, 2) = a2;
    L3(wave, i, 2, 2) = a2 * (ubar + cbar);
    L2(s, i, 2) = ubar + cbar;
  }
  if (!p->efix) {                                                              /* :80-92 */
    for (int m = 1; m <= 2; ++m)
      for (int i = 2 - mbc; i <= mx + mbc; ++i) {
        double am = 0.0, ap = 0.0;
        for (int mw = 1; mw <= mwaves; ++mw) {
          if (L2(s, i, mw) < 0.0) am = am + L2(s, i, mw) * L3(wave, i, m, mw);
          else ap = ap + L2(s, i, mw) * L3(wave, i, m, mw);
        }
        L2(amdq, i, m) = am;
        L2(apdq, i, m) = ap;
      }
    return;
  }
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {                                  /* :113-173 */
    const double *L = cell_internal ? ql : qr;
    const double *R = cell_internal ? qr : ql;
    const int il = cell_internal ? i : i - 1;
    double s0 = QLT(2) / QLT(1) - sqrt(grav * QLT(1));
    if (s0 >= 0.0 && L2(s, i, 1) > 0.0) {
      for (int m = 1; m <= 2; ++m) L2(amdq, i, m) = 0.0;
      continue;
    }
    double hr1 = QLT(1) + L3(wave, i, 1, 1);
    double uhr1 = QLT(2) + L3(wave, i, 2, 1);
    double s1 = uhr1 / hr1 - sqrt(grav * hr1);
    double sfract;
    if (s0 < 0.0 && s1 > 0.0) sfract = (s0 * (s1 - L2(s, i, 1))) / (s1 - s0);
    else if (L2(s, i, 1) < 0.0) sfract = L2(s, i, 1);
    else sfract = 0.0;
    for (int m = 1; m <= 2; ++m) L2(amdq, i, m) = sfract * L3(wave, i, m, 1);
    double s3 = QRT(2) / QRT(1) + sqrt(grav * QRT(1));
    double hl2 = QRT(1) - L3(wave, i, 1, 2);
    double uhl2 = QRT(2) - L3(wave, i, 2, 2);
    double s2 = uhl2 / hl2 + sqrt(grav * hl2);
    if (s2 < 0.0 && s3 > 0.0) sfract = (s2 * (s3 - L2(s, i, 2))) / (s3 - s2);
    else if (L2(s, i, 2) < 0.0) sfract = L2(s, i, 2);
    else continue;
    for (int m = 1; m <= 2; ++m) L2(amdq, i, m) = L2(amdq, i, m) + sfract * L3(wave, i, m, 2);
  }
#undef QLT
#undef QRT
  for (int m = 1; m <= 2; ++m)                                                 /* :176-183 */
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      double df = 0.0;
      for (int mw = 1; mw <= mwaves; ++mw) df = df + L2(s, i, mw) * L3(wave, i, m, mw);
      L2(apdq, i, m) = df - L2(amdq, i, m);
    }
  (void)meqn;
}

/* 1-D shallow-water Roe eigenvectors at interface i-1/2 (new; the reference
 * has none): averages as rp1sw.f:47-49 from q(i-1), q(i); the left
 * eigenvectors are the rows rp1sw.f:56-57 uses for a1, a2. */
static void evec_sw1d(const ocl_params *p, int mx, const double *q, double *evl, double *evr) {
  const int mbc = p->mbc, meqn = 2;
  const long ld = mx + 2 * mbc;
  const double grav = p->grav;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    double ubar = (L2(q, i - 1, 2) / sqrt(L2(q, i - 1, 1)) + L2(q, i, 2) / sqrt(L2(q, i, 1))) /
                  (sqrt(L2(q, i - 1, 1)) + sqrt(L2(q, i, 1)));
    double cbar = sqrt((0.5 * grav) * (L2(q, i - 1, 1) + L2(q, i, 1)));
    double ha = 0.5 / cbar;
    L3(evr, i, 1, 1) = 1.0;          L3(evr, i, 1, 2) = 1.0;
    L3(evr, i, 2, 1) = ubar - cbar;  L3(evr, i, 2, 2) = ubar + cbar;
    L3(evl, i, 1, 1) = (ubar + cbar) * ha;     L3(evl, i, 1, 2) = -ha;
    L3(evl, i, 2, 1) = -((ubar - cbar) * ha);  L3(evl, i, 2, 2) = ha;
  }
}

/* The f-wave shallow-water solvers of apps/shallowWater/1dPerturbSteady and
 * 2dRadialDam/1dRadialSymm-fwave{,-kappa} (rpf-wave.f90:55-122,
 * tfluctf-wave.f90:55-126 of each): Roe averages, the flux difference of the
 * app (with its source or area terms) split on the Roe eigenvectors into two
 * f-waves, amdq/apdq by the sign of the speeds (half each for a NaN speed).
 * cell_internal: the tfluct variant, left ql(i), right qr(i), which returns
 * the total fluctuation in amdq (adq = amdq + apdq). */
static void rp_swf(const ocl_params *p, int mx, const double *ql, const double *qr, const double *auxl,
                   const double *auxr, double *wave, double *s, double *amdq, double *apdq,
                   int cell_internal) {
  const int mbc = p->mbc, meqn = 2;
  const long ld = mx + 2 * mbc;
  const double grav = p->grav;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    double hl, ul, hr, ur;
    if (cell_internal) {
      hl = L2(ql, i, 1); ul = L2(ql, i, 2) / hl;
      hr = L2(qr, i, 1); ur = L2(qr, i, 2) / hr;
    } else {
      hl = L2(qr, i - 1, 1); ul = L2(qr, i - 1, 2) / hl;
      hr = L2(ql, i, 1); ur = L2(ql, i, 2) / hr;
    }
    double hbar = 0.5 * (hr + hl);
    double uhat = (sqrt(hl) * ul + sqrt(hr) * ur) / (sqrt(hl) + sqrt(hr));
    double chat = sqrt(grav * hbar);
    double f1, f2;
    if (p->rp == OCL_RP_SWF_BATHY && !cell_internal) {            /* 1dPerturbSteady/rpf-wave.f90:67-68 */
      f1 = (hr * ur) - (hl * ul);
      f2 = ((hr * ur) * ur + (0.5 * grav) * (hr * hr)) - ((hl * ul) * ul + (0.5 * grav) * (hl * hl));
    } else if (p->rp == OCL_RP_SWF_BATHY) {                       /* tfluctf-wave.f90:56-70 */
      double bl = L2(auxl, i - 1, 1), br = L2(auxr, i + 1, 1);
      f1 = (hr * ur) - (hl * ul);
      f2 = (((hr * ur) * ur + ((0.5 * grav) * hr) * hr) - ((hl * ul) * ul + ((0.5 * grav) * hl) * hl)) +
           ((grav * hbar) * (br - bl)) / 2.0;
    } else if (p->rp == OCL_RP_SWF_RADIAL && !cell_internal) {    /* 1dRadialSymm-fwave/rpf-wave.f90:69-70 */
      f1 = ((hr * ur) - (hl * ul)) + ((hbar * uhat) / L2(auxl, i, 1)) * L2(auxl, i, 2);
      f2 = (((hr * ur) * ur + (0.5 * grav) * (hr * hr)) - ((hl * ul) * ul + (0.5 * grav) * (hl * hl))) +
           ((hbar * (uhat * uhat)) / L2(auxl, i, 1)) * L2(auxl, i, 2);
    } else if (p->rp == OCL_RP_SWF_RADIAL) {                      /* tfluctf-wave.f90:68-69 */
      f1 = (hr * ur) - (hl * ul);
      f2 = ((hr * ur) * ur + ((0.5 * grav) * hr) * hr) - ((hl * ul) * ul + ((0.5 * grav) * hl) * hl);
    } else if (!cell_internal) {                                  /* -kappa/rpf-wave.f90:69-70 */
      f1 = L2(auxl, i, 1) * (hr * ur) - L2(auxr, i - 1, 1) * (hl * ul);
      f2 = (L2(auxl, i, 1) * ((hr * ur) * ur + ((0.5 * grav) * hr) * hr) -
            L2(auxr, i - 1, 1) * ((hl * ul) * ul + ((0.5 * grav) * hl) * hl)) -
           (((0.5 * grav) * hbar) * hbar) * L2(auxl, i, 4);
    } else {                                                      /* -kappa/tfluctf-wave.f90:68-69 */
      f1 = L2(auxr, i, 2) * (hr * ur) - L2(auxl, i, 2) * (hl * ul);
      f2 = L2(auxr, i, 2) * ((hr * ur) * ur + ((0.5 * grav) * hr) * hr) -
           L2(auxl, i, 3) * ((hl * ul) * ul + ((0.5 * grav) * hl) * hl);
    }
    double sp[2] = {uhat - chat, uhat + chat};
    double R[2][2] = {{1.0, 1.0}, {uhat - chat, uhat + chat}};          /* R(j,k) */
    double Lm[2][2] = {{(chat + uhat) / (2.0 * chat), -(1.0 / (2.0 * chat))},
                       {(chat - uhat) / (2.0 * chat), 1.0 / (2.0 * chat)}};   /* L(j,k) */
    double fd[2] = {f1, f2}, beta[2];
    for (int j = 0; j < 2; ++j) {
      double b = 0.0;
      for (int k = 0; k < 2; ++k) b = b + Lm[j][k] * fd[k];
      beta[j] = b;
    }
    L2(s, i, 1) = sp[0];
    L2(s, i, 2) = sp[1];
    for (int j = 0; j < 2; ++j) {
      double am = 0.0, ap = 0.0;
      for (int k = 0; k < 2; ++k) {
        double fw = beta[k] * R[j][k];
        L3(wave, i, j + 1, k + 1) = fw;
        if (sp[k] < 0.0) am = am + fw;
        else if (sp[k] >= 0.0) ap = ap + fw;
        else { am = am + 0.5 * fw; ap = ap + 0.5 * fw; }
      }
      L2(amdq, i, j + 1) = am;
      L2(apdq, i, j + 1) = ap;
    }
  }
}

/* Roe eigenvectors of the f-wave solvers from q(i-1), q(i) (their R and L,
 * rpf-wave.f90:71-88). */
static void evec_swf(const ocl_params *p, int mx, const double *q, double *evl, double *evr) {
  const int mbc = p->mbc, meqn = 2;
  const long ld = mx + 2 * mbc;
  const double grav = p->grav;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    double hl = L2(q, i - 1, 1), ul = L2(q, i - 1, 2) / hl;
    double hr = L2(q, i, 1), ur = L2(q, i, 2) / hr;
    double hbar = 0.5 * (hr + hl);
    double uhat = (sqrt(hl) * ul + sqrt(hr) * ur) / (sqrt(hl) + sqrt(hr));
    double chat = sqrt(grav * hbar);
    L3(evr, i, 1, 1) = 1.0;          L3(evr, i, 1, 2) = 1.0;
    L3(evr, i, 2, 1) = uhat - chat;  L3(evr, i, 2, 2) = uhat + chat;
    L3(evl, i, 1, 1) = (chat + uhat) / (2.0 * chat);  L3(evl, i, 1, 2) = -(1.0 / (2.0 * chat));
    L3(evl, i, 2, 1) = (chat - uhat) / (2.0 * chat);  L3(evl, i, 2, 2) = 1.0 / (2.0 * chat);
  }
}

/* apps/acoustics/1d/homogeneous: rp1.f:50-76 and tfluct.f (cell_internal:
 * left ql(i), right qr(i), adq = amdq + apdq), cc = sqrt(bulk/rho), zz =
 * cc*rho as setprob.f computes them. */
static void rp_acconst(const ocl_params *p, int mx, const double *ql, const double *qr, double *wave,
                       double *s, double *amdq, double *apdq, int cell_internal) {
  const int mbc = p->mbc, meqn = 2;
  const long ld = mx + 2 * mbc;
  const double cc = sqrt(p->bulk / p->rho), zz = cc * p->rho;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    double d1, d2;
    if (cell_internal) { d1 = L2(qr, i, 1) - L2(ql, i, 1); d2 = L2(qr, i, 2) - L2(ql, i, 2); }
    else { d1 = L2(ql, i, 1) - L2(qr, i - 1, 1); d2 = L2(ql, i, 2) - L2(qr, i - 1, 2); }
    double a1 = ((-d1) + zz * d2) / (2.0 * zz);
    double a2 = (d1 + zz * d2) / (2.0 * zz);
    L3(wave, i, 1, 1) = -(a1 * zz);
    L3(wave, i, 2, 1) = a1;
    L2(s, i, 1) = -cc;
    L3(wave, i, 1, 2) = a2 * zz;
    L3(wave, i, 2, 2) = a2;
    L2(s, i, 2) = cc;
  }
  for (int m = 1; m <= 2; ++m)
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      L2(amdq, i, m) = L2(s, i, 1) * L3(wave, i, m, 1);
      L2(apdq, i, m) = L2(s, i, 2) * L3(wave, i, m, 2);
    }
}

/* apps/acoustics/1d/homogeneous/evec.f */
static void evec_acconst(const ocl_params *p, int mx, double *evl, double *evr) {
  const int mbc = p->mbc, meqn = 2;
  const long ld = mx + 2 * mbc;
  const double cc = sqrt(p->bulk / p->rho), zz = cc * p->rho;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    L3(evr, i, 1, 1) = -zz;
    L3(evr, i, 1, 2) = zz;
    L3(evr, i, 2, 1) = 1.0;
    L3(evr, i, 2, 2) = 1.0;
    double z = 1.0 / (zz + zz);
    L3(evl, i, 1, 1) = -z;
    L3(evl, i, 1, 2) = zz * z;
    L3(evl, i, 2, 1) = 1.0 * z;
    L3(evl, i, 2, 2) = zz * z;
  }
}

/* Stress laws: apps/acoustics/1d/fwave/rp1acfw.f:116-140 (sigma = bulk*eps)
 * and apps/elasticity/stegoton/rp1nel.f:116-175 (exp(A eps) - 1 for A > 0,
 * else B eps), with their derivatives. */
static double sigma_el(const ocl_params *p, double eps, double a, double b) {
  if (p->rp == OCL_RP_STEGOTON) return a > 0.0 ? exp(a * eps) - 1.0 : b * eps;
  return a * eps;
}
static double sigmap_el(const ocl_params *p, double eps, double a, double b) {
  if (p->rp == OCL_RP_STEGOTON) return a > 0.0 ? a * exp(a * eps) : b;
  (void)eps;
  return a;
}

/* apps/acoustics/1d/fwave: rp1acfw.f:53-109 and tfluct1.f (cell_internal:
 * both sides use aux(i), left ql(i), right qr(i)); the same for
 * apps/elasticity/stegoton (rp1nel.f:53-109, tfluct1.f:56-113) with its stress law. */
static void rp_acfwave(const ocl_params *p, int mx, const double *ql, const double *qr, const double *auxl,
                       const double *auxr, double *wave, double *s, double *amdq, double *apdq,
                       int cell_internal) {
  const int mbc = p->mbc, meqn = 2;
  const long ld = mx + 2 * mbc;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    double rhoi, rhoim, epsi, epsim, urhoi, urhoim, ai, aim, bi = 0.0, bim = 0.0;
    const int nl = p->rp == OCL_RP_STEGOTON;
    if (cell_internal) {
      rhoi = L2(auxr, i, 1); rhoim = L2(auxl, i, 1);
      epsi = L2(qr, i, 1); epsim = L2(ql, i, 1);
      urhoi = L2(qr, i, 2); urhoim = L2(ql, i, 2);
      ai = L2(auxr, i, 2); aim = L2(auxl, i, 2);
      if (nl) { bi = L2(auxr, i, 3); bim = L2(auxl, i, 3); }
    } else {
      rhoi = L2(auxl, i, 1); rhoim = L2(auxr, i - 1, 1);
      epsi = L2(ql, i, 1); epsim = L2(qr, i - 1, 1);
      urhoi = L2(ql, i, 2); urhoim = L2(qr, i - 1, 2);
      ai = L2(auxl, i, 2); aim = L2(auxr, i - 1, 2);
      if (nl) { bi = L2(auxl, i, 3); bim = L2(auxr, i - 1, 3); }
    }
    double ki = sigmap_el(p, epsi, ai, bi);
    double kim = sigmap_el(p, epsim, aim, bim);
    double ci = sqrt(ki / rhoi);
    double cim = sqrt(kim / rhoim);
    double zi = ci * rhoi;
    double zim = cim * rhoim;
    double du = urhoi / rhoi - urhoim / rhoim;
    double dsig = sigma_el(p, epsi, ai, bi) - sigma_el(p, epsim, aim, bim);
    double b1 = -((zi * du + dsig) / (zim + zi));
    double b2 = -((zim * du - dsig) / (zim + zi));
    L3(wave, i, 1, 1) = b1;
    L3(wave, i, 2, 1) = b1 * zim;
    L2(s, i, 1) = -cim;
    L3(wave, i, 1, 2) = b2;
    L3(wave, i, 2, 2) = b2 * (-zi);
    L2(s, i, 2) = ci;
  }
  for (int m = 1; m <= 2; ++m)
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      L2(amdq, i, m) = L3(wave, i, m, 1);
      L2(apdq, i, m) = L3(wave, i, m, 2);
    }
}

/* apps/acoustics/1d/fwave/evec.f:40-63 (as the app writes it: evl holds the
 * rows (1, 1) and (zim, -zi), evr their inverse) */
static void evec_acfwave(const ocl_params *p, int mx, const double *q, const double *auxl, const double *auxr,
                         double *evl, double *evr) {
  const int mbc = p->mbc, meqn = 2;
  const long ld = mx + 2 * mbc;
  const int nl = p->rp == OCL_RP_STEGOTON;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    double ki = sigmap_el(p, L2(q, i, 1), L2(auxl, i, 2), nl ? L2(auxl, i, 3) : 0.0);
    double kim = sigmap_el(p, L2(q, i - 1, 1), L2(auxr, i - 1, 2), nl ? L2(auxr, i - 1, 3) : 0.0);
    double ci = sqrt(ki / L2(auxl, i, 1));
    double cim = sqrt(kim / L2(auxr, i - 1, 1));
    double zi = ci * L2(auxl, i, 1);
    double zim = cim * L2(auxr, i - 1, 1);
    L3(evl, i, 1, 1) = 1.0;
    L3(evl, i, 1, 2) = 1.0;
    L3(evl, i, 2, 1) = zim;
    L3(evl, i, 2, 2) = -zi;
    double zh = 1.0 / (zim + zi);
    L3(evr, i, 1, 1) = zi * zh;
    L3(evr, i, 1, 2) = zh;
    L3(evr, i, 2, 1) = zim * zh;
    L3(evr, i, 2, 2) = -zh;
  }
}

/* apps/traffic/congTraffic/rpf-wave.f90:42-90: f-wave for the flux
 * umax(x) q (1-q) with the entropy-satisfying split of its four sign cases;
 * tfluct1.f90:39-49: the cell's flux difference (both sides aux(i)). */
static void rp_traffic(const ocl_params *p, int mx, const double *ql, const double *qr, const double *auxl,
                       const double *auxr, double *wave, double *s, double *amdq, double *apdq) {
  const int mbc = p->mbc, meqn = 1;
  const long ld = mx + 2 * mbc;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    double fim1 = (L2(auxr, i - 1, 1) * L2(qr, i - 1, 1)) * (1.0 - L2(qr, i - 1, 1));
    double fi = (L2(auxl, i, 1) * L2(ql, i, 1)) * (1.0 - L2(ql, i, 1));
    L3(wave, i, 1, 1) = fi - fim1;
    double sim1 = L2(auxr, i - 1, 1) * (1.0 - 2.0 * L2(qr, i - 1, 1));
    double si = L2(auxl, i, 1) * (1.0 - 2.0 * L2(ql, i, 1));
    if (sim1 < 0.0 && si <= 0.0) {
      L2(s, i, 1) = sim1; L2(amdq, i, 1) = L3(wave, i, 1, 1); L2(apdq, i, 1) = 0.0;
    } else if (sim1 >= 0.0 && si > 0.0) {
      L2(s, i, 1) = si; L2(amdq, i, 1) = 0.0; L2(apdq, i, 1) = L3(wave, i, 1, 1);
    } else if (sim1 < 0.0 && si > 0.0) {                      /* transonic rarefaction */
      L2(s, i, 1) = 0.5 * (sim1 + si);
      double f0 = dmin1(L2(auxr, i - 1, 1), L2(auxl, i, 1)) * 0.25;
      L2(amdq, i, 1) = f0 - fim1;
      L2(apdq, i, 1) = fi - f0;
    } else {
      L2(s, i, 1) = 0.5 * (sim1 + si);
      if (L2(s, i, 1) < 0.0) { L2(amdq, i, 1) = L3(wave, i, 1, 1); L2(apdq, i, 1) = 0.0; }
      else if (L2(s, i, 1) > 0.0) { L2(amdq, i, 1) = 0.0; L2(apdq, i, 1) = L3(wave, i, 1, 1); }
      else { L2(amdq, i, 1) = 0.5 * L3(wave, i, 1, 1); L2(apdq, i, 1) = 0.5 * L3(wave, i, 1, 1); }
    }
  }
}

static void tfluct_traffic(const ocl_params *p, int mx, const double *ql, const double *qr, const double *auxl,
                           const double *auxr, double *adq) {
  const int mbc = p->mbc;
  const long ld = mx + 2 * mbc;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    double fim1 = (L2(auxl, i, 1) * L2(ql, i, 1)) * (1.0 - L2(ql, i, 1));
    double fi = (L2(auxr, i, 1) * L2(qr, i, 1)) * (1.0 - L2(qr, i, 1));
    L2(adq, i, 1) = fi - fim1;
  }
}

/* apps/traffic/flux-uq/rpf-wave.f90:43-64: conservative advection with cell
 * velocities, f-wave u(i) q(i) - u(i-1) q(i-1) to the side of u(i)'s sign. */
static void rp_advcons(const ocl_params *p, int mx, const double *ql, const double *qr, const double *auxl,
                       const double *auxr, double *wave, double *s, double *amdq, double *apdq) {
  const int mbc = p->mbc, meqn = 1;
  const long ld = mx + 2 * mbc;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    double ui = L2(auxl, i, 1), uim = L2(auxr, i - 1, 1);
    double fim = uim * L2(qr, i - 1, 1);
    double fi = ui * L2(ql, i, 1);
    L3(wave, i, 1, 1) = fi - fim;
    if (ui > 0.0) { L2(s, i, 1) = ui; L2(amdq, i, 1) = 0.0; L2(apdq, i, 1) = L3(wave, i, 1, 1); }
    else { L2(s, i, 1) = uim; L2(amdq, i, 1) = L3(wave, i, 1, 1); L2(apdq, i, 1) = 0.0; }
  }
}

/* apps/acoustics/1d/interface/rp1acv.f:49-80; with ixy it is also the new 2-D
 * normal solver (mu = normal velocity, tangential components carry 0). */
static void rp_acoustics(const ocl_params *p, int ixy, int mx, const double *ql, const double *qr,
                         const double *auxl, const double *auxr, double *wave, double *s,
                         double *amdq, double *apdq) {
  const int mbc = p->mbc, meqn = p->meqn;
  const long ld = mx + 2 * mbc;
  const int mu = (ixy == 1) ? 2 : 3, mv = (ixy == 1) ? 3 : 2;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    double d1 = L2(ql, i, 1) - L2(qr, i - 1, 1);
    double d2 = L2(ql, i, mu) - L2(qr, i - 1, mu);
    double zi = L2(auxl, i, 1);
    double zim = L2(auxr, i - 1, 1);
    double a1 = ((-d1) + zi * d2) / (zim + zi);
    double a2 = (d1 + zim * d2) / (zim + zi);
    L3(wave, i, 1, 1) = -(a1 * zim);
    L3(wave, i, mu, 1) = a1;
    L2(s, i, 1) = -L2(auxr, i - 1, 2);
    L3(wave, i, 1, 2) = a2 * zi;
    L3(wave, i, mu, 2) = a2;
    L2(s, i, 2) = L2(auxl, i, 2);
    if (meqn == 3) { L3(wave, i, mv, 1) = 0.0; L3(wave, i, mv, 2) = 0.0; }
  }
  for (int m = 1; m <= meqn; ++m)
    for (int i = 2 - mbc; i <= mx + mbc; ++i) {
      L2(amdq, i, m) = L2(s, i, 1) * L3(wave, i, m, 1);
      L2(apdq, i, m) = L2(s, i, 2) * L3(wave, i, m, 2);
    }
}

/* apps/acoustics/1d/interface/tfluct1acv.f:134-166 (2-D: normal by ixy) */
static void tfluct_acoustics(const ocl_params *p, int ixy, int mx, const double *ql, const double *qr,
                             const double *auxl, double *s, double *adq) {
  const int mbc = p->mbc, meqn = p->meqn;
  const long ld = mx + 2 * mbc;
  const int mu = (ixy == 1) ? 2 : 3, mv = (ixy == 1) ? 3 : 2;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    double d1 = L2(qr, i, 1) - L2(ql, i, 1);
    double d2 = L2(qr, i, mu) - L2(ql, i, mu);
    double zi = L2(auxl, i, 1);
    double zim = L2(auxl, i, 1);
    double a1 = ((-d1) + zi * d2) / (zim + zi);
    double a2 = (d1 + zim * d2) / (zim + zi);
    double w[3][2];
    w[0][0] = -(a1 * zim); w[0][1] = a2 * zi;
    w[mu - 1][0] = a1;     w[mu - 1][1] = a2;
    if (meqn == 3) { w[mv - 1][0] = 0.0; w[mv - 1][1] = 0.0; }
    double s1 = -L2(auxl, i, 2), s2 = L2(auxl, i, 2);
    L2(s, i, 1) = s1;
    L2(s, i, 2) = s2;
    for (int m = 1; m <= meqn; ++m) {
      double am = s1 * w[m - 1][0];
      double ap = s2 * w[m - 1][1];
      L2(adq, i, m) = am + ap;
    }
  }
}

/* apps/acoustics/1d/interface/evec.f90:196-206; 2-D adds the tangential
 * velocity as a third, zero-speed field (new). */
static void evec_acoustics(const ocl_params *p, int ixy, int mx, const double *auxl,
                           double *evl, double *evr) {
  const int mbc = p->mbc, meqn = p->meqn;
  const long ld = mx + 2 * mbc;
  const int mu = (ixy == 1) ? 2 : 3, mv = (ixy == 1) ? 3 : 2;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    L3(evr, i, 1, 1) = -L2(auxl, i - 1, 1);
    L3(evr, i, 1, 2) = L2(auxl, i, 1);
    L3(evr, i, mu, 1) = 1.0;
    L3(evr, i, mu, 2) = 1.0;
    double z = 1.0 / (L2(auxl, i - 1, 1) + L2(auxl, i, 1));
    L3(evl, i, 1, 1) = -1.0 * z;
    L3(evl, i, 1, mu) = L2(auxl, i, 1) * z;
    L3(evl, i, 2, 1) = 1.0 * z;
    L3(evl, i, 2, mu) = L2(auxl, i - 1, 1) * z;
    if (meqn == 3) {
      L3(evr, i, mv, 1) = 0.0; L3(evr, i, mv, 2) = 0.0;
      L3(evr, i, 1, 3) = 0.0;  L3(evr, i, mu, 3) = 0.0; L3(evr, i, mv, 3) = 1.0;
      L3(evl, i, 1, mv) = 0.0; L3(evl, i, 2, mv) = 0.0;
      L3(evl, i, 3, 1) = 0.0;  L3(evl, i, 3, mu) = 0.0; L3(evl, i, 3, mv) = 1.0;
    }
  }
}

/* apps/advection/1d/evec.f:118-121 */
static void evec_advection(const ocl_params *p, int mx, double *evl, double *evr) {
  const int mbc = p->mbc, meqn = 1;
  const long ld = mx + 2 * mbc;
  for (int i = 2 - mbc; i <= mx + mbc; ++i) {
    L3(evr, i, 1, 1) = 1.0;
    L3(evl, i, 1, 1) = 1.0;
  }
}

int ocl_rp(const ocl_params *p, int ixy, int mx, const double *ql, const double *qr,
           const double *auxl, const double *auxr, double *wave, double *s,
           double *amdq, double *apdq) {
  switch (p->rp) {
    case OCL_RP_ADVECTION: rp_advection(p, mx, ql, qr, wave, s, amdq, apdq); return 0;
    case OCL_RP_ADVECTION2D: rp_advedge(p, ixy, mx, ql, qr, auxl, wave, s, amdq, apdq); return 0;
    case OCL_RP_EULER: rp_euler(p, mx, ql, qr, wave, s, amdq, apdq); return 0;
    case OCL_RP_SW2D: rp_sw(p, ixy, mx, ql, qr, wave, s, amdq, apdq, 0); return 0;
    case OCL_RP_SW1D: rp_sw1d(p, mx, ql, qr, wave, s, amdq, apdq, 0); return 0;
    case OCL_RP_SWF_BATHY:
    case OCL_RP_SWF_RADIAL:
    case OCL_RP_SWF_KAPPA: rp_swf(p, mx, ql, qr, auxl, auxr, wave, s, amdq, apdq, 0); return 0;
    case OCL_RP_ACOUSTICS_CONST: rp_acconst(p, mx, ql, qr, wave, s, amdq, apdq, 0); return 0;
    case OCL_RP_ACOUSTICS_FWAVE:
    case OCL_RP_STEGOTON: rp_acfwave(p, mx, ql, qr, auxl, auxr, wave, s, amdq, apdq, 0); return 0;
    case OCL_RP_TRAFFIC: rp_traffic(p, mx, ql, qr, auxl, auxr, wave, s, amdq, apdq); return 0;
    case OCL_RP_ADVECTION_CONS: rp_advcons(p, mx, ql, qr, auxl, auxr, wave, s, amdq, apdq); return 0;
    case OCL_RP_ACOUSTICS1D:
    case OCL_RP_ACOUSTICS2D:
      rp_acoustics(p, ixy, mx, ql, qr, auxl, auxr, wave, s, amdq, apdq); return 0;
  }
  return -4;
}

int ocl_tfluct(const ocl_params *p, int ixy, int mx, const double *ql, const double *qr,
               const double *auxl, const double *auxr, double *s, double *adq) {
  (void)auxr;
  switch (p->rp) {
    case OCL_RP_ADVECTION: tfluct_advection(p, mx, ql, qr, s, adq); return 0;
    case OCL_RP_SW2D: {
      /* tfluct1sw.f: the Roe solve with left ql(i), right qr(i); adq = amdq+apdq */
      const long ld = mx + 2L * p->mbc;
      double *wave = (double *)calloc((size_t)ld * p->meqn * p->mwaves, sizeof(double));
      double *am = (double *)calloc((size_t)ld * p->meqn, sizeof(double));
      double *ap = (double *)calloc((size_t)ld * p->meqn, sizeof(double));
      rp_sw(p, ixy, mx, ql, qr, wave, s, am, ap, 1);
      for (long k = 0; k < ld * p->meqn; ++k) adq[k] = am[k] + ap[k];
      free(wave); free(am); free(ap);
      return 0;
    }
    case OCL_RP_SW1D: {
      /* 1dRadialSymm-qwave/tfluct1sw.f:44-186: left ql(i), right qr(i) */
      const long ld = mx + 2L * p->mbc;
      double *wave = (double *)calloc((size_t)ld * 4, sizeof(double));
      double *am = (double *)calloc((size_t)ld * 2, sizeof(double));
      double *ap = (double *)calloc((size_t)ld * 2, sizeof(double));
      rp_sw1d(p, mx, ql, qr, wave, s, am, ap, 1);
      for (long k = 0; k < ld * 2; ++k) adq[k] = am[k] + ap[k];
      free(wave); free(am); free(ap);
      return 0;
    }
    case OCL_RP_SWF_BATHY:
    case OCL_RP_SWF_RADIAL:
    case OCL_RP_SWF_KAPPA: {
      const long ld = mx + 2L * p->mbc;
      double *wave = (double *)calloc((size_t)ld * 4, sizeof(double));
      double *am = (double *)calloc((size_t)ld * 2, sizeof(double));
      double *ap = (double *)calloc((size_t)ld * 2, sizeof(double));
      rp_swf(p, mx, ql, qr, auxl, auxr, wave, s, am, ap, 1);
      for (long k = 0; k < ld * 2; ++k) adq[k] = am[k] + ap[k];     /* tfluctf-wave.f90:121-123 */
      free(wave); free(am); free(ap);
      return 0;
    }
    case OCL_RP_TRAFFIC: tfluct_traffic(p, mx, ql, qr, auxl, auxr, adq); return 0;
    case OCL_RP_ACOUSTICS_CONST:
    case OCL_RP_ACOUSTICS_FWAVE:
    case OCL_RP_STEGOTON: {
      const long ld = mx + 2L * p->mbc;
      double *wave = (double *)calloc((size_t)ld * 4, sizeof(double));
      double *am = (double *)calloc((size_t)ld * 2, sizeof(double));
      double *ap = (double *)calloc((size_t)ld * 2, sizeof(double));
      if (p->rp == OCL_RP_ACOUSTICS_CONST) rp_acconst(p, mx, ql, qr, wave, s, am, ap, 1);
      else rp_acfwave(p, mx, ql, qr, auxl, auxr, wave, s, am, ap, 1);
      for (long k = 0; k < ld * 2; ++k) adq[k] = am[k] + ap[k];
      free(wave); free(am); free(ap);
      return 0;
    }
    case OCL_RP_ACOUSTICS1D:
    case OCL_RP_ACOUSTICS2D:
      tfluct_acoustics(p, ixy, mx, ql, qr, auxl, s, adq); return 0;
  }
  return -4;  /* src/tfluct.f90: no tfluct for this family */
}

int ocl_evec(const ocl_params *p, int ixy, int mx, const double *q, const double *auxl,
             const double *auxr, double *evl, double *evr) {
  (void)auxr;
  switch (p->rp) {
    case OCL_RP_ADVECTION:
    case OCL_RP_ADVECTION2D:
    case OCL_RP_TRAFFIC:
    case OCL_RP_ADVECTION_CONS: evec_advection(p, mx, evl, evr); return 0;
    case OCL_RP_EULER: evec_euler(p, mx, q, evl, evr); return 0;
    case OCL_RP_SW2D: evec_sw(p, ixy, mx, q, evl, evr); return 0;
    case OCL_RP_SW1D: evec_sw1d(p, mx, q, evl, evr); return 0;
    case OCL_RP_SWF_BATHY:
    case OCL_RP_SWF_RADIAL:
    case OCL_RP_SWF_KAPPA: evec_swf(p, mx, q, evl, evr); return 0;
    case OCL_RP_ACOUSTICS_CONST: evec_acconst(p, mx, evl, evr); return 0;
    case OCL_RP_ACOUSTICS_FWAVE:
    case OCL_RP_STEGOTON: evec_acfwave(p, mx, q, auxl, auxr, evl, evr); return 0;
    case OCL_RP_ACOUSTICS1D:
    case OCL_RP_ACOUSTICS2D: evec_acoustics(p, ixy, mx, auxl, evl, evr); return 0;
  }
  return -4;
}

/* ======================================================================== */
/* src/flux1.f90:55-190                                                      */
/* ======================================================================== */
int ocl_flux1(const ocl_params *p, const double *q1d, double *dq1d, const double *aux1d,
              double dt, double *cfl, int ixy, int mx) {
  const int mbc = p->mbc, meqn = p->meqn, mwaves = p->mwaves, maux = p->maux;
  const long ld = mx + 2 * mbc;
  const int mx2 = (int)ld;
  int rc = 0;
  if (p->lim_type < 0 || p->lim_type > 2) return -5;
  double dx = (ixy == 1) ? p->dx : p->dy;
  double *dtdx = (double *)calloc((size_t)ld, sizeof(double));
  double *ql = (double *)calloc((size_t)ld * meqn, sizeof(double));
  double *qr = (double *)calloc((size_t)ld * meqn, sizeof(double));
  double *wave = (double *)calloc((size_t)ld * meqn * mwaves, sizeof(double));
  double *s = (double *)calloc((size_t)ld * mwaves, sizeof(double));
  double *amdq = (double *)calloc((size_t)ld * meqn, sizeof(double));
  double *apdq = (double *)calloc((size_t)ld * meqn, sizeof(double));
  double *amdq2 = (double *)calloc((size_t)ld * meqn, sizeof(double));
  double *apdq2 = (double *)calloc((size_t)ld * meqn, sizeof(double));
  double *evl = (double *)calloc((size_t)ld * meqn * meqn, sizeof(double));
  double *evr = (double *)calloc((size_t)ld * meqn * meqn, sizeof(double));
  double *auxl = (double *)calloc((size_t)ld * (maux > 0 ? maux : 1), sizeof(double));
  double *auxr = (double *)calloc((size_t)ld * (maux > 0 ? maux : 1), sizeof(double));
  if (!dtdx || !ql || !qr || !wave || !s || !amdq || !apdq || !amdq2 || !apdq2 || !evl ||
      !evr || !auxl || !auxr) { rc = -3; goto done; }

  for (int i = 1 - mbc; i <= mx + mbc; ++i) {                                 /* :57-61 */
    if (p->mcapa > 0) dtdx[i + mbc - 1] = dt / (dx * L2(aux1d, i, p->mcapa));
    else dtdx[i + mbc - 1] = dt / dx;
  }
  if (p->ndim > 1)                                                            /* :62 */
    for (long k = 0; k < ld * meqn; ++k) dq1d[k] = 0.0;

  if (p->lim_type == 0) {                                                    /* :65-76 */
    switch (p->char_decomp) {
      case 0: rc = ocl_poly(mx2, meqn, q1d, p->mthlim[0], ql, qr); break;
      case 1:
        rc = ocl_rp(p, ixy, mx, q1d, q1d, aux1d, aux1d, wave, s, amdq, apdq);
        if (!rc) rc = ocl_poly_wave(mx2, meqn, mwaves, q1d, p->mthlim[0], wave, ql, qr);
        break;
      default: rc = -5;
    }
  } else if (p->lim_type == 1) {                                             /* :78-91 */
    switch (p->char_decomp) {
      case 0: rc = ocl_tvd2(mx2, meqn, q1d, p->mthlim, ql, qr); break;
      case 1:
        rc = ocl_rp(p, ixy, mx, q1d, q1d, aux1d, aux1d, wave, s, amdq, apdq);
        if (!rc) rc = ocl_tvd2_wave(mx2, meqn, mwaves, q1d, p->mthlim, wave, s, ql, qr);
        break;
      case 2:
        rc = ocl_evec(p, ixy, mx, q1d, aux1d, aux1d, evl, evr);
        if (!rc) rc = ocl_tvd2_char(mx2, meqn, q1d, p->mthlim, evl, evr, ql, qr);
        break;
      default: rc = -5;
    }
  } else
  switch (p->char_decomp) {                                                   /* :92-116 */
    case 0: rc = ocl_weno5(mx2, meqn, q1d, ql, qr); break;
    case 1:                                                                   /* :97-101 */
      rc = ocl_rp(p, ixy, mx, q1d, q1d, aux1d, aux1d, wave, s, amdq, apdq);
      if (!rc) rc = ocl_weno5_wave(mx2, meqn, mwaves, q1d, wave, ql, qr);
      break;
    case 2:
      rc = ocl_evec(p, ixy, mx, q1d, aux1d, aux1d, evl, evr);
      if (!rc) rc = ocl_weno5_char(mx2, meqn, q1d, evl, evr, ql, qr);
      break;
    case 3:                                                                   /* :107-110 */
      rc = ocl_evec(p, ixy, mx, q1d, aux1d, aux1d, evl, evr);
      if (!rc) rc = ocl_weno5_trans(mx2, meqn, q1d, evl, evr, ql, qr);
      break;
    default: rc = -5;
  }
  if (rc) goto done;

  rc = ocl_rp(p, ixy, mx, ql, qr, aux1d, aux1d, wave, s, amdq, apdq);        /* :122-123 */
  if (rc) goto done;

  {
    double c = 0.0;                                                           /* :126-133 */
    for (int mw = 1; mw <= mwaves; ++mw)
      for (int i = 1; i <= mx + 1; ++i) {
        double a = dtdx[i + mbc - 1] * L2(s, i, mw);
        double b = -dtdx[i + mbc - 2] * L2(s, i, mw);
        c = dmax1(c, dmax1(a, b));
      }
    *cfl = c;
  }

  if (p->tfluct_solver == 1) {                                                /* :136-153 */
    rc = ocl_tfluct(p, ixy, mx, ql, qr, aux1d, aux1d, s, amdq2);
    if (rc) goto done;
    for (int m = 1; m <= meqn; ++m)
      for (int i = 1; i <= mx; ++i)
        L2(dq1d, i, m) = L2(dq1d, i, m) -
            dtdx[i + mbc - 1] * ((L2(apdq, i, m) + L2(amdq2, i, m)) + L2(amdq, i + 1, m));
  } else {                                                                    /* :155-188 */
    for (int i = 1 - mbc + 1; i <= mx + mbc; ++i)
      for (int m = 1; m <= meqn; ++m) {
        L2(qr, i - 1, m) = L2(ql, i, m);
        L2(ql, i, m) = L2(qr, i, m);
      }
    if (maux > 0)
      for (int i = 1 - mbc + 1; i <= mx + mbc; ++i)
        for (int m = 1; m <= maux; ++m) {
          L2(auxr, i - 1, m) = L2(aux1d, i, m);
          L2(auxl, i, m) = L2(aux1d, i, m);
        }
    rc = ocl_rp(p, ixy, mx, ql, qr, auxl, auxr, wave, s, amdq2, apdq2);
    if (rc) goto done;
    for (int m = 1; m <= meqn; ++m)
      for (int i = 1; i <= mx; ++i)
        L2(dq1d, i, m) = L2(dq1d, i, m) -
            dtdx[i + mbc - 1] * (((L2(amdq, i + 1, m) + L2(apdq, i, m)) + L2(amdq2, i, m)) + L2(apdq2, i, m));
  }
done:
  free(dtdx); free(ql); free(qr); free(wave); free(s); free(amdq); free(apdq);
  free(amdq2); free(apdq2); free(evl); free(evr); free(auxl); free(auxr);
  return rc;
}

/* ======================================================================== */
/* src/2d/flux2.f90:30-92                                                    */
/* ======================================================================== */
static int flux2(const ocl_params *p, const double *q, double *dq, const double *aux,
                 double dt, double *cfl) {
  const int mbc = p->mbc, nx = p->mx, ny = p->my, meqn = p->meqn, maux = p->maux;
  const long ldx = nx + 2 * mbc, ldy = ny + 2 * mbc;
  const long lmax = (ldx > ldy ? ldx : ldy);
  double *q1d = (double *)calloc((size_t)lmax * meqn, sizeof(double));
  double *dq1d = (double *)calloc((size_t)lmax * meqn, sizeof(double));
  double *a1d = (double *)calloc((size_t)lmax * (maux > 0 ? maux : 1), sizeof(double));
  int rc = 0;
  if (!q1d || !dq1d || !a1d) { rc = -3; goto out; }
  *cfl = 0.0;
  for (int j = 0; j <= ny + 1; ++j) {                                          /* :36-62 */
    for (int m = 1; m <= meqn; ++m)
      for (int i = 1 - mbc; i <= nx + mbc; ++i) q1d[(i + mbc - 1) + (m - 1) * ldx] = G3(q, i, j, m);
    for (int m = 1; m <= maux; ++m)
      for (int i = 1 - mbc; i <= nx + mbc; ++i) a1d[(i + mbc - 1) + (m - 1) * ldx] = G3(aux, i, j, m);
    double c1d;
    rc = ocl_flux1(p, q1d, dq1d, a1d, dt, &c1d, 1, nx);
    if (rc) goto out;
    *cfl = dmax1(*cfl, c1d);
    for (int m = 1; m <= meqn; ++m)
      for (int i = 1; i <= nx; ++i) G3(dq, i, j, m) = G3(dq, i, j, m) + dq1d[(i + mbc - 1) + (m - 1) * ldx];
  }
  for (int i = 0; i <= nx + 1; ++i) {                                          /* :68-92 */
    for (int m = 1; m <= meqn; ++m)
      for (int j = 1 - mbc; j <= ny + mbc; ++j) q1d[(j + mbc - 1) + (m - 1) * ldy] = G3(q, i, j, m);
    for (int m = 1; m <= maux; ++m)
      for (int j = 1 - mbc; j <= ny + mbc; ++j) a1d[(j + mbc - 1) + (m - 1) * ldy] = G3(aux, i, j, m);
    double c1d;
    rc = ocl_flux1(p, q1d, dq1d, a1d, dt, &c1d, 2, ny);
    if (rc) goto out;
    *cfl = dmax1(*cfl, c1d);
    for (int m = 1; m <= meqn; ++m)
      for (int j = 1; j <= ny; ++j) G3(dq, i, j, m) = G3(dq, i, j, m) + dq1d[(j + mbc - 1) + (m - 1) * ldy];
  }
out:
  free(q1d); free(dq1d); free(a1d);
  return rc;
}

/* The app's src(q,dq,aux,t,dt) on a 1-D grid: dq(i,:) for i = 1..mx.
 *   OCL_SRC_RADIAL_SW     apps/shallowWater/2dRadialDam/1dRadialSymm-qwave/src1.f90:24-28
 *   OCL_SRC_BATHYMETRY_SW apps/shallowWater/1dPerturbSteady/src1.f90:31-34 */
static void src1(const ocl_params *p, const double *q, double *dq, const double *aux, double dt) {
  const int mbc = p->mbc, mx = p->mx;
  const long ld = mx + 2 * mbc;
  for (int i = 1; i <= mx; ++i) {
    if (p->src_term == OCL_SRC_RADIAL_SW) {
      double rad_pos = p->xlower + ((double)i - 0.5) * p->dx;
      L2(dq, i, 1) = -(((1.0 * dt) * L2(q, i, 2)) / rad_pos);
      L2(dq, i, 2) = -((((1.0 * dt) * (L2(q, i, 2) * L2(q, i, 2))) / L2(q, i, 1)) / rad_pos);
    } else if (p->src_term == OCL_SRC_BATHYMETRY_SW) {
      L2(dq, i, 1) = 0.0;
      L2(dq, i, 2) = -(((((1.0 * p->grav) * L2(q, i, 1)) * (L2(aux, i, 1) - L2(aux, i - 1, 1))) / p->dx) * dt);
    }
  }
}

/* src/1d/step1d.f90:2-31, src/2d/step2d.f90:2-41 (with src1/src2 zeroing,
 * or the app's 1-D source hook) */
static int step_st(ocl_params *p, double *q, double *dq, double *aux, double dt, double t,
                   double *cfl) {
  int rc = (p->ndim == 1 && p->bc_user) ? bc1_user(p, q, aux, t) : ocl_bc(p, q);
  if (rc) return rc;
  const long n = ocl_plane(p) * p->meqn;
  for (long k = 0; k < n; ++k) dq[k] = 0.0;   /* src: interior zeroed; ghosts unused */
  if (p->ndim == 1 && p->src_term != OCL_SRC_NONE) {
    if (p->meqn != 2) return -5;
    if (p->src_term == OCL_SRC_BATHYMETRY_SW && p->maux < 1) return -5;
    if (p->src_term != OCL_SRC_RADIAL_SW && p->src_term != OCL_SRC_BATHYMETRY_SW) return -5;
    src1(p, q, dq, aux, dt);
  }
  if (p->ndim == 1) return ocl_flux1(p, q, dq, aux, dt, cfl, 1, p->mx);
  return flux2(p, q, dq, aux, dt, cfl);
}

/* a working copy of aux for the user bc, which rewrites aux ghost cells */
static double *aux_copy(const ocl_params *p, const double *aux) {
  if (!p->bc_user || !aux) return NULL;
  const size_t na = (size_t)ocl_plane(p) * (size_t)(p->maux > 0 ? p->maux : 1);
  double *w = (double *)malloc(sizeof(double) * na);
  if (w) memcpy(w, aux, sizeof(double) * na);
  return w;
}

int ocl_step(const ocl_params *p, double *q, double *dq, const double *aux, double dt,
             double t, double *cfl) {
  ocl_params pl = *p;
  double *auxw = aux_copy(p, aux);
  if (p->bc_user && aux && !auxw) return -3;
  int rc = step_st(&pl, q, dq, auxw ? auxw : (double *)aux, dt, t, cfl);
  free(auxw);
  return rc;
}

/* ======================================================================== */
/* SSP-RK stages, src/sharpclaw.f90:247-464 (whole-array updates).           */
/* ======================================================================== */
static int rk_step_st(ocl_params *p, int ti, double *q, const double *qold, double *aux, double dt,
                      double told, double *cfl) {
  const long n = ocl_plane(p) * p->meqn;
  double *r1 = (double *)calloc((size_t)n, sizeof(double));
  double *r2 = (ti == 4) ? (double *)calloc((size_t)n, sizeof(double)) : NULL;
  int rc = 0;
  if (!r1 || (ti == 4 && !r2)) { free(r1); free(r2); return -3; }
#define STEP(dst, tt) do { rc = step_st(p, q, (dst), aux, dt, (tt), cfl); if (rc) goto out; } while (0)
  if (ti == 1) {                                           /* ts_ssp22 :247-276 */
    const double c2 = 1.0;
    STEP(r1, told);
    for (long k = 0; k < n; ++k) q[k] = q[k] + r1[k];
    STEP(r1, told + c2 * dt);
    for (long k = 0; k < n; ++k) q[k] = 0.5 * ((qold[k] + q[k]) + r1[k]);
  } else if (ti == 2) {                                    /* ts_ssp42 :280-333 */
    const double third = 1.0 / 3.0, a21 = third, b4 = 0.25;
    STEP(r1, told);
    for (long k = 0; k < n; ++k) q[k] = q[k] + a21 * r1[k];
    STEP(r1, told + third * dt);
    for (long k = 0; k < n; ++k) q[k] = q[k] + third * r1[k];
    STEP(r1, told + (2.0 * third) * dt);
    for (long k = 0; k < n; ++k) q[k] = q[k] + third * r1[k];
    STEP(r1, told + 1.0 * dt);
    for (long k = 0; k < n; ++k) q[k] = (0.25 * qold[k] + 0.75 * q[k]) + b4 * r1[k];
  } else if (ti == 3) {                                    /* ts_ssp33 :337-376 */
    STEP(r1, told);
    for (long k = 0; k < n; ++k) q[k] = q[k] + r1[k];
    STEP(r1, told + 1.0 * dt);
    for (long k = 0; k < n; ++k) q[k] = 0.75 * qold[k] + 0.25 * (q[k] + r1[k]);
    STEP(r1, told + 0.5 * dt);
    for (long k = 0; k < n; ++k) q[k] = (qold[k] + 2.0 * (q[k] + r1[k])) / 3.0;
  } else if (ti == 4) {                                    /* ts_ssp104 :380-464 */
    const double c6 = 1.0 / 6.0;
    double that = told;
    STEP(r1, that);
    for (long k = 0; k < n; ++k) q[k] = q[k] + c6 * r1[k];
    that = told + dt / 6.0;
    STEP(r1, that);
    for (long k = 0; k < n; ++k) q[k] = q[k] + c6 * r1[k];
    that = told + dt / 3.0;
    STEP(r1, that);
    for (long k = 0; k < n; ++k) q[k] = q[k] + c6 * r1[k];
    that = told + 0.5 * dt;
    STEP(r1, that);
    for (long k = 0; k < n; ++k) q[k] = q[k] + c6 * r1[k];
    that = told + (2.0 / 3.0) * dt;
    STEP(r1, that);
    for (long k = 0; k < n; ++k) {
      r2[k] = q[k] + c6 * r1[k];
      r1[k] = 0.04 * qold[k] + 0.36 * r2[k];
      q[k] = 0.6 * qold[k] + 0.4 * r2[k];
    }
    that = told + (1.0 / 3.0) * dt;
    STEP(r2, that);
    for (long k = 0; k < n; ++k) q[k] = q[k] + c6 * r2[k];
    that = told + 0.5 * dt;
    STEP(r2, that);
    for (long k = 0; k < n; ++k) q[k] = q[k] + c6 * r2[k];
    that = told + (2.0 / 3.0) * dt;
    STEP(r2, that);
    for (long k = 0; k < n; ++k) q[k] = q[k] + c6 * r2[k];
    that = told + (5.0 / 6.0) * dt;
    STEP(r2, that);
    for (long k = 0; k < n; ++k) q[k] = q[k] + c6 * r2[k];
    that = told + dt;
    STEP(r2, that);
    for (long k = 0; k < n; ++k) q[k] = (r1[k] + 0.6 * q[k]) + 0.1 * r2[k];
  } else {
    rc = -6;
  }
#undef STEP
out:
  free(r1);
  free(r2);
  return rc;
}

int ocl_rk_step(const ocl_params *p, int ti, double *q, const double *qold,
                const double *aux, double dt, double told, double *cfl) {
  ocl_params pl = *p;
  double *auxw = aux_copy(p, aux);
  if (p->bc_user && aux && !auxw) return -3;
  int rc = rk_step_st(&pl, ti, q, qold, auxw ? auxw : (double *)aux, dt, told, cfl);
  free(auxw);
  return rc;
}

/* ======================================================================== */
/* src/sharpclaw.f90:2-243 driver                                            */
/* ======================================================================== */
/* apps/advection/2d/swirl/b4step.f90: aux = aux0 * cos(pi2 (time + dt/2) / tperiod),
   aux0 the stream-function velocities setaux.f computes (the app recomputes
   them each call; identical values) */
static void b4step_swirl(const ocl_params *p, const double *aux0, double *aux, long n, double time, double dt) {
  if (p->tperiod == 0.0) return;
  const double pi2 = 2.0 * (4.0 * atan(1.0));
  const double vt = cos(pi2 * (time + dt / 2.0) / p->tperiod);
  for (long k = 0; k < n; ++k) aux[k] = vt * aux0[k];
}

int ocl_sharpclaw(const ocl_params *p, const ocl_run *run, double *q, const double *aux_in,
                  ocl_result *res) {
  const long n = ocl_plane(p) * p->meqn;
  const long na = ocl_plane(p) * (p->maux > 0 ? p->maux : 1);
  double *auxw = NULL;          /* the hooks' working aux */
  const double *aux = aux_in;
  ocl_params pl = *p;           /* the user bc's switch state evolves */
  if ((p->b4step == 1 || p->bc_user) && aux_in) {
    auxw = (double *)malloc(sizeof(double) * (size_t)na);
    if (!auxw) return -3;
    memcpy(auxw, aux_in, sizeof(double) * (size_t)na);
    aux = auxw;
  }
  double tstart = run->tstart, tend = run->tend;
  double t = tstart, told = tstart, dt = run->dt_initial, cfl = 0.0, cflmax = 0.0;
  double dtmin = dt, dtmax = dt;
  int maxn = run->max_steps, info = 0, steps = 0, rejected = 0, retake = 0, rc = 0;
  memset(res, 0, sizeof(*res));
  if (run->dt_variable == 0) {                                                 /* :44-58 */
    if (tend < tstart) maxn = 1;
    else {
      maxn = (int)((tend - tstart + 1e-10) / dt);
      if (fabs(maxn * dt - (tend - tstart)) > 1e-5 * (tend - tstart)) { res->info = 2; free(auxw); return 0; }
    }
  }
  if (run->dt_variable == 1 && run->cfl_desired > run->cfl_max) { res->info = 3; free(auxw); return 0; }
  double *qold = (double *)malloc(sizeof(double) * (size_t)n);
  if (!qold) { free(auxw); return -3; }
  for (int it = 1; it <= maxn; ++it) {                                          /* :118-222 */
    if (!retake) {
      told = t;
      if (told + dt > tend && tstart < tend) dt = tend - told;
      if (auxw && p->b4step == 1) b4step_swirl(p, aux_in, auxw, na, told, dt);                 /* :129 */
      /* apps/elasticity/stegoton/b4step1.f:15-21 (1.e-10 is REAL(4)) */
      if (p->b4step == 2 && p->ndim == 1 && !pl.b4_done && told + (double)1.0e-10f >= p->trtime) {
        const long ld = p->mx + 2 * p->mbc;
        for (long i = 0; i < ld; ++i) q[ld + i] = -q[ld + i];
        pl.b4_done = 1;
      }
      memcpy(qold, q, sizeof(double) * (size_t)n);
    }
    retake = 0;
    t = told + dt;
    if (p->ndim == 1) {                                                        /* :153 */
      rc = pl.bc_user ? bc1_user(&pl, q, auxw, told) : ocl_bc(p, q);
      if (rc) break;
    }
    rc = rk_step_st(&pl, run->time_integrator, q, qold, (double *)aux, dt, told, &cfl);
    if (rc) break;
    if (run->dt_variable == 1) {                                               /* :184-192 */
      if (cfl > 0.0) {
        dt = dmin1(run->dt_max, dt * run->cfl_desired / cfl);
        dtmin = dmin1(dt, dtmin);
        dtmax = dmax1(dt, dtmax);
      } else {
        dt = run->dt_max;
      }
    }
    if (cfl <= run->cfl_max) {                                                 /* :195-216 */
      cflmax = dmax1(cfl, cflmax);
    } else {
      t = told;
      memcpy(q, qold, sizeof(double) * (size_t)n);
      ++rejected;
      if (run->dt_variable == 1) retake = 1;
      else { cflmax = dmax1(cfl, cflmax); break; }
    }
    steps = steps + 1;
    if (t >= tend) break;
  }
  free(qold);
  free(auxw);
  if (rc) return rc;
  if (run->dt_variable == 1 && t < tend && steps == maxn) info = 11;           /* :225 */
  if (run->dt_variable == 0 && cflmax > run->cfl_max) info = 12;               /* :228 */
  res->tend = t;
  res->cfl_maxused = cflmax;
  res->cfl_last = cfl;
  res->dt_minused = dtmin;
  res->dt_maxused = dtmax;
  res->dt_last = dt;
  res->steps_taken = steps;
  res->info = info;
  res->rejected = rejected;
  res->bc_switched = pl.bc_switched;
  return 0;
}

/* ======================================================================== */
/* src/1d/out1.f90 and src/2d/out2.f90: frame files fort.qNNNN/tNNNN/aNNNN  */
/* ======================================================================== */

/* Fortran Ew.d: [-]0.<d digits>E+xx (or +xxx), right-justified in w */
static void fmt_e(char *out, double v, int w, int d) {
  char body[64], dig[40], raw[64];
  int e = 0;
  if (v != v) { snprintf(body, sizeof body, "NaN"); }
  else if (isinf(v)) { snprintf(body, sizeof body, "%s", v < 0 ? "-Infinity" : "Infinity"); }
  else {
    if (v == 0.0) {
      memset(dig, '0', (size_t)d); dig[d] = 0;
    } else {
      int k = 0;
      snprintf(raw, sizeof raw, "%.*e", d - 1, fabs(v));
      for (const char *c = raw; *c && *c != 'e'; ++c) if (*c >= '0' && *c <= '9') dig[k++] = *c;
      dig[k] = 0;
      e = atoi(strchr(raw, 'e') + 1) + 1;
    }
    int ae = e < 0 ? -e : e;
    if (ae <= 99) snprintf(body, sizeof body, "%s0.%sE%c%02d", signbit(v) ? "-" : "", dig, e < 0 ? '-' : '+', ae);
    else snprintf(body, sizeof body, "%s0.%s%c%03d", signbit(v) ? "-" : "", dig, e < 0 ? '-' : '+', ae);
  }
  int n = (int)strlen(body);
  if (n > w) { memset(out, '*', (size_t)w); out[w] = 0; return; }
  memset(out, ' ', (size_t)(w - n));
  memcpy(out + (w - n), body, (size_t)n + 1);
}

static FILE *open_frame(const char *dir, char kind, int iframe) {
  char name[16], path[4096];
  int nstp = iframe;
  strcpy(name, "fort.xxxxx");
  name[5] = kind;                                   /* out1.f90:30-42 */
  for (int ipos = 10; ipos >= 7; --ipos) { name[ipos - 1] = (char)('0' + nstp % 10); nstp /= 10; }
  name[10] = 0;
  if (dir && dir[0]) snprintf(path, sizeof path, "%s/%s", dir, name);
  else snprintf(path, sizeof path, "%s", name);
  return fopen(path, "w");
}

static void write_grid(FILE *f, const ocl_params *p, const double *a, int ncomp, int nblank1d) {
  char b[64];
  const int mbc = p->mbc, mx = p->mx, my = p->ndim == 2 ? p->my : 1;
  const long ld = mx + 2 * mbc, plane = ld * (p->ndim == 2 ? my + 2 * mbc : 1);
  fprintf(f, "%5d                 grid_number\n%5d                 AMR_level\n%5d                 mx\n", 1, 1, mx);
  if (p->ndim == 2) {
    fprintf(f, "%5d                 my\n", my);
    fmt_e(b, p->xlower, 26, 16); fprintf(f, "%s    xlow\n", b);
    fmt_e(b, p->ylower, 26, 16); fprintf(f, "%s    ylow\n", b);
    fmt_e(b, p->dx, 26, 16); fprintf(f, "%s    dx\n", b);
    fmt_e(b, p->dy, 26, 16); fprintf(f, "%s    dy\n\n", b);
  } else {
    fmt_e(b, p->xlower, 18, 8); fprintf(f, "%s    xlow\n", b);
    fmt_e(b, p->dx, 18, 8); fprintf(f, "%s    dx\n\n", b);
  }
  const int w = p->ndim == 2 ? 26 : 16, d = p->ndim == 2 ? 16 : 8;
  for (int j = 1; j <= my; ++j) {
    for (int i = 1; i <= mx; ++i) {
      for (int m = 1; m <= ncomp; ++m) {
        long k = (i + mbc - 1) + (p->ndim == 2 ? (long)(j + mbc - 1) * ld : 0) + (long)(m - 1) * plane;
        double v = a[k];
        if (fabs(v) < 1e-99) v = 0.0;                 /* out1.f90:63-66 */
        fmt_e(b, v, w, d);
        fputs(b, f);
        if (m % 4 == 0 || m == ncomp) fputc('\n', f);  /* format (4ew.d) */
      }
    }
    if (p->ndim == 2) fputs("  \n", f);             /* out2.f90:68 */
  }
  for (int k = 0; k < (p->ndim == 2 ? 1 : nblank1d); ++k) fputs("  \n", f);
}

int ocl_output(const ocl_params *p, const double *q, const double *aux, double t, int iframe,
               const char *dir, int outaux) {
  FILE *fq = open_frame(dir, 'q', iframe), *ft = open_frame(dir, 't', iframe);
  if (!fq || !ft) { if (fq) fclose(fq); if (ft) fclose(ft); return -6; }
  write_grid(fq, p, q, p->meqn, 2);
  if (outaux && p->maux > 0 && aux) {
    FILE *fa = open_frame(dir, 'a', iframe);
    if (!fa) { fclose(fq); fclose(ft); return -6; }
    write_grid(fa, p, aux, p->maux, 1);
    fclose(fa);
  }
  char b[64];
  fmt_e(b, t, 26, 16);
  fprintf(ft, "%s    time\n%5d                 meqn\n%5d                 ngrids\n%5d                 maux\n"
              "%5d                 ndim\n\n\n", b, p->meqn, 1, p->maux, p->ndim);
  fclose(fq);
  fclose(ft);
  return 0;
}
