// scl_adjoint.cu -- discrete adjoint of the WENO step for the linear-Riemann
// plugins (2-D variable-coefficient acoustics), periodic bc: the VJP of one
// stage operator (componentwise or characteristic-wise WENO5) and the
// SSPRK(3,3) combinations (the other integrators' are in scl_capi.cu).
//
// The forward operator of one stage is D(q) = dt*L(q) of flux2
// (src/2d/flux2.f90): per line, WENO5 edge values (reconstruct.f90:77-143),
// the interface Riemann solve and the cell-internal tfluct (linear in the
// jumps for these plugins), dq(c) = -dtdx*(apdq(c) + adq(c) + amdq(c+1)),
// summed over the x and y sweeps.  Its vector-Jacobian product, for a given
// adjoint lam of dq:
//   mu(c)  = Ap(c)^T(-dtdx lam(c)) + Am(c)^T(-dtdx lam(c-1))   (interface c)
//   nu(c)  = T(c)^T(-dtdx lam(c))                              (cell c)
//   G_r(c) = -mu(c+1) + nu(c)    (adjoint of qr(c))
//   G_l(c) =  mu(c)   - nu(c)    (adjoint of ql(c))
// and both edge values of cell c depend on q(c-2..c+2), so each cell forms a
// five-entry contribution v_c = J_qr(c)^T G_r(c) + J_ql(c)^T G_l(c) and
// grad(k) = sum_j v_{k+2-j}[j] is a gather (no atomics).  Riemann and tfluct
// Jacobians are taken column by column from the plugin itself (unit jumps).
// SSPRK(3,3) (sharpclaw.f90:337-376) is then run backwards:
//   l2 = 2/3 (l3 + D'(q2)^T l3),  l1 = 1/4 (l2 + D'(q1)^T l2),
//   l0 = 1/3 l3 + 3/4 l2 + l1 + D'(q0)^T l1.
// Everything here is FP64.
#include <cuda_runtime.h>

#include <string>

#include "scl_kernels.cuh"
#include "scl_launch.h"

using namespace scl;

namespace {

// Reverse mode of weno_side (scl_weno.cuh): given ubar, accumulate the
// adjoints of its four jump inputs.
__device__ __forceinline__ void weno_side_vjp(double dm2, double dm1, double d0, double dp1, double im,
                                              double ub, double& gm2, double& gm1, double& g0,
                                              double& gp1) {
  const double ep = epweno();
  double t1 = im * (dm2 - dm1), t2 = im * (dm1 - d0), t3 = im * (d0 - dp1);
  double x1 = dm2 - 3.0 * dm1, x2 = dm1 + d0, x3 = 3.0 * d0 - dp1;
  double b1 = 13.0 * t1 * t1 + 3.0 * x1 * x1;
  double b2 = 13.0 * t2 * t2 + 3.0 * x2 * x2;
  double b3 = 13.0 * t3 * t3 + 3.0 * x3 * x3;
  double e1 = ep + b1, e2 = ep + b2, e3 = ep + b3;
  double tau1 = e1 * e1, tau2 = e2 * e2, tau3 = e3 * e3;
  double s1 = tau2 * tau3, s2 = 6.0 * tau1 * tau3, s3 = 3.0 * tau1 * tau2;
  double S = s1 + s2 + s3;
  double w1 = s1 / S, w3 = s3 / S;
  // u = (w1*(t2-t1) + (0.5*w3 - 0.25)*(t3-t2)) / 3
  double u3 = ub / 3.0;
  double wb1 = u3 * (t2 - t1);
  double wb3 = u3 * 0.5 * (t3 - t2);
  double tb1 = -u3 * w1;
  double tb2 = u3 * (w1 - (0.5 * w3 - 0.25));
  double tb3 = u3 * (0.5 * w3 - 0.25);
  // w1 = s1/S, w3 = s3/S
  double iS = 1.0 / S, iS2 = iS * iS;
  double sb1 = wb1 * (s2 + s3) * iS2 - wb3 * s3 * iS2;
  double sb2 = -(wb1 * s1 + wb3 * s3) * iS2;
  double sb3 = -wb1 * s1 * iS2 + wb3 * (s1 + s2) * iS2;
  double taub1 = sb2 * 6.0 * tau3 + sb3 * 3.0 * tau2;
  double taub2 = sb1 * tau3 + sb3 * 3.0 * tau1;
  double taub3 = sb1 * tau2 + sb2 * 6.0 * tau1;
  double bb1 = taub1 * 2.0 * e1, bb2 = taub2 * 2.0 * e2, bb3 = taub3 * 2.0 * e3;
  tb1 += bb1 * 26.0 * t1;
  tb2 += bb2 * 26.0 * t2;
  tb3 += bb3 * 26.0 * t3;
  double xb1 = bb1 * 6.0 * x1, xb2 = bb2 * 6.0 * x2, xb3 = bb3 * 6.0 * x3;
  // t1 = im(dm2-dm1), t2 = im(dm1-d0), t3 = im(d0-dp1); x1 = dm2-3dm1, x2 = dm1+d0, x3 = 3d0-dp1
  gm2 += im * tb1 + xb1;
  gm1 += -im * tb1 + im * tb2 - 3.0 * xb1 + xb2;
  g0 += -im * tb2 + im * tb3 + xb2 + 3.0 * xb3;
  gp1 += -im * tb3 - xb3;
}

constexpr int TA = 128;   // cells per adjoint tile

// VJP of one sweep direction of D over tiles of lines.  q, lam, out: pitched
// planes (double); periodic wrap is applied to every index, so ghost cells of
// q are not read.  out (+)= D_dir'(q)^T lam on interior cells.  CD 0:
// componentwise weno5; CD 2: weno5_char, whose eigenvectors depend on aux
// only for these plugins (so the projection is linear): the adjoint of an
// edge value is taken to the fields with evr^T, through weno_side's reverse
// mode, and back to the component jumps with evl^T, with the eigenvectors of
// the interface that reconstructs it (c+1 for qr(c), c for ql(c)).
template <class P, int CD>
__global__ void __launch_bounds__(TA) k_vjp_sweep(const double* q, const double* lam, const double* aux,
                                                   double* out, long pitch, long plane, int nx, int ny,
                                                   int dir, double dtdx, Phys ph, int accumulate) {
  constexpr int M = P::MEQN, MW = P::MWAVES, MA = P::MAUX;
  __shared__ double sq[M][TA + 8];        // cells i0-4 .. i0+TA+3
  __shared__ double sl[M][TA + 6];        // lam at cells i0-3 .. i0+TA+2
  __shared__ double sa[MA > 0 ? MA : 1][TA + 6];
  __shared__ double mu[M][TA + 5];        // interfaces i0-2 .. i0+TA+2
  __shared__ double vc[M][5][TA + 4];     // contributions of cells i0-2 .. i0+TA+1
  const int n = dir == 1 ? nx : ny;       // cells along the line
  const int line = blockIdx.y;            // row j (dir 1) or column i (dir 2), 1-based = line+1
  const int i0 = 1 + blockIdx.x * TA;
  const int tid = threadIdx.x;
  auto wrap = [&](int c) { int r = (c - 1) % n; if (r < 0) r += n; return r + 1; };
  auto off = [&](int c) -> long {          // element offset of cell c of this line
    const int w = wrap(c);
    return dir == 1 ? (long)(line + 3) * pitch + (w + 2) : (long)(w + 2) * pitch + (line + 3);
  };
  for (int k = tid; k < TA + 8; k += TA) {
    const long o = off(i0 - 4 + k);
#pragma unroll
    for (int m = 0; m < M; ++m) sq[m][k] = q[(long)m * plane + o];
  }
  for (int k = tid; k < TA + 6; k += TA) {
    const long o = off(i0 - 3 + k);
#pragma unroll
    for (int m = 0; m < M; ++m) sl[m][k] = lam[(long)m * plane + o];
#pragma unroll
    for (int a = 0; a < MA; ++a) sa[a][k] = aux[(long)a * plane + o];
  }
  __syncthreads();
  // mu at interfaces c = i0-2+k, k = 0..TA+4: needs lam(c-1), lam(c), aux(c-1), aux(c)
  for (int k = tid; k < TA + 5; k += TA) {
    const int kl = k;        // sl index of cell c-1 = (c-1) - (i0-3) = k
    double auxm[MA > 0 ? MA : 1], aux0[MA > 0 ? MA : 1];
#pragma unroll
    for (int a = 0; a < MA; ++a) { auxm[a] = sa[a][kl]; aux0[a] = sa[a][kl + 1]; }
    double r[M];
#pragma unroll
    for (int m = 0; m < M; ++m) r[m] = 0.0;
#pragma unroll
    for (int e = 0; e < M; ++e) {
      double z[M], dl[M], s[MW], am[M], ap[M];
#pragma unroll
      for (int m = 0; m < M; ++m) { z[m] = 0.0; dl[m] = (m == e) ? 1.0 : 0.0; }
      P::template rp<double>(ph, dir, z, z, dl, auxm, aux0, s, am, ap);
      double acc = 0.0;
#pragma unroll
      for (int m = 0; m < M; ++m) acc += ap[m] * (-dtdx * sl[m][kl + 1]) + am[m] * (-dtdx * sl[m][kl]);
      r[e] = acc;
    }
#pragma unroll
    for (int m = 0; m < M; ++m) mu[m][k] = r[m];
  }
  __syncthreads();
  // cells c = i0-2+k, k = 0..TA+3: G_r, G_l and the WENO VJP contributions
  for (int k = tid; k < TA + 4; k += TA) {
    const int kl = k + 1;    // sl index of cell c
    double auxc[MA > 0 ? MA : 1];
#pragma unroll
    for (int a = 0; a < MA; ++a) auxc[a] = sa[a][kl];
    double nu[M];
#pragma unroll
    for (int e = 0; e < M; ++e) {
      double z[M], dl[M], adq[M];
#pragma unroll
      for (int m = 0; m < M; ++m) { z[m] = 0.0; dl[m] = (m == e) ? 1.0 : 0.0; }
      P::template tfluct<double>(ph, dir, z, z, dl, auxc, adq);
      double acc = 0.0;
#pragma unroll
      for (int m = 0; m < M; ++m) acc += adq[m] * (-dtdx * sl[m][kl]);
      nu[e] = acc;
    }
    const int kq = k + 2;    // sq index of cell c
    if constexpr (CD == 2) {
      double Gr[M], Gl[M], D[M][4], gD[M][4];
#pragma unroll
      for (int m = 0; m < M; ++m) {
        Gr[m] = -mu[m][k + 1] + nu[m];
        Gl[m] = mu[m][k] - nu[m];
#pragma unroll
        for (int j = 0; j < 4; ++j) { D[m][j] = sq[m][kq - 1 + j] - sq[m][kq - 2 + j]; gD[m][j] = 0.0; }
      }
      // eigenvectors of interface c (cells c-1, c) and c+1 (cells c, c+1)
      double am1[MA > 0 ? MA : 1], a0[MA > 0 ? MA : 1], ap1[MA > 0 ? MA : 1], z[M];
#pragma unroll
      for (int a = 0; a < MA; ++a) { am1[a] = sa[a][kl - 1]; a0[a] = sa[a][kl]; ap1[a] = sa[a][kl + 1]; }
#pragma unroll
      for (int m = 0; m < M; ++m) z[m] = 0.0;
      double evlL[M][M], evrL[M][M], evlR[M][M], evrR[M][M];
      P::template evec<double>(ph, dir, z, z, am1, a0, evlL, evrL);
      P::template evec<double>(ph, dir, z, z, a0, ap1, evlR, evrR);
#pragma unroll
      for (int pf = 0; pf < M; ++pf) {
        double g1 = 0.0, g2 = 0.0, h1[4], h2[4], gh1[4] = {0.0, 0.0, 0.0, 0.0}, gh2[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int m = 0; m < M; ++m) { g1 += evrR[m][pf] * Gr[m]; g2 += evrL[m][pf] * Gl[m]; }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          double s1 = 0.0, s2 = 0.0;
#pragma unroll
          for (int m = 0; m < M; ++m) { s1 = s1 + evlR[pf][m] * D[m][j]; s2 = s2 + evlL[pf][m] * D[m][j]; }
          h1[j] = s1;
          h2[j] = s2;
        }
        weno_side_vjp(h1[0], h1[1], h1[2], h1[3], 1.0, g1, gh1[0], gh1[1], gh1[2], gh1[3]);
        weno_side_vjp(h2[3], h2[2], h2[1], h2[0], -1.0, g2, gh2[3], gh2[2], gh2[1], gh2[0]);
#pragma unroll
        for (int m = 0; m < M; ++m)
#pragma unroll
          for (int j = 0; j < 4; ++j) gD[m][j] += evlR[pf][m] * gh1[j] + evlL[pf][m] * gh2[j];
      }
#pragma unroll
      for (int m = 0; m < M; ++m) {
        double v[5];
        v[0] = -Gl[m] / 12.0;
        v[1] = -Gr[m] / 12.0 + 7.0 * Gl[m] / 12.0;
        v[2] = 7.0 * Gr[m] / 12.0 + 7.0 * Gl[m] / 12.0;
        v[3] = 7.0 * Gr[m] / 12.0 - Gl[m] / 12.0;
        v[4] = -Gr[m] / 12.0;
#pragma unroll
        for (int j = 0; j < 4; ++j) { v[j + 1] += gD[m][j]; v[j] -= gD[m][j]; }
#pragma unroll
        for (int j = 0; j < 5; ++j) vc[m][j][k] = v[j];
      }
      continue;
    }
#pragma unroll
    for (int m = 0; m < M; ++m) {
      const double Gr = -mu[m][k + 1] + nu[m];   // interface c+1 is mu index k+1
      const double Gl = mu[m][k] - nu[m];
      double qv[5];
#pragma unroll
      for (int j = 0; j < 5; ++j) qv[j] = sq[m][kq - 2 + j];
      double D[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) D[j] = qv[j + 1] - qv[j];
      double gD[4] = {0.0, 0.0, 0.0, 0.0};
      // qr(c) = side 1 on (D0,D1,D2,D3) + (-q(c-1) + 7q(c) + 7q(c+1) - q(c+2))/12
      weno_side_vjp(D[0], D[1], D[2], D[3], 1.0, Gr, gD[0], gD[1], gD[2], gD[3]);
      // ql(c) = side 2 on (D3,D2,D1,D0) + (-q(c-2) + 7q(c-1) + 7q(c) - q(c+1))/12
      weno_side_vjp(D[3], D[2], D[1], D[0], -1.0, Gl, gD[3], gD[2], gD[1], gD[0]);
      double v[5];
      v[0] = -Gl / 12.0;
      v[1] = -Gr / 12.0 + 7.0 * Gl / 12.0;
      v[2] = 7.0 * Gr / 12.0 + 7.0 * Gl / 12.0;
      v[3] = 7.0 * Gr / 12.0 - Gl / 12.0;
      v[4] = -Gr / 12.0;
#pragma unroll
      for (int j = 0; j < 4; ++j) { v[j + 1] += gD[j]; v[j] -= gD[j]; }
#pragma unroll
      for (int j = 0; j < 5; ++j) vc[m][j][k] = v[j];
    }
  }
  __syncthreads();
  // grad(c) for c = i0+t: sum_j v_{c+2-j}[j]; v index of cell c' is c' - (i0-2)
  const int c = i0 + tid;
  if (c <= n) {
    const long o = off(c);
#pragma unroll
    for (int m = 0; m < M; ++m) {
      double g = 0.0;
#pragma unroll
      for (int j = 0; j < 5; ++j) g += vc[m][j][tid + 4 - j];
      double* dst = out + (long)m * plane + o;
      *dst = accumulate ? *dst + g : g;
    }
  }
}

// elementwise combinations of the SSPRK(3,3) adjoint on interior cells
__global__ void k_adj_combine(int mode, double* a, const double* b, const double* c, long n) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x) {
    switch (mode) {
      case 0: a[k] = (2.0 / 3.0) * (b[k] + c[k]); break;                 // l2 = 2/3 (l3 + D2'l3)
      case 1: a[k] = 0.25 * (b[k] + c[k]); break;                        // l1 = 1/4 (l2 + D1'l2)
      default: break;
    }
  }
}

// l0 = 1/3 l3 + 3/4 l2 + l1 + D0'(l1)
__global__ void k_adj_final(double* l0, const double* l3, const double* l2, const double* l1, const double* t,
                            long n) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
    l0[k] = (1.0 / 3.0) * l3[k] + 0.75 * l2[k] + l1[k] + t[k];
}

// out = a x + b y (SSPRK(10,4) forward states and adjoint combinations)
__global__ void k_axpby(double* out, double a, const double* x, double b, const double* y, long n) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
    out[k] = a * x[k] + b * y[k];
}

}  // namespace

namespace scl {

bool adjoint_supported(int rp, int ndim, int cd, int ti, const int* mthbc) {
  if ((cd != 0 && cd != 2) || ti < 1 || ti > 4) return false;
  if (rp == SCL_RP_ACOUSTICS1D && ndim == 1) return mthbc[0] == 2 && mthbc[1] == 2;
  if (rp != SCL_RP_ACOUSTICS2D || ndim != 2) return false;
  for (int k = 0; k < 4; ++k) if (mthbc[k] != 2) return false;
  return true;
}

// out = D'(q)^T lam summed over both sweeps (q, lam, out pitched planes)
void launch_vjp2d(const double* q, const double* lam, const double* aux, double* out, long pitch, long plane,
                  int nx, int ny, double dx, double dy, double dt, const Phys& ph, int cd, cudaStream_t st,
                  int ndim) {
  if (ndim == 1) {
    // one line (apps/acoustics/1d/interface): row offset 0, so pitch 0
    using P1 = PAcoustics<2>;
    dim3 g((nx + TA - 1) / TA, 1);
    if (cd == 2) k_vjp_sweep<P1, 2><<<g, TA, 0, st>>>(q, lam, aux, out, 0, plane, nx, 1, 1, dt / dx, ph, 0);
    else k_vjp_sweep<P1, 0><<<g, TA, 0, st>>>(q, lam, aux, out, 0, plane, nx, 1, 1, dt / dx, ph, 0);
    return;
  }
  using P = PAcoustics<3>;
  dim3 gx((nx + TA - 1) / TA, ny), gy((ny + TA - 1) / TA, nx);
  if (cd == 2) {
    k_vjp_sweep<P, 2><<<gx, TA, 0, st>>>(q, lam, aux, out, pitch, plane, nx, ny, 1, dt / dx, ph, 0);
    k_vjp_sweep<P, 2><<<gy, TA, 0, st>>>(q, lam, aux, out, pitch, plane, nx, ny, 2, dt / dy, ph, 1);
  } else {
    k_vjp_sweep<P, 0><<<gx, TA, 0, st>>>(q, lam, aux, out, pitch, plane, nx, ny, 1, dt / dx, ph, 0);
    k_vjp_sweep<P, 0><<<gy, TA, 0, st>>>(q, lam, aux, out, pitch, plane, nx, ny, 2, dt / dy, ph, 1);
  }
}

void launch_adj_combine(int mode, double* a, const double* b, const double* c, long n, cudaStream_t st) {
  k_adj_combine<<<592, 256, 0, st>>>(mode, a, b, c, n);
}

void launch_adj_final(double* l0, const double* l3, const double* l2, const double* l1, const double* t, long n,
                      cudaStream_t st) {
  k_adj_final<<<592, 256, 0, st>>>(l0, l3, l2, l1, t, n);
}

void launch_axpby(double* out, double a, const double* x, double b, const double* y, long n, cudaStream_t st) {
  k_axpby<<<592, 256, 0, st>>>(out, a, x, b, y, n);
}

}  // namespace scl
