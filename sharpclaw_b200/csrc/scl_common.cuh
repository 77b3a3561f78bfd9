// scl_common.cuh -- shared device types for the SharpClaw B200 kernels.
//
// Layout in HBM: every field is a set of component planes ("structure of
// arrays"), exactly the column-major order of the reference
// (src/1d/qalloc1.f90:10, src/2d/qalloc2.f90:11) with the lower bound 1-mbc
// mapped to offset 0.  Rows are padded to `pitch` elements (a multiple of 32)
// so every row start is 256-byte aligned; a 2-D plane holds (my+2*mbc) rows.
#pragma once
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/sharpclaw_cuda.h"

namespace scl {

constexpr int MBC = 3;       // WENO5 needs three ghost cells (reconstruct.f90:85,158)
constexpr int MAXEQ = 3;     // largest meqn of the supported plugins
constexpr int MAXSTAGES = 10;

// Stage-update kinds: one per distinct Shu-Osher combination written in
// src/sharpclaw.f90 (ts_ssp22 247-276, ts_ssp42 280-333, ts_ssp33 337-376,
// ts_ssp104 380-464).  Each keeps the reference's evaluation order.
enum StageKind : int {
  SK_ADD = 0,        // q + dq                               ssp33 :356, ssp22 :264
  SK_SSP33_2 = 1,    // 0.75*qold + 0.25*(q + dq)            ssp33 :365
  SK_SSP33_3 = 2,    // (qold + 2*(q + dq))/3                ssp33 :374
  SK_ADD_SIXTH = 3,  // q + (1/6)*dq                         ssp104 :396 ...
  SK_SSP104_5 = 4,   // r2=q+dq/6; r1=.04qold+.36r2; q=.6qold+.4r2   ssp104 :424-426
  SK_SSP104_10 = 5,  // (r1 + 0.6*q) + 0.1*dq                ssp104 :462
  SK_SSP22_2 = 6,    // 0.5*((qold + q) + dq)                ssp22 :274
  SK_ADD_THIRD = 7,  // q + (1/3)*dq                         ssp42 :304,313,322
  SK_SSP42_4 = 8,    // (0.25*qold + 0.75*q) + 0.25*dq       ssp42 :331
  SK_DQ = 9          // write dq itself (step1d/step2d output, no combination)
};

// Buffer roles for the register rotation (no whole-array copies: the
// reference's qold=q (sharpclaw.f90:134) becomes "Q keeps q^n").
enum Role : int { ROLE_Q = 0, ROLE_A = 1, ROLE_B = 2, ROLE_R1 = 3, NROLES = 4 };

// One stage of an integrator: which roles it reads/writes and how it combines.
struct StageDesc {
  int kind;       // StageKind
  int in;         // role read with halo (the stage input q)
  int out;        // role written (new q, with ghost images)
  int out2;       // second output (SSP104 stage 5 writes r1), -1 if none
  int aux_in;     // pointwise extra input (qold role for most; r1 for SSP104 stage 10), -1 if none
};

// Device-resident controller state: the scalars of src/sharpclaw.f90:18-41 and
// the per-stage CFL numbers.  One per handle (or per batched instance).
struct __align__(16) Ctl {
  double t, told, dt, tstart, tend;
  double dt_max, cfl_max, cfl_desired;
  double cflmax, dtmin, dtmax, cfl_last;
  double stage_cfl[MAXSTAGES];  // written by the stage kernels (atomic max on bits)
  int role[NROLES];             // physical buffer index of each role
  int n_iter, maxn, steps_taken, rejected;
  int retake, done, info, dt_variable;
  int status;                   // OR of SCL_STATUS_* raised by kernels
  int accept_always;            // single-step mode (scl_rk_step): no dt update, always accept
  int fresh;                    // 1: the current step is a new one (b4step runs), 0: a retake
  int bc_switched;              // the user bc switched both sides to periodic (persistent)
  int b4_done;                  // the time-reversal b4step has fired (persistent)
  // conserved totals (scl_set_totals): per component, at the run's start, of
  // the accepted state, of the step's candidate, and the largest |tot - tot0|
  int totals;                   // 1: kept after every accepted step
  unsigned int tot_ticket;      // CTAs of the totals kernel that are done (self-resetting)
  double tot0[MAXEQ], tot[MAXEQ], tot_cand[MAXEQ], drift[MAXEQ];
};

// Physics constants of the plugins (COMMON blocks /comrp/, /param/).
struct Phys {
  double u;       // advection speed        apps/advection/1d/rp1.f:31
  double gamma;   // ratio of specific heats apps/euler/shockentropy/setprob.f:392
  double gamma1;  // gamma - 1
  double grav;    // gravity                apps/shallowWater/2dRadialDam/setprob.f90
  int efix;
  int mthlim[4];  // TVD limiters (ClawParams%mthlim)
  double cc, zz;  // homogeneous acoustics: sqrt(bulk/rho), cc*rho (apps/acoustics/1d/homogeneous/setprob.f)
};

// Host side: the constants setprob.f of apps/acoustics/1d/homogeneous derives
// from rho and bulk (cc = sqrt(bulk/rho), zz = cc*rho).
inline void set_acoustics_consts(const scl_params& p, Phys* ph) {
  ph->cc = 0.0;
  ph->zz = 0.0;
  if (p.rp == SCL_RP_ACOUSTICS_CONST && p.rho > 0 && p.bulk > 0) {
    ph->cc = std::sqrt(p.bulk / p.rho);
    ph->zz = ph->cc * p.rho;
  }
}

// Arguments of one stage launch (all by value; pointers are device pointers).
struct StageArgs {
  Ctl* ctl;
  void* buf[NROLES];        // physical buffers (storage type S), each meqn planes
  const void* aux;          // aux planes (storage type S), or nullptr
  double* dq_out;           // SK_DQ only: dt*L(q) in double, same layout
  StageDesc sd;
  int stage;                // stage index (slot in ctl->stage_cfl)
  int ixy;                  // normal direction of a 1-D line (flux1.f90 ixy)
  int mx, my;
  long pitch;               // row pitch (elements)
  long plane;               // elements per component plane
  double dx, dy;
  int mthbc[4];
  int mcapa;                // 1-based aux index of capacity, 0 if none
  Phys ph;
  int src_term;             // SCL_SRC_* (1-D single grids)
  double xlower;
  // user bc hook (SCL_BC_USER_*) and this stage's time: told + tc*dt (tform
  // 0), told + dt/tc (1), or tc itself (2), as sharpclaw.f90 writes `that`
  int bc_user, tform;
  double tc;
  double wall[6];
  // bulk-copy staging: the bound of each mbarrier wait (ns of device time; 0
  // means the default, 1 s) and extra bytes announced but never copied (0; a
  // failure-detection test sets 16 so that every wait runs out, see
  // scl_test_wait_timeout)
  unsigned long long wait_ns;
  unsigned int tx_extra;
};

// Arguments of a cluster-resident run of a 1-D grid (the whole controller
// loop in one launch): the stage arguments of stage 0 plus every stage's
// descriptor.
struct RunArgs {
  StageArgs st;
  StageDesc sd[MAXSTAGES];
  int nstages, final_role;
  int max_iters;            // controller iterations of one launch
  int totals;               // conserved totals are kept (Ctl::totals of the run)
};

// NaN-propagating maximum used for the CFL number: a NaN anywhere makes the
// block result NaN so the controller can flag a non-finite state.
template <class R>
__device__ __forceinline__ R nanmax(R a, R b) {
  return (b > a || b != b) ? b : a;
}

// The physical buffer of a role, buf[i] for a runtime i < NROLES, by selects:
// indexing a kernel parameter array with a runtime index makes the compiler
// copy the whole argument struct to local memory in every thread.
template <class T>
__device__ __forceinline__ T pick_buf(T const (&buf)[NROLES], int i) {
  static_assert(NROLES == 4, "pick_buf selects among four buffers");
  const T lo = i == 0 ? buf[0] : buf[1];
  const T hi = i == 2 ? buf[2] : buf[3];
  return i < 2 ? lo : hi;
}

// Atomic max of a non-negative double (or NaN) through its bit pattern:
// for +0.0 .. +inf and positive NaN, unsigned order equals value order.
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  if (!(v > 0.0) && v == v) return;  // +0/-0 never raise the max
  unsigned long long bits = __double_as_longlong(v);
  if (v != v) bits = 0x7ff8000000000000ULL;
  unsigned long long* p = reinterpret_cast<unsigned long long*>(addr);
  // Every tile of a smooth field carries nearly the same maximum, and one
  // atomic per tile on a single word serialises a large grid.  The slot only
  // grows during a launch, so a read that already shows >= bits makes the
  // atomic redundant; a stale read can only cost a redundant atomic.  A
  // volatile generic load (global or shared slot) bypasses L1.
  if (*reinterpret_cast<volatile unsigned long long*>(p) >= bits) return;
  atomicMax(p, bits);
}

template <class T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = nanmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Reciprocal of the FP32 forms: the hardware approximation (at most 1 ulp
// from the rounded reciprocal over the whole range; subnormal results flush
// to zero).  Every use is a scale factor (WENO stencil scaling and weight
// normalisation, Roe averages, 1/rho), so results stay within a few ulp of
// the correctly rounded ones, inside the rounding of those forms.
#ifndef SCL_FAST_RCP
#define SCL_FAST_RCP 1
#endif
__device__ __forceinline__ float rcp32(float x) {
#if SCL_FAST_RCP
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
#else
  return __frcp_rn(x);
#endif
}

}  // namespace scl
