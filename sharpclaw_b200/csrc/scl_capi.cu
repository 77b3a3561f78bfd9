// scl_capi.cu -- C ABI of the SharpClaw B200 step (include/sharpclaw_cuda.h).
//
// Host side of the drop-in boundary: handle lifetime, the device layout,
// host<->device transfers, the integrator stage tables of src/sharpclaw.f90
// and the device-resident time loop (controller kernels + CUDA graphs).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "scl_common.cuh"
#include "scl_ctl.cuh"
#include "scl_frames.h"
#include "scl_launch.h"
#include "scl_totals.cuh"

using namespace scl;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define CK(call)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return fail(SCL_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
  } while (0)

// Controller kernels: one thread each (the logic is in scl_ctl.cuh).
__global__ void k_begin_step(Ctl* c) { ctl_begin(c); }
__global__ void k_end_step(Ctl* c, int last_stage, int final_role) { ctl_end(c, last_stage, final_role); }
// the end of one step and the begin of the next in one launch (inside a graph)
__global__ void k_end_begin(Ctl* c, int last_stage, int final_role) {
  ctl_end(c, last_stage, final_role);
  ctl_begin(c);
}

// b4step of apps/advection/2d/swirl/b4step.f90 on the device: before a new
// step, aux = aux0 * cos(2 pi (told + dt/2) / tperiod) over every cell,
// ghost cells included (the app rebuilds aux0 from its stream function).
template <class S>
__global__ void k_b4step_swirl(const Ctl* c, S* aux, const S* aux0, long n, double tperiod) {
  if (c->done || !c->fresh || tperiod == 0.0) return;
  const double pi2 = 2.0 * 3.141592653589793;                       // setprob.f: 2*(4*datan(1))
  const double vt = cos(pi2 * (c->told + c->dt / 2.0) / tperiod);
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
    aux[k] = (S)(vt * (double)aux0[k]);
}

// bc1.f90 on device (initial fill after an upload); one thread per (m, ibc)
template <class S>
__global__ void k_bc1(S* q, long plane, int mx, int meqn, int bl, int br) {
  const int t = threadIdx.x;
  if (t >= meqn * 3) return;
  const int m = t / 3, ibc = t % 3 + 1;
  S* p = q + (long)m * plane;
  auto at = [&](int i) -> S& { return p[i + 2]; };
  if (bl == 1) at(1 - ibc) = at(1);
  else if (bl == 2) at(1 - ibc) = at(mx + 1 - ibc);
  else if (bl == 3) at(1 - ibc) = (m == 1) ? -at(ibc) : at(ibc);
  if (br == 1) at(mx + ibc) = at(mx);
  else if (br == 2) at(mx + ibc) = at(ibc);
  else if (br == 3) at(mx + ibc) = (m == 1) ? -at(mx + 1 - ibc) : at(mx + 1 - ibc);
}

// apps/elasticity/stegoton/b4step1.f: on a new step with told + 1e-10 >=
// trtime (1.e-10 is a REAL(4) literal), and only once (itrdone of
// /comtimereverse/), negate the momentum over every cell, ghosts included.
// One CTA: thread 0 decides, all flip, thread 0 records it.
template <class S>
__global__ void k_b4step_reverse(StageArgs a, int ld, double trtime) {
  Ctl* c = a.ctl;
  __shared__ int go;
  if (threadIdx.x == 0)
    go = !c->done && c->fresh && !c->b4_done && c->told + (double)1.0e-10f >= trtime;
  __syncthreads();
  if (!go) return;
  S* q = static_cast<S*>(pick_buf(a.buf, c->role[ROLE_Q])) + a.plane;   // component 2
  for (int i = threadIdx.x; i < ld; i += blockDim.x) q[i] = -q[i];
  if (threadIdx.x == 0) c->b4_done = 1;
}

// apps/elasticity/stegoton/bc1.f, g0: 1 + cos(pi s) on |s| < 1 (pi = 4 atan(1))
__device__ __forceinline__ double wall_g0(double s) {
  return fabs(s) < 1.0 ? 1.0 + cos(3.141592653589793 * s) : 0.0;
}

// The user bc of apps/elasticity/stegoton/bc1.f on the input of one stage, at
// the stage's time (step1d.f90:20 calls bc with it): the switch to periodic
// (bc1.f:31-35, remembered in ctl->bc_switched as bc1.f rewrites mthbc), the
// periodic ghosts of aux fields 1..3 when the left side is periodic
// (bc1.f:36-45), then each side.  One CTA; thread 0
// decides, then one thread per (m, ibc) writes q ghosts and one per (j, ibc)
// aux ghosts.  The moving wall's ghost momentum uses the density of the mirror
// cell, aux(ibc,1) (bc1.f:62 indexes aux with the unset loop variable i).
template <class S>
__global__ void k_bc_user1d(StageArgs a, int meqn, int maux) {
  Ctl* c = a.ctl;
  __shared__ int sw;
  __shared__ double vl, vr;
  if (c->done) return;
  if (threadIdx.x == 0) {
    const double told = c->told, dt = c->dt;
    const double t = a.tform == 0 ? told + a.tc * dt : a.tform == 1 ? told + dt / a.tc : a.tc;
    const double t1 = a.wall[0], a1 = a.wall[1], tw1 = a.wall[2];
    const double t2 = a.wall[3], a2 = a.wall[4], tw2 = a.wall[5];
    if (t > 5.0 * tw1 && t < 5.0 * tw1 + 1.0) c->bc_switched = 1;
    sw = c->bc_switched;
    vl = -(a1 * wall_g0((t - t1) / tw1));
    vr = a2 * wall_g0((t - t2) / tw2);
  }
  __syncthreads();
  S* q = static_cast<S*>(pick_buf(a.buf, c->role[a.sd.in]));
  S* aux = static_cast<S*>(const_cast<void*>(a.aux));
  const int mx = a.mx, k = threadIdx.x;
  const int bl = sw ? 2 : a.mthbc[0], br = sw ? 2 : a.mthbc[1];
  if (bl == 2 && k < 3 * (maux < 3 ? maux : 3)) {
    const int j = k / 3, ibc = k % 3 + 1;
    S* p = aux + (long)j * a.plane;
    p[1 - ibc + 2] = p[mx + 1 - ibc + 2];
    p[mx + ibc + 2] = p[ibc + 2];
  }
  if (k >= 3 * meqn) return;
  const int m = k / 3, ibc = k % 3 + 1;
  S* p = q + (long)m * a.plane;
  auto at = [&](int i) -> S& { return p[i + 2]; };
  auto rho = [&](int i) -> double { return (double)aux[i + 2]; };
  if (bl == 0) at(1 - ibc) = m == 1 ? (S)(2.0 * vl * rho(ibc) - (double)at(ibc)) : at(ibc);
  else if (bl == 1) at(1 - ibc) = at(1);
  else if (bl == 2) at(1 - ibc) = at(mx + 1 - ibc);
  else at(1 - ibc) = (m == 1) ? -at(ibc) : at(ibc);
  if (br == 0) at(mx + ibc) = m == 1 ? (S)(2.0 * vr * rho(mx + 1 - ibc) - (double)at(mx + 1 - ibc)) : at(mx + 1 - ibc);
  else if (br == 1) at(mx + ibc) = at(mx);
  else if (br == 2) at(mx + ibc) = at(ibc);
  else at(mx + ibc) = (m == 1) ? -at(mx + 1 - ibc) : at(mx + 1 - ibc);
}

// bc2.f90 x-sides (all rows j = 1-mbc..ny+mbc), then y-sides (all columns)
template <class S>
__global__ void k_bc2(S* q, long plane, long pitch, int nx, int ny, int meqn, int b0, int b1,
                      int ydir) {
  const int len = ydir ? nx + 6 : ny + 6;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= meqn * 3 * len) return;
  const int k = t % len, ibc = (t / len) % 3 + 1, m = t / (3 * len);
  S* p = q + (long)m * plane;
  const int n = ydir ? ny : nx;
  const int neg_m = ydir ? 2 : 1;
  auto at = [&](int c) -> S& {
    return ydir ? p[(long)(c + 2) * pitch + k] : p[(long)(k) * pitch + c + 2];
  };
  if (b0 == 1) at(1 - ibc) = at(1);
  else if (b0 == 2) at(1 - ibc) = at(n + 1 - ibc);
  else if (b0 == 3) at(1 - ibc) = (m == neg_m) ? -at(ibc) : at(ibc);
  if (b1 == 1) at(n + ibc) = at(n);
  else if (b1 == 2) at(n + ibc) = at(ibc);
  else if (b1 == 3) at(n + ibc) = (m == neg_m) ? -at(n + 1 - ibc) : at(n + 1 - ibc);
}

__global__ void k_f64_to_f32(const double* a, float* b, long n) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
    b[k] = (float)a[k];
}
__global__ void k_f32_to_f64(const float* a, double* b, long n) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < n; k += (long)gridDim.x * blockDim.x)
    b[k] = (double)a[k];
}

// Reconstruction code of the stage kernels' CD parameter: char_decomp for
// WENO5 (lim_type 2), 10 + char_decomp for TVD (lim_type 1), 20 +
// char_decomp for the unlimited polynomial (lim_type 0).
int recon_code(const scl_params& p) {
  return p.lim_type == 1 ? 10 + p.char_decomp : p.lim_type == 0 ? 20 + p.char_decomp : p.char_decomp;
}

bool get_launchers(int prec, int rp, int ndim, int cd, int tf, int variant, Launchers* L) {
  switch (prec) {
    case SCL_FP64: return get_launchers_fp64(rp, ndim, cd, tf, variant, L);
    case SCL_FP64_STRICT: return get_launchers_fp64s(rp, ndim, cd, tf, variant, L);
    case SCL_MIXED: return get_launchers_mixed(rp, ndim, cd, tf, variant, L);
    case SCL_FP32: return get_launchers_fp32(rp, ndim, cd, tf, variant, L);
  }
  return false;
}

// Stage tables of ts_ssp22/42/33/104 (src/sharpclaw.f90:247-464) with the
// register rotation; `final` is the role holding q^{n+1}.
int stage_table(int ti, StageDesc* sd, int* final_role) {
  auto S = [](int k, int in, int out, int out2, int ai) { return StageDesc{k, in, out, out2, ai}; };
  int n = 0;
  switch (ti) {
    case 1:
      sd[n++] = S(SK_ADD, ROLE_Q, ROLE_A, -1, -1);
      sd[n++] = S(SK_SSP22_2, ROLE_A, ROLE_B, -1, ROLE_Q);
      *final_role = ROLE_B;
      break;
    case 2:
      sd[n++] = S(SK_ADD_THIRD, ROLE_Q, ROLE_A, -1, -1);
      sd[n++] = S(SK_ADD_THIRD, ROLE_A, ROLE_B, -1, -1);
      sd[n++] = S(SK_ADD_THIRD, ROLE_B, ROLE_A, -1, -1);
      sd[n++] = S(SK_SSP42_4, ROLE_A, ROLE_B, -1, ROLE_Q);
      *final_role = ROLE_B;
      break;
    case 3:
      sd[n++] = S(SK_ADD, ROLE_Q, ROLE_A, -1, -1);
      sd[n++] = S(SK_SSP33_2, ROLE_A, ROLE_B, -1, ROLE_Q);
      sd[n++] = S(SK_SSP33_3, ROLE_B, ROLE_A, -1, ROLE_Q);
      *final_role = ROLE_A;
      break;
    case 4:
      sd[n++] = S(SK_ADD_SIXTH, ROLE_Q, ROLE_A, -1, -1);
      sd[n++] = S(SK_ADD_SIXTH, ROLE_A, ROLE_B, -1, -1);
      sd[n++] = S(SK_ADD_SIXTH, ROLE_B, ROLE_A, -1, -1);
      sd[n++] = S(SK_ADD_SIXTH, ROLE_A, ROLE_B, -1, -1);
      sd[n++] = S(SK_SSP104_5, ROLE_B, ROLE_A, ROLE_R1, ROLE_Q);
      sd[n++] = S(SK_ADD_SIXTH, ROLE_A, ROLE_B, -1, -1);
      sd[n++] = S(SK_ADD_SIXTH, ROLE_B, ROLE_A, -1, -1);
      sd[n++] = S(SK_ADD_SIXTH, ROLE_A, ROLE_B, -1, -1);
      sd[n++] = S(SK_ADD_SIXTH, ROLE_B, ROLE_A, -1, -1);
      sd[n++] = S(SK_SSP104_10, ROLE_A, ROLE_B, -1, ROLE_R1);
      *final_role = ROLE_B;
      break;
    default:
      return 0;
  }
  return n;
}

}  // namespace

static_assert(N2D_VARIANTS == SCL_TILE_SHAPES, "tile shape count of the C interface");

struct scl_handle {
  scl_params p{};
  int device = 0;
  cudaStream_t stream = nullptr;
  size_t ssize = 8;      // bytes per stored value
  long ld = 0;           // reference row length (mx+2mbc)
  long rows = 1;         // rows per plane (my+2mbc in 2-D)
  long pitch = 0;        // device row pitch (elements)
  long plane = 0;        // elements per component plane
  void* buf[NROLES] = {nullptr, nullptr, nullptr, nullptr};
  void* aux = nullptr;
  double* stage64 = nullptr;   // double staging (FP32 storage) and dq output
  Ctl* ctl = nullptr;          // device controller
  Ctl* hctl = nullptr;         // pinned host mirror
  int* hdone = nullptr;        // pinned flag
  Launchers L{};                    // launchers in use (LV[variant])
  Launchers LV[N2D_VARIANTS]{};     // every tile shape (LV[0] only in 1-D)
  int nvariants = 1;
  int variant = 0;
  int tiles_fixed = 0;              // 1: shape set by scl_select_tiles
  int tiles_tuned = 0;              // 1: shape chosen by timing
  float tile_ms[N2D_VARIANTS] = {0.f, 0.f, 0.f};
  StageDesc sd[MAXSTAGES];
  int nstages = 0, final_role = ROLE_A;
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t evq[2] = {nullptr, nullptr};
  double* adj = nullptr;       // adjoint work fields (5 x meqn planes), allocated on first use
  // frame output: pinned copy of the state, the copy's event, the writer thread
  double* fbuf = nullptr;
  size_t fbuf_n = 0;
  cudaEvent_t fev = nullptr;
  std::thread fthread;
  int frc = SCL_OK;
  std::string ferr;
  // b4step hook: kind, its constant, the base aux field it scales
  int b4kind = SCL_B4STEP_NONE;
  double b4param = 0.0;
  void* aux0 = nullptr;
  // time-loop mode (SCL_RUN_*) and what the last run used
  int run_mode = SCL_RUN_AUTO;
  int last_mode = SCL_RUN_AUTO;
  long long last_launches = 0;
  // conserved totals (scl_set_totals): on/off and the totals kernel's per-CTA partial sums
  int totals_on = 0;
  double* tot_partials = nullptr;
  // failure-detection test hook (scl_test_wait_timeout)
  int test_timeout = 0;
};

namespace {

// The time of stage s of integrator ti, `that` of sharpclaw.f90 in its
// written form: told + tc*dt (form 0) or told + dt/tc (form 1).
void stage_time_form(int ti, int s, int* form, double* tc) {
  *form = 0;
  *tc = 0.0;                                               // stage 1: told
  if (s == 0) return;
  if (ti == 1) { *tc = 1.0; return; }                      // :268 c2 = 1
  if (ti == 2) {                                           // :307-325
    const double third = 1.0 / 3.0;
    *tc = s == 1 ? third : s == 2 ? 2.0 * third : 1.0;
    return;
  }
  if (ti == 3) { *tc = s == 1 ? 1.0 : 0.5; return; }       // :359, :368
  static const double c104[10] = {0.0, 6.0, 3.0, 0.5, 2.0 / 3.0, 1.0 / 3.0, 0.5, 2.0 / 3.0, 5.0 / 6.0, 1.0};
  *tc = c104[s];                                           // :397-456
  *form = (s == 1 || s == 2) ? 1 : 0;                      // dt/6.d0, dt/3.d0
}

StageArgs make_args(const scl_handle* h, int s) {
  StageArgs a{};
  a.ctl = h->ctl;
  for (int r = 0; r < NROLES; ++r) a.buf[r] = h->buf[r];
  a.aux = h->aux;
  a.dq_out = h->stage64;
  a.sd = h->sd[s];
  a.stage = s;
  a.ixy = 1;
  a.mx = h->p.mx;
  a.my = h->p.ndim == 2 ? h->p.my : 1;
  a.pitch = h->pitch;
  a.plane = h->plane;
  a.dx = h->p.dx;
  a.dy = h->p.dy;
  for (int k = 0; k < 4; ++k) a.mthbc[k] = h->p.mthbc[k];
  a.mcapa = h->p.mcapa;
  a.src_term = h->p.src_term;
  a.xlower = h->p.xlower;
  a.ph.u = h->p.u;
  a.ph.gamma = h->p.gamma;
  a.ph.gamma1 = h->p.gamma - 1.0;
  a.ph.grav = h->p.grav;
  a.ph.efix = h->p.efix;
  for (int k = 0; k < 4; ++k) a.ph.mthlim[k] = h->p.mthlim[k];
  set_acoustics_consts(h->p, &a.ph);
  a.bc_user = h->p.bc_user;
  for (int k = 0; k < 6; ++k) a.wall[k] = h->p.wall[k];
  stage_time_form(h->p.time_integrator, s, &a.tform, &a.tc);
  // bulk-copy waits: the default bound, or under the test hook a 1 ms bound
  // and 16 bytes announced that no copy delivers
  a.wait_ns = h->test_timeout ? 1000000ull : 0ull;
  a.tx_extra = h->test_timeout ? 16u : 0u;
  return a;
}

// the user bc hook on the input of the stage `a` describes
void launch_bc_user(scl_handle* h, const StageArgs& a) {
  if (h->ssize == sizeof(double)) k_bc_user1d<double><<<1, 32, 0, h->stream>>>(a, h->p.meqn, h->p.maux);
  else k_bc_user1d<float><<<1, 32, 0, h->stream>>>(a, h->p.meqn, h->p.maux);
}

int upload_ctl(scl_handle* h) {
  CK(cudaMemcpyAsync(h->ctl, h->hctl, sizeof(Ctl), cudaMemcpyHostToDevice, h->stream));
  return SCL_OK;
}
int download_ctl(scl_handle* h) {
  CK(cudaMemcpyAsync(h->hctl, h->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return SCL_OK;
}

// CTAs of the totals kernel: at most four per SM (each takes the ticket with
// one same-address atomic, which serialise in L2), fewer for small grids
constexpr int TOT_BLOCKS = TOT_BLOCKS_MAX;

template <class S, bool CAP>
void launch_totals_m(int meqn, int nb, cudaStream_t st, const TotalsArgs& t) {
  if (meqn == 1) k_totals<S, 1, CAP><<<nb, TOT_NT, 0, st>>>(t);
  else if (meqn == 2) k_totals<S, 2, CAP><<<nb, TOT_NT, 0, st>>>(t);
  else k_totals<S, 3, CAP><<<nb, TOT_NT, 0, st>>>(t);
}

// Totals of the state in `role` (scl_totals.cuh): mode 0 -> the step's
// candidate (tot_cand), mode 1 -> the run's start (tot0 = tot, drift = 0).
void launch_totals(scl_handle* h, int role, int mode) {
  TotalsArgs t{};
  t.ctl = h->ctl;
  for (int r = 0; r < NROLES; ++r) t.buf[r] = h->buf[r];
  t.role = role;
  t.mode = mode;
  t.mx = h->p.mx;
  t.my = h->p.ndim == 2 ? h->p.my : 1;
  t.ndim = h->p.ndim;
  t.meqn = h->p.meqn;
  t.pitch = h->pitch;
  t.plane = h->plane;
  t.capa = h->p.mcapa > 0 ? static_cast<const char*>(h->aux) + h->ssize * h->plane * (h->p.mcapa - 1) : nullptr;
  t.area = h->p.ndim == 2 ? h->p.dx * h->p.dy : h->p.dx;
  t.partials = h->tot_partials;
  const long cells = (long)t.mx * t.my;
  long nb = (cells + (long)TOT_U * TOT_NT - 1) / ((long)TOT_U * TOT_NT);
  if (t.ndim == 2 && nb > t.my) nb = t.my;
  nb = std::max(1L, std::min(nb, (long)TOT_BLOCKS));
  const bool cap = t.capa != nullptr;
  if (h->ssize == sizeof(double)) {
    if (cap) launch_totals_m<double, true>(t.meqn, (int)nb, h->stream, t);
    else launch_totals_m<double, false>(t.meqn, (int)nb, h->stream, t);
  } else {
    if (cap) launch_totals_m<float, true>(t.meqn, (int)nb, h->stream, t);
    else launch_totals_m<float, false>(t.meqn, (int)nb, h->stream, t);
  }
}

// enqueue the stages of one RK step on the handle's stream
int enqueue_stages(scl_handle* h) {
  for (int s = 0; s < h->nstages; ++s) {
    StageArgs a = make_args(h, s);
    if (h->p.bc_user) launch_bc_user(h, a);
    h->L.stage(a, h->stream);
    if (h->L.ghost && s == h->nstages - 1) h->L.ghost(a, h->stream);
  }
  CK(cudaGetLastError());
  return SCL_OK;
}

// One controller step: begin (only for the first step of a sequence; later
// steps are begun by the previous step's k_end_begin), the b4step hook, the
// stages, end (last step) or end + the next begin.
int enqueue_step(scl_handle* h, bool first = true, bool last = true) {
  if (first) k_begin_step<<<1, 1, 0, h->stream>>>(h->ctl);
  if (h->b4kind == SCL_B4STEP_SWIRL) {
    const long n = h->plane * h->p.maux;
    if (h->ssize == sizeof(double))
      k_b4step_swirl<double><<<148, 256, 0, h->stream>>>(h->ctl, static_cast<double*>(h->aux),
                                                         static_cast<const double*>(h->aux0), n, h->b4param);
    else
      k_b4step_swirl<float><<<148, 256, 0, h->stream>>>(h->ctl, static_cast<float*>(h->aux),
                                                        static_cast<const float*>(h->aux0), n, h->b4param);
  } else if (h->b4kind == SCL_B4STEP_TIME_REVERSAL) {
    const StageArgs a = make_args(h, 0);
    if (h->ssize == sizeof(double)) k_b4step_reverse<double><<<1, 256, 0, h->stream>>>(a, (int)h->ld, h->b4param);
    else k_b4step_reverse<float><<<1, 256, 0, h->stream>>>(a, (int)h->ld, h->b4param);
  }
  int rc = enqueue_stages(h);
  if (rc) return rc;
  if (h->totals_on) launch_totals(h, h->final_role, 0);   // the candidate q^{n+1}; kept if accepted
  if (last) k_end_step<<<1, 1, 0, h->stream>>>(h->ctl, h->nstages - 1, h->final_role);
  else k_end_begin<<<1, 1, 0, h->stream>>>(h->ctl, h->nstages - 1, h->final_role);
  CK(cudaGetLastError());
  return SCL_OK;
}

// launches per step inside a graph (plus one begin per graph replay)
int kernels_per_step(const scl_handle* h) {
  return h->nstages * (h->p.bc_user ? 2 : 1) + 1 + (h->L.ghost ? 1 : 0) + (h->b4kind != SCL_B4STEP_NONE ? 1 : 0) +
         (h->totals_on ? 1 : 0);
}

// Capture `steps` controller steps (begin, stages, end) into one executable
// graph; rebuilt only when a different step count is asked for.
int build_graph(scl_handle* h, int steps) {
  if (h->graph && h->graph_steps == steps) return SCL_OK;
  if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
  h->graph_steps = steps;
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int rc = SCL_OK;
  for (int k = 0; k < steps && rc == SCL_OK; ++k) rc = enqueue_step(h, k == 0, k == steps - 1);
  cudaError_t e = cudaStreamEndCapture(h->stream, &g);
  if (rc) { if (g) cudaGraphDestroy(g); return rc; }
  if (e != cudaSuccess) return fail(SCL_E_CUDA, std::string("capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&h->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(SCL_E_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
  return SCL_OK;
}

int default_graph_steps(const scl_handle* h) { return std::max(1, 160 / kernels_per_step(h)); }

// Switch the stage launchers to tile shape v; a captured graph holds the old
// kernel, so it is dropped and rebuilt by the next run.
void use_variant(scl_handle* h, int v) {
  if (v == h->variant) return;
  h->variant = v;
  h->L = h->LV[v];
  if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
}

// Time the first RK stage of every 2-D tile shape on the current state and
// keep the fastest.  The trials run against a copy of the controller (ctl[1]),
// so the run's CFL record and status are untouched, and stage 0 writes only
// register A, which every step overwrites before reading.
int tune_tiles(scl_handle* h) {
  Ctl* trial = h->ctl + 1;
  CK(cudaMemcpyAsync(trial, h->ctl, sizeof(Ctl), cudaMemcpyDeviceToDevice, h->stream));
  StageArgs a = make_args(h, 0);
  a.ctl = trial;
  int best = 0;
  for (int v = 0; v < h->nvariants; ++v) {
    h->LV[v].stage(a, h->stream);  // warm-up (first launch of a kernel)
    CK(cudaEventRecord(h->ev0, h->stream));
    h->LV[v].stage(a, h->stream);
    CK(cudaEventRecord(h->ev1, h->stream));
    CK(cudaEventSynchronize(h->ev1));
    float one = 0.f;
    CK(cudaEventElapsedTime(&one, h->ev0, h->ev1));
    // about 2 ms of launches per shape, 3 to 50 of them
    const int reps = std::min(50, std::max(3, (int)(2.0f / std::max(one, 1e-3f))));
    CK(cudaEventRecord(h->ev0, h->stream));
    for (int r = 0; r < reps; ++r) h->LV[v].stage(a, h->stream);
    CK(cudaGetLastError());
    CK(cudaEventRecord(h->ev1, h->stream));
    CK(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    h->tile_ms[v] = ms / reps;
    if (h->tile_ms[v] < h->tile_ms[best]) best = v;
  }
  // near-ties keep shape 0, so that timing noise does not flip the choice
  // (in the FMA forms a different shape can change the last bits)
  if (!(h->tile_ms[best] < 0.98f * h->tile_ms[0])) best = 0;
  use_variant(h, best);
  h->tiles_tuned = 1;
  return SCL_OK;
}

template <class S>
void launch_bc(scl_handle* h, S* q) {
  const scl_params& p = h->p;
  if (p.ndim == 1) {
    k_bc1<S><<<1, 32, 0, h->stream>>>(q, h->plane, p.mx, p.meqn, p.mthbc[0], p.mthbc[1]);
  } else {
    int n = p.meqn * 3 * (p.my + 6);
    k_bc2<S><<<(n + 255) / 256, 256, 0, h->stream>>>(q, h->plane, h->pitch, p.mx, p.my, p.meqn,
                                                      p.mthbc[0], p.mthbc[1], 0);
    n = p.meqn * 3 * (p.mx + 6);
    k_bc2<S><<<(n + 255) / 256, 256, 0, h->stream>>>(q, h->plane, h->pitch, p.mx, p.my, p.meqn,
                                                      p.mthbc[2], p.mthbc[3], 1);
  }
}

// host (reference layout, double) -> device buffer (storage type, pitched)
int upload_field(scl_handle* h, void* dst, const double* src, int ncomp, bool from_device) {
  const cudaMemcpyKind kind = from_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const size_t w = sizeof(double) * h->ld;
  const size_t nrows = (size_t)h->rows * ncomp;
  if (h->ssize == sizeof(double)) {
    CK(cudaMemcpy2DAsync(dst, sizeof(double) * h->pitch, src, w, w, nrows, kind, h->stream));
  } else {
    CK(cudaMemcpy2DAsync(h->stage64, sizeof(double) * h->pitch, src, w, w, nrows, kind, h->stream));
    const long n = h->plane * ncomp;
    k_f64_to_f32<<<592, 256, 0, h->stream>>>(h->stage64, static_cast<float*>(dst), n);
    CK(cudaGetLastError());
  }
  return SCL_OK;
}

int download_field(scl_handle* h, double* dst, const void* src, int ncomp, bool to_device) {
  const cudaMemcpyKind kind = to_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const size_t w = sizeof(double) * h->ld;
  const size_t nrows = (size_t)h->rows * ncomp;
  const void* from = src;
  if (h->ssize != sizeof(double)) {
    const long n = h->plane * ncomp;
    k_f32_to_f64<<<592, 256, 0, h->stream>>>(static_cast<const float*>(src), h->stage64, n);
    CK(cudaGetLastError());
    from = h->stage64;
  }
  CK(cudaMemcpy2DAsync(dst, w, from, sizeof(double) * h->pitch, w, nrows, kind, h->stream));
  return SCL_OK;
}

int validate(const scl_params* p) {
  if (!p) return fail(SCL_E_INVALID, "null params");
  if (p->ndim != 1 && p->ndim != 2) return fail(SCL_E_INVALID, "ndim must be 1 or 2");
  if (p->mbc != 3) return fail(SCL_E_INVALID, "WENO5 requires mbc = 3 (reconstruct.f90:85)");
  if (p->mx < 3 || (p->ndim == 2 && p->my < 3)) return fail(SCL_E_INVALID, "need at least 3 cells per direction");
  if (p->lim_type < 0 || p->lim_type > 2)
    return fail(SCL_E_INVALID, "lim_type must be 0 (polynomial), 1 (TVD) or 2 (WENO5)");
  if (p->char_decomp < 0 || p->char_decomp > (p->lim_type == 2 ? 3 : p->lim_type == 1 ? 2 : 1))
    return fail(SCL_E_UNSUPPORTED,
                "char_decomp must be 0..3 with WENO5, 0..2 with TVD, 0..1 with the polynomial (flux1.f90:65-116)");
  if (p->lim_type == 0 && p->mthlim[0] != 3) {
    if (p->mthlim[0] == 7)
      return fail(SCL_E_UNSUPPORTED, "polynomial order 7 needs four ghost cells (mbc = 3 here)");
    return fail(SCL_E_INVALID, "Invalid reconstruction order: mthlim(1) must be 3 (polyrecon.f90:23-39)");
  }
  if (p->lim_type == 1)
    for (int k = 0; k < std::max(p->meqn, p->mwaves) && k < 4; ++k)
      if (p->mthlim[k] < 1 || p->mthlim[k] > 5) return fail(SCL_E_INVALID, "mthlim must be 1..5 (reconstruct.f90:551-571)");
  if (p->tfluct_solver != 0 && p->tfluct_solver != 1) return fail(SCL_E_INVALID, "tfluct_solver must be 0 or 1");
  if (p->bc_user < SCL_BC_USER_NONE || p->bc_user > SCL_BC_USER_OSCILLATING_WALL)
    return fail(SCL_E_INVALID, "bc_user must be SCL_BC_USER_NONE or SCL_BC_USER_OSCILLATING_WALL");
  if (p->bc_user && (p->ndim != 1 || p->meqn < 2 || p->meqn > 10 || p->maux < 1 || p->maux > 10))
    return fail(SCL_E_UNSUPPORTED, "the oscillating-wall bc is 1-D with 2..10 components and 1..10 aux fields");
  for (int k = 0; k < 2 * p->ndim; ++k) {
    if (p->mthbc[k] == 0 && !p->bc_user)
      return fail(SCL_E_INVALID, "mthbc(k)=0 and no BCs specified in bc1 (set bc_user)");
    if (p->mthbc[k] < 0 || p->mthbc[k] > 3)
      return fail(SCL_E_INVALID, "mthbc must be 0 (user bc), 1, 2 or 3");
  }
  for (int k = 0; k < 2 * p->ndim; ++k)
    if (p->mthbc[k] == 3 && p->meqn < (k < 2 ? 2 : 3))
      return fail(SCL_E_INVALID, "solid wall bc negates component 2 (x) / 3 (y): meqn too small");
  if ((p->mthbc[0] == 2) != (p->mthbc[1] == 2) ||
      (p->ndim == 2 && (p->mthbc[2] == 2) != (p->mthbc[3] == 2)))
    return fail(SCL_E_INVALID, "periodic bc must be set on both sides");
  if (p->time_integrator < 1 || p->time_integrator > 4)
    return fail(SCL_E_INVALID, "time_integrator should be between 1 and 4");
  if (p->precision < SCL_FP64 || p->precision > SCL_FP32) return fail(SCL_E_INVALID, "bad precision");
  if (!(p->dx > 0) || (p->ndim == 2 && !(p->dy > 0))) return fail(SCL_E_INVALID, "dx, dy must be > 0");
  struct { int rp, meqn, mwaves, maux, ndim; } tab[] = {
      {SCL_RP_ADVECTION, 1, 1, 0, 1}, {SCL_RP_EULER, 3, 3, 0, 1}, {SCL_RP_SW2D, 3, 3, 0, 2},
      {SCL_RP_ACOUSTICS1D, 2, 2, 2, 1}, {SCL_RP_ACOUSTICS2D, 3, 2, 2, 2},
      {SCL_RP_ADVECTION2D, 1, 1, 2, 2}, {SCL_RP_SW1D, 2, 2, 0, 1}, {SCL_RP_SWF_BATHY, 2, 2, 1, 1},
      {SCL_RP_SWF_RADIAL, 2, 2, 2, 1}, {SCL_RP_SWF_KAPPA, 2, 2, 4, 1}, {SCL_RP_ACOUSTICS_CONST, 2, 2, 0, 1},
      {SCL_RP_ACOUSTICS_FWAVE, 2, 2, 2, 1}, {SCL_RP_TRAFFIC, 1, 1, 1, 1}, {SCL_RP_ADVECTION_CONS, 1, 1, 1, 1},
      {SCL_RP_STEGOTON, 2, 2, 3, 1}};
  if (p->rp == SCL_RP_ADVECTION_CONS && p->tfluct_solver == 1)
    return fail(SCL_E_INVALID, "the flux-uq app has no tfluct: use tfluct_solver 0");
  if (p->rp == SCL_RP_ACOUSTICS_CONST && !(p->rho > 0 && p->bulk > 0))
    return fail(SCL_E_INVALID, "homogeneous acoustics needs rho > 0 and bulk > 0 (setprob.f)");
  if (p->src_term != SCL_SRC_NONE) {
    if (p->src_term != SCL_SRC_RADIAL_SW && p->src_term != SCL_SRC_BATHYMETRY_SW)
      return fail(SCL_E_INVALID, "src_term must be SCL_SRC_NONE, SCL_SRC_RADIAL_SW or SCL_SRC_BATHYMETRY_SW");
    if (p->rp != SCL_RP_SW1D || p->ndim != 1)
      return fail(SCL_E_UNSUPPORTED, "the source-term hooks are the 1-D shallow-water apps' (SCL_RP_SW1D)");
    if (p->src_term == SCL_SRC_BATHYMETRY_SW && p->maux < 1)
      return fail(SCL_E_INVALID, "the bathymetry source reads b from aux(:,1): maux >= 1");
  }
  for (auto& t : tab)
    if (t.rp == p->rp) {
      if (p->meqn != t.meqn || p->mwaves != t.mwaves)
        return fail(SCL_E_INVALID, "meqn/mwaves do not match the plugin");
      if (p->maux < t.maux) return fail(SCL_E_INVALID, "plugin needs more aux fields");
      if (p->ndim != t.ndim) return fail(SCL_E_INVALID, "plugin dimension does not match ndim");
      if (p->mcapa < 0 || p->mcapa > p->maux) return fail(SCL_E_INVALID, "mcapa out of range");
      if (p->rp == SCL_RP_EULER && p->tfluct_solver == 1)
        return fail(SCL_E_INVALID, "no tfluct exists for the Euler plugin (src/tfluct.f90 stub)");
      return SCL_OK;
    }
  return fail(SCL_E_INVALID, "unknown rp id");
}

}  // namespace

extern "C" {

const char* scl_version(void) { return "sharpclaw_b200 0.1 (sm_100a)"; }
const char* scl_last_error(void) { return g_err.c_str(); }
void* scl_stream(scl_handle* h) { return h ? (void*)h->stream : nullptr; }

int scl_create(const scl_params* p, scl_handle** out) {
  if (!out) return fail(SCL_E_INVALID, "null out");
  *out = nullptr;
  int rc = validate(p);
  if (rc) return rc;
  scl_handle* h = new scl_handle();
  h->p = *p;
  CK(cudaGetDevice(&h->device));
  h->ssize = (p->precision == SCL_FP32) ? sizeof(float) : sizeof(double);
  h->ld = p->mx + 2 * p->mbc;
  h->rows = p->ndim == 2 ? p->my + 2 * p->mbc : 1;
  h->pitch = (h->ld + 31) / 32 * 32;
  h->plane = h->pitch * h->rows;
  if (!get_launchers(p->precision, p->rp, p->ndim, recon_code(*p), p->tfluct_solver, 0, &h->LV[0])) {
    delete h;
    return fail(SCL_E_UNSUPPORTED, "no kernel for this plugin / char_decomp / tfluct_solver");
  }
  h->L = h->LV[0];
  if (p->ndim == 2)
    while (h->nvariants < N2D_VARIANTS &&
           get_launchers(p->precision, p->rp, p->ndim, recon_code(*p), p->tfluct_solver, h->nvariants,
                         &h->LV[h->nvariants]))
      h->nvariants += 1;
  h->nstages = stage_table(p->time_integrator, h->sd, &h->final_role);
  auto cleanup = [&](int code) { scl_destroy(h); return code; };
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(fail(SCL_E_CUDA, "stream create failed"));
  const size_t fbytes = h->ssize * h->plane * p->meqn;
  for (int r = 0; r < NROLES; ++r) {
    if (cudaMalloc(&h->buf[r], fbytes) != cudaSuccess) return cleanup(fail(SCL_E_CUDA, "cudaMalloc q buffers"));
    cudaMemsetAsync(h->buf[r], 0, fbytes, h->stream);
  }
  const size_t abytes = h->ssize * h->plane * std::max(1, p->maux);
  if (cudaMalloc(&h->aux, abytes) != cudaSuccess) return cleanup(fail(SCL_E_CUDA, "cudaMalloc aux"));
  cudaMemsetAsync(h->aux, 0, abytes, h->stream);
  const size_t sbytes = sizeof(double) * h->plane * std::max(p->meqn, std::max(1, p->maux));
  if (cudaMalloc(&h->stage64, sbytes) != cudaSuccess) return cleanup(fail(SCL_E_CUDA, "cudaMalloc staging"));
  cudaMemsetAsync(h->stage64, 0, sbytes, h->stream);
  // ctl[0] is the controller, ctl[1] a copy the tile-shape trials write into
  if (cudaMalloc(&h->ctl, 2 * sizeof(Ctl)) != cudaSuccess) return cleanup(fail(SCL_E_CUDA, "cudaMalloc ctl"));
  if (cudaMallocHost(&h->hctl, sizeof(Ctl)) != cudaSuccess) return cleanup(fail(SCL_E_CUDA, "cudaMallocHost"));
  if (cudaMallocHost(&h->hdone, 2 * sizeof(int)) != cudaSuccess) return cleanup(fail(SCL_E_CUDA, "cudaMallocHost"));
  memset(h->hctl, 0, sizeof(Ctl));
  for (int r = 0; r < NROLES; ++r) h->hctl->role[r] = r;
  h->hctl->done = 0;
  cudaEventCreate(&h->ev0);
  cudaEventCreate(&h->ev1);
  cudaEventCreateWithFlags(&h->evq[0], cudaEventDisableTiming);
  cudaEventCreateWithFlags(&h->evq[1], cudaEventDisableTiming);
  rc = upload_ctl(h);
  if (rc) return cleanup(rc);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return cleanup(fail(SCL_E_CUDA, "create sync"));
  *out = h;
  return SCL_OK;
}

int scl_destroy(scl_handle* h) {
  if (!h) return SCL_OK;
  if (h->fthread.joinable()) h->fthread.join();
  if (h->fbuf) cudaFreeHost(h->fbuf);
  if (h->fev) cudaEventDestroy(h->fev);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->graph) cudaGraphExecDestroy(h->graph);
  for (int r = 0; r < NROLES; ++r) if (h->buf[r]) cudaFree(h->buf[r]);
  if (h->aux) cudaFree(h->aux);
  if (h->stage64) cudaFree(h->stage64);
  if (h->adj) cudaFree(h->adj);
  if (h->aux0) cudaFree(h->aux0);
  if (h->tot_partials) cudaFree(h->tot_partials);
  if (h->ctl) cudaFree(h->ctl);
  if (h->hctl) cudaFreeHost(h->hctl);
  if (h->hdone) cudaFreeHost(h->hdone);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  for (int k = 0; k < 2; ++k) if (h->evq[k]) cudaEventDestroy(h->evq[k]);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return SCL_OK;
}

int scl_set_q(scl_handle* h, const double* q) {
  if (!h || !q) return fail(SCL_E_INVALID, "null argument");
  void* dst = h->buf[h->hctl->role[ROLE_Q]];
  int rc = upload_field(h, dst, q, h->p.meqn, false);
  if (rc) return rc;
  if (h->ssize == sizeof(double)) launch_bc<double>(h, static_cast<double*>(dst));
  else launch_bc<float>(h, static_cast<float*>(dst));
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(h->stream));
  return SCL_OK;
}

int scl_get_q(scl_handle* h, double* q) {
  if (!h || !q) return fail(SCL_E_INVALID, "null argument");
  int rc = download_field(h, q, h->buf[h->hctl->role[ROLE_Q]], h->p.meqn, false);
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->stream));
  return SCL_OK;
}

int scl_set_aux(scl_handle* h, const double* aux) {
  if (!h || !aux) return fail(SCL_E_INVALID, "null argument");
  if (h->p.maux == 0) return SCL_OK;
  int rc = upload_field(h, h->aux, aux, h->p.maux, false);
  if (rc) return rc;
  if (h->aux0)   // the b4step hook's base field follows the aux the caller sets
    CK(cudaMemcpyAsync(h->aux0, h->aux, h->ssize * h->plane * h->p.maux, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return SCL_OK;
}

int scl_set_b4step(scl_handle* h, int kind, double param) {
  if (!h) return fail(SCL_E_INVALID, "null handle");
  if (kind != SCL_B4STEP_NONE && kind != SCL_B4STEP_SWIRL && kind != SCL_B4STEP_TIME_REVERSAL)
    return fail(SCL_E_UNSUPPORTED, "unknown b4step hook");
  if (kind == SCL_B4STEP_SWIRL && (h->p.rp != SCL_RP_ADVECTION2D || h->p.maux < 2))
    return fail(SCL_E_INVALID, "the swirl b4step scales the edge velocities of SCL_RP_ADVECTION2D");
  if (kind == SCL_B4STEP_TIME_REVERSAL && (h->p.ndim != 1 || h->p.meqn < 2))
    return fail(SCL_E_INVALID, "the time-reversal b4step negates component 2 of a 1-D grid");
  CK(cudaStreamSynchronize(h->stream));
  if (kind == SCL_B4STEP_SWIRL && !h->aux0) {
    const size_t bytes = h->ssize * h->plane * h->p.maux;
    CK(cudaMalloc(&h->aux0, bytes));
    CK(cudaMemcpyAsync(h->aux0, h->aux, bytes, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
  }
  h->b4kind = kind;
  h->b4param = param;
  if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }   // captured steps change
  return SCL_OK;
}

int scl_step_dq(scl_handle* h, double* q, double* dq, double dt, double t, double* cfl) {
  if (!h || !q || !dq) return fail(SCL_E_INVALID, "null argument");
  int rc = scl_set_q(h, q);   // upload + bc
  if (rc) return rc;
  h->hctl->dt = dt;
  h->hctl->done = 0;
  for (int s = 0; s < MAXSTAGES; ++s) h->hctl->stage_cfl[s] = 0.0;
  rc = upload_ctl(h);
  if (rc) return rc;
  CK(cudaMemsetAsync(h->stage64, 0, sizeof(double) * h->plane * h->p.meqn, h->stream));
  StageArgs a = make_args(h, 0);
  a.sd = StageDesc{SK_DQ, ROLE_Q, -1, -1, -1};
  if (h->p.bc_user) {   // step1d.f90:20: bc at the step's time t
    a.tform = 2;
    a.tc = t;
    launch_bc_user(h, a);
    CK(cudaMemcpyAsync(&h->hctl->bc_switched, &h->ctl->bc_switched, sizeof(int), cudaMemcpyDeviceToHost,
                       h->stream));
  }
  h->L.stage(a, h->stream);
  if (h->L.ghost) h->L.ghost(a, h->stream);
  CK(cudaGetLastError());
  // dq in double, pitched -> reference layout
  const size_t w = sizeof(double) * h->ld;
  CK(cudaMemcpy2DAsync(dq, w, h->stage64, sizeof(double) * h->pitch, w, (size_t)h->rows * h->p.meqn,
                       cudaMemcpyDeviceToHost, h->stream));
  rc = download_field(h, q, h->buf[h->hctl->role[ROLE_Q]], h->p.meqn, false);
  if (rc) return rc;
  rc = download_ctl(h);
  if (rc) return rc;
  if (cfl) *cfl = h->hctl->stage_cfl[0];
  if (h->hctl->status & SCL_STATUS_TIMEOUT) return fail(SCL_E_TIMEOUT, "a bounded wait for staged data ran out");
  return SCL_OK;
}

int scl_flux1(scl_handle* h, const double* q1d, const double* aux1d, double* dq1d, double dt,
              int ixy, int mx, double* cfl) {
  if (!h || !q1d || !dq1d) return fail(SCL_E_INVALID, "null argument");
  if (ixy != 1 && ixy != 2) return fail(SCL_E_INVALID, "ixy must be 1 or 2");
  if (mx < 3) return fail(SCL_E_INVALID, "mx too small");
  if (h->p.maux > 0 && !aux1d) return fail(SCL_E_INVALID, "aux1d required");
  // A one-line problem of the same plugin: a temporary 1-D handle.
  scl_params p1 = h->p;
  p1.ndim = 1;
  p1.mx = mx;
  p1.my = 1;
  p1.dx = (ixy == 1) ? h->p.dx : h->p.dy;
  p1.mthbc[0] = p1.mthbc[1] = 1;
  Launchers L1{};
  if (!get_launchers(p1.precision, p1.rp, 1, recon_code(p1), p1.tfluct_solver, 0, &L1))
    return fail(SCL_E_UNSUPPORTED, "no 1-D kernel for this plugin");
  const long ld = mx + 2 * p1.mbc, pitch = (ld + 31) / 32 * 32;
  const size_t ss = h->ssize;
  void *dq_in = nullptr, *dq_aux = nullptr;
  double* d64 = nullptr;
  Ctl* dctl = nullptr;
  auto cleanup = [&]() {
    cudaFree(dq_in); cudaFree(dq_aux); cudaFree(d64); cudaFree(dctl);
  };
  if (cudaMalloc(&dq_in, ss * pitch * p1.meqn) != cudaSuccess ||
      cudaMalloc(&dq_aux, ss * pitch * std::max(1, p1.maux)) != cudaSuccess ||
      cudaMalloc(&d64, sizeof(double) * pitch * std::max(p1.meqn, std::max(1, p1.maux))) != cudaSuccess ||
      cudaMalloc(&dctl, sizeof(Ctl)) != cudaSuccess) {
    cleanup();
    return fail(SCL_E_CUDA, "cudaMalloc in scl_flux1");
  }
  int rc = SCL_OK;
  auto put = [&](void* dst, const double* src, int nc) -> int {
    const size_t w = sizeof(double) * ld;
    if (ss == sizeof(double)) {
      CK(cudaMemcpy2DAsync(dst, sizeof(double) * pitch, src, w, w, nc, cudaMemcpyHostToDevice, h->stream));
    } else {
      CK(cudaMemcpy2DAsync(d64, sizeof(double) * pitch, src, w, w, nc, cudaMemcpyHostToDevice, h->stream));
      k_f64_to_f32<<<64, 256, 0, h->stream>>>(d64, static_cast<float*>(dst), pitch * nc);
    }
    return SCL_OK;
  };
  Ctl c{};
  c.dt = dt;
  for (int r = 0; r < NROLES; ++r) c.role[r] = r;
  rc = put(dq_in, q1d, p1.meqn);
  if (!rc && p1.maux > 0) rc = put(dq_aux, aux1d, p1.maux);
  if (!rc && cudaMemcpyAsync(dctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
    rc = fail(SCL_E_CUDA, "ctl upload");
  if (!rc && cudaMemsetAsync(d64, 0, sizeof(double) * pitch * p1.meqn, h->stream) != cudaSuccess)
    rc = fail(SCL_E_CUDA, "memset");
  if (!rc) {
    StageArgs a{};
    a.ctl = dctl;
    a.buf[0] = dq_in;
    a.aux = dq_aux;
    a.dq_out = d64;
    a.sd = StageDesc{SK_DQ, 0, -1, -1, -1};
    a.stage = 0;
    a.ixy = ixy;
    a.mx = mx;
    a.my = 1;
    a.pitch = pitch;
    a.plane = pitch;
    a.dx = p1.dx;
    a.dy = p1.dx;
    for (int k = 0; k < 4; ++k) a.mthbc[k] = 1;
    a.mcapa = p1.mcapa;
    a.ph.u = p1.u; a.ph.gamma = p1.gamma; a.ph.gamma1 = p1.gamma - 1.0; a.ph.grav = p1.grav;
    a.ph.efix = p1.efix;
    for (int k = 0; k < 4; ++k) a.ph.mthlim[k] = p1.mthlim[k];
    set_acoustics_consts(p1, &a.ph);
    L1.stage(a, h->stream);
    if (cudaGetLastError() != cudaSuccess) rc = fail(SCL_E_CUDA, "flux1 launch");
  }
  if (!rc) {
    const size_t w = sizeof(double) * ld;
    if (cudaMemcpy2DAsync(dq1d, w, d64, sizeof(double) * pitch, w, p1.meqn, cudaMemcpyDeviceToHost,
                          h->stream) != cudaSuccess ||
        cudaMemcpyAsync(&c, dctl, sizeof(Ctl), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
      rc = fail(SCL_E_CUDA, "flux1 download");
    else if (c.status & SCL_STATUS_TIMEOUT)
      rc = fail(SCL_E_TIMEOUT, "a bounded wait for staged data ran out");
    else if (cfl)
      *cfl = c.stage_cfl[0];
  }
  cudaStreamSynchronize(h->stream);
  cleanup();
  return rc;
}

int scl_rk_step(scl_handle* h, double dt, double told, double* cfl) {
  if (!h) return fail(SCL_E_INVALID, "null handle");
  Ctl* c = h->hctl;
  c->dt = dt;
  c->told = told;
  c->t = told + dt;
  c->done = 0;
  c->status = 0;
  for (int s = 0; s < MAXSTAGES; ++s) c->stage_cfl[s] = 0.0;
  int rc = upload_ctl(h);
  if (rc) return rc;
  rc = enqueue_stages(h);
  if (rc) return rc;
  rc = download_ctl(h);
  if (rc) return rc;
  const double cv = c->stage_cfl[h->nstages - 1];
  if (c->status & SCL_STATUS_TIMEOUT) return fail(SCL_E_TIMEOUT, "a bounded wait for staged data ran out");
  std::swap(c->role[ROLE_Q], c->role[h->final_role]);
  if (cfl) *cfl = cv;
  if ((c->status & SCL_STATUS_NONFINITE) || cv != cv) return fail(SCL_E_NONFINITE, "non-finite stage output");
  return SCL_OK;
}

}  // extern "C"

namespace {

// Initialise the controller from sharpclaw()'s arguments (sharpclaw.f90:35-64).
int init_run(scl_handle* h, const scl_run* run, int max_steps, scl_result* res, bool* early) {
  *early = false;
  Ctl* c = h->hctl;
  c->t = run->tstart;
  c->told = run->tstart;
  c->tstart = run->tstart;
  c->tend = run->tend;
  c->dt = run->dt_initial;
  c->dt_max = run->dt_max;
  c->cfl_max = run->cfl_max;
  c->cfl_desired = run->cfl_desired;
  c->cflmax = 0.0;
  c->dtmin = run->dt_initial;
  c->dtmax = run->dt_initial;
  c->cfl_last = 0.0;
  c->n_iter = 0;
  c->maxn = max_steps;
  c->steps_taken = 0;
  c->rejected = 0;
  c->retake = 0;
  c->done = 0;
  c->info = 0;
  c->status = 0;
  c->dt_variable = run->dt_variable;
  c->totals = h->totals_on;
  memset(res, 0, sizeof(*res));
  if (run->dt_variable == 0) {
    if (run->tend < run->tstart) {
      c->maxn = 1;
    } else {
      c->maxn = (int)((run->tend - run->tstart + 1e-10) / run->dt_initial);
      if (std::fabs(c->maxn * run->dt_initial - (run->tend - run->tstart)) > 1e-5 * (run->tend - run->tstart)) {
        res->info = SCL_INFO_DT_NOT_DIVIDING;
        *early = true;
        return SCL_OK;
      }
    }
  }
  if (run->dt_variable == 1 && run->cfl_desired > run->cfl_max) {
    res->info = SCL_INFO_CFL_DESIRED_GT_MAX;
    *early = true;
    return SCL_OK;
  }
  int rc = upload_ctl(h);
  if (rc == SCL_OK && h->totals_on) {
    launch_totals(h, ROLE_Q, 1);   // the run's starting totals
    CK(cudaGetLastError());
  }
  if (rc == SCL_OK && h->nvariants > 1 && !h->tiles_fixed && !h->tiles_tuned) rc = tune_tiles(h);
  return rc;
}

void finish_run(scl_handle* h, scl_result* res) {
  const Ctl* c = h->hctl;
  int info = c->info;
  if (!info) {
    if (c->dt_variable == 1 && c->t < c->tend && c->steps_taken == c->maxn) info = SCL_INFO_TOO_MANY_STEPS;
    if (c->dt_variable == 0 && c->cflmax > c->cfl_max) info = SCL_INFO_CFL_FIXED_DT;
  }
  res->tend = c->t;
  res->cfl_maxused = c->cflmax;
  res->cfl_last = c->cfl_last;
  res->dt_minused = c->dtmin;
  res->dt_maxused = c->dtmax;
  res->dt_last = c->dt;
  res->steps_taken = c->steps_taken;
  res->info = info;
  res->rejected = c->rejected;
  res->status = c->status;
}

// Replay the K-step graph until the controller reports done.  The done flag
// of replay k is copied to pinned memory behind replay k+1, so the device
// never idles waiting for the host.
int run_loop(scl_handle* h, int graph_steps, long max_replays, float* ms) {
  int rc = build_graph(h, graph_steps);
  if (rc) return rc;
  if (ms) CK(cudaEventRecord(h->ev0, h->stream));
  h->hdone[0] = h->hdone[1] = 0;
  h->last_mode = SCL_RUN_GRAPH;
  h->last_launches = 0;
  for (long r = 0; r < max_replays; ++r) {
    CK(cudaGraphLaunch(h->graph, h->stream));
    h->last_launches += (long long)graph_steps * kernels_per_step(h) + 1;
    if (max_replays == 1) break;
    CK(cudaMemcpyAsync(&h->hdone[r & 1], &h->ctl->done, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaEventRecord(h->evq[r & 1], h->stream));
    if (r > 0) {  // replay r is already queued while we look at replay r-1
      CK(cudaEventSynchronize(h->evq[(r - 1) & 1]));
      if (h->hdone[(r - 1) & 1]) break;
    }
  }
  if (ms) {
    CK(cudaEventRecord(h->ev1, h->stream));
    CK(cudaEventSynchronize(h->ev1));
    CK(cudaEventElapsedTime(ms, h->ev0, h->ev1));
  }
  return download_ctl(h);
}

int resident_tiles(const scl_handle* h) { return (h->p.mx + RES_NT - 2) / (RES_NT - 1); }

// A resident run needs a 1-D grid of at most RES_MAX_TILES tiles and no
// b4step hook (the hooks run as kernels of the step graph).
bool resident_possible(const scl_handle* h) {
  return h->p.ndim == 1 && h->L.run != nullptr && h->b4kind == SCL_B4STEP_NONE && !h->p.bc_user &&
         resident_tiles(h) <= RES_MAX_TILES;
}

int use_resident(const scl_handle* h, bool* yes) {
  *yes = false;
  if (h->run_mode == SCL_RUN_GRAPH) return SCL_OK;
  if (h->run_mode == SCL_RUN_RESIDENT) {
    if (!resident_possible(h))
      return fail(SCL_E_UNSUPPORTED, "resident run: needs a 1-D grid of at most 64 tiles, no b4step hook and no user bc");
    *yes = true;
    return SCL_OK;
  }
  *yes = resident_possible(h) && resident_tiles(h) <= RES_AUTO_TILES;
  return SCL_OK;
}

// The controller loop as cluster-resident launches of RES_ITERS iterations
// each, relaunched until the controller is done (after maxn iterations at
// the latest).
int run_resident(scl_handle* h, float* ms) {
  RunArgs ra{};
  ra.st = make_args(h, 0);
  for (int s = 0; s < h->nstages; ++s) ra.sd[s] = h->sd[s];
  ra.nstages = h->nstages;
  ra.final_role = h->final_role;
  ra.max_iters = RES_ITERS;
  ra.totals = h->totals_on ? 1 : 0;
  const long max_launches = (long)h->hctl->maxn / RES_ITERS + 1;
  if (ms) CK(cudaEventRecord(h->ev0, h->stream));
  h->last_mode = SCL_RUN_RESIDENT;
  h->last_launches = 0;
  for (long r = 0; r < max_launches; ++r) {
    CK(h->L.run(ra, h->stream));
    h->last_launches += 1;
    if (r + 1 == max_launches) break;
    CK(cudaMemcpyAsync(&h->hdone[0], &h->ctl->done, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (h->hdone[0]) break;
  }
  if (ms) {
    CK(cudaEventRecord(h->ev1, h->stream));
    CK(cudaEventSynchronize(h->ev1));
    CK(cudaEventElapsedTime(ms, h->ev0, h->ev1));
  }
  return download_ctl(h);
}

}  // namespace

extern "C" {

int scl_sharpclaw(scl_handle* h, const scl_run* run, scl_result* res) {
  if (!h || !run || !res) return fail(SCL_E_INVALID, "null argument");
  bool resident = false;
  int rc = use_resident(h, &resident);
  if (rc) return rc;
  bool early = false;
  rc = init_run(h, run, run->max_steps, res, &early);
  if (rc || early) return rc;
  if (resident) {
    rc = run_resident(h, nullptr);
  } else {
    // a graph replay runs gs controller steps; after maxn iterations the
    // controller is done, so no more than ceil(maxn/gs) replays are launched
    const int gs = std::min(std::max(1, h->hctl->maxn), default_graph_steps(h));
    const long replays = ((long)h->hctl->maxn + gs - 1) / gs;
    rc = run_loop(h, gs, replays, nullptr);
  }
  if (rc) return rc;
  finish_run(h, res);
  if (res->status & SCL_STATUS_TIMEOUT) return fail(SCL_E_TIMEOUT, "a bounded wait for staged data ran out");
  if (res->status & SCL_STATUS_NONFINITE) return fail(SCL_E_NONFINITE, "non-finite CFL number");
  return SCL_OK;
}

int scl_sharpclaw_device(scl_handle* h, const scl_run* run, double* q_dev, scl_result* res) {
  if (!h || !run || !res || !q_dev) return fail(SCL_E_INVALID, "null argument");
  void* dst = h->buf[h->hctl->role[ROLE_Q]];
  int rc = upload_field(h, dst, q_dev, h->p.meqn, true);
  if (rc) return rc;
  if (h->ssize == sizeof(double)) launch_bc<double>(h, static_cast<double*>(dst));
  else launch_bc<float>(h, static_cast<float*>(dst));
  rc = scl_sharpclaw(h, run, res);
  if (rc && rc != SCL_E_NONFINITE) return rc;
  int rc2 = download_field(h, q_dev, h->buf[h->hctl->role[ROLE_Q]], h->p.meqn, true);
  if (rc2) return rc2;
  CK(cudaStreamSynchronize(h->stream));
  return rc;
}

int scl_time_steps(scl_handle* h, const scl_run* run, int nsteps, float* ms, scl_result* res) {
  if (!h || !run || !ms || !res || nsteps < 1) return fail(SCL_E_INVALID, "bad argument");
  bool resident = false;
  int rc = use_resident(h, &resident);
  if (rc) return rc;
  bool early = false;
  rc = init_run(h, run, nsteps, res, &early);
  if (rc || early) return rc ? rc : fail(SCL_E_INVALID, "run parameters rejected (info set)");
  if (resident) {
    rc = run_resident(h, ms);
  } else {
    const int gs = nsteps <= 64 ? nsteps : default_graph_steps(h);
    const long replays = (nsteps + gs - 1) / gs;
    rc = run_loop(h, gs, replays, ms);
  }
  if (rc) return rc;
  finish_run(h, res);
  if (res->status & SCL_STATUS_TIMEOUT) return fail(SCL_E_TIMEOUT, "a bounded wait for staged data ran out");
  return SCL_OK;
}

int scl_time_stages(scl_handle* h, double dt, int reps, float* ms, long long* launches) {
  if (!h || !ms || reps < 1) return fail(SCL_E_INVALID, "bad argument");
  Ctl* c = h->hctl;
  c->dt = dt;
  c->done = 0;
  c->status = 0;
  for (int s = 0; s < MAXSTAGES; ++s) c->stage_cfl[s] = 0.0;
  int rc = upload_ctl(h);
  if (rc) return rc;
  rc = enqueue_stages(h);  // warm-up pass
  if (rc) return rc;
  CK(cudaEventRecord(h->ev0, h->stream));
  for (int r = 0; r < reps; ++r) {
    for (int s = 0; s < h->nstages; ++s) {
      const StageArgs a = make_args(h, s);
      if (h->p.bc_user) launch_bc_user(h, a);
      h->L.stage(a, h->stream);
    }
  }
  CK(cudaGetLastError());
  CK(cudaEventRecord(h->ev1, h->stream));
  CK(cudaEventSynchronize(h->ev1));
  CK(cudaEventElapsedTime(ms, h->ev0, h->ev1));
  if (launches) *launches = (long long)reps * h->nstages;
  return SCL_OK;
}

int scl_kernels_per_step(scl_handle* h) { return h ? kernels_per_step(h) : 0; }

int scl_set_run_mode(scl_handle* h, int mode) {
  if (!h) return fail(SCL_E_INVALID, "null handle");
  if (mode != SCL_RUN_AUTO && mode != SCL_RUN_GRAPH && mode != SCL_RUN_RESIDENT)
    return fail(SCL_E_INVALID, "run mode must be SCL_RUN_AUTO, SCL_RUN_GRAPH or SCL_RUN_RESIDENT");
  if (mode == SCL_RUN_RESIDENT && !resident_possible(h))
    return fail(SCL_E_UNSUPPORTED, "resident run: needs a 1-D grid of at most 64 tiles, no b4step hook and no user bc");
  h->run_mode = mode;
  return SCL_OK;
}

int scl_set_totals(scl_handle* h, int on) {
  if (!h) return fail(SCL_E_INVALID, "null handle");
  if (on != 0 && on != 1) return fail(SCL_E_INVALID, "on must be 0 or 1");
  if (on && !h->tot_partials) {
    if (cudaMalloc(&h->tot_partials, sizeof(double) * TOT_BLOCKS * MAXEQ * 2) != cudaSuccess)
      return fail(SCL_E_CUDA, "cudaMalloc totals partials");
  }
  if (h->totals_on != on && h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }   // one kernel more or less per step
  h->totals_on = on;
  return SCL_OK;
}

int scl_test_wait_timeout(scl_handle* h, int on) {
  if (!h) return fail(SCL_E_INVALID, "null handle");
  if (on != 0 && on != 1) return fail(SCL_E_INVALID, "on must be 0 or 1");
  if (h->test_timeout != on && h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }   // captured arguments change
  h->test_timeout = on;
  return SCL_OK;
}

int scl_conserved_totals(scl_handle* h, double* tot0, double* tot, double* drift) {
  if (!h) return fail(SCL_E_INVALID, "null handle");
  if (!h->totals_on) return fail(SCL_E_INVALID, "totals are off (scl_set_totals)");
  const Ctl* c = h->hctl;   // as the last run left it (downloaded at its end)
  for (int m = 0; m < h->p.meqn; ++m) {
    if (tot0) tot0[m] = c->tot0[m];
    if (tot) tot[m] = c->tot[m];
    if (drift) drift[m] = c->drift[m];
  }
  return SCL_OK;
}

int scl_last_run(scl_handle* h, int* mode, long long* launches) {
  if (!h) return fail(SCL_E_INVALID, "null handle");
  if (mode) *mode = h->last_mode;
  if (launches) *launches = h->last_launches;
  return SCL_OK;
}

int scl_wait_frames(scl_handle* h) {
  if (!h) return fail(SCL_E_INVALID, "null handle");
  if (h->fthread.joinable()) h->fthread.join();
  const int rc = h->frc;
  h->frc = SCL_OK;
  if (rc) return fail(rc, h->ferr);
  return SCL_OK;
}

int scl_write_frame(scl_handle* h, double t, int iframe, const char* dir, int write_aux) {
  if (!h || iframe < 0) return fail(SCL_E_INVALID, "null handle or negative frame number");
  int rc = scl_wait_frames(h);   // the pinned buffer holds one frame at a time
  if (rc) return rc;
  const scl_params& p = h->p;
  const long plane_ref = h->ld * h->rows;
  const bool aux_out = write_aux && p.maux > 0;
  const size_t n = (size_t)plane_ref * (p.meqn + (aux_out ? p.maux : 0));
  if (n > h->fbuf_n) {
    if (h->fbuf) cudaFreeHost(h->fbuf);
    h->fbuf = nullptr;
    h->fbuf_n = 0;
    CK(cudaMallocHost(&h->fbuf, n * sizeof(double)));
    h->fbuf_n = n;
  }
  if (!h->fev) CK(cudaEventCreateWithFlags(&h->fev, cudaEventDisableTiming));
  rc = download_field(h, h->fbuf, h->buf[h->hctl->role[ROLE_Q]], p.meqn, false);
  if (rc) return rc;
  const double* aq = nullptr;
  if (aux_out) {
    rc = download_field(h, h->fbuf + plane_ref * p.meqn, h->aux, p.maux, false);
    if (rc) return rc;
    aq = h->fbuf + plane_ref * p.meqn;
  }
  CK(cudaEventRecord(h->fev, h->stream));
  FrameSpec f{p.ndim, p.mx, p.ndim == 2 ? p.my : 1, p.mbc, p.meqn, p.maux, p.xlower, p.ylower,
              p.dx, p.dy, t, iframe, aux_out, dir ? std::string(dir) : std::string()};
  const double* qq = h->fbuf;
  h->fthread = std::thread([h, f, qq, aq]() {
    cudaSetDevice(h->device);
    const cudaError_t e = cudaEventSynchronize(h->fev);
    if (e != cudaSuccess) {
      h->frc = SCL_E_CUDA;
      h->ferr = std::string("frame copy: ") + cudaGetErrorString(e);
      return;
    }
    std::string err;
    if (write_frame_files(f, qq, aq, &err)) {
      h->frc = SCL_E_IO;
      h->ferr = err;
    }
  });
  return SCL_OK;
}

int scl_format_frame(const scl_params* p, const double* q, const double* aux, double t, int iframe,
                     const char* dir, int write_aux) {
  if (!p || !q || iframe < 0) return fail(SCL_E_INVALID, "null argument or negative frame number");
  if ((p->ndim != 1 && p->ndim != 2) || p->mx < 1 || (p->ndim == 2 && p->my < 1) || p->mbc < 0 ||
      p->meqn < 1 || p->maux < 0)
    return fail(SCL_E_INVALID, "bad grid parameters");
  const bool aux_out = write_aux && p->maux > 0;
  if (aux_out && !aux) return fail(SCL_E_INVALID, "write_aux needs aux");
  FrameSpec f{p->ndim, p->mx, p->ndim == 2 ? p->my : 1, p->mbc, p->meqn, p->maux, p->xlower, p->ylower,
              p->dx, p->dy, t, iframe, aux_out, dir ? std::string(dir) : std::string()};
  std::string err;
  if (write_frame_files(f, q, aux_out ? aux : nullptr, &err)) return fail(SCL_E_IO, err);
  return SCL_OK;
}

int scl_select_tiles(scl_handle* h, int variant) {
  if (!h) return fail(SCL_E_INVALID, "null handle");
  if (variant < -1 || variant >= h->nvariants) return fail(SCL_E_UNSUPPORTED, "no such tile shape for this handle");
  for (int v = 0; v < N2D_VARIANTS; ++v) h->tile_ms[v] = 0.f;
  h->tiles_tuned = 0;
  h->tiles_fixed = variant >= 0;
  if (variant >= 0) {
    CK(cudaStreamSynchronize(h->stream));  // no launch of the old graph in flight
    use_variant(h, variant);
  }
  return SCL_OK;
}

int scl_tiles(scl_handle* h, int* variant, int* tuned, float* trial_ms) {
  if (!h) return fail(SCL_E_INVALID, "null handle");
  if (variant) *variant = h->variant;
  if (tuned) *tuned = h->tiles_tuned;
  if (trial_ms)
    for (int v = 0; v < N2D_VARIANTS; ++v) trial_ms[v] = h->tile_ms[v];
  return SCL_OK;
}

}  // extern "C"

namespace scl {
void set_last_error(const char* msg) { g_err = msg ? msg : ""; }
}  // namespace scl

namespace {

// Discrete adjoint of one SSPRK(10,4), SSPRK(2,2) or SSPRK(4,2) step
// (src/sharpclaw.f90:380-464, 247-276, 280-333) with D(q) = dt L(q).  The
// forward evaluates D at the stage states with SK_DQ launches of the
// handle's own stage kernel (in FP64_STRICT these are the solver's states
// bit for bit) and keeps them; the backward applies D'(s)^T in reverse:
//   SSPRK(10,4): s_{k+1} = s_k + D(s_k)/6 (k = 0..4, s5 = r2),
//     r1 = 0.04 s0 + 0.36 s5, s5' = 0.6 s0 + 0.4 s5, s6..s9 from s5',
//     q_new = (r1 + 0.6 s9) + 0.1 D(s9);
//     l9 = 0.6 l + 0.1 D'(s9)^T l, l_k = l_{k+1} + D'(s_k)^T l_{k+1} / 6,
//     l5 = 0.4 l5' + 0.36 l, acc = 0.6 l5' + 0.04 l, l0 = acc + l1 + D'(s0)^T l1 / 6;
//   SSPRK(2,2): s1 = s0 + D(s0), q_new = 0.5 ((s0 + s1) + D(s1));
//     l1 = 0.5 l + 0.5 D'(s1)^T l, l0 = 0.5 l + l1 + D'(s0)^T l1;
//   SSPRK(4,2): s_{k+1} = s_k + D(s_k)/3 (k = 0..2),
//     q_new = (0.25 s0 + 0.75 s3) + 0.25 D(s3);
//     l3 = 0.75 l + 0.25 D'(s3)^T l, l_k = l_{k+1} + D'(s_k)^T l_{k+1} / 3,
//     l0 = 0.25 l + l1 + D'(s0)^T l1 / 3.
int adjoint_rk(scl_handle* h, const double* q_dev, const double* lam_in_dev, double* lam_out_dev, double dt) {
  const scl_params& p = h->p;
  const int ti = p.time_integrator;
  const long nfield = h->plane * p.meqn;
  double* S[10];
  for (int k = 0; k < 10; ++k) S[k] = h->adj + k * nfield;    // stage states
  double* DQ = h->adj + 10 * nfield;
  double* LIN = h->adj + 11 * nfield;
  double* LA = h->adj + 12 * nfield;
  double* LB = h->adj + 13 * nfield;
  double* T = h->adj + 14 * nfield;
  double* ACC = h->adj + 15 * nfield;
  // a controller with identity roles and this dt for the SK_DQ evaluations
  Ctl c{};
  c.dt = dt;
  for (int r = 0; r < NROLES; ++r) c.role[r] = r;
  Ctl* dctl = h->ctl + 1;
  CK(cudaMemcpyAsync(dctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, h->stream));
  auto evalD = [&](double* s) {
    launch_bc<double>(h, s);
    StageArgs a = make_args(h, 0);
    a.ctl = dctl;
    for (int r = 0; r < NROLES; ++r) a.buf[r] = s;
    a.dq_out = DQ;
    a.sd = StageDesc{SK_DQ, ROLE_Q, -1, -1, -1};
    a.stage = 0;
    h->L.stage(a, h->stream);
  };
  const double sixth = 1.0 / 6.0, third = 1.0 / 3.0;
  int rc = upload_field(h, S[0], q_dev, p.meqn, true);
  if (rc) return rc;
  int last = 0;   // index of the last stage state
  if (ti == 4) {
    for (int k = 0; k < 4; ++k) {                                // stages 1-4 (:396-419)
      evalD(S[k]);
      launch_axpby(S[k + 1], 1.0, S[k], sixth, DQ, nfield, h->stream);
    }
    evalD(S[4]);                                                 // stage 5 (:421-429)
    launch_axpby(T, 1.0, S[4], sixth, DQ, nfield, h->stream);    // s5 (r2)
    launch_axpby(S[5], 0.6, S[0], 0.4, T, nfield, h->stream);    // s5'
    for (int k = 5; k < 9; ++k) {                                // stages 6-9 (:431-455)
      evalD(S[k]);
      launch_axpby(S[k + 1], 1.0, S[k], sixth, DQ, nfield, h->stream);
    }
    last = 9;
  } else if (ti == 1) {
    evalD(S[0]);                                                 // :262-264
    launch_axpby(S[1], 1.0, S[0], 1.0, DQ, nfield, h->stream);
    last = 1;
  } else {
    for (int k = 0; k < 3; ++k) {                                // :296-322
      evalD(S[k]);
      launch_axpby(S[k + 1], 1.0, S[k], third, DQ, nfield, h->stream);
    }
    last = 3;
  }
  launch_bc<double>(h, S[last]);   // the VJP reads the periodic images of the last state too
  CK(cudaGetLastError());
  const size_t w = sizeof(double) * h->ld;
  CK(cudaMemcpy2DAsync(LIN, sizeof(double) * h->pitch, lam_in_dev, w, w, (size_t)h->rows * p.meqn,
                       cudaMemcpyDeviceToDevice, h->stream));
  Phys ph{};
  ph.u = p.u; ph.gamma = p.gamma; ph.gamma1 = p.gamma - 1.0; ph.grav = p.grav; ph.efix = p.efix;
  const double* aux = static_cast<const double*>(h->aux);
  auto vjp = [&](const double* s, const double* lam) {
    launch_vjp2d(s, lam, aux, T, h->pitch, h->plane, p.mx, p.my, p.dx, p.dy, dt, ph, p.char_decomp, h->stream, p.ndim);
  };
  double *cur = LA, *nxt = LB;
  if (ti == 4) {
    vjp(S[9], LIN);                                              // stage 10 (:457-462)
    launch_axpby(cur, 0.6, LIN, 0.1, T, nfield, h->stream);      // l9
    for (int k = 8; k >= 5; --k) {                               // s8, s7, s6, s5'
      vjp(S[k], cur);
      launch_axpby(nxt, 1.0, cur, sixth, T, nfield, h->stream);
      std::swap(cur, nxt);
    }
    launch_axpby(ACC, 0.6, cur, 0.04, LIN, nfield, h->stream);   // the s0 share of s5' and r1
    launch_axpby(nxt, 0.4, cur, 0.36, LIN, nfield, h->stream);   // l5
    std::swap(cur, nxt);
    for (int k = 4; k >= 1; --k) {                               // s4 .. s1
      vjp(S[k], cur);
      launch_axpby(nxt, 1.0, cur, sixth, T, nfield, h->stream);
      std::swap(cur, nxt);
    }
    vjp(S[0], cur);
    launch_axpby(nxt, 1.0, ACC, 1.0, cur, nfield, h->stream);
    launch_axpby(cur, 1.0, nxt, sixth, T, nfield, h->stream);    // l0
  } else if (ti == 1) {
    vjp(S[1], LIN);
    launch_axpby(cur, 0.5, LIN, 0.5, T, nfield, h->stream);      // l1
    vjp(S[0], cur);
    launch_axpby(nxt, 0.5, LIN, 1.0, cur, nfield, h->stream);
    launch_axpby(cur, 1.0, nxt, 1.0, T, nfield, h->stream);      // l0
  } else {
    vjp(S[3], LIN);
    launch_axpby(cur, 0.75, LIN, 0.25, T, nfield, h->stream);    // l3
    for (int k = 2; k >= 1; --k) {                               // s2, s1
      vjp(S[k], cur);
      launch_axpby(nxt, 1.0, cur, third, T, nfield, h->stream);
      std::swap(cur, nxt);
    }
    vjp(S[0], cur);
    launch_axpby(nxt, 0.25, LIN, 1.0, cur, nfield, h->stream);
    launch_axpby(cur, 1.0, nxt, third, T, nfield, h->stream);    // l0
  }
  CK(cudaGetLastError());
  CK(cudaMemcpy2DAsync(lam_out_dev, w, cur, sizeof(double) * h->pitch, w, (size_t)h->rows * p.meqn,
                       cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return SCL_OK;
}

}  // namespace

extern "C" int scl_adjoint_step(scl_handle* h, const double* q_dev, const double* lam_in_dev,
                                double* lam_out_dev, double dt) {
  if (!h || !q_dev || !lam_in_dev || !lam_out_dev) return fail(SCL_E_INVALID, "null argument");
  const scl_params& p = h->p;
  if (p.lim_type != 2 || !adjoint_supported(p.rp, p.ndim, p.char_decomp, p.time_integrator, p.mthbc))
    return fail(SCL_E_UNSUPPORTED,
                "the adjoint covers the acoustics plugins (1-D interface, 2-D), WENO5 componentwise or char-wise, periodic bc");
  if (h->ssize != sizeof(double)) return fail(SCL_E_UNSUPPORTED, "the adjoint needs double state");
  const long nfield = h->plane * p.meqn;
  const int nf = p.time_integrator == 3 ? 5 : 16;   // work fields
  if (!h->adj) {
    if (cudaMalloc(&h->adj, sizeof(double) * nfield * nf) != cudaSuccess)
      return fail(SCL_E_CUDA, "cudaMalloc adjoint fields");
    CK(cudaMemsetAsync(h->adj, 0, sizeof(double) * nfield * nf, h->stream));
  }
  if (p.time_integrator != 3) return adjoint_rk(h, q_dev, lam_in_dev, lam_out_dev, dt);
  double* L3 = h->adj;
  double* L2 = L3 + nfield;
  double* L1 = L2 + nfield;
  double* T = L1 + nfield;
  double* L0 = T + nfield;
  // q^n into the Q register, ghost cells filled, then the forward stages
  // q1 = q + D(q) (role A) and q2 = 3/4 q + 1/4 (q1 + D(q1)) (role B)
  Ctl* c = h->hctl;
  c->dt = dt;
  c->done = 0;
  c->status = 0;
  for (int s = 0; s < MAXSTAGES; ++s) c->stage_cfl[s] = 0.0;
  int rc = upload_ctl(h);
  if (rc) return rc;
  double* Q = static_cast<double*>(h->buf[c->role[ROLE_Q]]);
  rc = upload_field(h, Q, q_dev, p.meqn, true);
  if (rc) return rc;
  launch_bc<double>(h, Q);
  for (int s = 0; s < 2; ++s) h->L.stage(make_args(h, s), h->stream);
  CK(cudaGetLastError());
  const double* A = static_cast<const double*>(h->buf[c->role[ROLE_A]]);
  const double* B = static_cast<const double*>(h->buf[c->role[ROLE_B]]);
  const size_t w = sizeof(double) * h->ld;
  CK(cudaMemcpy2DAsync(L3, sizeof(double) * h->pitch, lam_in_dev, w, w, (size_t)h->rows * p.meqn,
                       cudaMemcpyDeviceToDevice, h->stream));
  Phys ph{};
  ph.u = p.u; ph.gamma = p.gamma; ph.gamma1 = p.gamma - 1.0; ph.grav = p.grav; ph.efix = p.efix;
  const double* aux = static_cast<const double*>(h->aux);
  launch_vjp2d(B, L3, aux, T, h->pitch, h->plane, p.mx, p.my, p.dx, p.dy, dt, ph, p.char_decomp, h->stream, p.ndim);
  launch_adj_combine(0, L2, L3, T, nfield, h->stream);          // l2 = 2/3 (l3 + D'(q2) l3)
  launch_vjp2d(A, L2, aux, T, h->pitch, h->plane, p.mx, p.my, p.dx, p.dy, dt, ph, p.char_decomp, h->stream, p.ndim);
  launch_adj_combine(1, L1, L2, T, nfield, h->stream);          // l1 = 1/4 (l2 + D'(q1) l2)
  launch_vjp2d(Q, L1, aux, T, h->pitch, h->plane, p.mx, p.my, p.dx, p.dy, dt, ph, p.char_decomp, h->stream, p.ndim);
  launch_adj_final(L0, L3, L2, L1, T, nfield, h->stream);       // l0 = l3/3 + 3/4 l2 + l1 + D'(q0) l1
  CK(cudaGetLastError());
  CK(cudaMemcpy2DAsync(lam_out_dev, w, L0, sizeof(double) * h->pitch, w, (size_t)h->rows * p.meqn,
                       cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return SCL_OK;
}
