// scl_batch.cu -- C ABI of the batched solver: many independent 1-D problems
// of uneven size advanced together, each with its own sharpclaw() controller.
//
// Device layout: four state arenas (register roles Q, A, B, R1); instance k
// occupies meqn planes of plane_k = round_up(mx_k + 6, 32) elements starting at
// off_k in every arena (256-byte aligned), so all of an instance's registers
// share one offset and a role swap is an index swap in ctl[k].
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "scl_batch.cuh"
#include "scl_launch.h"

using namespace scl;

namespace {

int bfail(int code, const std::string& m) {
  scl::set_last_error(m.c_str());
  return code;
}

#define BCK(call)                                                                       \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return bfail(SCL_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

// concatenated reference layout (double) -> arena (storage type), one CTA per instance
template <class S>
__global__ void k_scatter(const double* src, S* dst, const long* hoff, const long* off, const long* plane,
                          const int* mx, int meqn) {
  const int k = blockIdx.x;
  const long ld = mx[k] + 6;
  for (long e = threadIdx.x; e < ld * meqn; e += blockDim.x) {
    const long m = e / ld, i = e % ld;
    dst[off[k] + m * plane[k] + i] = (S)src[hoff[k] + e];
  }
}

// arena of role Q of each instance -> concatenated reference layout (double)
template <class S>
__global__ void k_gather(double* dst, void* const* arena, const Ctl* ctl, const long* hoff, const long* off,
                         const long* plane, const int* mx, int meqn) {
  const int k = blockIdx.x;
  const long ld = mx[k] + 6;
  const S* src = static_cast<const S*>(arena[ctl[k].role[ROLE_Q]]);
  for (long e = threadIdx.x; e < ld * meqn; e += blockDim.x) {
    const long m = e / ld, i = e % ld;
    dst[hoff[k] + e] = (double)src[off[k] + m * plane[k] + i];
  }
}

// bc1.f90 ghost fill of every instance's Q register (after an upload)
template <class S>
__global__ void k_batch_bc(void* const* arena, const Ctl* ctl, const long* off, const long* plane,
                           const int* mx, int meqn, int bl, int br) {
  const int k = blockIdx.x, t = threadIdx.x;
  if (t >= meqn * 3) return;
  const int m = t / 3, ibc = t % 3 + 1, n = mx[k];
  S* p = static_cast<S*>(arena[ctl[k].role[ROLE_Q]]) + off[k] + (long)m * plane[k];
  auto at = [&](int i) -> S& { return p[i + 2]; };
  if (bl == 1) at(1 - ibc) = at(1);
  else if (bl == 2) at(1 - ibc) = at(n + 1 - ibc);
  else if (bl == 3) at(1 - ibc) = (m == 1) ? -at(ibc) : at(ibc);
  if (br == 1) at(n + ibc) = at(n);
  else if (br == 2) at(n + ibc) = at(ibc);
  else if (br == 3) at(n + ibc) = (m == 1) ? -at(n + 1 - ibc) : at(n + 1 - ibc);
}

bool batch_launchers(int prec, int rp, int cd, int tf, int v, BatchLaunchers* L) {
  switch (prec) {
    case SCL_FP64: return get_batch_launchers_fp64(rp, cd, tf, v, L);
    case SCL_FP64_STRICT: return get_batch_launchers_fp64s(rp, cd, tf, v, L);
    case SCL_MIXED: return get_batch_launchers_mixed(rp, cd, tf, v, L);
    case SCL_FP32: return get_batch_launchers_fp32(rp, cd, tf, v, L);
  }
  return false;
}

// Stage tables of ts_ssp22/42/33/104 (src/sharpclaw.f90:247-464), the same as
// the single-grid solver's.
int batch_stage_table(int ti, StageDesc* sd, int* final_role) {
  int n = 0;
  auto S = [&](int k, int in, int out, int out2, int ai) { sd[n++] = StageDesc{k, in, out, out2, ai}; };
  switch (ti) {
    case 1: S(SK_ADD, ROLE_Q, ROLE_A, -1, -1); S(SK_SSP22_2, ROLE_A, ROLE_B, -1, ROLE_Q); *final_role = ROLE_B; break;
    case 2:
      S(SK_ADD_THIRD, ROLE_Q, ROLE_A, -1, -1); S(SK_ADD_THIRD, ROLE_A, ROLE_B, -1, -1);
      S(SK_ADD_THIRD, ROLE_B, ROLE_A, -1, -1); S(SK_SSP42_4, ROLE_A, ROLE_B, -1, ROLE_Q);
      *final_role = ROLE_B;
      break;
    case 3:
      S(SK_ADD, ROLE_Q, ROLE_A, -1, -1); S(SK_SSP33_2, ROLE_A, ROLE_B, -1, ROLE_Q);
      S(SK_SSP33_3, ROLE_B, ROLE_A, -1, ROLE_Q);
      *final_role = ROLE_A;
      break;
    case 4:
      S(SK_ADD_SIXTH, ROLE_Q, ROLE_A, -1, -1); S(SK_ADD_SIXTH, ROLE_A, ROLE_B, -1, -1);
      S(SK_ADD_SIXTH, ROLE_B, ROLE_A, -1, -1); S(SK_ADD_SIXTH, ROLE_A, ROLE_B, -1, -1);
      S(SK_SSP104_5, ROLE_B, ROLE_A, ROLE_R1, ROLE_Q); S(SK_ADD_SIXTH, ROLE_A, ROLE_B, -1, -1);
      S(SK_ADD_SIXTH, ROLE_B, ROLE_A, -1, -1); S(SK_ADD_SIXTH, ROLE_A, ROLE_B, -1, -1);
      S(SK_ADD_SIXTH, ROLE_B, ROLE_A, -1, -1); S(SK_SSP104_10, ROLE_A, ROLE_B, -1, ROLE_R1);
      *final_role = ROLE_B;
      break;
    default: return 0;
  }
  return n;
}

}  // namespace

struct scl_batch {
  scl_params p{};
  int ninst = 0;
  cudaStream_t stream = nullptr;
  size_t ss = 4;
  std::vector<int> mx;
  std::vector<double> dx;
  std::vector<long> off, aoff, plane, hoff, ahoff;
  long arena_elems = 0, aux_elems = 0, host_elems = 0, aux_host_elems = 0;
  void* arena[NROLES] = {nullptr, nullptr, nullptr, nullptr};
  void** d_arena = nullptr;
  void* aux = nullptr;
  double* staging = nullptr;   // concatenated reference layout, double
  Ctl* ctl = nullptr;
  Ctl* hctl = nullptr;         // pinned mirror
  long *d_off = nullptr, *d_aoff = nullptr, *d_plane = nullptr, *d_hoff = nullptr, *d_ahoff = nullptr;
  int* d_mx = nullptr;
  double* d_dx = nullptr;
  int *d_active = nullptr, *d_prefix = nullptr, *d_nact = nullptr, *h_nact = nullptr;
  BatchLaunchers L[NBATCH_VARIANTS];
  int nvariants = 0, variant = -1, grid[NBATCH_VARIANTS] = {};
  float tune_ms[NBATCH_VARIANTS] = {};
  long long last_launches = 0;   // kernel launches of the last scl_batch_run's replays
  StageDesc sd[MAXSTAGES];
  int nstages = 0, final_role = ROLE_A;
  cudaGraphExec_t graph = nullptr;
  int graph_steps = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evq[2] = {nullptr, nullptr};
};

namespace {

BatchArgs make_bargs(const scl_batch* b, int s) {
  BatchArgs a{};
  a.ctl = b->ctl;
  a.off = b->d_off;
  a.aoff = b->d_aoff;
  a.plane = b->d_plane;
  a.mx = b->d_mx;
  a.dx = b->d_dx;
  a.active = b->d_active;
  a.prefix = b->d_prefix;
  a.nact = b->d_nact;
  for (int r = 0; r < NROLES; ++r) a.arena[r] = b->arena[r];
  a.aux = b->p.maux > 0 ? b->aux : nullptr;
  a.sd = b->sd[s];
  a.stage = s;
  a.mthbc[0] = b->p.mthbc[0];
  a.mthbc[1] = b->p.mthbc[1];
  a.mcapa = b->p.mcapa;
  a.ph.u = b->p.u;
  a.ph.gamma = b->p.gamma;
  a.ph.gamma1 = b->p.gamma - 1.0;
  a.ph.grav = b->p.grav;
  a.ph.efix = b->p.efix;
  for (int k = 0; k < 4; ++k) a.ph.mthlim[k] = b->p.mthlim[k];
  return a;
}

// One batch step.  Inside a graph of several steps, a step after the first
// ends its predecessor in its begin kernel (first = false) and only the last
// step launches k_batch_end.
int enqueue_batch_step(scl_batch* b, int v, bool first = true, bool last = true) {
  const BatchLaunchers& L = b->L[v];
  L.begin(b->ctl, b->d_mx, b->ninst, b->d_active, b->d_prefix, b->d_nact, first ? -1 : b->nstages - 1,
          b->final_role, b->stream);
  for (int s = 0; s < b->nstages; ++s) L.stage(make_bargs(b, s), b->grid[v], b->stream);
  if (last)
    k_batch_end<<<(b->ninst + 255) / 256, 256, 0, b->stream>>>(b->ctl, b->ninst, b->nstages - 1, b->final_role);
  BCK(cudaGetLastError());
  return SCL_OK;
}

int upload_batch_ctl(scl_batch* b) {
  BCK(cudaMemcpyAsync(b->ctl, b->hctl, sizeof(Ctl) * b->ninst, cudaMemcpyHostToDevice, b->stream));
  return SCL_OK;
}

int download_batch_ctl(scl_batch* b) {
  BCK(cudaMemcpyAsync(b->hctl, b->ctl, sizeof(Ctl) * b->ninst, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return SCL_OK;
}

template <class S>
void launch_scatter_bc(scl_batch* b) {
  k_scatter<S><<<b->ninst, 256, 0, b->stream>>>(b->staging, static_cast<S*>(b->arena[0]), b->d_hoff, b->d_off,
                                                 b->d_plane, b->d_mx, b->p.meqn);
  k_batch_bc<S><<<b->ninst, 32, 0, b->stream>>>(b->d_arena, b->ctl, b->d_off, b->d_plane, b->d_mx, b->p.meqn,
                                                 b->p.mthbc[0], b->p.mthbc[1]);
}

// put the staging copy (concatenated layout, device) into arena 0 with
// identity roles and filled ghost cells
int restore_from_staging(scl_batch* b) {
  for (int k = 0; k < b->ninst; ++k)
    for (int r = 0; r < NROLES; ++r) b->hctl[k].role[r] = r;
  int rc = upload_batch_ctl(b);
  if (rc) return rc;
  if (b->ss == sizeof(double)) launch_scatter_bc<double>(b);
  else launch_scatter_bc<float>(b);
  BCK(cudaGetLastError());
  return SCL_OK;
}

int gather_to_staging(scl_batch* b) {
  if (b->ss == sizeof(double))
    k_gather<double><<<b->ninst, 256, 0, b->stream>>>(b->staging, b->d_arena, b->ctl, b->d_hoff, b->d_off,
                                                       b->d_plane, b->d_mx, b->p.meqn);
  else
    k_gather<float><<<b->ninst, 256, 0, b->stream>>>(b->staging, b->d_arena, b->ctl, b->d_hoff, b->d_off,
                                                      b->d_plane, b->d_mx, b->p.meqn);
  BCK(cudaGetLastError());
  return SCL_OK;
}

// controller start values of every instance (sharpclaw.f90:35-64); roles kept
void init_batch_ctl(scl_batch* b, const scl_run* run, const double* dt0, std::vector<int>& early_info) {
  early_info.assign(b->ninst, 0);
  for (int k = 0; k < b->ninst; ++k) {
    Ctl& c = b->hctl[k];
    int roles[NROLES];
    memcpy(roles, c.role, sizeof(roles));
    const double dti = dt0 ? dt0[k] : run->dt_initial;
    memset(&c, 0, sizeof(Ctl));
    memcpy(c.role, roles, sizeof(roles));
    c.t = c.told = c.tstart = run->tstart;
    c.tend = run->tend;
    c.dt = dti;
    c.dt_max = run->dt_max;
    c.cfl_max = run->cfl_max;
    c.cfl_desired = run->cfl_desired;
    c.dtmin = c.dtmax = dti;
    c.maxn = run->max_steps;
    c.dt_variable = run->dt_variable;
    if (run->dt_variable == 0) {
      if (run->tend < run->tstart) {
        c.maxn = 1;
      } else {
        c.maxn = (int)((run->tend - run->tstart + 1e-10) / dti);
        if (std::fabs(c.maxn * dti - (run->tend - run->tstart)) > 1e-5 * (run->tend - run->tstart)) {
          early_info[k] = SCL_INFO_DT_NOT_DIVIDING;
          c.done = 1;
        }
      }
    }
    if (run->dt_variable == 1 && run->cfl_desired > run->cfl_max) {
      early_info[k] = SCL_INFO_CFL_DESIRED_GT_MAX;
      c.done = 1;
    }
  }
}

int build_batch_graph(scl_batch* b, int steps) {
  if (b->graph && b->graph_steps == steps) return SCL_OK;
  if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
  cudaGraph_t g = nullptr;
  BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int rc = SCL_OK;
  for (int k = 0; k < steps && rc == SCL_OK; ++k) rc = enqueue_batch_step(b, b->variant, k == 0, k == steps - 1);
  cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (rc) { if (g) cudaGraphDestroy(g); return rc; }
  if (e != cudaSuccess) return bfail(SCL_E_CUDA, std::string("capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return bfail(SCL_E_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
  b->graph_steps = steps;
  return SCL_OK;
}

// Autotuner: time a few steps of each tile width from the same start state
// and keep the faster (the start state and controllers are restored after
// every trial).
int autotune(scl_batch* b, const std::vector<Ctl>& start, int trial_steps) {
  int rc = gather_to_staging(b);
  if (rc) return rc;
  float best = 1e30f;
  int bestv = 0;
  for (int v = 0; v < b->nvariants; ++v) {
    memcpy(b->hctl, start.data(), sizeof(Ctl) * b->ninst);
    rc = restore_from_staging(b);
    if (rc) return rc;
    rc = enqueue_batch_step(b, v);   // warm-up step
    if (rc) return rc;
    BCK(cudaEventRecord(b->ev0, b->stream));
    for (int s = 0; s < trial_steps && rc == SCL_OK; ++s) rc = enqueue_batch_step(b, v);
    if (rc) return rc;
    BCK(cudaEventRecord(b->ev1, b->stream));
    BCK(cudaEventSynchronize(b->ev1));
    float ms = 0;
    BCK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    b->tune_ms[v] = ms;
    if (ms < best) { best = ms; bestv = v; }
  }
  memcpy(b->hctl, start.data(), sizeof(Ctl) * b->ninst);
  rc = restore_from_staging(b);
  if (rc) return rc;
  b->variant = bestv;
  return SCL_OK;
}

}  // namespace

extern "C" {

int scl_batch_destroy(scl_batch* b) {
  if (!b) return SCL_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  for (int r = 0; r < NROLES; ++r) cudaFree(b->arena[r]);
  cudaFree(b->d_arena);
  cudaFree(b->aux);
  cudaFree(b->staging);
  cudaFree(b->ctl);
  cudaFree(b->d_off); cudaFree(b->d_aoff); cudaFree(b->d_plane); cudaFree(b->d_hoff); cudaFree(b->d_ahoff);
  cudaFree(b->d_mx); cudaFree(b->d_dx);
  cudaFree(b->d_active); cudaFree(b->d_prefix); cudaFree(b->d_nact);
  if (b->hctl) cudaFreeHost(b->hctl);
  if (b->h_nact) cudaFreeHost(b->h_nact);
  for (cudaEvent_t e : {b->ev0, b->ev1, b->evq[0], b->evq[1]}) if (e) cudaEventDestroy(e);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return SCL_OK;
}

int scl_batch_create(const scl_params* p, int ninst, const int* mx, const double* dx, scl_batch** out) {
  if (!p || !mx || !dx || !out || ninst < 1) return bfail(SCL_E_INVALID, "bad argument");
  *out = nullptr;
  if (p->ndim != 1) return bfail(SCL_E_INVALID, "batched solver takes 1-D problems");
  if (p->lim_type == 0) return bfail(SCL_E_UNSUPPORTED, "no polynomial reconstruction (lim_type 0) in the batched solver");
  if (p->mbc != 3 || (p->lim_type != 1 && p->lim_type != 2)) return bfail(SCL_E_INVALID, "need mbc = 3 and lim_type 1 or 2");
  if (p->char_decomp < 0 || p->char_decomp > (p->lim_type == 2 ? 3 : 2)) return bfail(SCL_E_UNSUPPORTED, "char_decomp out of range");
  if (p->precision < SCL_FP64 || p->precision > SCL_FP32) return bfail(SCL_E_INVALID, "bad precision");
  for (int k = 0; k < 2; ++k)
    if (p->mthbc[k] < 1 || p->mthbc[k] > 3 || (p->mthbc[k] == 3 && p->meqn < 2))
      return bfail(SCL_E_INVALID, "mthbc must be 1, 2 or 3 (a wall needs meqn >= 2)");
  if ((p->mthbc[0] == 2) != (p->mthbc[1] == 2)) return bfail(SCL_E_INVALID, "periodic bc on one side only");
  struct { int rp, meqn, mwaves, maux; } tab[] = {
      {SCL_RP_ADVECTION, 1, 1, 0}, {SCL_RP_EULER, 3, 3, 0}, {SCL_RP_ACOUSTICS1D, 2, 2, 2}};
  bool ok = false;
  for (auto& t : tab)
    if (t.rp == p->rp) {
      ok = p->meqn == t.meqn && p->mwaves == t.mwaves && p->maux >= t.maux;
      if (!ok) return bfail(SCL_E_INVALID, "meqn/mwaves/maux do not match the plugin");
    }
  if (!ok) return bfail(SCL_E_INVALID, "batched solver takes the 1-D plugins");
  if (p->mcapa < 0 || p->mcapa > p->maux) return bfail(SCL_E_INVALID, "mcapa out of range");
  if (p->src_term != SCL_SRC_NONE) return bfail(SCL_E_UNSUPPORTED, "no source-term hooks in the batched solver");
  if (p->bc_user != SCL_BC_USER_NONE) return bfail(SCL_E_UNSUPPORTED, "no user bc in the batched solver");
  for (int k = 0; k < ninst; ++k) {
    if (mx[k] < 3) return bfail(SCL_E_INVALID, "every instance needs mx >= 3");
    if (!(dx[k] > 0)) return bfail(SCL_E_INVALID, "every instance needs dx > 0");
  }
  scl_batch* b = new scl_batch();
  b->p = *p;
  b->ninst = ninst;
  b->ss = p->precision == SCL_FP32 ? sizeof(float) : sizeof(double);
  b->nstages = batch_stage_table(p->time_integrator, b->sd, &b->final_role);
  if (!b->nstages) { delete b; return bfail(SCL_E_INVALID, "time_integrator should be between 1 and 4"); }
  for (int v = 0; v < NBATCH_VARIANTS; ++v)
    if ((v < 2 || p->mcapa == 0) &&   // the paired tile (variant 2) has no capacity form
        batch_launchers(p->precision, p->rp, p->lim_type == 1 ? 10 + p->char_decomp : p->char_decomp,
                        p->tfluct_solver, v, &b->L[v]))
      b->nvariants = v + 1;
  if (b->nvariants == 0) { delete b; return bfail(SCL_E_UNSUPPORTED, "no batched kernel for this plugin / options"); }
  b->mx.assign(mx, mx + ninst);
  b->dx.assign(dx, dx + ninst);
  const int maux = std::max(1, p->maux);
  for (int k = 0; k < ninst; ++k) {
    const long ld = mx[k] + 6, pl = (ld + 31) / 32 * 32;
    b->plane.push_back(pl);
    b->off.push_back(b->arena_elems);
    b->aoff.push_back(b->aux_elems);
    b->hoff.push_back(b->host_elems);
    b->ahoff.push_back(b->aux_host_elems);
    b->arena_elems += pl * p->meqn;
    b->aux_elems += pl * maux;
    b->host_elems += ld * p->meqn;
    b->aux_host_elems += ld * maux;
  }
  auto cleanup = [&](int code) { scl_batch_destroy(b); return code; };
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
    return cleanup(bfail(SCL_E_CUDA, "stream create"));
  bool okm = true;
  for (int r = 0; r < NROLES; ++r) okm &= cudaMalloc(&b->arena[r], b->ss * b->arena_elems) == cudaSuccess;
  okm &= cudaMalloc(&b->d_arena, sizeof(void*) * NROLES) == cudaSuccess;
  okm &= cudaMalloc(&b->aux, b->ss * b->aux_elems) == cudaSuccess;
  okm &= cudaMalloc(&b->staging, sizeof(double) * std::max(b->host_elems, b->aux_host_elems)) == cudaSuccess;
  okm &= cudaMalloc(&b->ctl, sizeof(Ctl) * ninst) == cudaSuccess;
  okm &= cudaMalloc(&b->d_off, sizeof(long) * ninst) == cudaSuccess;
  okm &= cudaMalloc(&b->d_aoff, sizeof(long) * ninst) == cudaSuccess;
  okm &= cudaMalloc(&b->d_plane, sizeof(long) * ninst) == cudaSuccess;
  okm &= cudaMalloc(&b->d_hoff, sizeof(long) * ninst) == cudaSuccess;
  okm &= cudaMalloc(&b->d_ahoff, sizeof(long) * ninst) == cudaSuccess;
  okm &= cudaMalloc(&b->d_mx, sizeof(int) * ninst) == cudaSuccess;
  okm &= cudaMalloc(&b->d_dx, sizeof(double) * ninst) == cudaSuccess;
  okm &= cudaMalloc(&b->d_active, sizeof(int) * ninst) == cudaSuccess;
  okm &= cudaMalloc(&b->d_prefix, sizeof(int) * (ninst + 1)) == cudaSuccess;
  okm &= cudaMalloc(&b->d_nact, sizeof(int)) == cudaSuccess;
  okm &= cudaMallocHost(&b->hctl, sizeof(Ctl) * ninst) == cudaSuccess;
  okm &= cudaMallocHost(&b->h_nact, 2 * sizeof(int)) == cudaSuccess;
  if (!okm) return cleanup(bfail(SCL_E_CUDA, "device allocation for the batch failed"));
  for (int r = 0; r < NROLES; ++r) cudaMemsetAsync(b->arena[r], 0, b->ss * b->arena_elems, b->stream);
  cudaMemsetAsync(b->aux, 0, b->ss * b->aux_elems, b->stream);
  cudaMemcpyAsync(b->d_arena, b->arena, sizeof(void*) * NROLES, cudaMemcpyHostToDevice, b->stream);
  cudaMemcpyAsync(b->d_off, b->off.data(), sizeof(long) * ninst, cudaMemcpyHostToDevice, b->stream);
  cudaMemcpyAsync(b->d_aoff, b->aoff.data(), sizeof(long) * ninst, cudaMemcpyHostToDevice, b->stream);
  cudaMemcpyAsync(b->d_plane, b->plane.data(), sizeof(long) * ninst, cudaMemcpyHostToDevice, b->stream);
  cudaMemcpyAsync(b->d_hoff, b->hoff.data(), sizeof(long) * ninst, cudaMemcpyHostToDevice, b->stream);
  cudaMemcpyAsync(b->d_ahoff, b->ahoff.data(), sizeof(long) * ninst, cudaMemcpyHostToDevice, b->stream);
  cudaMemcpyAsync(b->d_mx, b->mx.data(), sizeof(int) * ninst, cudaMemcpyHostToDevice, b->stream);
  cudaMemcpyAsync(b->d_dx, b->dx.data(), sizeof(double) * ninst, cudaMemcpyHostToDevice, b->stream);
  memset(b->hctl, 0, sizeof(Ctl) * ninst);
  for (int k = 0; k < ninst; ++k) {
    for (int r = 0; r < NROLES; ++r) b->hctl[k].role[r] = r;
    b->hctl[k].done = 1;
  }
  int rc = upload_batch_ctl(b);
  if (rc) return cleanup(rc);
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  for (int v = 0; v < b->nvariants; ++v) b->grid[v] = std::max(1, b->L[v].blocks_per_sm()) * nsm;
  cudaEventCreate(&b->ev0);
  cudaEventCreate(&b->ev1);
  cudaEventCreateWithFlags(&b->evq[0], cudaEventDisableTiming);
  cudaEventCreateWithFlags(&b->evq[1], cudaEventDisableTiming);
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return cleanup(bfail(SCL_E_CUDA, "batch create sync"));
  *out = b;
  return SCL_OK;
}

int scl_batch_set_q(scl_batch* b, const double* q) {
  if (!b || !q) return bfail(SCL_E_INVALID, "null argument");
  BCK(cudaMemcpyAsync(b->staging, q, sizeof(double) * b->host_elems, cudaMemcpyHostToDevice, b->stream));
  int rc = restore_from_staging(b);
  if (rc) return rc;
  BCK(cudaStreamSynchronize(b->stream));
  return SCL_OK;
}

int scl_batch_get_q(scl_batch* b, double* q) {
  if (!b || !q) return bfail(SCL_E_INVALID, "null argument");
  int rc = gather_to_staging(b);
  if (rc) return rc;
  BCK(cudaMemcpyAsync(q, b->staging, sizeof(double) * b->host_elems, cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return SCL_OK;
}

int scl_batch_set_aux(scl_batch* b, const double* aux) {
  if (!b || !aux) return bfail(SCL_E_INVALID, "null argument");
  if (b->p.maux == 0) return SCL_OK;
  BCK(cudaMemcpyAsync(b->staging, aux, sizeof(double) * b->aux_host_elems, cudaMemcpyHostToDevice, b->stream));
  if (b->ss == sizeof(double))
    k_scatter<double><<<b->ninst, 256, 0, b->stream>>>(b->staging, static_cast<double*>(b->aux), b->d_ahoff,
                                                        b->d_aoff, b->d_plane, b->d_mx, b->p.maux);
  else
    k_scatter<float><<<b->ninst, 256, 0, b->stream>>>(b->staging, static_cast<float*>(b->aux), b->d_ahoff,
                                                       b->d_aoff, b->d_plane, b->d_mx, b->p.maux);
  BCK(cudaGetLastError());
  BCK(cudaStreamSynchronize(b->stream));
  return SCL_OK;
}

int scl_batch_run(scl_batch* b, const scl_run* run, const double* dt_initial, scl_result* res, float* ms) {
  if (!b || !run || !res) return bfail(SCL_E_INVALID, "null argument");
  int rc = download_batch_ctl(b);   // current roles
  if (rc) return rc;
  std::vector<int> early;
  init_batch_ctl(b, run, dt_initial, early);
  std::vector<Ctl> start(b->hctl, b->hctl + b->ninst);
  if (b->variant < 0) {
    rc = autotune(b, start, 3);
    if (rc) return rc;
  } else {
    rc = upload_batch_ctl(b);
    if (rc) return rc;
  }
  const int K = std::max(1, 160 / (b->nstages + 1));
  rc = build_batch_graph(b, K);
  if (rc) return rc;
  int maxn = 0;
  for (int k = 0; k < b->ninst; ++k) maxn = std::max(maxn, b->hctl[k].maxn);
  const long max_replays = (long)maxn / K + 2;
  BCK(cudaEventRecord(b->ev0, b->stream));
  b->h_nact[0] = b->h_nact[1] = 1;
  long replays = 0;
  for (long r = 0; r < max_replays; ++r) {
    BCK(cudaGraphLaunch(b->graph, b->stream));
    ++replays;
    BCK(cudaMemcpyAsync(&b->h_nact[r & 1], b->d_nact, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaEventRecord(b->evq[r & 1], b->stream));
    if (r > 0) {
      BCK(cudaEventSynchronize(b->evq[(r - 1) & 1]));
      if (b->h_nact[(r - 1) & 1] == 0) break;
    }
  }
  BCK(cudaEventRecord(b->ev1, b->stream));
  BCK(cudaEventSynchronize(b->ev1));
  if (ms) BCK(cudaEventElapsedTime(ms, b->ev0, b->ev1));
  // per replay: K begins (each but the first also ends a step), K * nstages stages, one end
  b->last_launches = (long long)replays * (K * (b->nstages + 1) + 1);
  rc = download_batch_ctl(b);
  if (rc) return rc;
  for (int k = 0; k < b->ninst; ++k) {
    const Ctl& c = b->hctl[k];
    scl_result& r = res[k];
    int info = early[k] ? early[k] : c.info;
    if (!info) {
      if (c.dt_variable == 1 && c.t < c.tend && c.steps_taken == c.maxn) info = SCL_INFO_TOO_MANY_STEPS;
      if (c.dt_variable == 0 && c.cflmax > c.cfl_max) info = SCL_INFO_CFL_FIXED_DT;
    }
    r.tend = c.t;
    r.cfl_maxused = c.cflmax;
    r.cfl_last = c.cfl_last;
    r.dt_minused = c.dtmin;
    r.dt_maxused = c.dtmax;
    r.dt_last = c.dt;
    r.steps_taken = c.steps_taken;
    r.info = info;
    r.rejected = c.rejected;
    r.status = c.status;
  }
  return SCL_OK;
}

long long scl_batch_launches(scl_batch* b) { return b ? b->last_launches : 0; }

int scl_batch_select(scl_batch* b, int variant) {
  if (!b) return bfail(SCL_E_INVALID, "null argument");
  if (variant < -1 || variant >= b->nvariants) return bfail(SCL_E_UNSUPPORTED, "no such tile variant");
  BCK(cudaStreamSynchronize(b->stream));
  b->variant = variant;
  for (int v = 0; v < NBATCH_VARIANTS; ++v) b->tune_ms[v] = 0.0f;
  if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
  return SCL_OK;
}

int scl_batch_tuning(scl_batch* b, int* variant, int* threads, int* grid, float* trial_ms) {
  if (!b) return bfail(SCL_E_INVALID, "null argument");
  if (variant) *variant = b->variant;
  if (threads) *threads = b->variant >= 0 ? b->L[b->variant].nt : 0;
  if (grid) *grid = b->variant >= 0 ? b->grid[b->variant] : 0;
  if (trial_ms)
    for (int v = 0; v < NBATCH_VARIANTS; ++v) trial_ms[v] = v < b->nvariants ? b->tune_ms[v] : 0.0f;
  return SCL_OK;
}

}  // extern "C"
