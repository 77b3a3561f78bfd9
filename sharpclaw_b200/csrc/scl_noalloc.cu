// scl_noalloc.cu -- one SSP-RK time step of a 1-D grid that allocates nothing.
//
// Some callers cannot call cudaMalloc: a Fortran time loop that calls the
// step from inside code that must not synchronise the device (cudaMalloc and
// cudaFree can stall every stream of the device), hosts that give each
// library a fixed memory budget decided at start-up, and callers that hand us
// memory from their own pool and forbid any other device allocation after
// initialisation.  scl_rk_step_noalloc serves them: the caller passes its own
// device array q (in and out) and aux, and the stage registers the Runge-Kutta
// stages need live in a file-scope device array of fixed size that exists as
// soon as the library's device code is loaded on a GPU.  It has no counterpart
// in the reference.
//
// Rules of use:
//  * at most SCL_NOALLOC_MAX_VALUES = meqn*(mx+2*mbc) values per grid; larger
//    grids are rejected with SCL_E_INVALID;
//  * all calls on one GPU share the one scratch array, so two calls whose work
//    overlaps on that GPU (different streams, or threads) race and corrupt
//    each other: serialise them;
//  * the first call on each device looks up the scratch array's device
//    address with cudaGetSymbolAddress (with that device current); make this
//    first call before any stream capture is started on that thread.  The
//    address is kept for the life of the process: a device reset
//    (cudaDeviceReset) after the first call invalidates it, so do not reset
//    a device this library has stepped on;
//  * q_dev and aux_dev must be device (or managed) allocations of the current
//    device; any other pointer is refused before anything is launched;
//  * a CUDA error left pending by the caller's earlier work is reported (and
//    left in place) instead of being taken for a failure of this call;
//  * with cfl == NULL the call returns once the step is enqueued: it then
//    reports neither a non-finite state nor an asynchronous kernel error.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "scl_common.cuh"
#include "scl_launch.h"

using namespace scl;

namespace {

// Three stage registers (A, B, R1) of at most SCL_NOALLOC_MAX_VALUES doubles
// each, plus the controller block that carries dt, the buffer roles and the
// per-stage CFL numbers: 3 * 196608 * 8 B + 512 B = 4.5 MiB + 512 B per GPU.
constexpr long kMaxValues = SCL_NOALLOC_MAX_VALUES;
constexpr size_t kCtlBytes = 512;
static_assert(sizeof(Ctl) <= kCtlBytes, "controller block does not fit its scratch slot");
constexpr size_t kScratchBytes = kCtlBytes + 3 * sizeof(double) * kMaxValues;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};   // device address of g_noalloc_scratch per device

// errors are reported through scl_last_error(), like every other entry point
int fail_na(int code, const std::string& m) {
  scl::set_last_error(m.c_str());
  return code;
}

// Resolve the scratch array's device address once per device.
int scratch_for_current_device(void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail_na(SCL_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail_na(SCL_E_INVALID, "device index out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail_na(SCL_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return SCL_OK;
}

// Controller block for a single step: dt, identity roles, zeroed CFL slots
// and status (the scratch keeps the previous call's contents).
__global__ void k_noalloc_init(Ctl* c, double dt) {
  Ctl z{};
  z.dt = dt;
  z.t = dt;
  for (int r = 0; r < NROLES; ++r) z.role[r] = r;
  *c = z;
}

// bc1.f90 ghost fill of the caller's q before the first stage.
__global__ void k_noalloc_bc1(double* q, long plane, int mx, int meqn, int bl, int br) {
  const int t = threadIdx.x;
  if (t >= meqn * 3) return;
  const int m = t / 3, ibc = t % 3 + 1;
  double* p = q + (long)m * plane;
  auto at = [&](int i) -> double& { return p[i + 2]; };
  if (bl == 1) at(1 - ibc) = at(1);
  else if (bl == 2) at(1 - ibc) = at(mx + 1 - ibc);
  else if (bl == 3) at(1 - ibc) = (m == 1) ? -at(ibc) : at(ibc);
  if (br == 1) at(mx + ibc) = at(mx);
  else if (br == 2) at(mx + ibc) = at(ibc);
  else if (br == 3) at(mx + ibc) = (m == 1) ? -at(mx + 1 - ibc) : at(mx + 1 - ibc);
}

// The same stage sequences as ts_ssp22/42/33/104 (src/sharpclaw.f90:247-464)
// on roles Q (the caller's q), A, B, R1; the final stage writes back into Q,
// which it only reads pointwise (as qold) or not at all.
int noalloc_table(int ti, StageDesc* sd) {
  int n = 0;
  auto S = [&](int k, int in, int out, int out2, int ai) { sd[n++] = StageDesc{k, in, out, out2, ai}; };
  switch (ti) {
    case 1:
      S(SK_ADD, ROLE_Q, ROLE_A, -1, -1);
      S(SK_SSP22_2, ROLE_A, ROLE_Q, -1, ROLE_Q);
      break;
    case 2:
      S(SK_ADD_THIRD, ROLE_Q, ROLE_A, -1, -1);
      S(SK_ADD_THIRD, ROLE_A, ROLE_B, -1, -1);
      S(SK_ADD_THIRD, ROLE_B, ROLE_A, -1, -1);
      S(SK_SSP42_4, ROLE_A, ROLE_Q, -1, ROLE_Q);
      break;
    case 3:
      S(SK_ADD, ROLE_Q, ROLE_A, -1, -1);
      S(SK_SSP33_2, ROLE_A, ROLE_B, -1, ROLE_Q);
      S(SK_SSP33_3, ROLE_B, ROLE_Q, -1, ROLE_Q);
      break;
    case 4:
      S(SK_ADD_SIXTH, ROLE_Q, ROLE_A, -1, -1);
      S(SK_ADD_SIXTH, ROLE_A, ROLE_B, -1, -1);
      S(SK_ADD_SIXTH, ROLE_B, ROLE_A, -1, -1);
      S(SK_ADD_SIXTH, ROLE_A, ROLE_B, -1, -1);
      S(SK_SSP104_5, ROLE_B, ROLE_A, ROLE_R1, ROLE_Q);
      S(SK_ADD_SIXTH, ROLE_A, ROLE_B, -1, -1);
      S(SK_ADD_SIXTH, ROLE_B, ROLE_A, -1, -1);
      S(SK_ADD_SIXTH, ROLE_A, ROLE_B, -1, -1);
      S(SK_ADD_SIXTH, ROLE_B, ROLE_A, -1, -1);
      S(SK_SSP104_10, ROLE_A, ROLE_Q, -1, ROLE_R1);
      break;
    default:
      return 0;
  }
  return n;
}

// A caller pointer the stage kernels may dereference: a device or managed
// allocation of the current device.  Host memory (pageable or pinned) and
// other devices' memory are refused with SCL_E_INVALID before any launch.
int check_device_pointer(const void* p, const char* name) {
  cudaPointerAttributes at{};
  cudaError_t e = cudaPointerGetAttributes(&at, p);
  if (e != cudaSuccess) {
    cudaGetLastError();   // the query's own error (none was pending before it)
    return fail_na(SCL_E_INVALID, std::string(name) + " is not a device allocation (cudaPointerGetAttributes: " +
                                      cudaGetErrorString(e) + ")");
  }
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return fail_na(SCL_E_INVALID, "no current CUDA device");
  }
  if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)
    return fail_na(SCL_E_INVALID, std::string(name) + " is not device or managed memory");
  if (at.type == cudaMemoryTypeDevice && at.device != dev)
    return fail_na(SCL_E_INVALID, std::string(name) + " belongs to another device");
  return SCL_OK;
}

bool launchers_for(int prec, int rp, int cd, int tf, Launchers* L) {
  switch (prec) {
    case SCL_FP64: return get_launchers_fp64(rp, 1, cd, tf, 0, L);
    case SCL_FP64_STRICT: return get_launchers_fp64s(rp, 1, cd, tf, 0, L);
    case SCL_MIXED: return get_launchers_mixed(rp, 1, cd, tf, 0, L);
  }
  return false;
}

}  // namespace

extern "C" int scl_rk_step_noalloc(const scl_params* p, double* q_dev, const double* aux_dev,
                                   double dt, double* cfl, void* stream) {
  if (!p || !q_dev) return fail_na(SCL_E_INVALID, "null argument");
  if (p->ndim != 1) return fail_na(SCL_E_INVALID, "scl_rk_step_noalloc takes 1-D grids only");
  if (p->mbc != 3 || p->mx < 3) return fail_na(SCL_E_INVALID, "need mbc = 3 and mx >= 3");
  if (p->precision == SCL_FP32)
    return fail_na(SCL_E_UNSUPPORTED, "scl_rk_step_noalloc works on double state (FP64, FP64_STRICT, MIXED)");
  if (p->lim_type != 2 || (p->char_decomp != 0 && p->char_decomp != 2))
    return fail_na(SCL_E_UNSUPPORTED, "only WENO5 with char_decomp 0 or 2");
  for (int k = 0; k < 2; ++k)
    if (p->mthbc[k] < 1 || p->mthbc[k] > 3 || (p->mthbc[k] == 3 && p->meqn < 2))
      return fail_na(SCL_E_INVALID, "mthbc must be 1, 2 or 3 (a wall needs meqn >= 2)");
  if ((p->mthbc[0] == 2) != (p->mthbc[1] == 2)) return fail_na(SCL_E_INVALID, "periodic bc on one side only");
  if (p->maux > 0 && !aux_dev) return fail_na(SCL_E_INVALID, "aux_dev required when maux > 0");
  if (p->mcapa < 0 || p->mcapa > p->maux) return fail_na(SCL_E_INVALID, "mcapa out of range");
  if (p->src_term != SCL_SRC_NONE) return fail_na(SCL_E_UNSUPPORTED, "no source-term hooks in scl_rk_step_noalloc");
  if (p->bc_user != SCL_BC_USER_NONE) return fail_na(SCL_E_UNSUPPORTED, "no user bc in scl_rk_step_noalloc");
  const long ld = (long)p->mx + 2 * p->mbc;
  // the kernels read exactly the plugin's number of components and aux fields
  struct { int rp, meqn, mwaves, maux; } tab[] = {
      {SCL_RP_ADVECTION, 1, 1, 0}, {SCL_RP_EULER, 3, 3, 0}, {SCL_RP_ACOUSTICS1D, 2, 2, 2}};
  bool known = false;
  for (auto& t : tab)
    if (t.rp == p->rp) {
      known = true;
      if (p->meqn != t.meqn || p->mwaves != t.mwaves || p->maux < t.maux)
        return fail_na(SCL_E_INVALID, "meqn/mwaves/maux do not match the plugin");
    }
  if (!known) return fail_na(SCL_E_INVALID, "scl_rk_step_noalloc takes the 1-D plugins only");
  if (p->rp == SCL_RP_EULER && p->tfluct_solver == 1)
    return fail_na(SCL_E_INVALID, "no tfluct exists for the Euler plugin");
  if ((long)p->meqn * ld > kMaxValues)
    return fail_na(SCL_E_INVALID, "grid too large for scl_rk_step_noalloc: meqn*(mx+2*mbc) = " +
                                      std::to_string((long)p->meqn * ld) + " exceeds " +
                                      std::to_string(kMaxValues) + " values");
  Launchers L{};
  if (!launchers_for(p->precision, p->rp, p->char_decomp, p->tfluct_solver, &L))
    return fail_na(SCL_E_UNSUPPORTED, "no kernel for this plugin / char_decomp / tfluct_solver");
  StageDesc sd[MAXSTAGES];
  const int ns = noalloc_table(p->time_integrator, sd);
  if (ns == 0) return fail_na(SCL_E_INVALID, "time_integrator should be between 1 and 4");

  // an error left by the caller's earlier work stays the caller's
  cudaError_t pend = cudaPeekAtLastError();
  if (pend == cudaErrorNoDevice || pend == cudaErrorInsufficientDriver)
    return fail_na(SCL_E_CUDA, std::string("no usable CUDA device: ") + cudaGetErrorString(pend));
  if (pend != cudaSuccess)
    return fail_na(SCL_E_CUDA, std::string("a CUDA error was pending before this call (left in place): ") +
                                   cudaGetErrorString(pend));
  int rc0 = check_device_pointer(q_dev, "q_dev");
  if (rc0 == SCL_OK && p->maux > 0) rc0 = check_device_pointer(aux_dev, "aux_dev");
  if (rc0) return rc0;

  void* base = nullptr;
  int rc = scratch_for_current_device(&base);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  Ctl* ctl = static_cast<Ctl*>(base);
  double* regs = reinterpret_cast<double*>(static_cast<unsigned char*>(base) + kCtlBytes);
  const long nval = (long)p->meqn * ld;

  k_noalloc_init<<<1, 1, 0, st>>>(ctl, dt);
  k_noalloc_bc1<<<1, 32, 0, st>>>(q_dev, ld, p->mx, p->meqn, p->mthbc[0], p->mthbc[1]);
  for (int s = 0; s < ns; ++s) {
    StageArgs a{};
    a.ctl = ctl;
    a.buf[ROLE_Q] = q_dev;
    a.buf[ROLE_A] = regs;
    a.buf[ROLE_B] = regs + nval;
    a.buf[ROLE_R1] = regs + 2 * nval;
    a.aux = aux_dev;
    a.dq_out = nullptr;
    a.sd = sd[s];
    a.stage = s;
    a.ixy = 1;
    a.mx = p->mx;
    a.my = 1;
    a.pitch = ld;
    a.plane = ld;
    a.dx = p->dx;
    a.dy = p->dx;
    for (int k = 0; k < 4; ++k) a.mthbc[k] = p->mthbc[k];
    a.mcapa = p->mcapa;
    a.ph.u = p->u;
    a.ph.gamma = p->gamma;
    a.ph.gamma1 = p->gamma - 1.0;
    a.ph.grav = p->grav;
    a.ph.efix = p->efix;
    L.stage(a, st);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail_na(SCL_E_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  if (cfl) {
    Ctl h{};
    e = cudaMemcpyAsync(&h, ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail_na(SCL_E_CUDA, std::string("cfl readback: ") + cudaGetErrorString(e));
    *cfl = h.stage_cfl[ns - 1];
    if (h.status & SCL_STATUS_TIMEOUT) return fail_na(SCL_E_TIMEOUT, "a bounded wait for staged data ran out");
    if ((h.status & SCL_STATUS_NONFINITE) || *cfl != *cfl)
      return fail_na(SCL_E_NONFINITE, "non-finite stage output");
  }
  return SCL_OK;
}
