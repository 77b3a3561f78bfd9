// scl_dispatch.cuh -- instantiates the stage kernels of one arithmetic form.
// Included by two translation units per form (scl_prec_*.cu: the 1-D and
// batched kernels, SCL_PART 1; scl_prec_*_2d.cu: the 2-D kernels, SCL_PART 2)
// with SCL_PREC_VALUE defined, so the build compiles them in parallel; the
// FP64_STRICT units are compiled without FMA contraction so their arithmetic
// follows the reference's evaluation order.
#pragma once
#include <algorithm>
#include <type_traits>

#include "scl_batch.cuh"
#include "scl_kernels.cuh"
#include "scl_launch.h"
#include "scl_pair.cuh"
#include "scl_resident.cuh"

#ifndef SCL_PREC_VALUE
#error "SCL_PREC_VALUE must be defined"
#endif
#ifndef SCL_PART
#error "SCL_PART must be defined (1: 1-D and batched kernels, 2: 2-D kernels)"
#endif

namespace scl {
namespace SCL_PREC_NS {

constexpr int PREC = SCL_PREC_VALUE;
using R = typename Prec<PREC>::R;
using S = typename Prec<PREC>::S;

constexpr int NT1 = 128;

// Bulk-copy staging needs every role buffer on a 16-byte boundary and a
// component stride that keeps the planes there (handles pad it to 32
// elements; caller-owned arrays may not).
inline bool bulk_staging_ok(const StageArgs& a) {
  constexpr long AL = 16 / (long)sizeof(S);
  if (a.plane % AL != 0) return false;
  for (int r = 0; r < NROLES; ++r)
    if (reinterpret_cast<uintptr_t>(a.buf[r]) % 16 != 0) return false;
  return true;
}

// The Euler plugin in the FP64 forms: 118 registers unbounded (4 CTAs, 16
// warps per SM); bounded to 6 CTAs per SM it spills a little and runs 9-12 %
// faster, and its tiles are staged by bulk copies (measured at 2^20 and 2^23
// cells).  Lighter plugins keep the compiler's register choice and stage by
// the threads: their CTAs are short, and a bulk copy's latency then shows
// (1-D advection at 2^26 cells: 777 us per stage staged by the threads,
// 1027 us by bulk copies).
template <class P>
constexpr bool heavy1d() {
  return std::is_same_v<P, PEuler> && Prec<PREC>::EXACT;
}

template <class P, int CD, int TF>
void launch1d(const StageArgs& a, cudaStream_t st) {
  const int nb = (a.mx + NT1 - 2) / (NT1 - 1);
  if constexpr (heavy1d<P>()) {
    if (bulk_staging_ok(a)) {
      k_stage1d<P, CD, TF, PREC, NT1, true, 6><<<nb, NT1, 0, st>>>(a);
      return;
    }
    k_stage1d<P, CD, TF, PREC, NT1, false, 6><<<nb, NT1, 0, st>>>(a);
  } else {
    k_stage1d<P, CD, TF, PREC, NT1><<<nb, NT1, 0, st>>>(a);
  }
}

// One cluster of nc CTAs, T tiles each (T the fewest tiles per CTA with
// nc <= RES_CLUSTER), runs the controller loop with the rows of every
// buffer in shared memory.
template <class P, int CD, int TF>
cudaError_t launch_run1d(const RunArgs& a, cudaStream_t st) {
  using S = typename Prec<PREC>::S;
  const int ntiles = (a.st.mx + RES_NT - 2) / (RES_NT - 1);
  const int T = (ntiles + RES_CLUSTER - 1) / RES_CLUSTER;
  const int nc = (ntiles + T - 1) / T;
  const size_t rows = run1d_rows_bytes<S>(P::MEQN, T, RES_NT);
  bool gen = a.st.mcapa > 0 || a.totals;
  for (int s = 0; s < a.nstages; ++s) gen = gen || a.sd[s].out2 >= 0;
  auto k = gen ? k_run1d<P, CD, TF, PREC, RES_NT, true> : k_run1d<P, CD, TF, PREC, RES_NT, false>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rows);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nc, 1, 1);
  cfg.blockDim = dim3(run1d_threads<RES_NT>(), 1, 1);
  cfg.dynamicSmemBytes = rows;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = nc;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, a);
}

// 1-D Euler in the FP32 forms: two interfaces per thread in packed FP32
// (scl_pair.cuh); capacity grids take the one-interface kernel.
#ifndef SCL_PAIR
#define SCL_PAIR 1
#endif
constexpr int NTP = 128;

template <int CD>
void launch1d_pair(const StageArgs& a, cudaStream_t st) {
  if (a.mcapa > 0) {
    launch1d<PEuler, CD, 0>(a, st);
    return;
  }
  const int nb = a.mx / PairGeom<PREC, NTP>::STRIDE + 1;
  if (bulk_staging_ok(a)) k_stage1d_pair<CD, PREC, NTP, true><<<nb, NTP, 0, st>>>(a);
  else k_stage1d_pair<CD, PREC, NTP, false><<<nb, NTP, 0, st>>>(a);
}

template <class P, int CD, int TF, int TX, int TY, int NT>
constexpr size_t smem2d() {
  using T = Tile2D<TX, TY>;
  return sizeof(S) * P::MEQN * T::WX * T::WY + sizeof(R) * 4 * P::MEQN * (T::NXI + T::NYI);
}

// CTAs per SM the 2-D kernel's registers are budgeted for: in the FP64 forms
// the shallow-water kernel needs 120 registers unbounded (2 CTAs of 256
// threads per SM); bounded to 3 (6 for the 128-thread shape) it spills a
// little and runs 3.5-4 % faster at 4096^2 (16x15: 2196 -> 2119 us, 16x7:
// 2438 -> 2340 us, 32x7: 2297 -> 2211 us).  The FP32 forms fit in 64
// registers and keep the compiler's choice.
template <int NT>
constexpr int stage2d_minb() {
  return Prec<PREC>::EXACT ? (NT == 256 ? 3 : 6) : 0;
}

template <class P, int CD, int TF, int TX, int TY, int NT>
void launch2d(const StageArgs& a, cudaStream_t st) {
  dim3 grid((a.mx + TX - 1) / TX, (a.my + TY - 1) / TY);
  k_stage2d<P, CD, TF, PREC, TX, TY, NT, stage2d_minb<NT>()><<<grid, NT, smem2d<P, CD, TF, TX, TY, NT>(), st>>>(a);
}

// dynamic shared memory above 48 KB must be opted into before launch (and
// outside any stream capture), so it is done when the kernel is picked
template <class P, int CD, int TF, int TX, int TY, int NT>
bool prepare2d(Launchers* L) {
  if (cudaFuncSetAttribute(k_stage2d<P, CD, TF, PREC, TX, TY, NT, stage2d_minb<NT>()>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem2d<P, CD, TF, TX, TY, NT>()) != cudaSuccess)
    return false;
  L->stage = &launch2d<P, CD, TF, TX, TY, NT>;
  return true;
}

template <class P, int CD>
void launch_ghost2d(const StageArgs& a, cudaStream_t st) {
  const int n = 2 * (a.mx + 1) + 2 * (a.my + 1);
  k_ghost_cfl2d<P, CD, PREC><<<(n + 127) / 128, 128, 0, st>>>(a);
}

template <class P, int CD, int TF>
bool fill2d(int variant, Launchers* L) {
  switch (variant) {
    case 0: if (!prepare2d<P, CD, TF, 16, 7, 128>(L)) return false; break;
    case 1: if (!prepare2d<P, CD, TF, 32, 7, 256>(L)) return false; break;
    case 2: if (!prepare2d<P, CD, TF, 16, 15, 256>(L)) return false; break;
    default: return false;
  }
  L->ghost = &launch_ghost2d<P, CD>;
  return true;
}

template <class P, int CD, int TF>
void fill1d(Launchers* L) {
  L->stage = &launch1d<P, CD, TF>;
  L->run = &launch_run1d<P, CD, TF>;
}

template <class P>
bool pick(int ndim, int cd, int tf, int variant, Launchers* L) {
  L->stage = nullptr;
  L->ghost = nullptr;
  L->run = nullptr;
  if (ndim == 1) {
#if SCL_PART == 1
    if (variant != 0) return false;
    if (cd == 0 && tf == 0) fill1d<P, 0, 0>(L);
    if (cd == 1 && tf == 0) fill1d<P, 1, 0>(L);
    if (cd == 2 && tf == 0) fill1d<P, 2, 0>(L);
    if (cd == 3 && tf == 0) fill1d<P, 3, 0>(L);
    if (cd == 10 && tf == 0) fill1d<P, 10, 0>(L);
    if (cd == 11 && tf == 0) fill1d<P, 11, 0>(L);
    if (cd == 12 && tf == 0) fill1d<P, 12, 0>(L);
    if (cd == 20 && tf == 0) fill1d<P, 20, 0>(L);
    if (cd == 21 && tf == 0) fill1d<P, 21, 0>(L);
    if constexpr (P::HAS_TFLUCT) {
      if (cd == 0 && tf == 1) fill1d<P, 0, 1>(L);
      if (cd == 1 && tf == 1) fill1d<P, 1, 1>(L);
      if (cd == 2 && tf == 1) fill1d<P, 2, 1>(L);
      if (cd == 3 && tf == 1) fill1d<P, 3, 1>(L);
      if (cd == 10 && tf == 1) fill1d<P, 10, 1>(L);
      if (cd == 11 && tf == 1) fill1d<P, 11, 1>(L);
      if (cd == 12 && tf == 1) fill1d<P, 12, 1>(L);
      if (cd == 20 && tf == 1) fill1d<P, 20, 1>(L);
      if (cd == 21 && tf == 1) fill1d<P, 21, 1>(L);
    }
    // the FP32 forms of 1-D Euler step large grids with the paired kernel;
    // a resident run keeps the one-interface tile code
    if constexpr (SCL_PAIR && std::is_same_v<P, PEuler> && !Prec<PREC>::EXACT) {
      if (cd == 0 && tf == 0) L->stage = &launch1d_pair<0>;
      if (cd == 2 && tf == 0) L->stage = &launch1d_pair<2>;
    }
    return L->stage != nullptr;
#else
    return false;
#endif
  }
#if SCL_PART == 2
  if constexpr (P::NDIM == 2) {
    if (cd == 0 && tf == 0) return fill2d<P, 0, 0>(variant, L);
    if (cd == 1 && tf == 0) return fill2d<P, 1, 0>(variant, L);
    if (cd == 2 && tf == 0) return fill2d<P, 2, 0>(variant, L);
    if (cd == 3 && tf == 0) return fill2d<P, 3, 0>(variant, L);
    if (cd == 10 && tf == 0) return fill2d<P, 10, 0>(variant, L);
    if (cd == 11 && tf == 0) return fill2d<P, 11, 0>(variant, L);
    if (cd == 12 && tf == 0) return fill2d<P, 12, 0>(variant, L);
    if (cd == 20 && tf == 0) return fill2d<P, 20, 0>(variant, L);
    if (cd == 21 && tf == 0) return fill2d<P, 21, 0>(variant, L);
    if constexpr (P::HAS_TFLUCT) {
      if (cd == 0 && tf == 1) return fill2d<P, 0, 1>(variant, L);
      if (cd == 1 && tf == 1) return fill2d<P, 1, 1>(variant, L);
      if (cd == 2 && tf == 1) return fill2d<P, 2, 1>(variant, L);
      if (cd == 3 && tf == 1) return fill2d<P, 3, 1>(variant, L);
      if (cd == 10 && tf == 1) return fill2d<P, 10, 1>(variant, L);
      if (cd == 11 && tf == 1) return fill2d<P, 11, 1>(variant, L);
      if (cd == 12 && tf == 1) return fill2d<P, 12, 1>(variant, L);
      if (cd == 20 && tf == 1) return fill2d<P, 20, 1>(variant, L);
      if (cd == 21 && tf == 1) return fill2d<P, 21, 1>(variant, L);
    }
  }
#endif
  return false;
}

#if SCL_PART == 1
// ---- batched persistent launchers ----
template <class P, int CD, int TF, int NT>
void launch_batch_stage(const BatchArgs& a, int grid, cudaStream_t st) {
  k_batch_stage<P, CD, TF, PREC, NT><<<grid, NT, 0, st>>>(a);
}
template <int STRIDE, int FIRST>
void launch_batch_begin(Ctl* ctl, const int* mx, int ninst, int* active, int* prefix, int* nact,
                        int end_stage, int final_role, cudaStream_t st) {
  k_batch_begin<STRIDE, FIRST><<<1, 1024, 0, st>>>(ctl, mx, ninst, active, prefix, nact, end_stage, final_role);
}
template <class P, int CD, int TF, int NT>
int batch_blocks_per_sm() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_stage<P, CD, TF, PREC, NT>, NT, 0);
  return n;
}
template <class P, int CD, int TF, int NT>
void fill_batch(BatchLaunchers* L) {
  L->stage = &launch_batch_stage<P, CD, TF, NT>;
  L->begin = &launch_batch_begin<NT - 1, 1>;
  L->blocks_per_sm = &batch_blocks_per_sm<P, CD, TF, NT>;
  L->nt = NT;
}
// (capacity batches do not get this variant: scl_batch_create skips it)
template <int CD>
void launch_batch_stage_pair(const BatchArgs& a, int grid, cudaStream_t st) {
  k_batch_stage_pair<CD, PREC, NTP><<<grid, NTP, 0, st>>>(a);
}
template <int CD>
int batch_blocks_per_sm_pair() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_stage_pair<CD, PREC, NTP>, NTP, 0);
  return n;
}

template <class P, int CD, int TF>
bool pick_batch_nt(int variant, BatchLaunchers* L) {
  // variants 0 and 1: one interface per thread, tiles of 127 / 255 cells;
  // variant 2 (1-D Euler in the FP32 forms): the paired tile of 254 cells
  if constexpr (SCL_PAIR && std::is_same_v<P, PEuler> && !Prec<PREC>::EXACT && TF == 0 && (CD == 0 || CD == 2)) {
    if (variant == 2) {
      L->stage = &launch_batch_stage_pair<CD>;
      L->begin = &launch_batch_begin<PairGeom<PREC, NTP>::STRIDE, 0>;
      L->blocks_per_sm = &batch_blocks_per_sm_pair<CD>;
      L->nt = NTP;
      return true;
    }
  }
  if (variant == 0) { fill_batch<P, CD, TF, 128>(L); return true; }
  if (variant == 1) { fill_batch<P, CD, TF, 256>(L); return true; }
  return false;
}
template <class P>
bool pick_batch(int cd, int tf, int variant, BatchLaunchers* L) {
  if (cd == 0 && tf == 0) return pick_batch_nt<P, 0, 0>(variant, L);
  if (cd == 1 && tf == 0) return pick_batch_nt<P, 1, 0>(variant, L);
  if (cd == 2 && tf == 0) return pick_batch_nt<P, 2, 0>(variant, L);
  if (cd == 3 && tf == 0) return pick_batch_nt<P, 3, 0>(variant, L);
  if (cd == 10 && tf == 0) return pick_batch_nt<P, 10, 0>(variant, L);
  if (cd == 11 && tf == 0) return pick_batch_nt<P, 11, 0>(variant, L);
  if (cd == 12 && tf == 0) return pick_batch_nt<P, 12, 0>(variant, L);
  if constexpr (P::HAS_TFLUCT) {
    if (cd == 0 && tf == 1) return pick_batch_nt<P, 0, 1>(variant, L);
    if (cd == 1 && tf == 1) return pick_batch_nt<P, 1, 1>(variant, L);
    if (cd == 2 && tf == 1) return pick_batch_nt<P, 2, 1>(variant, L);
    if (cd == 3 && tf == 1) return pick_batch_nt<P, 3, 1>(variant, L);
    if (cd == 10 && tf == 1) return pick_batch_nt<P, 10, 1>(variant, L);
    if (cd == 11 && tf == 1) return pick_batch_nt<P, 11, 1>(variant, L);
    if (cd == 12 && tf == 1) return pick_batch_nt<P, 12, 1>(variant, L);
  }
  return false;
}

#endif  // SCL_PART == 1

}  // namespace SCL_PREC_NS

#if SCL_PART == 1
bool SCL_BATCH_GETTER(int rp, int cd, int tf, int variant, BatchLaunchers* L) {
  using namespace SCL_PREC_NS;
  switch (rp) {
    case SCL_RP_ADVECTION: return pick_batch<PAdvection>(cd, tf, variant, L);
    case SCL_RP_EULER: return pick_batch<PEuler>(cd, tf, variant, L);
    case SCL_RP_ACOUSTICS1D: return pick_batch<PAcoustics<2>>(cd, tf, variant, L);
  }
  return false;
}

bool SCL_PREC_GETTER_2D(int rp, int cd, int tf, int variant, Launchers* L);   // the form's 2-D unit

bool SCL_PREC_GETTER(int rp, int ndim, int cd, int tf, int variant, Launchers* L) {
  using namespace SCL_PREC_NS;
  if (ndim == 2) return SCL_PREC_GETTER_2D(rp, cd, tf, variant, L);
  switch (rp) {
    case SCL_RP_ADVECTION: return pick<PAdvection>(ndim, cd, tf, variant, L);
    case SCL_RP_EULER: return pick<PEuler>(ndim, cd, tf, variant, L);
    case SCL_RP_SW2D: return pick<PShallow2D>(ndim, cd, tf, variant, L);
    case SCL_RP_ACOUSTICS1D: return pick<PAcoustics<2>>(ndim, cd, tf, variant, L);
    case SCL_RP_ACOUSTICS2D: return pick<PAcoustics<3>>(ndim, cd, tf, variant, L);
    case SCL_RP_ADVECTION2D: return pick<PAdvEdge2D>(ndim, cd, tf, variant, L);
    case SCL_RP_SW1D: return pick<PShallow1D>(ndim, cd, tf, variant, L);
    case SCL_RP_SWF_BATHY: return pick<PShallowF1D<0>>(ndim, cd, tf, variant, L);
    case SCL_RP_SWF_RADIAL: return pick<PShallowF1D<1>>(ndim, cd, tf, variant, L);
    case SCL_RP_SWF_KAPPA: return pick<PShallowF1D<2>>(ndim, cd, tf, variant, L);
    case SCL_RP_ACOUSTICS_CONST: return pick<PAcousticsConst>(ndim, cd, tf, variant, L);
    case SCL_RP_ACOUSTICS_FWAVE: return pick<PElasticFwave<0>>(ndim, cd, tf, variant, L);
    case SCL_RP_STEGOTON: return pick<PElasticFwave<1>>(ndim, cd, tf, variant, L);
    case SCL_RP_TRAFFIC: return pick<PTraffic>(ndim, cd, tf, variant, L);
    case SCL_RP_ADVECTION_CONS: return pick<PAdvCons>(ndim, cd, tf, variant, L);
  }
  return false;
}
#else
bool SCL_PREC_GETTER_2D(int rp, int cd, int tf, int variant, Launchers* L) {
  using namespace SCL_PREC_NS;
  switch (rp) {
    case SCL_RP_SW2D: return pick<PShallow2D>(2, cd, tf, variant, L);
    case SCL_RP_ACOUSTICS2D: return pick<PAcoustics<3>>(2, cd, tf, variant, L);
    case SCL_RP_ADVECTION2D: return pick<PAdvEdge2D>(2, cd, tf, variant, L);
  }
  return false;
}
#endif

}  // namespace scl
