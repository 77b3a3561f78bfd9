// scl_launch.h -- launcher table shared by the C ABI and the per-precision
// kernel translation units.
#pragma once
#include "scl_common.cuh"

namespace scl {

struct Launchers {
  void (*stage)(const StageArgs&, cudaStream_t);  // one fused RK stage over the grid
  void (*ghost)(const StageArgs&, cudaStream_t);  // 2-D ghost-line CFL (nullptr in 1-D)
  cudaError_t (*run)(const RunArgs&, cudaStream_t);  // cluster-resident run (1-D), or nullptr
};

// Cluster-resident runs: tile width, largest cluster (portable size), the
// tile counts up to which the automatic mode picks them and up to which they
// are allowed, and controller iterations per launch.
constexpr int RES_NT = 128;
constexpr int RES_CLUSTER = 8;
constexpr int RES_AUTO_TILES = 8;   // one tile per CTA: beyond it the graphs are faster
constexpr int RES_MAX_TILES = 64;
constexpr int RES_TILES_PER_CTA = RES_MAX_TILES / RES_CLUSTER;   // tiles one CTA holds at most
constexpr int RES_ITERS = 4096;

// One getter per arithmetic form; `variant` selects a tile shape (2-D).
bool get_launchers_fp64(int rp, int ndim, int cd, int tf, int variant, Launchers* L);
bool get_launchers_fp64s(int rp, int ndim, int cd, int tf, int variant, Launchers* L);
bool get_launchers_mixed(int rp, int ndim, int cd, int tf, int variant, Launchers* L);
bool get_launchers_fp32(int rp, int ndim, int cd, int tf, int variant, Launchers* L);

constexpr int N2D_VARIANTS = 3;

// Sets the message returned by scl_last_error() on this thread.
void set_last_error(const char* msg);

}  // namespace scl

namespace scl {

struct BatchArgs;

// Batched persistent launchers of one plugin / precision / tile width.
struct BatchLaunchers {
  void (*stage)(const BatchArgs&, int grid, cudaStream_t);
  // end_stage >= 0: run the previous step's end (that last stage, final_role) first
  void (*begin)(Ctl* ctl, const int* mx, int ninst, int* active, int* prefix, int* nact, int end_stage,
                int final_role, cudaStream_t);
  int (*blocks_per_sm)();
  int nt;   // threads per CTA = interfaces per tile
};

constexpr int NBATCH_VARIANTS = 3;   // tile width 128 or 256; 2: paired 1-D Euler tile (FP32 forms)

bool get_batch_launchers_fp64(int rp, int cd, int tf, int variant, BatchLaunchers* L);
bool get_batch_launchers_fp64s(int rp, int cd, int tf, int variant, BatchLaunchers* L);
bool get_batch_launchers_mixed(int rp, int cd, int tf, int variant, BatchLaunchers* L);
bool get_batch_launchers_fp32(int rp, int cd, int tf, int variant, BatchLaunchers* L);

}  // namespace scl

namespace scl {
// Discrete adjoint pieces (FP64, 2-D acoustics, periodic bc).
bool adjoint_supported(int rp, int ndim, int cd, int ti, const int* mthbc);
void launch_vjp2d(const double* q, const double* lam, const double* aux, double* out, long pitch, long plane,
                  int nx, int ny, double dx, double dy, double dt, const Phys& ph, int cd, cudaStream_t st,
                  int ndim = 2);
void launch_adj_combine(int mode, double* a, const double* b, const double* c, long n, cudaStream_t st);
void launch_adj_final(double* l0, const double* l3, const double* l2, const double* l1, const double* t, long n,
                      cudaStream_t st);
void launch_axpby(double* out, double a, const double* x, double b, const double* y, long n, cudaStream_t st);
}  // namespace scl
