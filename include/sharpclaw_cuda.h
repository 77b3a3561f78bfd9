/*
 * sharpclaw_cuda.h -- C ABI of the B200 SharpClaw semi-discrete WENO step.
 *
 * Drop-in boundary for the reference's hot path.  The reference binds these
 * operations as Fortran subroutines; a Fortran host replaces them with
 * bind(C) shims that forward here (the iso_c_binding module and the shims
 * flux1, flux2, step and sharpclaw are in fortran/sharpclaw_cuda.f90).
 * Every entry point returns an int status (0 = ok,
 * negative = SCL_E_*) and never calls exit/abort, replacing the reference's
 * `stop` statements.
 *
 * Arrays crossing the boundary are host (or, for the *_device variants,
 * device) arrays of double in the reference layout: Fortran column-major
 * q(1-mbc:mx+mbc[,1-mbc:my+mbc], meqn) (src/1d/qalloc1.f90:10,
 * src/2d/qalloc2.f90:11), i.e. element (i[,j],m) at
 *   (i+mbc-1) [+ (j+mbc-1)*(mx+2mbc)] + (m-1)*plane.
 * No torch types appear here.
 */
#ifndef SHARPCLAW_CUDA_H
#define SHARPCLAW_CUDA_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define SCL_OK 0
#define SCL_E_INVALID (-1)      /* bad parameter (the reference would `stop`)      */
#define SCL_E_CUDA (-2)         /* a CUDA call failed; see scl_last_error()         */
#define SCL_E_UNSUPPORTED (-3)  /* valid in the reference, not built here           */
#define SCL_E_NONFINITE (-4)    /* NaN/Inf met in the CFL number                    */
#define SCL_E_TIMEOUT (-5)      /* a bounded device wait ran out                    */
#define SCL_E_IO (-6)           /* a frame file could not be written                */

/* device status bits (scl_result.status) */
#define SCL_STATUS_NONFINITE 1
#define SCL_STATUS_TIMEOUT 2
#define SCL_STATUS_BOUNDS 4

/* sharpclaw() info codes (src/sharpclaw.f90:35-63,225-228) plus one new one */
#define SCL_INFO_DT_NOT_DIVIDING 2
#define SCL_INFO_CFL_DESIRED_GT_MAX 3
#define SCL_INFO_TOO_MANY_STEPS 11
#define SCL_INFO_CFL_FIXED_DT 12
#define SCL_INFO_NONFINITE 20

/* ---- plugins (device Riemann solvers selected by id) ------------------- */
#define SCL_RP_ADVECTION 1    /* apps/advection/1d/{rp1.f,tfluct1.f,evec.f}                 */
#define SCL_RP_EULER 2        /* apps/euler/shockentropy/rp1eu.f (+ Roe evec, new)           */
#define SCL_RP_SW2D 3         /* apps/shallowWater/2dRadialDam/{rpn2sw.f,tfluct1sw.f} (+evec) */
#define SCL_RP_ACOUSTICS1D 4  /* apps/acoustics/1d/interface/{rp1acv.f,tfluct1acv.f,evec.f90} */
#define SCL_RP_ACOUSTICS2D 5  /* 2-D variable-coefficient acoustics rpn2/tfluct/evec (new)    */
#define SCL_RP_ADVECTION2D 6  /* apps/advection/2d/swirl/rpn2ad1.f: edge velocities in aux      */
#define SCL_RP_SW1D 7         /* apps/shallowWater/2dRadialDam/1dRadialSymm-qwave/{rp1sw.f,
                                 tfluct1sw.f}, entropy fix on by default (+ Roe evec, new)  */
/* f-wave shallow water (rpf-wave.f90, tfluctf-wave.f90 of each app):        */
#define SCL_RP_SWF_BATHY 8    /* apps/shallowWater/1dPerturbSteady: bathymetry b = aux(:,1),
                                 its source in the cell's total fluctuation (maux >= 1)     */
#define SCL_RP_SWF_RADIAL 9   /* 2dRadialDam/1dRadialSymm-fwave: aux = (r, dx), the radial
                                 source in the interface flux difference (maux >= 2)       */
#define SCL_RP_SWF_KAPPA 10   /* 2dRadialDam/1dRadialSymm-fwave-kappa: aux = (r(i-1/2), r, r,
                                 dx), area-weighted fluxes, capacity aux(:,2) (maux >= 4)  */
#define SCL_RP_ACOUSTICS_CONST 11  /* apps/acoustics/1d/homogeneous/{rp1.f,tfluct.f,evec.f}:
                                      constant rho, bulk (scl_params.rho, .bulk)          */
#define SCL_RP_ACOUSTICS_FWAVE 12  /* apps/acoustics/1d/fwave/{rp1acfw.f,tfluct1.f,evec.f}:
                                      q = (strain, momentum), aux = (rho, bulk)          */
#define SCL_RP_TRAFFIC 13          /* apps/traffic/congTraffic/{rpf-wave.f90,tfluct1.f90}:
                                      flux umax(x) q (1-q), aux = umax                   */
#define SCL_RP_ADVECTION_CONS 14   /* apps/traffic/flux-uq/rpf-wave.f90: (u(x) q)_x with
                                      cell velocities aux = u; no tfluct                 */
#define SCL_RP_STEGOTON 15         /* apps/elasticity/stegoton/{rp1nel.f,tfluct1.f}: stress
                                      exp(A eps) - 1 (A > 0) or B eps, aux = (rho, A, B)
                                      (+ evec of the form of acoustics/1d/fwave, new)    */

/* ---- source terms: the src(q,dq,aux,t,dt) an app links (src/1d/step1d.f90:23),
 * evaluated in the stage kernel before the fluctuations are subtracted;
 * 1-D, SCL_RP_SW1D only ---------------------------------------------------- */
#define SCL_SRC_NONE 0           /* src/1d/src1.f90: dq = 0                                */
#define SCL_SRC_RADIAL_SW 1      /* apps/shallowWater/2dRadialDam/1dRadialSymm-qwave/src1.f90:
                                    dq = -dt (hu, hu^2/h) / r, r = xlower + (i-1/2) dx     */
#define SCL_SRC_BATHYMETRY_SW 2  /* apps/shallowWater/1dPerturbSteady/src1.f90:
                                    dq(2) = -g h (b(i) - b(i-1)) / dx * dt, b = aux(:,1)   */

/* ---- b4step hooks (src/b4step.f90 and the apps' own, run on the device) - */
#define SCL_B4STEP_NONE 0     /* src/b4step.f90: no-op                                      */
#define SCL_B4STEP_SWIRL 1    /* apps/advection/2d/swirl/b4step.f90: aux = aux0 *
                                 cos(2 pi (t + dt/2) / tperiod); no-op for tperiod = 0     */
#define SCL_B4STEP_TIME_REVERSAL 2  /* apps/elasticity/stegoton/b4step1.f: once, at the
                                 first step with told + 1e-10 >= trtime (param), q(:,2) =
                                 -q(:,2) over every cell; 1-D.  Its time traces
                                 (fort.17/18/28) are host I/O and are not written      */

/* ---- user boundary conditions (mthbc = 0: the app's own bc1.f, run on the
 * device before every stage, with the stage time) -------------------------- */
#define SCL_BC_USER_NONE 0              /* src/1d/bc1.f90: mthbc = 0 stops      */
#define SCL_BC_USER_OSCILLATING_WALL 1  /* apps/elasticity/stegoton/bc1.f: a wall
   at x = xlower (mthbc[0] = 0) moving with v = -a1 g0((t - t1)/tw1), at
   x = xupper (mthbc[1] = 0) with v = a2 g0((t - t2)/tw2), g0(s) = 1 + cos(pi s)
   for |s| < 1, else 0; ghost momentum 2 v rho - q2 of the mirror cell.  Once
   a stage time lies in (5 tw1, 5 tw1 + 1) both sides become periodic (q and
   aux ghosts) for the rest of the handle's life, as bc1.f rewrites mthbc.   */

/* ---- arithmetic ---------------------------------------------------------- */
#define SCL_FP64 0         /* plain FP64 (FMA contraction allowed)                       */
#define SCL_FP64_STRICT 1  /* FP64, no FMA contraction: the reference's evaluation order */
#define SCL_MIXED 2        /* FP32 reconstruction/Riemann, FP64 state and RK accumulation */
#define SCL_FP32 3         /* FP32 throughout (FP32 state)                               */

/* Mirrors module ClawParams (src/ClawParams.f90:1-16) plus the plugin COMMON
 * blocks (/comrp/ u or g, /param/ gamma) and the integrator choice. */
typedef struct scl_params {
  int ndim;             /* 1 or 2                                                  */
  int mx, my;           /* nx(1), nx(2)                                            */
  int meqn, mwaves, mbc, maux, mcapa;
  int lim_type;         /* 2 = WENO5, 1 = second-order TVD (reconstruct.f90),
                           0 = unlimited polynomial of order mthlim(1) = 3
                           (polyrecon.f90; single grids, not the batched solver)  */
  int char_decomp;      /* 0 weno5, 1 weno5_wave, 2 weno5_char, 3 weno5_trans
                           (TVD: 0..2, polynomial: 0 q2qlqr_poly, 1 _poly_wave)   */
  int tfluct_solver;    /* 1 tfluct plugin, 0 swap + second rp (flux1.f90:136-188) */
  int mthbc[4];         /* 1 extrapolation, 2 periodic, 3 solid wall,
                           0 the user bc named by bc_user (1-D)                   */
  double dx, dy, xlower, ylower;
  int rp;               /* SCL_RP_*                                                */
  int efix;             /* entropy fix (rp1eu.f:40 .true., rpn2sw.f:48 .false.)    */
  double u, gamma, grav;
  int time_integrator;  /* 1 SSP22, 2 SSP42, 3 SSP33, 4 SSP104 (sharpclaw.f90:159) */
  int precision;        /* SCL_FP64, SCL_FP64_STRICT, SCL_MIXED, SCL_FP32          */
  int mthlim[4];        /* TVD limiter per component / field / wave (lim_type = 1):
                           1 minmod, 2 superbee, 3 van Leer, 4 MC, 5 Cada-Torrilhon
                           (ClawParams%mthlim, reconstruct.f90:551-571); with
                           lim_type = 0, mthlim[0] is the order (3)              */
  int src_term;         /* SCL_SRC_* (ClawParams%src_term; the reference links the
                           app's src1.f90 instead)                                */
  double rho, bulk;     /* SCL_RP_ACOUSTICS_CONST: common /cparam/ rho, bulk       */
  int bc_user;          /* SCL_BC_USER_* for the sides with mthbc = 0              */
  double wall[6];       /* SCL_BC_USER_OSCILLATING_WALL: t1, a1, tw1 (common
                           /comwall/, setprob.data) and t2, a2, tw2 of the right
                           wall                                                    */
} scl_params;

/* Arguments of sharpclaw() (src/sharpclaw.f90:2-5). */
typedef struct scl_run {
  double tstart, tend;
  double dt_initial, dt_max, cfl_max, cfl_desired;
  int max_steps, dt_variable;
} scl_run;

/* Outputs of sharpclaw() (cfl_maxused, cfl_last, dt_minused, dt_maxused,
 * dt_last, steps_taken, info) plus rejected-step and device status counts. */
typedef struct scl_result {
  double tend, cfl_maxused, cfl_last, dt_minused, dt_maxused, dt_last;
  int steps_taken, info, rejected, status;
} scl_result;

typedef struct scl_handle scl_handle;

/* Library identification and the last error message of this thread. */
const char* scl_version(void);
const char* scl_last_error(void);

/* Create a solver for one grid; allocates its device buffers on the current
 * device and one stream.  Replaces module allocation in src/main.f90:128-133
 * (qalloc, alloc_recon_workspace) and the griddat allocation in
 * src/sharpclaw.f90:66-111. */
int scl_create(const scl_params* p, scl_handle** out);
int scl_destroy(scl_handle* h);

/* Copy q / aux (reference layout, double, ghost cells included) to and from
 * the device state.  scl_set_q also fills ghost cells as bc1/bc2 would. */
int scl_set_q(scl_handle* h, const double* q);
int scl_get_q(scl_handle* h, double* q);
int scl_set_aux(scl_handle* h, const double* aux);

/* One evaluation of dq = dt*L(q): bc + src + flux1 (1-D) or flux2 (2-D),
 * step1d.f90:2-31 / step2d.f90:2-41.  q is updated in place with its ghost
 * cells (as bc does), dq receives the interior update, cfl the CFL number
 * (flux1.f90:126-133, flux2.f90:47,80).  Host arrays. */
int scl_step_dq(scl_handle* h, double* q, double* dq, double dt, double t, double* cfl);

/* flux1.f90:2 on one line of mx cells (ixy = 1 or 2 selects the normal
 * direction for the 2-D plugins): q1d(1-mbc:mx+mbc,meqn) in, dq1d out
 * (interior cells), cfl out.  aux1d may be NULL when maux == 0. */
int scl_flux1(scl_handle* h, const double* q1d, const double* aux1d, double* dq1d,
              double dt, int ixy, int mx, double* cfl);

/* One SSP-RK time step on the device-resident q (ts_ssp22/42/33/104,
 * sharpclaw.f90:247-464), qold = q on entry; returns the last stage's CFL. */
int scl_rk_step(scl_handle* h, double dt, double told, double* cfl);

/* The time loop of sharpclaw() (src/sharpclaw.f90:118-228) run on the
 * device: dt control, rejection/retake and stopping are decided by a
 * one-thread controller kernel between steps, captured in CUDA graphs, so the
 * host does not synchronise per step.  b4step is the default no-op. */
int scl_sharpclaw(scl_handle* h, const scl_run* run, scl_result* res);

/* Same with device pointers: q_dev holds the initial data / receives the
 * final state in the reference layout (double). */
int scl_sharpclaw_device(scl_handle* h, const scl_run* run, double* q_dev, scl_result* res);

/* Timing helper for benchmarks: replays `nsteps` steps of the controller on
 * the device-resident state with stage kernels only (no host copies) and
 * returns the elapsed device time in milliseconds, measured with CUDA events
 * on the handle's stream. */
int scl_time_steps(scl_handle* h, const scl_run* run, int nsteps, float* ms, scl_result* res);

/* Roofline helper: launches the integrator's stage kernels (one pass of all
 * stages = one time step's worth, no controller) `reps` times back to back on
 * the device-resident state with step size dt and returns the elapsed device
 * time (CUDA events on the handle's stream) and the number of launches.  The
 * state is not advanced (every pass restarts from q^n). */
int scl_time_stages(scl_handle* h, double dt, int reps, float* ms, long long* launches);

/* Kernel launches per controller step inside a step graph (stages + one
 * controller kernel that ends the step and begins the next, + 1 ghost-line
 * CFL kernel in 2-D, + 1 b4step kernel when set); each graph replay adds
 * one begin kernel. */
int scl_kernels_per_step(scl_handle* h);

/* How scl_sharpclaw and scl_time_steps run the controller loop (no
 * counterpart in the reference, whose loop is sharpclaw.f90:118-221 on the
 * host).  SCL_RUN_GRAPH: CUDA graphs of stage and controller kernels, any
 * grid.  SCL_RUN_RESIDENT: one thread-block cluster of up to 8 CTAs keeps the
 * whole loop in one launch (per 4096 iterations), for 1-D grids of at most
 * 64 tiles of 127 cells (8128 cells) without a b4step hook; SCL_E_UNSUPPORTED
 * otherwise.  SCL_RUN_AUTO (the default): resident for 1-D grids of at most
 * 8 tiles (1016 cells: one tile per CTA), graphs for the rest.  Both modes run the same tile
 * arithmetic and controller, so their results are identical, except in the
 * FP32 forms of 1-D Euler (char_decomp 0/2, tfluct_solver 0), whose graph
 * path uses a paired kernel with a different FP32 contraction order. */
#define SCL_RUN_AUTO 0
#define SCL_RUN_GRAPH 1
#define SCL_RUN_RESIDENT 2
int scl_set_run_mode(scl_handle* h, int mode);

/* Conserved totals (no counterpart in the reference, which keeps none).
 * With on = 1, scl_sharpclaw and scl_time_steps keep for every component m
 *   T_m = sum over interior cells of q(i[,j],m) [* aux(i[,j],mcapa)] * dx [* dy]
 * in FP64 with compensated (error-free two-sum) accumulation, whatever the
 * arithmetic form of the stages: at the start of the run and after every
 * accepted step, with the largest |T_m - T_m(start)| over the run's accepted
 * steps.  Step graphs add one kernel per step (one read of q); a
 * cluster-resident run sums the last stage's outputs in its tile code. */
int scl_set_totals(scl_handle* h, int on);

/* The totals of the last scl_sharpclaw / scl_time_steps: at its start (tot0),
 * of the current state (tot) and the largest drift |tot - tot0| over its
 * accepted steps (drift); meqn values each, any pointer may be NULL.
 * SCL_E_INVALID when totals are off. */
int scl_conserved_totals(scl_handle* h, double* tot0, double* tot, double* drift);

/* Failure-detection test hook (no counterpart in the reference).  The 1-D
 * Euler stage kernels stage their tiles by bulk copies completed on an
 * mbarrier, and every wait on it is bounded (1 s of device time): a thread whose wait runs
 * out raises SCL_STATUS_TIMEOUT, waits once more (bounded) for copies still
 * in flight and finishes; the controller then discards the step and stops
 * the run (q = qold), and the call returns SCL_E_TIMEOUT.  With on = 1 the
 * handle's stage launches announce 16 bytes more than they copy and bound
 * each wait at 1 ms, so every wait runs out: this exercises that path on a
 * GPU without faulting or hanging it (tests only; on = 0 restores normal
 * operation). */
int scl_test_wait_timeout(scl_handle* h, int on);

/* The mode the last scl_sharpclaw / scl_time_steps ran in (SCL_RUN_GRAPH or
 * SCL_RUN_RESIDENT) and the kernels it launched (graph nodes counted one by
 * one); either out pointer may be NULL. */
int scl_last_run(scl_handle* h, int* mode, long long* launches);

/* Frame output in the reference's format (src/1d/out1.f90, src/2d/out2.f90):
 * fort.qNNNN (interior cells, 4 values per record, e16.8 in 1-D and e26.16 in
 * 2-D), fort.tNNNN, and with write_aux fort.aNNNN, in directory dir (NULL or
 * "" = the working directory); NNNN = the last four digits of iframe.  Values
 * below 1e-99 in magnitude are written as 0 (the reference also zeroes them in
 * its state array; the state here is left as it is).
 *
 * scl_write_frame writes the handle's current state without stalling the
 * device: it enqueues a copy into a pinned host buffer on the handle's stream
 * and returns; a host thread formats and writes the files once the copy is
 * done.  One frame is in flight per handle: the next scl_write_frame, and
 * scl_wait_frames, wait for it and return its error, if any (SCL_E_IO). */
int scl_write_frame(scl_handle* h, double t, int iframe, const char* dir, int write_aux);
int scl_wait_frames(scl_handle* h);

/* The same files from host arrays in the reference layout (synchronous; needs
 * no GPU).  aux may be NULL when write_aux == 0 or maux == 0. */
int scl_format_frame(const scl_params* p, const double* q, const double* aux, double t, int iframe,
                     const char* dir, int write_aux);

/* Select the b4step hook that scl_sharpclaw / scl_time_steps run on the
 * device before every new (not retaken) time step, as sharpclaw.f90:129 calls
 * b4step; param is the hook's constant (SCL_B4STEP_SWIRL: tperiod, and the
 * aux set by scl_set_aux, now or later, is the hook's base field aux0;
 * SCL_B4STEP_TIME_REVERSAL: trtime, and the handle remembers that the flip
 * has happened, as the app's itrdone). */
int scl_set_b4step(scl_handle* h, int kind, double param);

/* Tile shape of the fused 2-D stage kernel (no counterpart in the reference;
 * flux2.f90 sweeps whole lines).  Shapes: 0 = 16x7 cells on 128 threads,
 * 1 = 32x7 on 256, 2 = 16x15 on 256.  variant -1 (the default) makes the next
 * scl_sharpclaw / scl_time_steps time one stage of every shape on the current
 * state and keep the fastest; 0..SCL_TILE_SHAPES-1 fixes a shape.  Every
 * shape evaluates each interface and cell with the same arithmetic, so the
 * results are bitwise identical.  1-D handles accept -1 and 0 only. */
#define SCL_TILE_SHAPES 3
int scl_select_tiles(scl_handle* h, int variant);

/* Shape in use (0 until a run has tuned or one was fixed), whether it was
 * chosen by timing (1) or not (0), and the trial time in ms of one stage per
 * shape (SCL_TILE_SHAPES entries, 0 for shapes not timed); any out pointer
 * may be NULL. */
int scl_tiles(scl_handle* h, int* variant, int* tuned, float* trial_ms);

/* One SSP-RK time step of a 1-D grid that allocates nothing, for callers
 * that cannot call cudaMalloc (no counterpart in the reference).  The caller
 * owns every array: q_dev (device, reference layout, double, ghost cells
 * included) is stepped in place, aux_dev is read (NULL when maux == 0); the
 * Runge-Kutta stage registers live in a fixed device array inside the library
 * of 3 * SCL_NOALLOC_MAX_VALUES doubles (4.5 MiB per GPU, held while the
 * library is loaded).  Grids with meqn*(mx+2*mbc) > SCL_NOALLOC_MAX_VALUES are
 * rejected (SCL_E_INVALID).  Calls on one GPU share that array: calls whose
 * work overlaps on the same GPU race, so serialise them.  The first call on a
 * device resolves the array's address; make it before any stream capture, and
 * do not reset the device afterwards (the address is kept for the process).
 * q_dev and aux_dev must be device or managed allocations of the current
 * device (anything else: SCL_E_INVALID, nothing launched); a CUDA error the
 * caller left pending is reported as SCL_E_CUDA and left in place.
 * stream is a cudaStream_t (NULL = default stream); when cfl is not NULL the
 * call waits for the step, returns the last stage's CFL number and reports a
 * non-finite state (SCL_E_NONFINITE) or a kernel error (SCL_E_CUDA); with cfl
 * NULL it returns once the step is enqueued and reports neither.  Double
 * state only (FP64, FP64_STRICT, MIXED). */
#define SCL_NOALLOC_MAX_VALUES 196608
int scl_rk_step_noalloc(const scl_params* p, double* q_dev, const double* aux_dev, double dt,
                        double* cfl, void* stream);

/* Discrete adjoint of one step of the handle's integrator (ts_ssp22, ts_ssp42,
 * ts_ssp33, ts_ssp104: sharpclaw.f90:247-464)
 * of dq = dt*L(q) (flux1/flux2 with componentwise or characteristic-wise
 * WENO5 and a Riemann solver that is linear in the jumps): given q^n and
 * lam_in = dJ/dq^{n+1}, returns lam_out = dJ/dq^n.  Device arrays in the
 * reference layout (interior cells are meaningful).  Built for the 2-D
 * acoustics plugin and the 1-D interface acoustics plugin
 * (apps/acoustics/1d/interface), with periodic bc and double state;
 * computed in FP64.  No reference counterpart (the reference
 * has no adjoint). */
int scl_adjoint_step(scl_handle* h, const double* q_dev, const double* lam_in_dev, double* lam_out_dev,
                     double dt);

/* ---- batched solver: many independent 1-D problems of uneven size ------ */
/* Replaces a host loop that calls sharpclaw() once per problem: every
 * instance k (mx[k] cells, spacing dx[k]) has its own controller (t, dt,
 * CFL, rejections, info) and all of them advance together, one persistent
 * launch per RK stage walking the active instances' tiles, captured in CUDA
 * graphs.  The plugin, options, integrator and precision come from p (its
 * mx/dx are ignored).  1-D plugins only. */
typedef struct scl_batch scl_batch;
int scl_batch_create(const scl_params* p, int ninst, const int* mx, const double* dx, scl_batch** out);
int scl_batch_destroy(scl_batch* b);
/* q: all instances concatenated, instance k in the reference layout
 * q(1-mbc:mx[k]+mbc, meqn) (double), ghost cells included; set_q fills ghosts. */
int scl_batch_set_q(scl_batch* b, const double* q);
int scl_batch_get_q(scl_batch* b, double* q);
int scl_batch_set_aux(scl_batch* b, const double* aux);
/* sharpclaw() on every instance with the same run parameters; dt_initial
 * (nullable) gives a first step per instance.  res has ninst entries; ms
 * (nullable) receives the device time of the time loop (CUDA events).  The
 * first run picks the faster tile width by timing a few steps of each from
 * the same start state (autotuning), then restores that state. */
int scl_batch_run(scl_batch* b, const scl_run* run, const double* dt_initial, scl_result* res, float* ms);
/* The autotuner's choice: variant index, threads per CTA, persistent grid
 * size and the trial time of each variant (3 entries: tile widths 128 and 256,
 * and the paired two-interfaces-per-thread tile of 1-D Euler in the FP32
 * forms; 0 for variants a plugin does not have). */
int scl_batch_tuning(scl_batch* b, int* variant, int* threads, int* grid, float* trial_ms);

/* Kernel launches (begin, stages, end of every captured step) of the last
 * scl_batch_run, autotuning trials excluded. */
long long scl_batch_launches(scl_batch* b);

/* Fix the batched tile variant (0, 1 or 2, as scl_batch_tuning reports them), or
 * with -1 let the next scl_batch_run time both and keep the faster (the
 * default).  No counterpart in the reference. */
int scl_batch_select(scl_batch* b, int variant);

/* Stream of the handle (cudaStream_t as void*), for callers that overlap work. */
void* scl_stream(scl_handle* h);

#ifdef __cplusplus
}
#endif
#endif /* SHARPCLAW_CUDA_H */
