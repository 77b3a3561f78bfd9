/*
 * sclaw_oracle.h -- CPU oracle for the SharpClaw semi-discrete WENO step.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (sharpclaw_b200/, include/)
 * links or calls this code; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load it, as the checker.
 *
 * The oracle restates, array by array and loop by loop, the reference Fortran:
 *   src/flux1.f90, src/reconstruct.f90 (weno5, weno5_char), src/2d/flux2.f90,
 *   src/1d/bc1.f90, src/2d/bc2.f90, src/1d/src1.f90, src/2d/src2.f90,
 *   src/1d/step1d.f90, src/2d/step2d.f90, src/sharpclaw.f90 (driver + ts_ssp*),
 * and the application plugins named in sclaw_oracle.c.  Arrays use the
 * reference layout: Fortran column-major with lower bound 1-mbc, i.e. element
 * (i,m) of a 1-D field is at (i+mbc-1) + (m-1)*(mx+2*mbc), and element (i,j,m)
 * of a 2-D field is at (i+mbc-1) + (j+mbc-1)*(mx+2*mbc) + (m-1)*(mx+2*mbc)*(my+2*mbc).
 *
 * Parity status: the reference ships no golden vectors and no Fortran compiler
 * exists on this machine, so the restatement is pinned by the reference's own
 * known-answer test (the exact acoustics interface solution used by
 * apps/acoustics/1d/interface/sharpclawtest.py) and by analytic invariants.
 */
#ifndef SCLAW_ORACLE_H
#define SCLAW_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Plugin families (device and oracle share the numbering). */
enum {
  OCL_RP_ADVECTION = 1,     /* apps/advection/1d/{rp1.f,tfluct1.f,evec.f}            */
  OCL_RP_EULER = 2,         /* apps/euler/shockentropy/rp1eu.f + new Roe evec          */
  OCL_RP_SW2D = 3,          /* apps/shallowWater/2dRadialDam/{rpn2sw.f,tfluct1sw.f}   */
  OCL_RP_ACOUSTICS1D = 4,   /* apps/acoustics/1d/interface/{rp1acv,tfluct1acv,evec}   */
  OCL_RP_ACOUSTICS2D = 5,   /* new 2-D variable-coefficient acoustics rpn2/tfluct/evec */
  OCL_RP_ADVECTION2D = 6,   /* apps/advection/2d/swirl/rpn2ad1.f (edge velocities)     */
  OCL_RP_SW1D = 7,          /* apps/shallowWater/2dRadialDam/1dRadialSymm-qwave/
                               {rp1sw.f,tfluct1sw.f} + new Roe evec                    */
  OCL_RP_SWF_BATHY = 8,     /* apps/shallowWater/1dPerturbSteady/{rpf-wave.f90,
                               tfluctf-wave.f90}: f-waves, bathymetry b = aux(:,1)     */
  OCL_RP_SWF_RADIAL = 9,    /* 2dRadialDam/1dRadialSymm-fwave: aux = (r, dx)            */
  OCL_RP_SWF_KAPPA = 10,    /* 2dRadialDam/1dRadialSymm-fwave-kappa: aux = (r(i-1/2),
                               r(i), r(i), dx), capacity aux(:,2)                      */
  OCL_RP_ACOUSTICS_CONST = 11,  /* apps/acoustics/1d/homogeneous/{rp1.f,tfluct.f,evec.f},
                                   common /cparam/ rho, bulk                           */
  OCL_RP_ACOUSTICS_FWAVE = 12,  /* apps/acoustics/1d/fwave/{rp1acfw.f,tfluct1.f,evec.f}:
                                   q = (strain, momentum), aux = (rho, bulk)           */
  OCL_RP_TRAFFIC = 13,      /* apps/traffic/congTraffic/{rpf-wave.f90,tfluct1.f90}:
                               flux umax(x) q (1-q), aux = umax                        */
  OCL_RP_ADVECTION_CONS = 14, /* apps/traffic/flux-uq/rpf-wave.f90: (u(x) q)_x, aux = u */
  OCL_RP_STEGOTON = 15      /* apps/elasticity/stegoton/{rp1nel.f,tfluct1.f}: sigma =
                               exp(A eps) - 1 (A > 0) or B eps, aux = (rho, A, B)      */
};

/* Source-term hooks: the src(q,dq,aux,t,dt) an app links (src/1d/step1d.f90:23). */
enum {
  OCL_SRC_NONE = 0,         /* src/1d/src1.f90: dq = 0                                 */
  OCL_SRC_RADIAL_SW = 1,    /* 1dRadialSymm-qwave/src1.f90: radial shallow water        */
  OCL_SRC_BATHYMETRY_SW = 2 /* 1dPerturbSteady/src1.f90: -g h b_x, b = aux(:,1)         */
};

typedef struct {
  int ndim;             /* 1 or 2                                  ClawParams%ndim  */
  int mx, my;           /* interior cells                          ClawParams%nx    */
  int meqn, mwaves, mbc, maux, mcapa;
  int lim_type;         /* 2 WENO5, 1 TVD (reconstruct.f90:525-763), 0 unlimited
                           polynomial (polyrecon.f90, order mthlim(1) = 3)          */
  int char_decomp;      /* 0 componentwise, 2 characteristic-wise                   */
  int tfluct_solver;    /* 1: tfluct plugin, 0: swap + second rp                    */
  int mthbc[4];         /* 1 extrap, 2 periodic, 3 wall, 0 user bc (bc_user)         */
  double dx, dy, xlower, ylower;
  int rp;               /* OCL_RP_* */
  int efix;             /* entropy fix flag (Euler default 1, SW default 0)          */
  double u;             /* advection speed        common /comrp/ u                  */
  double gamma;         /* ratio of specific heats common /param/ gamma,gamma1       */
  double grav;          /* gravity                 common /comrp/ g                  */
  int mthlim[4];        /* TVD limiter per component/field/wave (lim_type = 1)       */
  int b4step;           /* 0 src/b4step.f90 (no-op), 1 apps/advection/2d/swirl,
                           2 apps/elasticity/stegoton/b4step1.f (time reversal)       */
  double tperiod;       /* swirl: common /comvt/ tperiod                              */
  int src_term;         /* OCL_SRC_* (1-D)                                            */
  double rho, bulk;     /* homogeneous acoustics: common /cparam/ rho, bulk           */
  int bc_user;          /* 1: apps/elasticity/stegoton/bc1.f replaces src/1d/bc1.f90  */
  double wall[6];       /* t1, a1, tw1 (common /comwall/), t2, a2, tw2                 */
  int bc_switched;      /* the switch to periodic of bc1.f:31-35 has happened         */
  double trtime;        /* stegoton b4step: common /comtimereverse/ trtime             */
  int b4_done;          /* ... and its itrdone                                         */
} ocl_params;

typedef struct {
  double tstart, tend;
  double dt_initial, dt_max, cfl_max, cfl_desired;
  int max_steps, dt_variable, time_integrator;
} ocl_run;

typedef struct {
  double tend;          /* time reached */
  double cfl_maxused, cfl_last, dt_minused, dt_maxused, dt_last;
  int steps_taken, info, rejected;
  int bc_switched;      /* state of the user bc's switch after the run                */
} ocl_result;

/* size of a field with ghost cells (number of doubles per component) */
long ocl_plane(const ocl_params *p);

int ocl_bc(const ocl_params *p, double *q);

/* reconstruct.f90 weno5 / weno5_char on one line of mx2 = mx+2*mbc cells.
 * q, ql, qr: (mx2, meqn); evl, evr: (mx2, meqn, meqn). */
int ocl_weno5(int mx2, int meqn, const double *q, double *ql, double *qr);
/* reconstruct.f90:350-428; wave(mx2, meqn, mwaves) from the rp pass on the
   cell averages (flux1.f90:99-100) */
int ocl_weno5_wave(int mx2, int meqn, int mwaves, const double *q, const double *wave,
                   double *ql, double *qr);
/* reconstruct.f90:525-761: second-order TVD reconstructions (lim_type = 1) */
int ocl_tvd2(int mx2, int meqn, const double *q, const int *mthlim, double *ql, double *qr);
int ocl_poly(int mx2, int meqn, const double *q, int order, double *ql, double *qr);
int ocl_poly_wave(int mx2, int meqn, int mwaves, const double *q, int order, const double *wave,
                  double *ql, double *qr);
int ocl_tvd2_char(int mx2, int meqn, const double *q, const int *mthlim, const double *evl,
                  const double *evr, double *ql, double *qr);
int ocl_tvd2_wave(int mx2, int meqn, int mwaves, const double *q, const int *mthlim, const double *wave,
                  const double *s, double *ql, double *qr);
/* reconstruct.f90:244-347 (transmission-based, char_decomp = 3) */
int ocl_weno5_trans(int mx2, int meqn, const double *q, const double *evl,
                    const double *evr, double *ql, double *qr);
int ocl_weno5_char(int mx2, int meqn, const double *q, const double *evl,
                   const double *evr, double *ql, double *qr);

/* plugin calls on one line (Fortran loop ranges i = 2-mbc .. mx+mbc) */
int ocl_rp(const ocl_params *p, int ixy, int mx, const double *ql, const double *qr,
           const double *auxl, const double *auxr, double *wave, double *s,
           double *amdq, double *apdq);
int ocl_tfluct(const ocl_params *p, int ixy, int mx, const double *ql, const double *qr,
               const double *auxl, const double *auxr, double *s, double *adq);
int ocl_evec(const ocl_params *p, int ixy, int mx, const double *q, const double *auxl,
             const double *auxr, double *evl, double *evr);

/* flux1.f90: one line of mx cells; dq1d (mx+2mbc, meqn) is accumulated into
 * exactly as the reference does (zeroed first when ndim > 1). */
int ocl_flux1(const ocl_params *p, const double *q1d, double *dq1d, const double *aux1d,
              double dt, double *cfl, int ixy, int mx);

/* step1d/step2d: bc (in place on q), src (zero interior dq), flux1/flux2 */
int ocl_step(const ocl_params *p, double *q, double *dq, const double *aux, double dt,
             double t, double *cfl);

/* one time step of the SSP-RK integrator (ts_ssp22/42/33/104), q updated in
 * place, qold must hold q on entry (sharpclaw.f90:132-135). */
int ocl_rk_step(const ocl_params *p, int time_integrator, double *q, const double *qold,
                const double *aux, double dt, double told, double *cfl);

/* sharpclaw.f90:2-243 driver (b4step is the default no-op). */
int ocl_sharpclaw(const ocl_params *p, const ocl_run *run, double *q, const double *aux,
                  ocl_result *res);

/* src/1d/out1.f90, src/2d/out2.f90: fort.qNNNN, fort.tNNNN (and fort.aNNNN
   with outaux) in directory dir */
int ocl_output(const ocl_params *p, const double *q, const double *aux, double t, int iframe,
               const char *dir, int outaux);

#ifdef __cplusplus
}
#endif
#endif
