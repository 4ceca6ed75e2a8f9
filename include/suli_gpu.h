/*
 * suli_gpu.h — C-ABI of libsuli_gpu.so, the B200 (sm_100a) implementation of the
 * per-time-step hot path of SuLi-IC (lacia-udesc/SuLi-OpenMP, directory SuLi-IC/).
 *
 * The reference exposes its hot path as argument-less Fortran subroutines that read and
 * write module arrays (SuLi-IC/0_modules.f90:87-201).  This header replaces each of them
 * with one extern "C" entry point that acts on a solver context whose fields live in HBM:
 *
 *   reference subroutine (file:line)                  entry point here
 *   ------------------------------------------------  ---------------------------------
 *   level_set()            14_level_set.f90:221-285    suli_level_set
 *   heaviside()            14_level_set.f90:612-707    suli_heaviside
 *   mod_ls1()              14_level_set.f90:709-805    suli_mod_ls1
 *   level_set_ini() tail   14_level_set.f90:205-217    suli_level_set_ini
 *   visco()                5_viscosidade.f90:12-219    suli_visco
 *   convdiff()+classico()  6_convdiff.f90:14-189,
 *                          7_advectivo.f90:3-290       suli_convdiff
 *   tempo()                11_diversos.f90:10-230      suli_tempo
 *   contorno(nlock)        3_contorno.f90:10-492       suli_contorno
 *   graddin()              9_grad.f90:10-278           suli_graddin
 *   posdin()               10_pos.f90:1-96             suli_posdin
 *   est(div)               4_plot.f90:500-525          suli_est
 *   time loop body         1_principal.f90:64-108      suli_step
 *   dt = a_dt(tt)          1_principal.f90:78          suli_set_dt
 *   iniciais() RK table    2_iniciais.f90:85-104       suli_iniciais
 *
 * Conventions
 *  - Every function returns an int status: 0 = OK, > 0 = warning (e.g. the Poisson
 *    solve hit its iteration cap, which the reference only prints, 9_grad.f90:178),
 *    < 0 = error.  suli_last_error() gives a message for the last failing call.
 *  - Host arrays passed to suli_upload/suli_download use the reference's Fortran layout:
 *    column-major, i fastest, with the extents of the module arrays (halos included);
 *    suli_field_extent() returns them.  A Fortran caller passes c_loc(u) directly.
 *  - One context = one CUDA stream; a context must be used from one host thread at a time.
 *  - Nothing here falls back to the CPU: a missing device or kernel is an error.
 */
#ifndef SULI_GPU_H
#define SULI_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------ */
#define SULI_OK                 0
#define SULI_WARN_CG_MAXIT      1   /* Poisson solve stopped at cg_maxit (9_grad.f90:175-178) */
#define SULI_ERR_ARG           -1   /* bad argument / unsupported parameter combination      */
#define SULI_ERR_CUDA          -2   /* a CUDA call failed                                     */
#define SULI_ERR_NAN           -3   /* NaN/Inf met in a reduction                             */
#define SULI_ERR_UNSUPPORTED   -4   /* option of the reference not built here                 */
#define SULI_ERR_NOMEM         -5
#define SULI_ERR_NODEVICE      -6
#define SULI_ERR_SIZE          -7   /* size beyond a stated maximum                           */

/* ---- run-time parameters (the reference's compile-time parameters, 0_modules.f90) ---- */
typedef struct suli_params {
    int    nx, ny, nz;              /* cells (disc, 0_modules.f90:15)                          */
    double dx, dy, dz;              /* cell sizes (0_modules.f90:7)                            */
    double dt;                      /* base time step (0_modules.f90:9)                        */
    int    ccx0, ccxf;              /* x walls: 0 periodic 1 free-slip 2 no-slip 3 prescribed 4 outflow(xf) (0_modules.f90:53-54) */
    int    ccy0, ccyf;              /* y walls: 0 periodic 1 free-slip 2 no-slip 3 prescribed  (0_modules.f90:58-59) */
    int    ccz0, cczf;              /* z walls: 1 free-slip 2 no-slip 3 prescribed; 0 periodic is an extension (both ends) */
    int    t_tempo;                 /* 0 Euler, 1 RK2, 2 RK3, 3 AB2 (0_modules.f90:24)         */
    int    der;                     /* advection scheme: 1 upwind, 2 centred, 3 2nd-order upwind (0_modules.f90:26) */
    int    adv_type;                /* advective form: 1 classico, 2 rotacional, 3 antissim (2, 3 with der = 1) (0_modules.f90:27) */
    int    m_turb;                  /* 0 none, 1 Smagorinsky, 2 directional Smagorinsky (0_modules.f90:31) */
    int    obst_t;                  /* 0 none; 1..10 the obstaculo presets, masks set by suli_set_obstacle (0_modules.f90:29) */
    int    t_hs;                    /* density/viscosity mix in H: 0 linear, 1 geometric (0_modules.f90:199) */
    double csmag;                   /* Smagorinsky constant (0_modules.f90:181)                */
    double gx, gz;                  /* gravity components, gz acts downward (0_modules.f90:143) */
    double chezy;                   /* wall-friction Chezy coefficient (0_modules.f90:141)     */
    double rho_f1, mi_f1;           /* fluid where ls < 0 (air)   (14_level_set.f90:26-27)     */
    double rho_f2, mi_f2;           /* fluid where ls > 0 (water) (14_level_set.f90:28-29)     */
    double sigma;                   /* surface tension (14_level_set.f90:30)                   */
    double alpha1;                  /* Heaviside half-width in cells (14_level_set.f90:25)     */
    double dt1;                     /* reinitialisation pseudo time step, 0.1*max(dx,dy,dz) (0_modules.f90:198) */
    int    reinit_maxit;            /* 3 (14_level_set.f90:397)                                */
    double vol_tol;                 /* volume-correction trigger, 0.1 (14_level_set.f90:257)   */
    /* Poisson solve (9_grad.f90:175): cg_stop 0 = the reference's test sum(r~^2) > cg_tol/(nx*ny*nz),
       checked on the residual at the start of the iteration (cg_tol = 1e-4 reproduces it);
       cg_stop 1 = relative test ||r~||_2 <= cg_tol * ||b~||_2 on the current residual. */
    int    cg_stop;
    double cg_tol;
    int    cg_maxit;                /* 10000 in the reference                                  */
    int    precision;               /* 0 = plain FP64; 1 = FP32 stencil arithmetic (convdiff, Smagorinsky, WENO
                                       level set) over FP64 fields, FP32 multigrid-preconditioned inner CG
                                       with FP64 residual/refinement, FP64 projection, divergence, volume */
    int    refine_maxit;            /* outer FP64 refinement sweeps for precision 1            */
    double inner_tol;               /* relative tolerance of each FP32 inner solve             */
    double mg_omega;                /* precision 1: damping of the multigrid Jacobi sweeps (0 = 0.9) */
    double mg_alpha;                /* precision 1: scale of the coarse-grid correction (0 = 1.8)     */
    int    mg_kernels;              /* precision 1: 0 = vectorised multigrid/PCG kernels (4 x cells a
                                       thread, float4 loads), every level its own kernels (default);
                                       1 = one cell a thread (same arithmetic, kept as the reference
                                       the tests compare with); 2 = vectorised, with the three
                                       coarsest levels in one 16-CTA cluster launch where their
                                       shapes allow (measured slower at 256x128x128) */
    int    wave_t;                  /* wave inflow at x = 0: 0 none, 1 Stokes I, 2 Stokes II, 5 Stokes V (0_modules.f90:35) */
    int    outflow_fix;             /* 0 = the reference's outflow copy (3_contorno.f90:193-197, 362-409);
                                       1 (extension, needs ccxf = 4) = contorno(2) then shifts the
                                       outflow plane u(nx+1,:,:) above the obstacle mask by one uniform
                                       value so that the net boundary flux is zero and graddin's
                                       all-Neumann system (9_grad.f90:96-116) is consistent */
    int    periodic_faces;          /* 0 = the reference: graddin and posdin take the face density of
                                       interp?_cf, whose end faces copy their neighbour (8_derivadas.f90:318-323);
                                       1 (extension) = on a periodic axis both end faces, one face of the
                                       periodic box, take the average across the wrap, which keeps the
                                       scaled Poisson operator symmetric when the density varies there */
    double mg_omega2;               /* precision 1: weight of the second pre-smoothing sweep and of the
                                       first post-smoothing one (0 = mg_omega); two different weights
                                       make the smoother a degree-2 polynomial (Chebyshev-like) */
    double div_tol;                 /* 0 = off (the reference); > 0 (extension): the Poisson solve also
                                       requires max |sqrt(d) r~| <= div_tol, the largest |div u| the
                                       projection leaves (the unscaled residual), and iterates on
                                       (FP64 CG: threshold lowered and the loop resumed; precision 1:
                                       another refinement pass) until both tests hold or the cap */
} suli_params;

/* ---- field identifiers (module arrays of 0_modules.f90) ------------------------------ */
enum suli_field {
    SULI_F_U = 0, SULI_F_V, SULI_F_W,                 /* velpre u,v,w   (0_modules.f90:92-94)  */
    SULI_F_PRD1, SULI_F_PRD0, SULI_F_PRD,             /* velpre (0_modules.f90:121)          */
    SULI_F_RHO, SULI_F_LS_NU,                         /* velpre (0_modules.f90:122)          */
    SULI_F_FU, SULI_F_U0, SULI_F_FU0, SULI_F_FU1,     /* vartempo (0_modules.f90:131)        */
    SULI_F_FV, SULI_F_V0, SULI_F_FV0, SULI_F_FV1,     /* vartempo (0_modules.f90:132)        */
    SULI_F_FW, SULI_F_W0, SULI_F_FW0, SULI_F_FW1,     /* vartempo (0_modules.f90:133)        */
    SULI_F_NUT, SULI_F_XNUT, SULI_F_YNUT, SULI_F_ZNUT,/* smag (0_modules.f90:182-185)        */
    SULI_F_LS, SULI_F_MOD_LS, SULI_F_KURV, SULI_F_HS, /* ls_param (0_modules.f90:193)        */
    SULI_F_DDLSDX, SULI_F_DDLSDY, SULI_F_DDLSDZ,
    SULI_F_HSX, SULI_F_HSY, SULI_F_HSZ,
    SULI_F_UB, SULI_F_VB, SULI_F_WB,                  /* obst (0_modules.f90:71-73)          */
    SULI_F_TF_U, SULI_F_TF_V, SULI_F_TF_W,            /* mms_m source terms (0_modules.f90:215-217) */
    /* prescribed-boundary planes (velpre, 0_modules.f90:96-118) */
    SULI_F_BXX0, SULI_F_BXX1, SULI_F_BXY0, SULI_F_BXZ0,
    SULI_F_BXXF, SULI_F_BXXF1, SULI_F_BXYF, SULI_F_BXZF,
    SULI_F_BYX0, SULI_F_BYY0, SULI_F_BYY1, SULI_F_BYZ0,
    SULI_F_BYXF, SULI_F_BYYF, SULI_F_BYYF1, SULI_F_BYZF,
    SULI_F_BZX0, SULI_F_BZY0, SULI_F_BZZ0, SULI_F_BZZ1,
    SULI_F_BZXF, SULI_F_BZYF, SULI_F_BZZF, SULI_F_BZZF1,
    SULI_F_COUNT
};

/* ---- scalar identifiers --------------------------------------------------------------- */
enum suli_scalar {
    SULI_S_DT = 0,      /* the global dt, mutated per RK stage (1_principal.f90:78) */
    SULI_S_VOL_INI,     /* ls_param vol_ini (14_level_set.f90:208-215) */
    SULI_S_VOL_INS,     /* ls_param vol_ins (14_level_set.f90:246-253) */
    SULI_S_DT1,         /* ls_param dt1 */
    SULI_S_T,           /* disc t */
    SULI_S_NTT,         /* number of RK stages (2_iniciais.f90:85-104) */
    SULI_S_A_DT1, SULI_S_A_DT2, SULI_S_A_DT3,
    SULI_S_FALLBACKS,   /* read only, no counterpart in the reference: precision-1 solves that the
                           plain FP64 CG finished because the FP32 refinement stopped converging */
    SULI_S_COUNT
};

/* Inclusive Fortran index ranges of a field (planes have lo[2] = hi[2] = 0). */
int suli_field_extent(const suli_params* p, int field, int lo[3], int hi[3]);
/* The reference's compiled defaults, 0_modules.f90 and 14_level_set.f90:25-31. */
int suli_params_default(suli_params* p);
/* sizeof(suli_params) and sizeof(suli_step_stats) as compiled, for binding checks
   (no counterpart in the reference, which has no foreign-language boundary). */
int suli_abi_sizes(int* params_bytes, int* stats_bytes);

/* ---- context ---------------------------------------------------------------------------- */
typedef struct suli_ctx suli_ctx;

/* Allocates every field in HBM of `device` and zeroes it.  Replaces the static module
   arrays of 0_modules.f90 (the reference's 30M-cell guard, 1_principal.f90:31-34, is lifted). */
int suli_create(const suli_params* p, int device, suli_ctx** out);
int suli_destroy(suli_ctx* c);
const char* suli_last_error(const suli_ctx* c);
int suli_synchronize(suli_ctx* c);

/* Fortran-layout copies (c_loc of the module array).  Synchronous.  The pointer may be host
   memory or device memory of any GPU (unified addressing decides the copy's direction). */
int suli_upload(suli_ctx* c, int field, const double* host);
int suli_download(suli_ctx* c, int field, double* host);
int suli_set_scalar(suli_ctx* c, int scalar, double v);
int suli_get_scalar(suli_ctx* c, int scalar, double* v);

/* iniciais() without the presets: u = u_init, v = w = 0, prd = 0, ub = 0, RK table
   (2_iniciais.f90:36-46, 85-104).  The level-set preset is written by the caller. */
int suli_iniciais(suli_ctx* c, double u_init);
/* The tail of level_set_ini after the caller's preset: ls += ls_m for t_hs = 1, heaviside();
   vol_ini = sum(hs) dV; mod_ls1() (14_level_set.f90:196-217). */
int suli_level_set_ini(suli_ctx* c);
/* The bottom-obstacle masks that obstaculo() computes (3_contorno.f90:494-762; module obst,
   0_modules.f90:76-79): for each column, the k up to which the velocities are zeroed.
   Host arrays in Fortran order: ku(0:nx+2, 0:ny+1), kv(0:nx+1, 0:ny+2), kw(0:nx+1, 0:ny+1);
   ku and kv within [-1, nz], kw within [-1, nz+1] (else SULI_ERR_ARG, as obstaculo clamps
   them).  Needs obst_t != 0.  Set them before suli_iniciais, which zeroes the inflow planes
   below ku (2_iniciais.f90:60-65); contorno(1), contorno(2) then zero the columns and capture
   the wall-friction velocities above them, contorno(3) extends the level set into the
   obstacle (3_contorno.f90:266-294, 445-487). */
int suli_set_obstacle(suli_ctx* c, const int* ku, const int* kv, const int* kw);

/* Hot-path subroutines. */
int suli_level_set(suli_ctx* c, double* vol_ins);          /* 14_level_set.f90:221-285 */
int suli_heaviside(suli_ctx* c);                           /* 14_level_set.f90:612-707 */
int suli_mod_ls1(suli_ctx* c);                             /* 14_level_set.f90:709-805 */
int suli_visco(suli_ctx* c);                               /* 5_viscosidade.f90:12-219 */
int suli_convdiff(suli_ctx* c);                            /* 6_convdiff.f90:14-189    */
int suli_tempo(suli_ctx* c, int tt, int it);               /* 11_diversos.f90:10-230   */
int suli_contorno(suli_ctx* c, int nlock);                 /* 3_contorno.f90:10-492    */
int suli_graddin(suli_ctx* c, int* iters, double* resid); /* 9_grad.f90:10-278; resid = ||r~||/||b~|| */
int suli_posdin(suli_ctx* c);                              /* 10_pos.f90:1-96          */
int suli_est(suli_ctx* c, double* max_div);                /* 4_plot.f90:500-525 (FP64) */
int suli_set_dt(suli_ctx* c, double dt);                   /* dt = a_dt(tt), 1_principal.f90:78 */
/* boundary_waves() (3_contorno.f90:952-1082): with wave_t != 0, the wave's inflow planes
   bxx0, bxx1, bxz0 at the context's time t, the level set of column i = 1, and the reference's
   single-precision round trip of the whole level set; the step calls it after tempo. */
int suli_boundary_waves(suli_ctx* c);

typedef struct suli_step_stats {
    int    cg_iters[3];     /* Poisson iterations of each RK stage (inner FP32 iterations for precision 1) */
    double cg_resid[3];     /* final relative FP64 residual of each stage */
    double vol_ins;
    double max_div;         /* max |div u| after the step (FP64) */
    int    status;
} suli_step_stats;

/* One time step it (1_principal.f90:64-108 without MMS/plot/restart), plus est(). */
int suli_step(suli_ctx* c, int it, suli_step_stats* st);

/* One time step whose state crosses from and back to host memory, for a time loop that keeps
   the module arrays on the host as the reference's loop does (1_principal.f90:64-108, every
   subroutine acting on the host arrays of 0_modules.f90).  The same as suli_upload of each
   in_fields[q] from in_host[q], suli_step, then suli_download of each out_fields[q] into
   out_host[q], with the same results, but the copies run on two copy streams and overlap the
   step where its order allows: prd1, which the step first reads in the first RK stage's
   convdiff (its prd0 = prd1 copy), is copied in while the level-set stage runs, and ls, which
   nothing after the level-set stage writes (without wave inflow), is copied out while the RK
   stages run.  Host buffers should be pinned for the overlap (pageable memory works, with the
   copies serialised).  At most SULI_STEP_HOST_MAX_FIELDS fields each way, no field twice in
   one list; planes and tf_u/v/w are copied synchronously before or after the step.  A field's
   output may use the same host array as its input; an output array must not overlap the
   input array of another field.  The call returns once every copy has landed; after an error
   the fields may hold a partly updated state.  The first call allocates one staging box per copied
   field and two streams; a later call allocates only for list positions that no earlier call
   used.
   No counterpart in the reference (an addition for a host-side driver of this library). */
#define SULI_STEP_HOST_MAX_FIELDS 8
int suli_step_host(suli_ctx* c, int it, int n_in, const int* in_fields, const double* const* in_host, int n_out,
                   const int* out_fields, double* const* out_host, suli_step_stats* st);

/* ---- learned initial guess / preconditioner of the pressure solve ------------------------
   No counterpart in the reference (an addition of this build for the variable-density
   Poisson solve of 9_grad.f90).  A 3-D U-Net (4 levels, 16/32/64/96 channels, 3x3x3
   convolutions, BF16 weights, FP32 accumulation on the tensor cores) maps three channels
   (scaled residual, density feature, scaled previous pressure) to the scaled correction of the
   pressure.  Grid dimensions must be multiples of 8.  Device buffers: in3 [V][3] FP32 and
   out/target [V] FP32, x fastest. */
typedef struct suli_nn suli_nn;
long long suli_nn_num_params(void);
int suli_nn_create(int nx, int ny, int nz, int device, suli_nn** out);
int suli_nn_destroy(suli_nn* n);
const char* suli_nn_last_error(const suli_nn* n);
int suli_nn_set_params(suli_nn* n, const float* host, long long count);   /* FP32 master weights */
int suli_nn_get_params(suli_nn* n, float* host, long long count);
int suli_nn_forward(suli_nn* n, const float* d_in3, float* d_out);
/* mean squared error against d_target and its gradient (copied to host_grad if not null) */
int suli_nn_loss_grad(suli_nn* n, const float* d_in3, const float* d_target, double* loss, float* host_grad);
int suli_nn_train_step(suli_nn* n, const float* d_in3, const float* d_target, float lr, double* loss);
/* the convolution primitive on caller buffers: channels-last BF16 x [V][cin], w [27][cout][cin]
   (tap = dx + 3 dy + 9 dz), bias [cout] FP32 or NULL, out [V][cout] BF16 = relu?(conv(x) + b) */
int suli_nn_conv3d(int nx, int ny, int nz, const void* x, int cin, const void* w, const float* bias, int cout,
                   int relu, void* out, int kernel);
/* as suli_nn_conv3d, plus what the network fuses into a convolution: pool_out (or NULL) gets the
   2x2x2 average of the BF16 output [V/8][cout] BF16 (even grid); head_w (17 floats: 16 weights,
   bias; cout = 16) and head_out [V] FP32 (or NULL) the 1x1x1 head of the BF16 output.  Kernel 0
   computes them in the convolution's epilogue, kernels 1 and 2 with separate kernels. */
int suli_nn_conv3d_ex(int nx, int ny, int nz, const void* x, int cin, const void* w, const float* bias, int cout,
                      int relu, void* out, void* pool_out, const float* head_w, float* head_out, int kernel);
/* convolution kernel of a network (and of suli_nn_conv3d's last argument): 0 = persistent
   tcgen05 pipeline (TMA loads, accumulators in TMEM; default), 1 = mma.sync tensor cores,
   2 = tcgen05 with one output tile per CTA */
int suli_nn_set_kernel(suli_nn* n, int kernel);

/* Attach a network to a context (same grid and device) for its pressure solves.
   mode 0 detaches; mode 1 (precision 1 only) uses the network as the initial guess: after
   graddin's set-up the network maps (r~0/s, H, (e0 - mean)/s_e) to a correction y of the
   scaled pressure, and e0 <- e0 + alpha s y with alpha = -(r~0 . y)/(y . A~ y), the
   energy-norm optimal step in FP64, so the guess never raises the A~-norm error of e0.  The
   solve then runs to the same FP64 stopping test as without the network.  Mode 2 (precision 1)
   also applies the network as the preconditioner of the outer FP64 iteration: after every
   refinement pass that has not met the stopping tests, the network maps the current residual
   and iterate to a correction, applied with the same energy-optimal step (a nonlinear
   preconditioner; the multigrid-preconditioned inner CG, and the plain FP64 CG as its fallback,
   still decide when the solve is done).  A network serves one context at a time (it keeps its
   activations). */
int suli_attach_nn(suli_ctx* c, suli_nn* net, int mode);
/* graddin() that also records a training pair of the network: d_in3 [V][3] receives the
   network's input features of the solve's starting state and d_target [V] the scaled
   correction (e* - e0)/s to the converged solution, less its component along sqrt(d) (the
   null vector of A~ for the all-Neumann pressure problem) (device FP32 buffers, x fastest
   over the nx x ny x nz cells).  Any precision; an attached network is not applied. */
int suli_graddin_record(suli_ctx* c, float* d_in3, float* d_target, int* iters, double* resid);

/* ---- divergence check that allocates nothing ---------------------------------------------
   No counterpart in the reference: an extra way to run est() for callers that may not let a
   library allocate device memory.  Typical callers: a driver whose u, v, w already live on
   the GPU under another runtime (OpenACC or CUDA Fortran device arrays, or a framework whose
   caching allocator has reserved the memory), where a cudaMalloc could fail for lack of
   unreserved memory and cudaMalloc/cudaFree would stall the device.  It needs no context.
   u, v, w: device pointers in the reference's Fortran layout u(0:nx+2,0:ny+1,0:nz+1),
   v(0:nx+1,0:ny+2,0:nz+1), w(0:nx+1,0:ny+1,0:nz+2); max_div: device pointer to one double;
   stream: a cudaStream_t (NULL = default stream).  Runs on the calling thread's current
   device and returns without waiting for the result.
   Scratch: a fixed array inside the library (SULI_EST_STATIC_MAX_BLOCKS block partials,
   about 64 KiB), held on every GPU that loads the library until the process exits.  Grids
   needing more blocks (one block per 32 x 8 x 16 cells; 512 x 256 x 256 fits exactly) are
   refused with SULI_ERR_SIZE.  The first call on a device looks up the array's device
   address; make that first call before any stream capture.  All calls share the array:
   calls that overlap on the GPU race and must be ordered by the caller. */
#define SULI_EST_STATIC_MAX_BLOCKS 8192
int suli_est_static(const double* u, const double* v, const double* w, int nx, int ny, int nz,
                    double dx, double dy, double dz, double* max_div, void* stream);

/* ---- tracing (replaces the wall-clock bookkeeping of 4_plot.f90:113-120, 253-257) ----- */
/* Kernel classes timed with CUDA events on the context's stream when profiling is on. */
enum suli_kernel {
    SULI_K_LS_ADVECT = 0,  /* conv_weno + intt_ls stage           */
    SULI_K_REINIT,         /* reinic_weno stages, S(phi0), error  */
    SULI_K_LSPROPS,        /* der_weno + mod_ls1 part A + heaviside + volume */
    SULI_K_CURV,           /* mod_ls1 part B (curvature)          */
    SULI_K_VOLFIX,         /* volume correction                   */
    SULI_K_VISCO,
    SULI_K_CONVDIFF,
    SULI_K_TEMPO,
    SULI_K_CONTORNO,
    SULI_K_CG_SETUP,
    SULI_K_CG_SPMV,        /* CG kernel A: p = r + beta p, q = A p, p.q */
    SULI_K_CG_UPDATE,      /* CG kernel B: e -= alpha p, r -= alpha q, r.r */
    SULI_K_CG_FINAL,
    SULI_K_POSDIN,
    SULI_K_EST,
    SULI_K_MG,             /* precision 1: FP32 inner PCG iterations (SpMV, update, multigrid
                              V-cycle), launched as one CUDA graph per iteration */
    SULI_K_REFINE,         /* precision 1: FP64 residual and correction of the refinement */
    SULI_K_NN,             /* learned initial guess: the network's forward pass (its input
                              features and the FP64 step count as CG_SETUP) */
    SULI_K_COUNT
};
/* The CUDA stream (cudaStream_t) this context launches on, for callers ordering their own
   work or events against it. */
int suli_stream(suli_ctx* c, void** stream);
/* Turn per-kernel timing on (clearing the counters) or off. */
int suli_profile_enable(suli_ctx* c, int on);
/* Totals since enable: device milliseconds and launches per kernel class, and the number of
   CG iterations actually performed (launches after convergence return at once). */
int suli_profile_read(suli_ctx* c, double ms[SULI_K_COUNT], long long launches[SULI_K_COUNT],
                      long long* cg_iterations);

#ifdef __cplusplus
}
#endif
#endif /* SULI_GPU_H */
