// ctx.cuh — the solver context: device field arena, scalars, scratch, and the kernel
// launchers shared by the host API (suli_gpu.cu) and the kernel translation units.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <string>
#include <vector>
#include "../../include/suli_gpu.h"
#include "geom.cuh"
#include "waves.cuh"

namespace suli {

// the coarsest multigrid solve's Chebyshev coefficients (formed on the host, k_mixed.cu)
constexpr int kCoarseMaxCheb = 64;   // most Chebyshev steps
struct CoarsePoly {
    float lo;                        // > 0: the Chebyshev polynomial over [lo, 2], else damped Jacobi sweeps
    float g0;
    float h[kCoarseMaxCheb], g[kCoarseMaxCheb];   // step m = 1 .. steps - 1 at index m - 1
};

// Device-resident state of the Poisson solve (graddin, 9_grad.f90:10-278).  Written by the
// last block of each reduction kernel; read by the next kernel and, at poll points, by the
// host through a pinned mirror.
struct CGState {
    double rr;        // r~.r~ of the current residual
    double rr_start;  // r~.r~ at the start of the current iteration (alfamupr)
    double alpha;
    double beta;
    double bb;        // b~.b~ (scaled right-hand side)
    double thr;       // stopping threshold on r~.r~
    double pq;        // last p.q
    int iters;
    int done;
    int maxit;
    int mode;         // suli_params.cg_stop
    int status;       // 0 ok, SULI_WARN_CG_MAXIT, SULI_ERR_NAN
    int pad;
    double div_tol;   // suli_params.div_tol (0: off)
    double rmax;      // max |sqrt(d) r~| of the last check: the max |div u| projection leaves
};

// State of the FP32 inner preconditioned CG of the mixed-precision solve (device resident).
struct PCGState {
    double rz;      // r.z of the current residual
    double rr;      // r.r
    double rr0;     // r.r of the right-hand side of this inner solve
    double pq;
    double alpha;
    double beta;
    double tol2;    // stop when r.r <= tol2
    int iters;
    int done;
    int maxit;
    int status;
};

// Scales of the learned initial guess (device resident): rms of the first scaled residual,
// mean and rms deviation of e0, the FP64 step length, the null-space coefficient of a
// recorded target, and whether the guess applies.
struct NNScale {
    double sigma_r;
    double mean_e;
    double sigma_e;
    double alpha;
    double proj;
    int active;
};

// One level of the FP32 multigrid hierarchy: face conductances, inverse Jacobi diagonal,
// vectors; level 0 also holds the FP32 density its kernels form the faces from, and the
// dt-dependent face constants.
struct MGLevel {
    Geo g;
    float *sx = nullptr, *sy = nullptr, *sz = nullptr, *idg = nullptr;
    float *f = nullptr, *x = nullptr, *y = nullptr;
    float *rho = nullptr, *c2 = nullptr;
};

// Boundary planes of prescribed walls (velpre, 0_modules.f90:96-118), Fortran layout.
struct Planes {
    const double *bxx0, *bxx1, *bxy0, *bxz0, *bxxf, *bxxf1, *bxyf, *bxzf;
    const double *byx0, *byy0, *byy1, *byz0, *byxf, *byyf, *byyf1, *byzf;
    const double *bzx0, *bzy0, *bzz0, *bzz1, *bzxf, *bzyf, *bzzf, *bzzf1;
};

// Deterministic reduction scratch: one slot of per-block partials plus a block counter.
struct RedSlot {
    double* partial;       // [max_blocks * 2]
    unsigned int* counter;
    double* out;           // [2] results
};

constexpr int kMaxRedBlocks = 1 << 16;

}  // namespace suli

struct suli_ctx {
    suli_params P;
    suli::Geo g;
    suli::BC bc;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    // one arena for all 3-D fields
    double* arena = nullptr;
    size_t arena_elems = 0;
    double* f[SULI_F_COUNT] = {nullptr};   // 3-D fields in the shared box; planes separate
    size_t plane_elems[SULI_F_COUNT] = {0};
    // work arrays (same box)
    double *ls1 = nullptr, *ls2 = nullptr, *funcs = nullptr;
    double *nrmx = nullptr, *nrmy = nullptr, *nrmz = nullptr;
    double *cg_d = nullptr, *cg_e = nullptr, *cg_r = nullptr, *cg_b = nullptr;
    double *cg_pa = nullptr, *cg_pb = nullptr, *cg_q = nullptr;
    double *cg_ax = nullptr, *cg_ay = nullptr, *cg_az = nullptr;
    // reductions
    double* red_partial = nullptr;
    unsigned int* red_counter = nullptr;
    double* red_out = nullptr;
    suli::CGState* cg = nullptr;        // device
    suli::CGState* cg_host = nullptr;   // pinned mirror
    double* host_scalars = nullptr;     // pinned, small
    // scalars of disc / ls_param
    double dt = 0, t = 0, dt1 = 0, vol_ini = 0, vol_ins = 0;
    int ntt = 1;
    double a_dt[3] = {0, 0, 0};
    bool tf_active = false;             // tf_u/v/w uploaded non-zero
    // obstacle masks (suli_set_obstacle): ku (nx+3)x(ny+2), kv (nx+2)x(ny+3), kw (nx+2)x(ny+2),
    // Fortran order, one device allocation; host copies for suli_iniciais
    int* obst_k = nullptr;
    const int *obst_ku = nullptr, *obst_kv = nullptr, *obst_kw = nullptr;   // into obst_k
    std::vector<int> obst_ku_host;
    suli::WaveCoef wave;                // waves_coef of the wave inflow (wave_t != 0)
    int last_reinit_iters = 0;
    int last_volfix_iters = 0;
    // mixed-precision solve (precision = 1)
    std::vector<suli::MGLevel> mg;
    float *pc_x = nullptr, *pc_r = nullptr, *pc_pa = nullptr, *pc_pb = nullptr, *pc_q = nullptr;
    float* pc_r2 = nullptr;   // the inner residual is updated from one buffer into the other
    double* cg_e2 = nullptr;
    double* cg_sd = nullptr;    // sqrt(d), stored once per solve (ghost values, the refinement's scaling)
    double* cg_isd = nullptr;   // 1/sqrt(d) (the coefficient scaling)
    suli::PCGState* pcg = nullptr;
    suli::PCGState* pcg_host = nullptr;
    float* f32_arena = nullptr;
    int coarse_sweeps = 20;     // steps of the coarsest solve
    float coarse_lo = 0.02f;    // > 0: the coarsest solve is a Chebyshev polynomial over [coarse_lo, 2]
    suli::CoarsePoly coarse_poly = {};
    bool cluster_ok = false;    // the device runs k_mg_cluster (16-CTA cluster with its shared memory)
    bool fuse_update = false;   // the inner PCG update runs inside the level-0 pre-smoothing kernel
    bool mg_fused = false;      // the coarse levels run one kernel a V-cycle leg (k_mg_fused.cuh)
    bool tail_ok = false;       // the device runs k_mg_tail (one CTA, the last two levels)
    int mg_kz = 2;              // cells along z a thread of the vectorised multigrid kernels owns (2 or 4)
    // level-0 kernels that stream z-planes through shared memory with TMA (k_mg_stream.cuh):
    // one tensor map per level-0 array they read, the planes a CTA computes, and whether they run
    bool stream_ok = false;
    bool stream_post_ok = false;   // also the post-smoothing (nx a multiple of 32)
    int stream_chunk = 16;
    int n_smap = 0;
    CUtensorMap smap_c;            // level 1's correction, the post-smoothing's prolongation source
    CUtensorMap smap[12];          // boxes with the halo
    CUtensorMap smap_own[12];      // the same arrays, boxes of the tile's own cells
    const float* smap_ptr[12] = {nullptr};
    int inner_maxit = 200;
    int inner_batch = 4;
    int last_outer_iters = 0;
    long long fallbacks = 0;   // mixed solves finished by the plain FP64 CG (the refinement stalled)
    // one CUDA graph per ping-pong parity holding a whole inner PCG iteration
    // the inner PCG loop as one graph: a WHILE node repeats two iterations (ping-pong) and a
    // kernel that clears the condition once the inner solve is done
    cudaGraphExec_t pcg_loop = nullptr;
    cudaGraphExec_t cg_loop = nullptr;   // the plain FP64 CG iterations as one device-side loop
    int pcg_graph_kernels = 0;   // kernels of one inner iteration
    // learned initial guess (suli_attach_nn) and training-pair recording (suli_graddin_record)
    suli_nn* nn = nullptr;
    int nn_mode = 0;
    float* nn_out = nullptr;   // the network's output [V]
    double* nn_e0 = nullptr;                     // e0 of a recorded solve (box layout)
    suli::NNScale* nn_scale = nullptr;
    float *rec_in = nullptr, *rec_target = nullptr;
    // false (environment SULI_EAGER_LOOPS=1, for per-kernel profiling): the CG and inner PCG
    // iterations are launched one by one from the host, two at a time with a check of the
    // device state after each pair, in place of the device-side graph loop; same kernels, same
    // order, same results
    bool use_graphs = true;
    // suli_step_host (allocated on its first call): one copy stream per direction, and per
    // copied field a staging box (Fortran layout) and the event that orders its copy
    cudaStream_t io_in = nullptr, io_out = nullptr;
    double* io_stage[2 * SULI_STEP_HOST_MAX_FIELDS] = {nullptr};
    cudaEvent_t io_ev[2 * SULI_STEP_HOST_MAX_FIELDS] = {nullptr};
    // tracing: CUDA-event pairs around each kernel class (suli_profile_*)
    struct Prof {
        bool on = false;
        std::vector<cudaEvent_t> ev;   // 2 per pair
        std::vector<int> kind;
        int used = 0;
        double ms[SULI_K_COUNT] = {0};
        long long launches[SULI_K_COUNT] = {0};
        long long cg_iters = 0;
    } prof;
    suli::Planes planes() const;
};

namespace suli {
// Accumulate the timed pairs recorded so far (synchronises the stream).
inline void prof_resolve(suli_ctx* c) {
    auto& P = c->prof;
    if (P.used == 0) return;
    cudaStreamSynchronize(c->stream);
    for (int q = 0; q < P.used; ++q) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, P.ev[2 * q], P.ev[2 * q + 1]) == cudaSuccess) P.ms[P.kind[q]] += t;
    }
    P.used = 0;
}
// RAII timer of one kernel class around `n` launches on the context's stream.
struct ProfScope {
    suli_ctx* c;
    int slot = -1;
    ProfScope(suli_ctx* ctx, int kind, int n) : c(ctx) {
        auto& P = c->prof;
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        cudaStreamIsCapturing(c->stream, &cs);
        if (cs != cudaStreamCaptureStatusNone) return;   // inside a graph capture: counted at launch
        P.launches[kind] += n;
        if (!P.on) return;
        if (P.used * 2 + 2 > (int)P.ev.size()) prof_resolve(c);
        slot = P.used++;
        P.kind[slot] = kind;
        cudaEventRecord(P.ev[2 * slot], c->stream);
    }
    ~ProfScope() {
        if (slot >= 0) cudaEventRecord(c->prof.ev[2 * slot + 1], c->stream);
    }
};
}  // namespace suli

inline suli::Planes suli_ctx::planes() const {
    suli::Planes pl;
    pl.bxx0 = f[SULI_F_BXX0]; pl.bxx1 = f[SULI_F_BXX1]; pl.bxy0 = f[SULI_F_BXY0]; pl.bxz0 = f[SULI_F_BXZ0];
    pl.bxxf = f[SULI_F_BXXF]; pl.bxxf1 = f[SULI_F_BXXF1]; pl.bxyf = f[SULI_F_BXYF]; pl.bxzf = f[SULI_F_BXZF];
    pl.byx0 = f[SULI_F_BYX0]; pl.byy0 = f[SULI_F_BYY0]; pl.byy1 = f[SULI_F_BYY1]; pl.byz0 = f[SULI_F_BYZ0];
    pl.byxf = f[SULI_F_BYXF]; pl.byyf = f[SULI_F_BYYF]; pl.byyf1 = f[SULI_F_BYYF1]; pl.byzf = f[SULI_F_BYZF];
    pl.bzx0 = f[SULI_F_BZX0]; pl.bzy0 = f[SULI_F_BZY0]; pl.bzz0 = f[SULI_F_BZZ0]; pl.bzz1 = f[SULI_F_BZZ1];
    pl.bzxf = f[SULI_F_BZXF]; pl.bzyf = f[SULI_F_BZYF]; pl.bzzf = f[SULI_F_BZZF]; pl.bzzf1 = f[SULI_F_BZZF1];
    return pl;
}

namespace suli {
// ---- kernel launchers (k_fp64.cu) ----
void launch_lsprops(suli_ctx* c, const double* ls, bool do_mod, bool do_hs, bool do_vol);
void launch_boundary_waves(suli_ctx* c);
void launch_curv(suli_ctx* c);
void launch_ls_advect(suli_ctx* c, const double* cur, const double* phi0, double* out,
                      double a, double b, double gd);
void launch_reinit_funcs(suli_ctx* c);
void launch_reinit_stage(suli_ctx* c, const double* cur, const double* phi0, double* out,
                         double a, double b, double gd);
void launch_reinit_err(suli_ctx* c, const double* after, const double* before, double band);
void launch_volfix(suli_ctx* c, double fac);
void launch_ls_shift(suli_ctx* c, double shift);
void launch_visco(suli_ctx* c);
void launch_convdiff(suli_ctx* c);
void launch_tempo(suli_ctx* c, int tt, int it);
void launch_contorno(suli_ctx* c, int nlock);
void launch_cg_setup(suli_ctx* c);
void launch_cg_iter(suli_ctx* c, const double* p_old, double* p_new);
void launch_cg_cond(suli_ctx* c, cudaGraphConditionalHandle h);
void launch_cg_divcheck(suli_ctx* c);
int cluster_ready(suli_ctx* c);
int stream_ready(suli_ctx* c);
int tail_ready(suli_ctx* c);
void launch_cg_final(suli_ctx* c, const double* e);
// ---- mixed-precision solve (k_mixed.cu) ----
void launch_mx_setup(suli_ctx* c);
void launch_mx_residual(suli_ctx* c, const double* e_in, double* e_out, bool apply);
void launch_pcg_init(suli_ctx* c, int maxit);
// the loop condition of the inner-solve graph: non-zero while the inner solve is not done
void launch_pcg_cond(suli_ctx* c, cudaGraphConditionalHandle h);
void launch_vcycle(suli_ctx* c, const float* f0, bool pre_done = false);
// ---- learned initial guess (k_learned.cu) ----
void launch_nn_features(suli_ctx* c, float* in3);
void launch_nn_features16(suli_ctx* c, void* in16);
void launch_nn_features16_at(suli_ctx* c, void* in16, const double* r, const double* e);
void launch_nn_step(suli_ctx* c, const float* out, double* e);
void launch_nn_target(suli_ctx* c, const double* e_star, float* target);
void launch_pcg_iter(suli_ctx* c, const float* p_old, float* p_new, const float* r_old, float* r_new,
                     bool x_zero = false);
int pcg_iter_kernels(const suli_ctx* c);
int vcycle_kernels(const suli_ctx* c);
void launch_posdin(suli_ctx* c);
void launch_est(suli_ctx* c);
void launch_fill(suli_ctx* c, double* a, double v);
}  // namespace suli
