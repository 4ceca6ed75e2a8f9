// suli_gpu.cu — host side of the C-ABI declared in include/suli_gpu.h.
//
// Owns the solver context (field arena in HBM, stream, reduction scratch) and sequences the
// kernels of k_fp64.cu in the order of the reference's subroutines.  Data-dependent control
// flow of the reference (the reinitialisation error loop, the volume-correction loop and the
// Poisson stopping test) is decided from device-resident scalars; the host reads them back
// only where the reference branches on them.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include "ctx.cuh"
#include "nn_api.cuh"

using namespace suli;

namespace {

int fail(suli_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

#define CUDA_TRY(c, expr)                                                                       \
    do {                                                                                        \
        cudaError_t e_ = (expr);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return fail((c), SULI_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define CHECK_LAUNCH(c)                                                                          \
    do {                                                                                         \
        cudaError_t e_ = cudaGetLastError();                                                     \
        if (e_ != cudaSuccess) return fail((c), SULI_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e_)); \
    } while (0)

bool is_plane(int f) { return f >= SULI_F_BXX0 && f < SULI_F_COUNT; }

// Fortran extents of each module array (0_modules.f90).
int extent(const suli_params* p, int f, int lo[3], int hi[3]) {
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    auto set = [&](int a, int b, int c, int d, int e, int g) {
        lo[0] = a; hi[0] = b; lo[1] = c; hi[1] = d; lo[2] = e; hi[2] = g;
        return 0;
    };
    switch (f) {
    case SULI_F_U: case SULI_F_UB: return set(0, nx + 2, 0, ny + 1, 0, nz + 1);
    case SULI_F_V: case SULI_F_VB: return set(0, nx + 1, 0, ny + 2, 0, nz + 1);
    case SULI_F_W: case SULI_F_WB: return set(0, nx + 1, 0, ny + 1, 0, nz + 2);
    case SULI_F_PRD1: case SULI_F_PRD0: case SULI_F_PRD: return set(0, nx + 1, 0, ny + 1, 0, nz + 1);
    case SULI_F_RHO: case SULI_F_LS_NU: case SULI_F_NUT: case SULI_F_LS: case SULI_F_MOD_LS: case SULI_F_KURV:
    case SULI_F_HS: case SULI_F_DDLSDX: case SULI_F_DDLSDY: case SULI_F_DDLSDZ: case SULI_F_HSX: case SULI_F_HSY:
    case SULI_F_HSZ:
        return set(1, nx, 1, ny, 1, nz);
    case SULI_F_FU: case SULI_F_U0: case SULI_F_FU0: case SULI_F_FU1: case SULI_F_XNUT: case SULI_F_TF_U:
        return set(1, nx + 1, 1, ny, 1, nz);
    case SULI_F_FV: case SULI_F_V0: case SULI_F_FV0: case SULI_F_FV1: case SULI_F_YNUT: case SULI_F_TF_V:
        return set(1, nx, 1, ny + 1, 1, nz);
    case SULI_F_FW: case SULI_F_W0: case SULI_F_FW0: case SULI_F_FW1: case SULI_F_ZNUT: case SULI_F_TF_W:
        return set(1, nx, 1, ny, 1, nz + 1);
    case SULI_F_BXX0: case SULI_F_BXX1: case SULI_F_BXXF: case SULI_F_BXXF1: return set(0, ny + 1, 0, nz + 1, 0, 0);
    case SULI_F_BXY0: case SULI_F_BXYF: return set(0, ny + 2, 0, nz + 1, 0, 0);
    case SULI_F_BXZ0: case SULI_F_BXZF: return set(0, ny + 1, 0, nz + 2, 0, 0);
    case SULI_F_BYX0: case SULI_F_BYXF: return set(0, nx + 2, 0, nz + 1, 0, 0);
    case SULI_F_BYY0: case SULI_F_BYY1: case SULI_F_BYYF: case SULI_F_BYYF1: return set(0, nx + 1, 0, nz + 1, 0, 0);
    case SULI_F_BYZ0: case SULI_F_BYZF: return set(0, nx + 1, 0, nz + 2, 0, 0);
    case SULI_F_BZX0: case SULI_F_BZXF: return set(0, nx + 2, 0, ny + 1, 0, 0);
    case SULI_F_BZY0: case SULI_F_BZYF: return set(0, nx + 1, 0, ny + 2, 0, 0);
    case SULI_F_BZZ0: case SULI_F_BZZ1: case SULI_F_BZZF: case SULI_F_BZZF1: return set(0, nx + 1, 0, ny + 1, 0, 0);
    default: return SULI_ERR_ARG;
    }
}

// Scatter a dense Fortran-layout block into the padded box and back.
__global__ void k_scatter(Geo G, const double* __restrict__ src, double* dst, int l0, int l1, int l2, int n0, int n1,
                          int n2) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long tot = (long long)n0 * n1 * n2;
    if (q >= tot) return;
    const int a = (int)(q % n0);
    const int b = (int)((q / n0) % n1);
    const int cc = (int)(q / ((long long)n0 * n1));
    dst[G.idx(l0 + a, l1 + b, l2 + cc)] = src[q];
}
__global__ void k_gather(Geo G, const double* __restrict__ src, double* dst, int l0, int l1, int l2, int n0, int n1,
                         int n2) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long tot = (long long)n0 * n1 * n2;
    if (q >= tot) return;
    const int a = (int)(q % n0);
    const int b = (int)((q / n0) % n1);
    const int cc = (int)(q / ((long long)n0 * n1));
    dst[q] = src[G.idx(l0 + a, l1 + b, l2 + cc)];
}

int sync_read(suli_ctx* c, const void* dev, void* host, size_t bytes) {
    CUDA_TRY(c, cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SULI_OK;
}

int validate(const suli_params* p, std::string& why) {
    if (p->nx < 4 || p->ny < 4 || p->nz < 4) { why = "nx, ny, nz must be >= 4 (WENO stencil)"; return SULI_ERR_ARG; }
    if (make_geo(p->nx, p->ny, p->nz).n >= (1LL << 31)) { why = "a field of this grid exceeds 2^31 elements"; return SULI_ERR_SIZE; }
    if (!(p->dx > 0 && p->dy > 0 && p->dz > 0)) { why = "dx, dy, dz must be positive"; return SULI_ERR_ARG; }
    if ((p->ccx0 == 0) != (p->ccxf == 0)) { why = "periodic x needs ccx0 = ccxf = 0 (0_modules.f90:56)"; return SULI_ERR_ARG; }
    if ((p->ccy0 == 0) != (p->ccyf == 0)) { why = "periodic y needs ccy0 = ccyf = 0"; return SULI_ERR_ARG; }
    if ((p->ccz0 == 0) != (p->cczf == 0)) { why = "periodic z needs ccz0 = cczf = 0"; return SULI_ERR_ARG; }
    if (p->ccx0 < 0 || p->ccx0 > 4 || p->ccxf < 0 || p->ccxf > 4) { why = "ccx0/ccxf out of range"; return SULI_ERR_ARG; }
    if (p->ccy0 < 0 || p->ccy0 > 3 || p->ccyf < 0 || p->ccyf > 3) { why = "ccy0/ccyf out of range"; return SULI_ERR_ARG; }
    if (p->ccz0 < 0 || p->ccz0 > 3 || p->cczf < 0 || p->cczf > 3) { why = "ccz0/cczf out of range"; return SULI_ERR_ARG; }
    if (p->obst_t < 0 || p->obst_t > 10) { why = "obst_t must be 0 (none) or an obstaculo preset 1..10"; return SULI_ERR_ARG; }
    if (p->wave_t != 0 && p->wave_t != 1 && p->wave_t != 2 && p->wave_t != 5) {
        why = "wave_t must be 0 (none), 1 (Stokes I), 2 (Stokes II) or 5 (Stokes V)"; return SULI_ERR_ARG;
    }
    if (p->periodic_faces != 0 && p->periodic_faces != 1) { why = "periodic_faces must be 0 or 1"; return SULI_ERR_ARG; }
    if (!(p->div_tol >= 0)) { why = "div_tol must be >= 0 (0: no divergence test)"; return SULI_ERR_ARG; }
    if (p->outflow_fix != 0 && p->outflow_fix != 1) { why = "outflow_fix must be 0 or 1"; return SULI_ERR_ARG; }
    if (p->outflow_fix == 1 && p->ccxf != 4) { why = "outflow_fix = 1 corrects the outflow plane: it needs ccxf = 4"; return SULI_ERR_ARG; }
    if (p->t_hs != 0 && p->t_hs != 1) { why = "t_hs must be 0 (linear) or 1 (geometric) (14_level_set.f90:696-703)"; return SULI_ERR_ARG; }
    if (p->adv_type < 1 || p->adv_type > 3) { why = "adv_type must be 1 (classico), 2 (rotacional) or 3 (antissim)"; return SULI_ERR_ARG; }
    if (p->der < 1 || p->der > 3) { why = "der must be 1 (upwind), 2 (centred) or 3 (2nd-order upwind)"; return SULI_ERR_ARG; }
    if (p->adv_type != 1 && p->der != 1) {   // the reference stops there (7_advectivo.f90:450-451, 646-647)
        why = "adv_type 2 and 3 exist only with der = 1"; return SULI_ERR_ARG;
    }
    if (p->m_turb < 0 || p->m_turb > 2) { why = "m_turb must be 0, 1 or 2"; return SULI_ERR_ARG; }
    if (p->t_tempo < 0 || p->t_tempo > 3) { why = "t_tempo out of range"; return SULI_ERR_ARG; }
    if (p->precision != 0 && p->precision != 1) { why = "precision must be 0 (FP64) or 1 (mixed)"; return SULI_ERR_ARG; }
    if (p->precision == 1) {
        if (p->cg_stop != 1) { why = "precision 1 stops on the relative FP64 residual (cg_stop = 1)"; return SULI_ERR_ARG; }
        if (p->refine_maxit < 1) { why = "refine_maxit must be >= 1"; return SULI_ERR_ARG; }
        if (!(p->inner_tol > 0 && p->inner_tol < 1)) { why = "inner_tol must lie in (0, 1)"; return SULI_ERR_ARG; }
        if (!(p->mg_omega >= 0 && p->mg_omega < 1)) { why = "mg_omega must lie in [0, 1)"; return SULI_ERR_ARG; }
        if (!(p->mg_alpha >= 0 && p->mg_alpha <= 2)) { why = "mg_alpha must lie in [0, 2]"; return SULI_ERR_ARG; }
        if (!(p->mg_omega2 >= 0 && p->mg_omega2 < 2)) { why = "mg_omega2 must lie in [0, 2)"; return SULI_ERR_ARG; }
        if (p->mg_kernels < 0 || p->mg_kernels > 2) { why = "mg_kernels must be 0, 1 or 2"; return SULI_ERR_ARG; }
        int nx = p->nx, ny = p->ny, nz = p->nz;
        while ((long long)nx * ny * nz > 1024 && nx % 2 == 0 && ny % 2 == 0 && nz % 2 == 0 && nx >= 4 && ny >= 4 && nz >= 4) {
            nx /= 2; ny /= 2; nz /= 2;
        }
        if ((long long)nx * ny * nz > 1024) {
            why = "precision 1: the grid must halve to <= 1024 cells for the multigrid coarsest level";
            return SULI_ERR_UNSUPPORTED;
        }
    }
    if (p->cg_stop != 0 && p->cg_stop != 1) { why = "cg_stop must be 0 or 1"; return SULI_ERR_ARG; }
    if (p->cg_maxit < 0) { why = "cg_maxit must be >= 0"; return SULI_ERR_ARG; }
    if (p->reinit_maxit < 1) { why = "reinit_maxit must be >= 1"; return SULI_ERR_ARG; }
    return SULI_OK;
}

}  // namespace


extern "C" {

int suli_field_extent(const suli_params* p, int field, int lo[3], int hi[3]) {
    if (!p || !lo || !hi) return SULI_ERR_ARG;
    return extent(p, field, lo, hi);
}

int suli_abi_sizes(int* params_bytes, int* stats_bytes) {
    if (params_bytes) *params_bytes = (int)sizeof(suli_params);
    if (stats_bytes) *stats_bytes = (int)sizeof(suli_step_stats);
    return SULI_OK;
}

int suli_params_default(suli_params* p) {
    if (!p) return SULI_ERR_ARG;
    std::memset(p, 0, sizeof(*p));
    p->dx = p->dy = p->dz = 0.02;
    p->nx = (int)(.5 / p->dx); p->ny = (int)(1. / p->dy); p->nz = (int)(0.9 / p->dz);
    p->dt = 0.001;
    p->ccx0 = p->ccxf = 0; p->ccy0 = p->ccyf = 2; p->ccz0 = 2; p->cczf = 1;
    p->t_tempo = 1; p->der = 1; p->adv_type = 1; p->m_turb = 0; p->obst_t = 0; p->t_hs = 0;
    p->csmag = 0.13;
    const double decliv = 0.0002;
    p->gx = 9.80665 * std::sin(std::atan(decliv));
    p->gz = 9.80665 * std::cos(std::atan(decliv));
    p->chezy = 44.5;
    p->rho_f1 = 1.204; p->mi_f1 = 0.000018253; p->rho_f2 = 998.0; p->mi_f2 = 0.00100798;
    p->sigma = 0.0728; p->alpha1 = 1.5;
    p->dt1 = 0.1 * std::fmax(p->dx, std::fmax(p->dy, p->dz));
    p->reinit_maxit = 3; p->vol_tol = 0.1;
    p->cg_stop = 0; p->cg_tol = 0.0001; p->cg_maxit = 10000;
    p->precision = 0; p->refine_maxit = 20; p->inner_tol = 1e-4;
    p->mg_omega = 0.9; p->mg_alpha = 1.8;
    return SULI_OK;
}

int suli_create(const suli_params* p, int device, suli_ctx** out) {
    if (!p || !out) return SULI_ERR_ARG;
    *out = nullptr;
    std::string why;
    const int v = validate(p, why);
    if (v != SULI_OK) { std::fprintf(stderr, "suli_create: %s\n", why.c_str()); return v; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0) {
        cudaGetLastError();
        std::fprintf(stderr, "suli_create: no CUDA device %d (there is no CPU fallback)\n", device);
        return SULI_ERR_NODEVICE;
    }
    suli_ctx* c = new suli_ctx();
    c->P = *p;
    if (c->P.mg_omega == 0.) c->P.mg_omega = 0.9;   // zero-initialised structs get the defaults
    if (c->P.mg_alpha == 0.) c->P.mg_alpha = 1.8;
    if (c->P.mg_omega2 == 0.) c->P.mg_omega2 = c->P.mg_omega;   // one weight for both sweeps
    c->device = device;
    c->g = make_geo(p->nx, p->ny, p->nz);
    c->bc.x0 = p->ccx0; c->bc.xf = p->ccxf; c->bc.y0 = p->ccy0; c->bc.yf = p->ccyf; c->bc.z0 = p->ccz0; c->bc.zf = p->cczf;
    c->bc.perx = (p->ccx0 == 0); c->bc.pery = (p->ccy0 == 0); c->bc.perz = (p->ccz0 == 0);
    c->bc.wrapf = p->periodic_faces;
    if (const char* ev = std::getenv("SULI_EAGER_LOOPS")) c->use_graphs = (std::strcmp(ev, "1") != 0);
    auto bail = [&](cudaError_t e, const char* what) {
        std::fprintf(stderr, "suli_create: %s: %s\n", what, cudaGetErrorString(e));
        suli_destroy(c);
        return (e == cudaErrorMemoryAllocation) ? SULI_ERR_NOMEM : SULI_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaSetDevice(device)) != cudaSuccess) return bail(e, "cudaSetDevice");
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "stream");
    // arena: 40 module fields + 18 work arrays, all in the shared padded box
    const int n3d = SULI_F_BXX0;
    const int nwork = 18;
    const size_t per = (size_t)c->g.n;
    c->arena_elems = per * (size_t)(n3d + nwork);
    if ((e = cudaMalloc(&c->arena, c->arena_elems * sizeof(double))) != cudaSuccess) return bail(e, "arena");
    if ((e = cudaMemsetAsync(c->arena, 0, c->arena_elems * sizeof(double), c->stream)) != cudaSuccess) return bail(e, "memset");
    for (int f = 0; f < n3d; ++f) c->f[f] = c->arena + per * f;
    double* wk = c->arena + per * n3d;
    double** work[18] = {&c->ls1, &c->ls2, &c->funcs, &c->nrmx, &c->nrmy, &c->nrmz, &c->cg_d, &c->cg_e,
                         &c->cg_r, &c->cg_b, &c->cg_pa, &c->cg_pb, &c->cg_q, &c->cg_ax, &c->cg_ay, &c->cg_az,
                         &c->cg_sd, &c->cg_isd};
    for (int q = 0; q < nwork; ++q) *work[q] = wk + per * q;
    for (int f = SULI_F_BXX0; f < SULI_F_COUNT; ++f) {
        int lo[3], hi[3];
        extent(p, f, lo, hi);
        const size_t n = (size_t)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1);
        c->plane_elems[f] = n;
        if ((e = cudaMalloc(&c->f[f], n * sizeof(double))) != cudaSuccess) return bail(e, "plane");
        if ((e = cudaMemsetAsync(c->f[f], 0, n * sizeof(double), c->stream)) != cudaSuccess) return bail(e, "memset");
    }
    const long long nb = (long long)((p->nx + 1 + 31) / 32) * ((p->ny + 1 + 7) / 8) * (p->nz + 1) + 64;
    if ((e = cudaMalloc(&c->red_partial, (size_t)nb * 3 * sizeof(double))) != cudaSuccess) return bail(e, "partial");
    if ((e = cudaMalloc(&c->red_counter, 64 * sizeof(unsigned int))) != cudaSuccess) return bail(e, "counter");
    if ((e = cudaMemsetAsync(c->red_counter, 0, 64 * sizeof(unsigned int), c->stream)) != cudaSuccess) return bail(e, "memset");
    if ((e = cudaMalloc(&c->red_out, 16 * sizeof(double))) != cudaSuccess) return bail(e, "red_out");
    if ((e = cudaMalloc(&c->cg, sizeof(CGState))) != cudaSuccess) return bail(e, "cg state");
    if ((e = cudaMemsetAsync(c->cg, 0, sizeof(CGState), c->stream)) != cudaSuccess) return bail(e, "memset");
    if ((e = cudaMallocHost(&c->cg_host, 2 * sizeof(CGState))) != cudaSuccess) return bail(e, "pinned");
    if ((e = cudaMallocHost(&c->host_scalars, 16 * sizeof(double))) != cudaSuccess) return bail(e, "pinned");
    if (p->precision == 1) {
        // FP32 multigrid hierarchy + inner PCG vectors, one float arena
        std::vector<Geo> gs;
        int nx = p->nx, ny = p->ny, nz = p->nz;
        gs.push_back(make_geo(nx, ny, nz));
        while ((long long)nx * ny * nz > 1024 && nx % 2 == 0 && ny % 2 == 0 && nz % 2 == 0 && nx >= 4 && ny >= 4 && nz >= 4) {
            nx /= 2; ny /= 2; nz /= 2;
            gs.push_back(make_geo(nx, ny, nz));
        }
        size_t tot = 7 * (size_t)gs[0].n + 64;
        for (auto& g : gs) tot += 7 * (size_t)g.n;
        if ((e = cudaMalloc(&c->f32_arena, tot * sizeof(float))) != cudaSuccess) return bail(e, "f32 arena");
        if ((e = cudaMemsetAsync(c->f32_arena, 0, tot * sizeof(float), c->stream)) != cudaSuccess) return bail(e, "memset");
        float* q = c->f32_arena;
        auto take = [&](size_t n) { float* r = q; q += n; return r; };
        c->pc_x = take(gs[0].n); c->pc_r = take(gs[0].n); c->pc_pa = take(gs[0].n); c->pc_pb = take(gs[0].n);
        c->pc_q = take(gs[0].n); c->pc_r2 = take(gs[0].n);
        for (auto& g : gs) {
            MGLevel L;
            L.g = g;
            L.sx = take(g.n); L.sy = take(g.n); L.sz = take(g.n); L.idg = take(g.n);
            L.f = take(g.n); L.x = take(g.n); L.y = take(g.n);
            if (c->mg.empty()) { L.rho = take(g.n); L.c2 = take(64); }
            c->mg.push_back(L);
        }
        if ((e = cudaMalloc(&c->cg_e2, per * sizeof(double))) != cudaSuccess) return bail(e, "e2");
        if ((e = cudaMemsetAsync(c->cg_e2, 0, per * sizeof(double), c->stream)) != cudaSuccess) return bail(e, "memset");
        if ((e = cudaMalloc(&c->pcg, sizeof(PCGState))) != cudaSuccess) return bail(e, "pcg state");
        if ((e = cudaMemsetAsync(c->pcg, 0, sizeof(PCGState), c->stream)) != cudaSuccess) return bail(e, "memset");
        if ((e = cudaMallocHost(&c->pcg_host, 2 * sizeof(PCGState))) != cudaSuccess) return bail(e, "pinned");
        cluster_ready(c);
        stream_ready(c);
        tail_ready(c);
    }
    if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) return bail(e, "sync");
    c->dt = p->dt;
    c->dt1 = p->dt1;
    c->ntt = 1;
    c->a_dt[0] = c->a_dt[1] = c->a_dt[2] = p->dt;
    *out = c;
    return SULI_OK;
}

int suli_destroy(suli_ctx* c) {
    if (!c) return SULI_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->pcg_loop) cudaGraphExecDestroy(c->pcg_loop);
    if (c->cg_loop) cudaGraphExecDestroy(c->cg_loop);
    for (auto& e : c->prof.ev) cudaEventDestroy(e);
    cudaFree(c->arena);
    cudaFree(c->obst_k);
    for (int f = SULI_F_BXX0; f < SULI_F_COUNT; ++f) cudaFree(c->f[f]);
    cudaFree(c->red_partial);
    cudaFree(c->red_counter);
    cudaFree(c->red_out);
    cudaFree(c->cg);
    cudaFree(c->f32_arena);
    cudaFree(c->cg_e2);
    cudaFree(c->pcg);
    cudaFree(c->nn_out);
    cudaFree(c->nn_e0);
    cudaFree(c->nn_scale);
    for (int q = 0; q < 2 * SULI_STEP_HOST_MAX_FIELDS; ++q) {
        cudaFree(c->io_stage[q]);
        if (c->io_ev[q]) cudaEventDestroy(c->io_ev[q]);
    }
    if (c->io_in) cudaStreamDestroy(c->io_in);
    if (c->io_out) cudaStreamDestroy(c->io_out);
    if (c->pcg_host) cudaFreeHost(c->pcg_host);
    if (c->cg_host) cudaFreeHost(c->cg_host);
    if (c->host_scalars) cudaFreeHost(c->host_scalars);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return SULI_OK;
}

const char* suli_last_error(const suli_ctx* c) { return c ? c->err.c_str() : "null context"; }

int suli_synchronize(suli_ctx* c) {
    if (!c) return SULI_ERR_ARG;
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SULI_OK;
}

// true for pageable or pinned host memory, false for device or managed memory
static bool host_memory(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered || a.type == cudaMemoryTypeHost;
}

int suli_upload(suli_ctx* c, int field, const double* host) {
    if (!c || !host || field < 0 || field >= SULI_F_COUNT) return fail(c, SULI_ERR_ARG, "upload: bad field");
    cudaSetDevice(c->device);
    int lo[3], hi[3];
    extent(&c->P, field, lo, hi);
    const int n0 = hi[0] - lo[0] + 1, n1 = hi[1] - lo[1] + 1, n2 = hi[2] - lo[2] + 1;
    const size_t n = (size_t)n0 * n1 * n2;
    if (is_plane(field)) {
        CUDA_TRY(c, cudaMemcpyAsync(c->f[field], host, n * sizeof(double), cudaMemcpyDefault, c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        return SULI_OK;
    }
    if (field == SULI_F_TF_U || field == SULI_F_TF_V || field == SULI_F_TF_W) {
        if (!host_memory(host)) {
            c->tf_active = true;   // device data is not scanned: adding zeros changes nothing
        } else {
            for (size_t q = 0; q < n; ++q)
                if (host[q] != 0.0) { c->tf_active = true; break; }
        }
    }
    // stage through the CG q buffer (same size class as any field, free between calls)
    double* stage = c->cg_q;
    CUDA_TRY(c, cudaMemcpyAsync(stage, host, n * sizeof(double), cudaMemcpyDefault, c->stream));
    k_scatter<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->g, stage, c->f[field], lo[0], lo[1], lo[2], n0, n1, n2);
    CHECK_LAUNCH(c);
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SULI_OK;
}

int suli_download(suli_ctx* c, int field, double* host) {
    if (!c || !host || field < 0 || field >= SULI_F_COUNT) return fail(c, SULI_ERR_ARG, "download: bad field");
    cudaSetDevice(c->device);
    int lo[3], hi[3];
    extent(&c->P, field, lo, hi);
    const int n0 = hi[0] - lo[0] + 1, n1 = hi[1] - lo[1] + 1, n2 = hi[2] - lo[2] + 1;
    const size_t n = (size_t)n0 * n1 * n2;
    if (is_plane(field)) {
        CUDA_TRY(c, cudaMemcpyAsync(host, c->f[field], n * sizeof(double), cudaMemcpyDefault, c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        return SULI_OK;
    }
    double* stage = c->cg_q;
    k_gather<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->g, c->f[field], stage, lo[0], lo[1], lo[2], n0, n1, n2);
    CHECK_LAUNCH(c);
    CUDA_TRY(c, cudaMemcpyAsync(host, stage, n * sizeof(double), cudaMemcpyDefault, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SULI_OK;
}

int suli_set_scalar(suli_ctx* c, int id, double v) {
    if (!c) return SULI_ERR_ARG;
    switch (id) {
    case SULI_S_DT: c->dt = v; return SULI_OK;
    case SULI_S_VOL_INI: c->vol_ini = v; return SULI_OK;
    case SULI_S_VOL_INS: c->vol_ins = v; return SULI_OK;
    case SULI_S_DT1: c->dt1 = v; return SULI_OK;
    case SULI_S_T: c->t = v; return SULI_OK;
    case SULI_S_NTT: if (v < 1 || v > 3) return fail(c, SULI_ERR_ARG, "ntt must be 1..3"); c->ntt = (int)v; return SULI_OK;
    case SULI_S_A_DT1: c->a_dt[0] = v; return SULI_OK;
    case SULI_S_A_DT2: c->a_dt[1] = v; return SULI_OK;
    case SULI_S_A_DT3: c->a_dt[2] = v; return SULI_OK;
    case SULI_S_FALLBACKS: return fail(c, SULI_ERR_ARG, "fallbacks is read only");
    default: return fail(c, SULI_ERR_ARG, "set_scalar: bad id");
    }
}

int suli_get_scalar(suli_ctx* c, int id, double* v) {
    if (!c || !v) return SULI_ERR_ARG;
    switch (id) {
    case SULI_S_DT: *v = c->dt; return SULI_OK;
    case SULI_S_VOL_INI: *v = c->vol_ini; return SULI_OK;
    case SULI_S_VOL_INS: *v = c->vol_ins; return SULI_OK;
    case SULI_S_DT1: *v = c->dt1; return SULI_OK;
    case SULI_S_T: *v = c->t; return SULI_OK;
    case SULI_S_NTT: *v = c->ntt; return SULI_OK;
    case SULI_S_A_DT1: *v = c->a_dt[0]; return SULI_OK;
    case SULI_S_A_DT2: *v = c->a_dt[1]; return SULI_OK;
    case SULI_S_A_DT3: *v = c->a_dt[2]; return SULI_OK;
    case SULI_S_FALLBACKS: *v = (double)c->fallbacks; return SULI_OK;
    default: return fail(c, SULI_ERR_ARG, "get_scalar: bad id");
    }
}

int suli_set_dt(suli_ctx* c, double dt) {
    if (!c) return SULI_ERR_ARG;
    c->dt = dt;
    return SULI_OK;
}

// iniciais (2_iniciais.f90:36-46 and 85-104), without obstacle/wave/level-set presets
int suli_set_obstacle(suli_ctx* c, const int* ku, const int* kv, const int* kw) {
    if (!c || !ku || !kv || !kw) return SULI_ERR_ARG;
    if (c->P.obst_t == 0) return fail(c, SULI_ERR_ARG, "set_obstacle: obst_t is 0");
    const int nx = c->P.nx, ny = c->P.ny, nz = c->P.nz;
    const size_t nu = (size_t)(nx + 3) * (ny + 2), nv = (size_t)(nx + 2) * (ny + 3), nw = (size_t)(nx + 2) * (ny + 2);
    // the column kernels index k from -1 + 1 = 0 up to mask + 1: keep it inside the halo
    for (size_t q = 0; q < nu; ++q) if (ku[q] < -1 || ku[q] > nz) return fail(c, SULI_ERR_ARG, "set_obstacle: ku outside [-1, nz]");
    for (size_t q = 0; q < nv; ++q) if (kv[q] < -1 || kv[q] > nz) return fail(c, SULI_ERR_ARG, "set_obstacle: kv outside [-1, nz]");
    for (size_t q = 0; q < nw; ++q) if (kw[q] < -1 || kw[q] > nz + 1) return fail(c, SULI_ERR_ARG, "set_obstacle: kw outside [-1, nz+1]");
    cudaSetDevice(c->device);
    if (!c->obst_k) {
        CUDA_TRY(c, cudaMalloc(&c->obst_k, (nu + nv + nw) * sizeof(int)));
        c->obst_ku = c->obst_k;
        c->obst_kv = c->obst_k + nu;
        c->obst_kw = c->obst_k + nu + nv;
    }
    CUDA_TRY(c, cudaMemcpyAsync(c->obst_k, ku, nu * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(c->obst_k + nu, kv, nv * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(c->obst_k + nu + nv, kw, nw * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->obst_ku_host.assign(ku, ku + nu);
    return SULI_OK;
}

int suli_boundary_waves(suli_ctx* c) {
    if (!c) return SULI_ERR_ARG;
    if (c->P.wave_t == 0) return fail(c, SULI_ERR_ARG, "boundary_waves: wave_t is 0");
    cudaSetDevice(c->device);
    if (c->wave.type != c->P.wave_t) c->wave = wave_coefficients(c->P.wave_t, c->P.gz);
    launch_boundary_waves(c);
    CHECK_LAUNCH(c);
    return SULI_OK;
}

int suli_iniciais(suli_ctx* c, double u_init) {
    if (!c) return SULI_ERR_ARG;
    cudaSetDevice(c->device);
    c->t = 0.;
    launch_fill(c, c->f[SULI_F_U], u_init);
    launch_fill(c, c->f[SULI_F_V], 0.);
    launch_fill(c, c->f[SULI_F_W], 0.);
    launch_fill(c, c->f[SULI_F_PRD0], 0.);
    launch_fill(c, c->f[SULI_F_PRD1], 0.);
    launch_fill(c, c->f[SULI_F_UB], 0.);
    launch_fill(c, c->f[SULI_F_VB], 0.);
    launch_fill(c, c->f[SULI_F_WB], 0.);
    CHECK_LAUNCH(c);
    std::vector<double> bx0(c->plane_elems[SULI_F_BXX0], u_init), bx1(bx0);
    if (c->P.wave_t > 0) {
        // 2_iniciais.f90:52-54: waves_coef instead of the uniform inflow; boundary_waves writes
        // the inflow planes at every stage
        c->wave = wave_coefficients(c->P.wave_t, c->P.gz);
    } else if (c->P.obst_t != 0) {
        // 2_iniciais.f90:60-65: bxx1(:,0:ku(1,j)) = 0 for every j zeroes whole rows of the
        // (0:ny+1, 0:nz+1) plane up to the highest ku(1,j) (likewise bxx0 with ku(0,j))
        if (c->obst_ku_host.empty()) return fail(c, SULI_ERR_ARG, "iniciais: obst_t != 0 needs suli_set_obstacle first");
        const int nx = c->P.nx, ny = c->P.ny, rows = ny + 2;
        for (int j = 0; j <= ny + 1; ++j) {
            const int k1 = c->obst_ku_host[1 + (size_t)(nx + 3) * j], k0 = c->obst_ku_host[0 + (size_t)(nx + 3) * j];
            for (int k = 0; k <= k1; ++k) std::fill_n(bx1.begin() + (size_t)rows * k, rows, 0.);
            for (int k = 0; k <= k0; ++k) std::fill_n(bx0.begin() + (size_t)rows * k, rows, 0.);
        }
    }
    if (c->P.wave_t == 0) {
        CUDA_TRY(c, cudaMemcpyAsync(c->f[SULI_F_BXX0], bx0.data(), bx0.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        CUDA_TRY(c, cudaMemcpyAsync(c->f[SULI_F_BXX1], bx1.data(), bx1.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    }
    const int tm = c->P.t_tempo;
    const double dt = c->P.dt;
    c->dt = dt;
    if (tm == 0 || tm == 3) { c->ntt = 1; c->a_dt[0] = c->a_dt[1] = c->a_dt[2] = 1.0 * dt; }
    else if (tm == 1) { c->ntt = 2; c->a_dt[0] = 0.5 * dt; c->a_dt[1] = 1.0 * dt; c->a_dt[2] = 1.0 * dt; }
    else { c->ntt = 3; c->a_dt[0] = 0.5 * dt; c->a_dt[1] = 1.0 * dt; c->a_dt[2] = 1.0 * dt; }
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return SULI_OK;
}

int suli_heaviside(suli_ctx* c) {
    if (!c) return SULI_ERR_ARG;
    cudaSetDevice(c->device);
    launch_lsprops(c, c->f[SULI_F_LS], false, true, false);
    CHECK_LAUNCH(c);
    return SULI_OK;
}

int suli_mod_ls1(suli_ctx* c) {
    if (!c) return SULI_ERR_ARG;
    cudaSetDevice(c->device);
    launch_lsprops(c, c->f[SULI_F_LS], true, false, false);
    launch_curv(c);
    CHECK_LAUNCH(c);
    return SULI_OK;
}

int suli_level_set_ini(suli_ctx* c) {
    if (!c) return SULI_ERR_ARG;
    cudaSetDevice(c->device);
    if (c->P.t_hs != 0) {   // the preset shifted by ls_m for the geometric mix (14_level_set.f90:47-51, 196-202)
        const double dx1 = fmax(c->P.dx, fmax(c->P.dy, c->P.dz));
        launch_ls_shift(c, 0.481803535 * dx1 * c->P.alpha1);
    }
    launch_lsprops(c, c->f[SULI_F_LS], true, true, true);
    launch_curv(c);
    CHECK_LAUNCH(c);
    int r = sync_read(c, c->red_out, c->host_scalars, sizeof(double));
    if (r != SULI_OK) return r;
    c->vol_ini = c->host_scalars[0];
    return SULI_OK;
}

// level_set (14_level_set.f90:221-285)
int suli_level_set(suli_ctx* c, double* vol_ins) {
    if (!c) return SULI_ERR_ARG;
    cudaSetDevice(c->device);
    const double adtl[3] = {1., 3. / 4., 1. / 3.}, bdtl[3] = {0., 1. / 4., 2. / 3.}, gdtl[3] = {1., 1. / 4., 2. / 3.};
    double* L0 = c->f[SULI_F_LS];
    double* L1 = c->ls1;
    double* L2 = c->ls2;
    // transport: three TVD-RK3 stages with dt1 := dt (:231-239)
    const double dta = c->dt;
    launch_ls_advect(c, L0, L0, L1, adtl[0], bdtl[0], gdtl[0] * dta);
    launch_ls_advect(c, L1, L0, L2, adtl[1], bdtl[1], gdtl[1] * dta);
    launch_ls_advect(c, L2, L0, L0, adtl[2], bdtl[2], gdtl[2] * dta);
    CHECK_LAUNCH(c);
    // reinitialisation (reinic_weno, :386-509)
    const double dt1 = c->dt1;
    const double dx1 = std::fmax(c->P.dx, std::fmax(c->P.dy, c->P.dz));
    launch_reinit_funcs(c);
    int il = 0;
    double error = 999.;
    while (error > dt1 * dx1 * dx1) {
        il = il + 1;
        launch_reinit_stage(c, L0, L0, L1, adtl[0], bdtl[0], gdtl[0] * dt1);
        launch_reinit_stage(c, L1, L0, L2, adtl[1], bdtl[1], gdtl[1] * dt1);
        launch_reinit_stage(c, L2, L0, L0, adtl[2], bdtl[2], gdtl[2] * dt1);
        CHECK_LAUNCH(c);
        if (il == c->P.reinit_maxit) {
            error = 0.;
        } else {
            launch_reinit_err(c, L0, L2, 2. * c->P.alpha1 * dx1);
            CHECK_LAUNCH(c);
            int r = sync_read(c, c->red_out, c->host_scalars, 2 * sizeof(double));
            if (r != SULI_OK) return r;
            error = c->host_scalars[0] / c->host_scalars[1];   // nr = 0 gives NaN and ends the loop
        }
    }
    c->last_reinit_iters = il;
    // mod_ls1 + heaviside + volume (:243-253)
    launch_lsprops(c, L0, true, true, true);
    launch_curv(c);
    CHECK_LAUNCH(c);
    int r = sync_read(c, c->red_out, c->host_scalars, sizeof(double));
    if (r != SULI_OK) return r;
    c->vol_ins = c->host_scalars[0];
    // volume correction (:257-278); the trailing mod_ls1/heaviside pair (:280-282) recomputes
    // identical values from an unchanged ls and is skipped.
    int passes = 0;
    while (std::fabs(c->vol_ins - c->vol_ini) / c->vol_ins > c->P.vol_tol && passes < 1000) {
        launch_volfix(c, dt1 * (c->vol_ins - c->vol_ini));
        launch_lsprops(c, L0, true, true, true);
        launch_curv(c);
        CHECK_LAUNCH(c);
        r = sync_read(c, c->red_out, c->host_scalars, sizeof(double));
        if (r != SULI_OK) return r;
        c->vol_ins = c->host_scalars[0];
        ++passes;
    }
    c->last_volfix_iters = passes;
    if (vol_ins) *vol_ins = c->vol_ins;
    return SULI_OK;
}

int suli_visco(suli_ctx* c) {
    if (!c) return SULI_ERR_ARG;
    cudaSetDevice(c->device);
    launch_visco(c);
    CHECK_LAUNCH(c);
    return SULI_OK;
}

int suli_convdiff(suli_ctx* c) {
    if (!c) return SULI_ERR_ARG;
    cudaSetDevice(c->device);
    launch_convdiff(c);
    CHECK_LAUNCH(c);
    return SULI_OK;
}

int suli_tempo(suli_ctx* c, int tt, int it) {
    if (!c) return SULI_ERR_ARG;
    if (tt < 1 || tt > 3) return fail(c, SULI_ERR_ARG, "tempo: tt must be 1..3");
    cudaSetDevice(c->device);
    launch_tempo(c, tt, it);
    CHECK_LAUNCH(c);
    return SULI_OK;
}

int suli_contorno(suli_ctx* c, int nlock) {
    if (!c) return SULI_ERR_ARG;
    if (nlock < 1 || nlock > 3) return fail(c, SULI_ERR_ARG, "contorno: nlock must be 1..3");
    if (c->P.obst_t != 0 && !c->obst_k) return fail(c, SULI_ERR_ARG, "contorno: obst_t != 0 needs suli_set_obstacle first");
    cudaSetDevice(c->device);
    launch_contorno(c, nlock);
    CHECK_LAUNCH(c);
    return SULI_OK;
}

// graddin (9_grad.f90:10-278)
}  // extern "C"

namespace {
// A solver's iterations as one graph launch: a WHILE conditional node whose body is two
// iterations (the direction vector ping-pongs between two buffers; every kernel reads its
// scalars from device memory, so the captured parameters never change) and a kernel that clears
// the condition once the solve has converged or hit its cap.  The GPU iterates without host
// round trips, and no iteration is launched after convergence except the rest of the last body
// (kernels that return at once).
template <class Body, class Cond>
int make_loop_graph(suli_ctx* c, cudaGraphExec_t* out, Body body, Cond cond, const char* what) {
    cudaGraph_t g = nullptr;
    CUDA_TRY(c, cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, nullptr, 0, &np);
    if (e == cudaSuccess)
        e = cudaStreamBeginCaptureToGraph(c->stream, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        body();
        cond(h);
        cudaGraph_t captured = nullptr;
        e = cudaStreamEndCapture(c->stream, &captured);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(c, SULI_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    }
    return SULI_OK;
}

// the inner FP32 PCG of the mixed path
int ensure_pcg_loop(suli_ctx* c) {
    if (c->pcg_loop) return SULI_OK;
    if (int r = make_loop_graph(
            c, &c->pcg_loop,
            [&] {
                launch_pcg_iter(c, c->pc_pa, c->pc_pb, c->pc_r2, c->pc_r);
                launch_pcg_iter(c, c->pc_pb, c->pc_pa, c->pc_r, c->pc_r2);
            },
            [&](cudaGraphConditionalHandle h) { launch_pcg_cond(c, h); }, "inner-solve graph"))
        return r;
    c->pcg_graph_kernels = pcg_iter_kernels(c);
    return SULI_OK;
}

// the plain FP64 CG
int ensure_cg_loop(suli_ctx* c) {
    if (c->cg_loop) return SULI_OK;
    return make_loop_graph(
        c, &c->cg_loop,
        [&] {
            launch_cg_iter(c, c->cg_pa, c->cg_pb);
            launch_cg_iter(c, c->cg_pb, c->cg_pa);
        },
        [&](cudaGraphConditionalHandle h) { launch_cg_cond(c, h); }, "CG graph");
}

// Mixed-precision solve: FP64 refinement around an FP32 multigrid-preconditioned CG.
// Buffers of the learned guess and of recorded solves (allocated on first use).
int ensure_nn_buffers(suli_ctx* c, bool net) {
    const long long V = (long long)c->P.nx * c->P.ny * c->P.nz;
    if (!c->nn_scale) CUDA_TRY(c, cudaMalloc(&c->nn_scale, sizeof(NNScale)));
    if (!c->nn_e0) CUDA_TRY(c, cudaMalloc(&c->nn_e0, c->g.n * sizeof(double)));
    if (net && !c->nn_out) CUDA_TRY(c, cudaMalloc(&c->nn_out, V * sizeof(float)));
    return SULI_OK;
}

// After graddin's set-up: record the features and e0, or apply the learned initial guess.
void nn_begin(suli_ctx* c) {
    const bool rec = c->rec_in != nullptr;
    const bool learn = !rec && c->nn && c->nn_mode >= 1;
    if (!rec && !learn) return;
    if (rec) {
        {
            ProfScope ps(c, SULI_K_CG_SETUP, 2);
            launch_nn_features(c, c->rec_in);
        }
        cudaMemcpyAsync(c->nn_e0, c->cg_e, c->g.n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
        return;
    }
    {   // the features go straight into the network's BF16 input
        ProfScope ps(c, SULI_K_CG_SETUP, 2);
        launch_nn_features16(c, suli::nn::input16(c->nn));
    }
    {
        ProfScope ps(c, SULI_K_NN, 0);
        c->prof.launches[SULI_K_NN] += suli::nn::forward_packed_on(c->nn, c->stream, c->nn_out);
    }
    ProfScope ps(c, SULI_K_CG_SETUP, 2);
    launch_nn_step(c, c->nn_out, c->cg_e);
}

// The plain FP64 Jacobi-scaled CG (9_grad.f90:118-264) from prd1: set-up, the device-side loop,
// the divergence test's resumptions, de-normalisation.  `record` takes a training pair
// (suli_graddin_record).
int graddin_fp64(suli_ctx* c, int* iters, double* resid, bool record) {
    if (int rg = ensure_cg_loop(c)) return rg;
    launch_cg_setup(c);
    if (record) nn_begin(c);   // recording only: the learned guess needs the refinement loop
    CHECK_LAUNCH(c);
    // iteration 1 uses p_old = r with beta = 0 (erroppr = erropr, :172); then the device loop
    launch_cg_iter(c, c->cg_r, c->cg_pa);
    auto run_loop = [&]() -> int {
        if (c->use_graphs) {
            ProfScope ps(c, SULI_K_CG_SPMV, 0);   // kernel launches are counted below, once known
            CUDA_TRY(c, cudaGraphLaunch(c->cg_loop, c->stream));
            return SULI_OK;
        }
        for (;;) {
            launch_cg_iter(c, c->cg_pa, c->cg_pb);
            launch_cg_iter(c, c->cg_pb, c->cg_pa);
            CHECK_LAUNCH(c);
            if (int rr = sync_read(c, c->cg, c->cg_host, sizeof(CGState))) return rr;
            if (c->cg_host[0].done) return SULI_OK;
        }
    };
    if (int rl = run_loop()) return rl;
    CHECK_LAUNCH(c);
    // div_tol > 0: resume the solve while the divergence the projection would leave is too large
    for (int pass = 0; c->P.div_tol > 0. && pass < 64; ++pass) {
        launch_cg_divcheck(c);
        CHECK_LAUNCH(c);
        int rr = sync_read(c, c->cg, c->cg_host, sizeof(CGState));
        if (rr != SULI_OK) return rr;
        const CGState& s = c->cg_host[0];
        if (s.done) break;
        // after n iterations the last direction is in cg_pa for odd n, cg_pb for even n; the loop
        // body starts from cg_pa
        if (s.iters == 0) {
            launch_cg_iter(c, c->cg_r, c->cg_pa);
        } else if (s.iters % 2 == 0) {
            CUDA_TRY(c, cudaMemcpyAsync(c->cg_pa, c->cg_pb, c->g.n * sizeof(double), cudaMemcpyDeviceToDevice,
                                        c->stream));
        }
        if (int rl = run_loop()) return rl;
        CHECK_LAUNCH(c);
    }
    launch_cg_final(c, c->cg_e);
    if (record && c->rec_in) launch_nn_target(c, c->cg_e, c->rec_target);
    CHECK_LAUNCH(c);
    int r = sync_read(c, c->cg, c->cg_host, sizeof(CGState));
    if (r != SULI_OK) return r;
    const CGState& s = c->cg_host[0];
    c->prof.cg_iters += s.iters;
    if (c->use_graphs) {   // the loop ran ceil((iters - 1) / 2) two-iteration bodies (at least one)
        const long long bodies = std::max(1, s.iters / 2);
        c->prof.launches[SULI_K_CG_SPMV] += 2 * bodies;
        c->prof.launches[SULI_K_CG_UPDATE] += 2 * bodies;
    }
    if (iters) *iters = s.iters;
    if (resid) *resid = (s.bb > 0.) ? std::sqrt(s.rr / s.bb) : 0.;
    if (s.status == SULI_ERR_NAN) return fail(c, SULI_ERR_NAN, "graddin: NaN/Inf in the Poisson solve");
    return s.status;
}

int graddin_mixed(suli_ctx* c, int* iters, double* resid) {
    if (int rg = ensure_pcg_loop(c)) return rg;
    launch_cg_setup(c);   // FP64 diagonal, coefficients, b~, first residual and threshold
    launch_mx_setup(c);   // FP32 faces of every multigrid level
    nn_begin(c);
    double* ecur = c->cg_e;
    double* enext = c->cg_e2;
    launch_mx_residual(c, ecur, enext, false);
    std::swap(ecur, enext);
    CHECK_LAUNCH(c);
    long long inner_total = 0;
    int outer = 0, status = SULI_OK;
    bool fallback = false;
    double rr_prev = -1.;
    bool inner_capped = false;
    // The inner solve's state is copied to the host right after its loop and read at the next
    // synchronisation, so the refinement residual is launched without waiting for the host.
    bool pcg_pending = false;
    auto take_inner = [&]() -> int {
        pcg_pending = false;
        if (c->pcg_host[0].status == SULI_ERR_NAN) return fail(c, SULI_ERR_NAN, "graddin: NaN/Inf in the inner solve");
        if (c->pcg_host[0].status == SULI_ERR_CUDA)
            return fail(c, SULI_ERR_CUDA, "graddin: a streaming multigrid kernel's wait for its loads ran out");
        inner_total += c->pcg_host[0].iters;
        inner_capped = (c->pcg_host[0].iters >= c->inner_maxit);
        if (c->use_graphs) {   // eager launches were counted as they went
            const long long bodies = std::max(1, (c->pcg_host[0].iters - 1 + 1) / 2);
            c->prof.launches[SULI_K_MG] += bodies * (2LL * c->pcg_graph_kernels + 1);
        }
        return SULI_OK;
    };
    while (true) {
        int r = sync_read(c, c->cg, c->cg_host, sizeof(CGState));
        if (r != SULI_OK) return r;
        if (pcg_pending)
            if (int ri = take_inner()) return ri;
        if (c->cg_host[0].status == SULI_ERR_NAN) return fail(c, SULI_ERR_NAN, "graddin: NaN/Inf in the Poisson solve");
        if (c->cg_host[0].done) break;
        // a pass that did not halve the FP64 residual, or an inner solve that hit its cap: the
        // FP32 inner solve no longer helps; the plain FP64 CG finishes from the better iterate
        const double rr_now = c->cg_host[0].rr;
        if (rr_prev >= 0. && (rr_now > 0.5 * rr_prev || inner_capped)) {
            if (rr_now > rr_prev) std::swap(ecur, enext);   // the pass made it worse: keep the one before
            fallback = true;
            break;
        }
        rr_prev = rr_now;
        if (outer >= c->P.refine_maxit) { status = SULI_WARN_CG_MAXIT; break; }
        launch_pcg_init(c, c->inner_maxit);
        {
            ProfScope ps(c, SULI_K_MG, vcycle_kernels(c));
            launch_vcycle(c, c->pc_r);
        }
        launch_pcg_iter(c, c->mg[0].y, c->pc_pa, c->pc_r, c->pc_r2, true);   // p_old = z with beta = 0, x = 0
        if (c->use_graphs) {
            ProfScope ps(c, SULI_K_MG, 0);   // kernel launches are counted below, once known
            CUDA_TRY(c, cudaGraphLaunch(c->pcg_loop, c->stream));
        } else {
            for (int pair = 0; pair < c->inner_maxit; ++pair) {
                launch_pcg_iter(c, c->pc_pa, c->pc_pb, c->pc_r2, c->pc_r);
                launch_pcg_iter(c, c->pc_pb, c->pc_pa, c->pc_r, c->pc_r2);
                CHECK_LAUNCH(c);
                if (int rr = sync_read(c, c->pcg, c->pcg_host, sizeof(PCGState))) return rr;
                if (c->pcg_host[0].done) break;
            }
        }
        CUDA_TRY(c, cudaMemcpyAsync(c->pcg_host, c->pcg, sizeof(PCGState), cudaMemcpyDeviceToHost, c->stream));
        pcg_pending = true;
        launch_mx_residual(c, ecur, enext, true);
        std::swap(ecur, enext);
        CHECK_LAUNCH(c);
        ++outer;
        if (c->nn && c->nn_mode == 2 && !c->rec_in) {
            // the network as the outer iteration's preconditioner: its correction of the current
            // residual, with the energy-optimal FP64 step, before the next pass (or the test)
            r = sync_read(c, c->cg, c->cg_host, sizeof(CGState));
            if (r != SULI_OK) return r;
            if (pcg_pending)
                if (int ri = take_inner()) return ri;
            if (!c->cg_host[0].done) {
                {
                    ProfScope ps(c, SULI_K_CG_SETUP, 2);
                    launch_nn_features16_at(c, suli::nn::input16(c->nn), c->cg_r, ecur);
                }
                {
                    ProfScope ps(c, SULI_K_NN, 0);
                    c->prof.launches[SULI_K_NN] += suli::nn::forward_packed_on(c->nn, c->stream, c->nn_out);
                }
                {
                    ProfScope ps(c, SULI_K_CG_SETUP, 2);
                    launch_nn_step(c, c->nn_out, ecur);
                }
                launch_mx_residual(c, ecur, enext, false);
                std::swap(ecur, enext);
                CHECK_LAUNCH(c);
            }
        }
    }
    c->last_outer_iters = outer;
    if (c->nn && c->nn_mode >= 1 && !c->rec_in && suli::nn::take_error(c->nn))
        return fail(c, SULI_ERR_CUDA, "graddin: the network's tensor-core convolution timed out");
    if (fallback) {   // prd1 from the iterate, then the FP64 CG to the same stopping tests
        launch_cg_final(c, ecur);
        int n64 = 0;
        double res64 = 0.;
        const int rf = graddin_fp64(c, &n64, &res64, false);
        ++c->fallbacks;
        if (rf < 0) return rf;
        if (c->rec_in) launch_nn_target(c, c->cg_e, c->rec_target);
        CHECK_LAUNCH(c);
        c->prof.cg_iters += inner_total;
        if (iters) *iters = (int)(inner_total + n64);
        if (resid) *resid = res64;
        return rf;
    }
    launch_cg_final(c, ecur);
    if (c->rec_in) launch_nn_target(c, ecur, c->rec_target);
    CHECK_LAUNCH(c);
    int r = sync_read(c, c->cg, c->cg_host, sizeof(CGState));
    if (r != SULI_OK) return r;
    const CGState& s = c->cg_host[0];
    c->prof.cg_iters += inner_total;
    if (iters) *iters = (int)inner_total;
    if (resid) *resid = (s.bb > 0.) ? std::sqrt(s.rr / s.bb) : 0.;
    return status;
}
}  // namespace

extern "C" {

int suli_graddin(suli_ctx* c, int* iters, double* resid) {
    if (!c) return SULI_ERR_ARG;
    cudaSetDevice(c->device);
    if (c->P.precision == 1) return graddin_mixed(c, iters, resid);
    return graddin_fp64(c, iters, resid, true);
}

int suli_attach_nn(suli_ctx* c, suli_nn* net, int mode) {
    if (!c) return SULI_ERR_ARG;
    cudaSetDevice(c->device);
    if (mode == 0) {
        c->nn = nullptr;
        c->nn_mode = 0;
        return SULI_OK;
    }
    if ((mode != 1 && mode != 2) || !net) return fail(c, SULI_ERR_ARG, "attach_nn: mode must be 0, 1 or 2 with a network");
    if (c->P.precision != 1) return fail(c, SULI_ERR_UNSUPPORTED, "attach_nn: the learned guess needs precision 1");
    int nx, ny, nz, dev;
    suli::nn::dims(net, &nx, &ny, &nz, &dev);
    if (nx != c->P.nx || ny != c->P.ny || nz != c->P.nz || dev != c->device)
        return fail(c, SULI_ERR_ARG, "attach_nn: network grid or device differs from the context's");
    if (int r = ensure_nn_buffers(c, true)) return r;
    c->nn = net;
    c->nn_mode = mode;
    return SULI_OK;
}

int suli_graddin_record(suli_ctx* c, float* d_in3, float* d_target, int* iters, double* resid) {
    if (!c || !d_in3 || !d_target) return SULI_ERR_ARG;
    cudaSetDevice(c->device);
    if (int r = ensure_nn_buffers(c, false)) return r;
    c->rec_in = d_in3;
    c->rec_target = d_target;
    const int r = suli_graddin(c, iters, resid);
    c->rec_in = nullptr;
    c->rec_target = nullptr;
    return r;
}

int suli_posdin(suli_ctx* c) {
    if (!c) return SULI_ERR_ARG;
    cudaSetDevice(c->device);
    launch_posdin(c);
    CHECK_LAUNCH(c);
    return SULI_OK;
}

int suli_est(suli_ctx* c, double* max_div) {
    if (!c) return SULI_ERR_ARG;
    cudaSetDevice(c->device);
    launch_est(c);
    CHECK_LAUNCH(c);
    int r = sync_read(c, c->red_out, c->host_scalars, sizeof(double));
    if (r != SULI_OK) return r;
    if (max_div) *max_div = c->host_scalars[0];
    return SULI_OK;
}

int suli_stream(suli_ctx* c, void** stream) {
    if (!c || !stream) return SULI_ERR_ARG;
    *stream = (void*)c->stream;
    return SULI_OK;
}

int suli_profile_enable(suli_ctx* c, int on) {
    if (!c) return SULI_ERR_ARG;
    cudaSetDevice(c->device);
    auto& P = c->prof;
    prof_resolve(c);
    if (on && P.ev.empty()) {
        const int pairs = 1 << 14;
        P.ev.resize(2 * pairs);
        P.kind.resize(pairs);
        for (auto& e : P.ev) CUDA_TRY(c, cudaEventCreate(&e));
    }
    for (int k = 0; k < SULI_K_COUNT; ++k) { P.ms[k] = 0.; P.launches[k] = 0; }
    P.cg_iters = 0;
    P.used = 0;
    P.on = (on != 0);
    return SULI_OK;
}

int suli_profile_read(suli_ctx* c, double ms[SULI_K_COUNT], long long launches[SULI_K_COUNT],
                      long long* cg_iterations) {
    if (!c) return SULI_ERR_ARG;
    cudaSetDevice(c->device);
    prof_resolve(c);
    for (int k = 0; k < SULI_K_COUNT; ++k) {
        if (ms) ms[k] = c->prof.ms[k];
        if (launches) launches[k] = c->prof.launches[k];
    }
    if (cg_iterations) *cg_iterations = c->prof.cg_iters;
    return SULI_OK;
}

// one time step (1_principal.f90:64-108, without MMS/plot/restart), then est()
// Copies of suli_step_host that overlap the step: the inputs not yet scattered into their
// fields (prd1), the outputs already gathered and on their way out (ls).
struct StepIO {
    int n_in, n_out;
    const int* fin;
    const int* fout;
    double* const* hout;
    bool late_in[SULI_STEP_HOST_MAX_FIELDS];    // copied in; scattered before the first convdiff
    bool early_out[SULI_STEP_HOST_MAX_FIELDS];  // gathered after the level-set stage
};

static int io_scatter(suli_ctx* c, int slot, int field) {
    int lo[3], hi[3];
    extent(&c->P, field, lo, hi);
    const int n0 = hi[0] - lo[0] + 1, n1 = hi[1] - lo[1] + 1, n2 = hi[2] - lo[2] + 1;
    const size_t n = (size_t)n0 * n1 * n2;
    CUDA_TRY(c, cudaStreamWaitEvent(c->stream, c->io_ev[slot], 0));
    k_scatter<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->g, c->io_stage[slot], c->f[field], lo[0], lo[1],
                                                                   lo[2], n0, n1, n2);
    CHECK_LAUNCH(c);
    return SULI_OK;
}

static int io_send(suli_ctx* c, int slot, int field, double* host) {
    int lo[3], hi[3];
    extent(&c->P, field, lo, hi);
    const int n0 = hi[0] - lo[0] + 1, n1 = hi[1] - lo[1] + 1, n2 = hi[2] - lo[2] + 1;
    const size_t n = (size_t)n0 * n1 * n2;
    k_gather<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->g, c->f[field], c->io_stage[slot], lo[0], lo[1],
                                                                  lo[2], n0, n1, n2);
    CHECK_LAUNCH(c);
    CUDA_TRY(c, cudaEventRecord(c->io_ev[slot], c->stream));
    CUDA_TRY(c, cudaStreamWaitEvent(c->io_out, c->io_ev[slot], 0));
    CUDA_TRY(c, cudaMemcpyAsync(host, c->io_stage[slot], n * sizeof(double), cudaMemcpyDefault, c->io_out));
    return SULI_OK;
}

// The time step (1_principal.f90:64-108); `io` (suli_step_host) places the overlapped copies.
static int step_body(suli_ctx* c, int it, suli_step_stats* st, const StepIO* io) {
    int status = SULI_OK;
    c->t = it * c->dt;
    int r = suli_level_set(c, nullptr);
    if (r < 0) return r;
    if (c->P.obst_t != 0 && (r = suli_contorno(c, 3)) < 0) return r;   // 1_principal.f90:75
    if (io)   // ls is final here unless the wave inflow rounds it in every stage
        for (int q = 0; q < io->n_out; ++q)
            if (io->early_out[q] && (r = io_send(c, SULI_STEP_HOST_MAX_FIELDS + q, io->fout[q], io->hout[q])) < 0)
                return r;
    for (int tt = 1; tt <= c->ntt; ++tt) {
        c->dt = c->a_dt[tt - 1];
        if ((r = suli_visco(c)) < 0) return r;
        if (io && tt == 1)   // convdiff's prd0 = prd1 copy is the step's first read of prd1
            for (int q = 0; q < io->n_in; ++q)
                if (io->late_in[q] && (r = io_scatter(c, q, io->fin[q])) < 0) return r;
        if ((r = suli_convdiff(c)) < 0) return r;
        if ((r = suli_tempo(c, tt, it)) < 0) return r;
        if (c->P.wave_t > 0 && (r = suli_boundary_waves(c)) < 0) return r;   // 1_principal.f90:84
        if ((r = suli_contorno(c, 2)) < 0) return r;
        int n = 0;
        double res = 0.;
        r = suli_graddin(c, &n, &res);
        if (r < 0) return r;
        if (r > 0) status = r;
        if (st) { st->cg_iters[tt - 1] = n; st->cg_resid[tt - 1] = res; }
        if ((r = suli_posdin(c)) < 0) return r;
        if ((r = suli_contorno(c, 1)) < 0) return r;
    }
    double md = 0.;
    if ((r = suli_est(c, &md)) < 0) return r;
    if (st) {
        for (int tt = c->ntt; tt < 3; ++tt) { st->cg_iters[tt] = 0; st->cg_resid[tt] = 0.; }
        st->vol_ins = c->vol_ins;
        st->max_div = md;
        st->status = status;
    }
    return status;
}

int suli_step(suli_ctx* c, int it, suli_step_stats* st) {
    if (!c) return SULI_ERR_ARG;
    return step_body(c, it, st, nullptr);
}

static int io_ready(suli_ctx* c, int slot) {
    if (!c->io_in) CUDA_TRY(c, cudaStreamCreateWithFlags(&c->io_in, cudaStreamNonBlocking));
    if (!c->io_out) CUDA_TRY(c, cudaStreamCreateWithFlags(&c->io_out, cudaStreamNonBlocking));
    if (!c->io_stage[slot]) CUDA_TRY(c, cudaMalloc(&c->io_stage[slot], c->g.n * sizeof(double)));
    if (!c->io_ev[slot]) CUDA_TRY(c, cudaEventCreateWithFlags(&c->io_ev[slot], cudaEventDisableTiming));
    return SULI_OK;
}

// a box field the overlapped copies handle (planes and the forcing arrays go through
// suli_upload / suli_download, which treat them specially)
static bool io_box_field(int f) {
    return f >= 0 && f < SULI_F_COUNT && !is_plane(f) && f != SULI_F_TF_U && f != SULI_F_TF_V && f != SULI_F_TF_W;
}

int suli_step_host(suli_ctx* c, int it, int n_in, const int* in_fields, const double* const* in_host, int n_out,
                   const int* out_fields, double* const* out_host, suli_step_stats* st) {
    if (!c) return SULI_ERR_ARG;
    if (n_in < 0 || n_in > SULI_STEP_HOST_MAX_FIELDS || n_out < 0 || n_out > SULI_STEP_HOST_MAX_FIELDS ||
        (n_in > 0 && (!in_fields || !in_host)) || (n_out > 0 && (!out_fields || !out_host)))
        return fail(c, SULI_ERR_ARG, "step_host: bad field lists");
    for (int a = 0; a < n_in; ++a) {
        if (in_fields[a] < 0 || in_fields[a] >= SULI_F_COUNT || !in_host[a])
            return fail(c, SULI_ERR_ARG, "step_host: bad input field");
        for (int b = 0; b < a; ++b)
            if (in_fields[b] == in_fields[a]) return fail(c, SULI_ERR_ARG, "step_host: input field listed twice");
    }
    for (int a = 0; a < n_out; ++a) {
        if (out_fields[a] < 0 || out_fields[a] >= SULI_F_COUNT || !out_host[a])
            return fail(c, SULI_ERR_ARG, "step_host: bad output field");
        for (int b = 0; b < a; ++b)
            if (out_fields[b] == out_fields[a]) return fail(c, SULI_ERR_ARG, "step_host: output field listed twice");
    }
    cudaSetDevice(c->device);
    StepIO io{};
    io.n_in = n_in; io.n_out = n_out; io.fin = in_fields; io.fout = out_fields; io.hout = out_host;
    for (int q = 0; q < n_in; ++q)
        if (io_box_field(in_fields[q]))
            if (int r = io_ready(c, q)) return r;
    for (int q = 0; q < n_out; ++q)
        if (io_box_field(out_fields[q]))
            if (int r = io_ready(c, SULI_STEP_HOST_MAX_FIELDS + q)) return r;
    // inputs: the special ones synchronously, the box fields on the copy stream, each scattered
    // as soon as it lands (prd1 only before the first convdiff)
    for (int q = 0; q < n_in; ++q)
        if (!io_box_field(in_fields[q]))
            if (int r = suli_upload(c, in_fields[q], in_host[q])) return r;
    int r = SULI_OK;
    for (int q = 0; q < n_in && r == SULI_OK; ++q) {
        const int f = in_fields[q];
        if (!io_box_field(f)) continue;
        int lo[3], hi[3];
        extent(&c->P, f, lo, hi);
        const size_t n = (size_t)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
        cudaError_t e = cudaMemcpyAsync(c->io_stage[q], in_host[q], n * sizeof(double), cudaMemcpyDefault, c->io_in);
        if (e == cudaSuccess) e = cudaEventRecord(c->io_ev[q], c->io_in);
        if (e != cudaSuccess) {
            r = fail(c, SULI_ERR_CUDA, std::string("step_host: copy in: ") + cudaGetErrorString(e));
            break;
        }
        io.late_in[q] = (f == SULI_F_PRD1);
        if (!io.late_in[q]) r = io_scatter(c, q, f);
    }
    for (int q = 0; q < n_out; ++q) io.early_out[q] = (out_fields[q] == SULI_F_LS && c->P.wave_t == 0);
    if (r == SULI_OK) r = step_body(c, it, st, &io);
    int status = r;
    // outputs: each box field gathered into its staging box and copied out while the next one
    // is gathered
    if (status >= 0)
        for (int q = 0; q < n_out; ++q) {
            if (!io_box_field(out_fields[q]) || io.early_out[q]) continue;
            if (int rs = io_send(c, SULI_STEP_HOST_MAX_FIELDS + q, out_fields[q], out_host[q])) { status = rs; break; }
        }
    // nothing may still read the caller's inputs or write its outputs once the call returns
    cudaError_t e1 = cudaStreamSynchronize(c->io_in);
    cudaError_t e2 = cudaStreamSynchronize(c->io_out);
    cudaError_t e3 = cudaStreamSynchronize(c->stream);
    if (status >= 0 && (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess))
        return fail(c, SULI_ERR_CUDA, std::string("step_host: ") +
                                          cudaGetErrorString(e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3)));
    if (status < 0) return status;
    for (int q = 0; q < n_out; ++q)
        if (!io_box_field(out_fields[q]))
            if (int rd = suli_download(c, out_fields[q], out_host[q])) return rd;
    return status;
}

}  // extern "C"
