// k_learned.cu — the network's place in the pressure solve (9_grad.f90:118-151 set-up).
//
// After graddin's set-up (scaled system A~ e = b~, first residual r~0 = A~ e0 - b~):
//   features  in3[v] = (r~0/s, H, (e0 - mean e0)/s_e),  s = rms(r~0), s_e = rms(e0 - mean),
//             H the smoothed Heaviside hs that heaviside() mixed rho from (0 in phase 1, 1 in
//             phase 2), read as stored, so that the feature is the same for the linear
//             (t_hs = 0) and the geometric (t_hs = 1) mix of rho (14_level_set.f90:696-703);
//   step      y = network output, alpha = -(r~0 . y)/(y . A~ y), e <- e0 + alpha y (FP64);
//   target    P(e* - e0)/s for training (e* the converged scaled solution), P removing the
//             component along n = sqrt(d): A~ n = 0 for the all-Neumann pressure problem, so
//             that component of e* is arbitrary (the FP32 inner solves may add some of it)
//             and neither the step nor the solution depends on it.
// Cells are enumerated v = (i-1) + nx ((j-1) + ny (k-1)).  All sums are FP64 block partials
// finished by the last block.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cmath>
#include "ctx.cuh"
#include "reduce.cuh"

namespace suli {

namespace {
__device__ __forceinline__ long long cell_v(const Geo& G, int i, int j, int k) {
    return (long long)(i - 1) + (long long)G.nx * ((j - 1) + (long long)G.ny * (k - 1));
}

// The reductions over the cells give a thread kColChunks chunks of kColZ cells of one column:
// each chunk's loads come from clamped plane indices and are issued together, and the grid has
// 16x fewer blocks than one cell a thread (whose launch, block reduction and counter update were
// most of those kernels' time).  Planes past nz are left out of the sums.
constexpr int kColZ = 4, kColChunks = 4;

// s = sqrt(rr/n) from graddin's set-up reduction; mean and rms deviation of e0
__global__ void __launch_bounds__(256) k_nn_stats(Geo G, const double* __restrict__ e, const CGState* cg,
                                                  NNScale* sc, double* partial, unsigned int* counter) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    double s1 = 0., s2 = 0.;
    if (i <= G.nx && j <= G.ny) {
        for (int ch = 0; ch < kColChunks; ++ch) {
            const int k0 = (blockIdx.z * kColChunks + ch) * kColZ + 1;
            if (k0 > G.nz) break;
            double v[kColZ];
#pragma unroll
            for (int q = 0; q < kColZ; ++q) v[q] = e[G.idx(i, j, min(k0 + q, G.nz))];
#pragma unroll
            for (int q = 0; q < kColZ; ++q)
                if (k0 + q <= G.nz) {
                    s1 += v[q];
                    s2 += v[q] * v[q];
                }
        }
    }
    double t1, t2;
    if (reduce2_last(s1, s2, partial, counter, t1, t2) && flat_tid() == 0) {
        const double n = (double)G.nx * G.ny * G.nz;
        const double mean = t1 / n;
        const double var = t2 / n - mean * mean;
        const double sr = sqrt(cg->rr / n);
        sc->mean_e = mean;
        sc->sigma_e = var > 0. ? sqrt(var) : 0.;
        sc->sigma_r = sr;
        sc->alpha = 0.;
        sc->active = (!cg->done && sr > 0. && isfinite(sr) && isfinite(mean) && isfinite(var)) ? 1 : 0;
    }
}

// the three features of cell c (FP32, as the network's input receives them)
struct Feat3 {
    float r, h, e;
};
__device__ __forceinline__ Feat3 features_at(const double* r, const double* e, const double* hs, const NNScale* sc,
                                             long long c) {
    const double sr = sc->sigma_r, se = sc->sigma_e;
    return Feat3{sc->active ? (float)(r[c] / sr) : 0.f, (float)hs[c], se > 0. ? (float)((e[c] - sc->mean_e) / se) : 0.f};
}
// FP32 [V][3] (recorded training inputs, suli_nn_forward's input format)
__global__ void __launch_bounds__(256) k_nn_features(Geo G, const double* __restrict__ r, const double* __restrict__ e,
                                                     const double* __restrict__ hs, const NNScale* __restrict__ sc,
                                                     float* __restrict__ in3) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z + 1;
    if (i > G.nx || j > G.ny || k > G.nz) return;
    const long long v = cell_v(G, i, j, k);
    const Feat3 f = features_at(r, e, hs, sc, G.idx(i, j, k));
    in3[3 * v + 0] = f.r;
    in3[3 * v + 1] = f.h;
    in3[3 * v + 2] = f.e;
}
// the network's own input layout, BF16 [V][16] with channels 3-15 zero: the same values the
// network's packing of the FP32 features produces, written once
__global__ void __launch_bounds__(256) k_nn_features16(Geo G, const double* __restrict__ r,
                                                       const double* __restrict__ e, const double* __restrict__ hs,
                                                       const NNScale* __restrict__ sc,
                                                       __nv_bfloat16* __restrict__ in16) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z + 1;
    if (i > G.nx || j > G.ny || k > G.nz) return;
    const long long v = cell_v(G, i, j, k);
    const Feat3 f = features_at(r, e, hs, sc, G.idx(i, j, k));
    __nv_bfloat16 t[16];
    t[0] = __float2bfloat16(f.r);
    t[1] = __float2bfloat16(f.h);
    t[2] = __float2bfloat16(f.e);
#pragma unroll
    for (int ch = 3; ch < 16; ++ch) t[ch] = __float2bfloat16(0.f);
    uint4* o = reinterpret_cast<uint4*>(in16 + v * 16);
    o[0] = *reinterpret_cast<const uint4*>(&t[0]);
    o[1] = *reinterpret_cast<const uint4*>(&t[8]);
}

// r.y and y.A~y with A~ the set-up's scaled operator (ghost rules as the refinement residual);
// y is the network output, read in place at the ghost-mapped neighbours.  A thread walks a
// column (kColChunks chunks of kColZ cells): the x and y neighbours are mapped once, and y
// below and at a cell are the values at and above the cell before it.
__global__ void __launch_bounds__(256) k_nn_dots(Geo G, BC bc, const float* __restrict__ out,
                                                 const double* __restrict__ r, const double* __restrict__ ax,
                                                 const double* __restrict__ ay, const double* __restrict__ az,
                                                 NNScale* sc, double* partial, unsigned int* counter) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int kb = blockIdx.z * kColChunks * kColZ + 1;
    double ry = 0., yay = 0.;
    if (i <= G.nx && j <= G.ny && kb <= G.nz) {
        const long long nxy = (long long)G.nx * G.ny;
        const long long v0 = cell_v(G, i, j, 1);
        const int dxm = map_any(i - 1, G.nx, bc.perx) - i, dxp = map_any(i + 1, G.nx, bc.perx) - i;
        const int dym = (map_any(j - 1, G.ny, bc.pery) - j) * G.nx, dyp = (map_any(j + 1, G.ny, bc.pery) - j) * G.nx;
        auto yz = [&](int kk) { return out[v0 + nxy * (map_any(kk, G.nz, bc.perz) - 1)]; };
        const int px = G.px, pxy = (int)G.pxy;
        float ym = yz(kb - 1), yc = yz(kb);
        for (int ch = 0; ch < kColChunks; ++ch) {
            const int k0 = kb + ch * kColZ;
            if (k0 > G.nz) break;
            float yxm[kColZ], yxp[kColZ], yym[kColZ], yyp[kColZ], yzp[kColZ];
            double rc[kColZ], axc[kColZ], axp[kColZ], ayc[kColZ], ayp[kColZ], azc[kColZ], azp[kColZ];
#pragma unroll
            for (int q = 0; q < kColZ; ++q) {
                const int k = min(k0 + q, G.nz);
                const long long v = v0 + nxy * (k - 1);
                const int c = G.idx32(i, j, k);
                yxm[q] = out[v + dxm]; yxp[q] = out[v + dxp]; yym[q] = out[v + dym]; yyp[q] = out[v + dyp];
                yzp[q] = yz(k + 1);
                rc[q] = r[c]; axc[q] = ax[c]; axp[q] = ax[c + 1]; ayc[q] = ay[c]; ayp[q] = ay[c + px];
                azc[q] = az[c]; azp[q] = az[c + pxy];
            }
#pragma unroll
            for (int q = 0; q < kColZ; ++q) {
                if (k0 + q > G.nz) break;
                const double ycd = yc;
                const double ayv = ycd - axp[q] * (double)yxp[q] - axc[q] * (double)yxm[q] -
                                   ayp[q] * (double)yyp[q] - ayc[q] * (double)yym[q] -
                                   azp[q] * (double)yzp[q] - azc[q] * (double)ym;
                ry += rc[q] * ycd;
                yay += ycd * ayv;
                ym = yc;
                yc = yzp[q];
            }
        }
    }
    double t1, t2;
    if (reduce2_last(ry, yay, partial, counter, t1, t2) && flat_tid() == 0) {
        const bool ok = sc->active && t2 > 0. && isfinite(t1) && isfinite(t2);
        sc->alpha = ok ? -t1 / t2 : 0.;
    }
}

__global__ void __launch_bounds__(256) k_nn_apply(Geo G, const float* __restrict__ out, const NNScale* __restrict__ sc,
                                                  double* __restrict__ e) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z + 1;
    if (i > G.nx || j > G.ny || k > G.nz) return;
    const double a = sc->alpha;
    if (a == 0.) return;
    const long long c = G.idx(i, j, k);
    e[c] += a * (double)out[cell_v(G, i, j, k)];
}

// n.(e* - e0) and n.n with n = sqrt(d) -> the projection coefficient
__global__ void __launch_bounds__(256) k_nn_nullproj(Geo G, const double* __restrict__ es, const double* __restrict__ e0,
                                                     const double* __restrict__ d, NNScale* sc, double* partial,
                                                     unsigned int* counter) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z + 1;
    double s1 = 0., s2 = 0.;
    if (i <= G.nx && j <= G.ny && k <= G.nz) {
        const long long c = G.idx(i, j, k);
        s1 = sqrt(d[c]) * (es[c] - e0[c]);
        s2 = d[c];
    }
    double t1, t2;
    if (reduce2_last(s1, s2, partial, counter, t1, t2) && flat_tid() == 0) sc->proj = t2 > 0. ? t1 / t2 : 0.;
}

__global__ void __launch_bounds__(256) k_nn_target(Geo G, const double* __restrict__ es, const double* __restrict__ e0,
                                                   const double* __restrict__ d, const NNScale* __restrict__ sc,
                                                   float* __restrict__ t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z + 1;
    if (i > G.nx || j > G.ny || k > G.nz) return;
    const long long c = G.idx(i, j, k);
    const double sr = sc->sigma_r;
    t[cell_v(G, i, j, k)] = sc->active ? (float)((es[c] - e0[c] - sc->proj * sqrt(d[c])) / sr) : 0.f;
}

const dim3 kBL(32, 8, 1);
inline dim3 grid_cells(const Geo& g) { return dim3((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz); }
// the column reductions (k_nn_stats, k_nn_dots)
inline dim3 grid_cols(const Geo& g) {
    return dim3((g.nx + 31) / 32, (g.ny + 7) / 8, (g.nz + kColChunks * kColZ - 1) / (kColChunks * kColZ));
}
}  // namespace

void launch_nn_features(suli_ctx* c, float* in3) {
    const Geo& G = c->g;
    k_nn_stats<<<grid_cols(G), kBL, 0, c->stream>>>(G, c->cg_e, c->cg, c->nn_scale, c->red_partial, c->red_counter);
    k_nn_features<<<grid_cells(G), kBL, 0, c->stream>>>(G, c->cg_r, c->cg_e, c->f[SULI_F_HS], c->nn_scale, in3);
}

void launch_nn_features16(suli_ctx* c, void* in16) { launch_nn_features16_at(c, in16, c->cg_r, c->cg_e); }

// the features of the FP64 scaled residual r and iterate e (the refinement's current ones)
void launch_nn_features16_at(suli_ctx* c, void* in16, const double* r, const double* e) {
    const Geo& G = c->g;
    k_nn_stats<<<grid_cols(G), kBL, 0, c->stream>>>(G, e, c->cg, c->nn_scale, c->red_partial, c->red_counter);
    k_nn_features16<<<grid_cells(G), kBL, 0, c->stream>>>(G, r, e, c->f[SULI_F_HS], c->nn_scale,
                                                           static_cast<__nv_bfloat16*>(in16));
}

void launch_nn_step(suli_ctx* c, const float* out, double* e) {
    const Geo& G = c->g;
    k_nn_dots<<<grid_cols(G), kBL, 0, c->stream>>>(G, c->bc, out, c->cg_r, c->cg_ax, c->cg_ay, c->cg_az, c->nn_scale,
                                                      c->red_partial, c->red_counter);
    k_nn_apply<<<grid_cells(G), kBL, 0, c->stream>>>(G, out, c->nn_scale, e);
}

void launch_nn_target(suli_ctx* c, const double* e_star, float* target) {
    const Geo& G = c->g;
    k_nn_nullproj<<<grid_cells(G), kBL, 0, c->stream>>>(G, e_star, c->nn_e0, c->cg_d, c->nn_scale, c->red_partial,
                                                        c->red_counter);
    k_nn_target<<<grid_cells(G), kBL, 0, c->stream>>>(G, e_star, c->nn_e0, c->cg_d, c->nn_scale, target);
}

}  // namespace suli
