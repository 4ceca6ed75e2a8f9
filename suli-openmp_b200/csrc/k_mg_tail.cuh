// k_mg_tail.cuh — the last level above the coarsest and the coarsest solve of the inner
// solve's V-cycle in one CTA (included by k_mixed.cu after the vectorised kernels).
//
// At 256x128x128 these are 32x16x16 (8192 cells) and 16x8x8 (1024 cells): five launches of the
// per-level path (pre-smoothing, restriction, coarsest solve, prolongation + post-smoothing,
// last sweep) with microseconds of work each, bound by launch and memory latency.  Here one CTA
// of 1024 threads runs them as phases separated by CTA barriers, with the level's smoothing
// iterates and the coarsest grid in shared memory; the level's faces, inverse diagonal and
// right-hand side come through L1/L2.  Per cell the arithmetic is the per-level kernels' (the
// same stored faces, apply_faces, update expressions and the restriction's children order), so
// the V-cycle is the same operator.  Used when that level has at most kTailM cells and the
// coarsest at most 1024, and SULI_TAIL=1 selects it: measured at 256x128x128 one CTA takes
// longer than the five launches it replaces, so the per-level kernels stay the default.
#pragma once

namespace suli {

constexpr int kTailM = 8192;
constexpr int kTailThreads = 1024;

static inline size_t tail_smem_bytes() { return (size_t)(3 * kTailM + 3 * 1024) * sizeof(float); }

struct TailArgs {
    Geo gm, gb;                 // the level M and the coarsest level B
    OpStored am, ab;            // their stored faces and inverse diagonals
    const float* fm;            // M's right-hand side (the restriction from the level above)
    float* ym;                  // M's result (the level above's coarse correction)
    float omega, omega2, alpha;
    int sweeps;
    CoarsePoly cp;              // the coarsest solve's polynomial (k_mg_coarsest)
};

// neighbour cell numbers (0-based, x fastest) of cell (i, j, k) under the unknowns' map
__device__ __forceinline__ void tail_nb(const Geo& G, const BC& bc, int i, int j, int k, int (&nb)[6]) {
    const int im = map_any(i - 1, G.nx, bc.perx), ip = map_any(i + 1, G.nx, bc.perx);
    const int jm = map_any(j - 1, G.ny, bc.pery), jp = map_any(j + 1, G.ny, bc.pery);
    const int km = map_any(k - 1, G.nz, bc.perz), kp = map_any(k + 1, G.nz, bc.perz);
    auto lin = [&](int a, int b, int d) { return (a - 1) + G.nx * ((b - 1) + G.ny * (d - 1)); };
    nb[0] = lin(im, j, k); nb[1] = lin(ip, j, k); nb[2] = lin(i, jm, k);
    nb[3] = lin(i, jp, k); nb[4] = lin(i, j, km); nb[5] = lin(i, j, kp);
}
__device__ __forceinline__ void tail_ijk(const Geo& G, int q, int& i, int& j, int& k) {
    i = q % G.nx + 1;
    j = (q / G.nx) % G.ny + 1;
    k = q / (G.nx * G.ny) + 1;
}
// A x at cell q of a level held in shared memory (x indexed by cell number)
__device__ __forceinline__ float tail_ax(const Faces& F, const float* x, int q, const int (&nb)[6]) {
    return apply_faces(F, x[q], x[nb[0]], x[nb[1]], x[nb[2]], x[nb[3]], x[nb[4]], x[nb[5]]);
}

__global__ void __launch_bounds__(kTailThreads) k_mg_tail(const __grid_constant__ TailArgs a, BC bc, const PCGState* st) {
    pdl_wait();
    if (st->done) return;
    extern __shared__ __align__(16) float t_smem[];
    float* x1 = t_smem;                // M: first sweep, later the prolongated x'
    float* ys = t_smem + kTailM;       // M: pre-smoothed y
    float* xo = t_smem + 2 * kTailM;   // M: post-smoothed x
    float* fb = t_smem + 3 * kTailM;   // B: right-hand side
    float* xb[2] = {fb + 1024, fb + 2048};
    const Geo& M = a.gm;
    const Geo& B = a.gb;
    const int nm = M.nx * M.ny * M.nz, nbc = B.nx * B.ny * B.nz;
    const int t = threadIdx.x;
    // pre-smoothing on M: x1 = w f/dg, y = x1 + w2 (f - A x1)/dg
    for (int q = t; q < nm; q += kTailThreads) {
        int i, j, k;
        tail_ijk(M, q, i, j, k);
        const int c = (int)M.idx(i, j, k);
        x1[q] = a.omega * a.fm[c] * a.am.inv_diag(c);
    }
    __syncthreads();
    for (int q = t; q < nm; q += kTailThreads) {
        int i, j, k, nb[6];
        tail_ijk(M, q, i, j, k);
        tail_nb(M, bc, i, j, k, nb);
        const int c = (int)M.idx(i, j, k);
        const float ax = tail_ax(a.am.cell(M, i, j, k, c), x1, q, nb);
        ys[q] = x1[q] + a.omega2 * (a.fm[c] - ax) * a.am.inv_diag(c);
    }
    __syncthreads();
    // restriction: f_B = (1/8) sum over the children of (f - A y), children in (z, y, x) order
    for (int p = t; p < nbc; p += kTailThreads) {
        int I, J, K;
        tail_ijk(B, p, I, J, K);
        float s = 0.f;
        for (int dz = 0; dz < 2; ++dz)
            for (int dy = 0; dy < 2; ++dy)
                for (int dx = 0; dx < 2; ++dx) {
                    const int i = 2 * I - 1 + dx, j = 2 * J - 1 + dy, k = 2 * K - 1 + dz;
                    int nb[6];
                    tail_nb(M, bc, i, j, k, nb);
                    const int q = (i - 1) + M.nx * ((j - 1) + M.ny * (k - 1));
                    const int c = (int)M.idx(i, j, k);
                    s += a.fm[c] - tail_ax(a.am.cell(M, i, j, k, c), ys, q, nb);
                }
        fb[p] = 0.125f * s;
    }
    __syncthreads();
    // coarsest: Jacobi sweeps from x = w f/dg or the Chebyshev polynomial (k_mg_coarsest)
    int cb = 0, nbb[6] = {0, 0, 0, 0, 0, 0};
    float fv = 0.f, idv = 1.f;
    Faces FB{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (t < nbc) {
        int i, j, k;
        tail_ijk(B, t, i, j, k);
        cb = (int)B.idx(i, j, k);
        fv = fb[t];
        idv = a.ab.inv_diag(cb);
        FB = a.ab.cell(B, i, j, k, cb);
        tail_nb(B, bc, i, j, k, nbb);
    }
    const bool cheb = a.cp.lo > 0.f;
    float dv = 0.f;
    if (t < nbc) {
        dv = cheb ? a.cp.g0 * fv * idv : 0.f;
        xb[0][t] = cheb ? dv : a.omega * fv * idv;
    }
    __syncthreads();
    int cur = 0;
    for (int sw = 1; sw < a.sweeps; ++sw) {
        const float h = cheb ? a.cp.h[sw - 1] : 0.f, g = cheb ? a.cp.g[sw - 1] : 0.f;
        if (t < nbc) {
            const float xc = xb[cur][t];
            float ax = 0.f;
            ax += FB.xm * (xc - xb[cur][nbb[0]]);
            ax += FB.xp * (xc - xb[cur][nbb[1]]);
            ax += FB.ym * (xc - xb[cur][nbb[2]]);
            ax += FB.yp * (xc - xb[cur][nbb[3]]);
            ax += FB.zm * (xc - xb[cur][nbb[4]]);
            ax += FB.zp * (xc - xb[cur][nbb[5]]);
            if (cheb) {
                dv = h * dv + g * (fv - ax) * idv;
                xb[cur ^ 1][t] = xc + dv;
            } else {
                xb[cur ^ 1][t] = xc + a.omega * (fv - ax) * idv;
            }
        }
        __syncthreads();
        cur ^= 1;
    }
    const float* xcb = xb[cur];
    // prolongation and post-smoothing on M: x' = y + alpha P x_B, x = x' + w2 (f - A x')/dg
    for (int q = t; q < nm; q += kTailThreads) {
        int i, j, k;
        tail_ijk(M, q, i, j, k);
        const int p = ((i + 1) / 2 - 1) + B.nx * (((j + 1) / 2 - 1) + B.ny * ((k + 1) / 2 - 1));
        x1[q] = ys[q] + a.alpha * xcb[p];
    }
    __syncthreads();
    for (int q = t; q < nm; q += kTailThreads) {
        int i, j, k, nb[6];
        tail_ijk(M, q, i, j, k);
        tail_nb(M, bc, i, j, k, nb);
        const int c = (int)M.idx(i, j, k);
        const float ax = tail_ax(a.am.cell(M, i, j, k, c), x1, q, nb);
        xo[q] = x1[q] + a.omega2 * (a.fm[c] - ax) * a.am.inv_diag(c);
    }
    __syncthreads();
    // last sweep: y = x + w (f - A x)/dg, to global memory
    for (int q = t; q < nm; q += kTailThreads) {
        int i, j, k, nb[6];
        tail_ijk(M, q, i, j, k);
        tail_nb(M, bc, i, j, k, nb);
        const int c = (int)M.idx(i, j, k);
        const float ax = tail_ax(a.am.cell(M, i, j, k, c), xo, q, nb);
        a.ym[c] = xo[q] + a.omega * (a.fm[c] - ax) * a.am.inv_diag(c);
    }
}

}  // namespace suli
