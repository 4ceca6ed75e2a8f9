// k_mg_cluster.cuh — the three coarsest levels of the inner solve's V-cycle in one launch of a
// 16-CTA thread-block cluster (included by k_mixed.cu after the vectorised kernels).
//
// Below about 65k cells a level's kernels are launch- and latency-bound: at 256x128x128 the
// levels 64x32x32, 32x16x16 and the 16x8x8 coarsest grid took nine launches per inner iteration
// that moved a few MB between them.  Here one cluster holds those levels in its distributed
// shared memory: CTA r owns z-slab r of the level M = b (pb planes) and of its coarse level
// C = b + 1 (pb/2 planes); the coarsest level B = b + 2 is solved inside CTA 0.  A neighbour in
// another CTA's slab is read through distributed shared memory after a cluster barrier.  The
// host uses it when level M has 32 planes (two per CTA, so C has one per CTA and B eight) and at
// most 2048 cells a plane.
//
// The stages and the per-cell arithmetic are those of the per-level kernels (k_mgv_pre,
// k_mgv_restrict, k_mg_coarsest, k_mgv_post, k_mgv_jacc on stored faces): two damped Jacobi
// sweeps from zero, restriction of (f - A y)/8, the coarsest solve (k_mg_coarsest), prolongation
// y + alpha P x_c, then two sweeps.  Only the restriction to B sums its 8 children in two
// halves (one per CTA holding them) before adding.  The level M's right-hand side comes from,
// and its result returns to, global memory (mg[b].f, mg[b].y): the finer levels' kernels are
// unchanged.
//
// Every CTA takes every cluster barrier (the done test at entry reads one value written before
// the launch, the same for all), and a last barrier keeps each CTA's shared memory alive until
// the other CTAs' reads of it have finished.
#pragma once
#include <cooperative_groups.h>

namespace suli {

namespace cg = cooperative_groups;

constexpr int kClCTAs = 16;
constexpr int kClThreads = 1024;
constexpr int kClMaxM = 4096;    // cells of level M in one CTA
constexpr int kClMaxB = 1024;    // cells of the coarsest level

struct ClLevel {
    Geo g;
    const float *sx, *sy, *sz, *idg;
};
struct ClArgs {
    ClLevel M, C, B;
    BC bc;
    const float* fM;   // level M's right-hand side (the restriction from the level above)
    float* yM;         // level M's result (read by the prolongation into the level above)
    float omega, alpha;
    float omega2;      // weight of the second pre-smoothing sweep, of the first post-smoothing one
    int sweeps;        // steps of the coarsest solve
    CoarsePoly cp;     // the coarsest solve's polynomial (k_mg_coarsest)
};

// one level's slab in shared memory: pl planes of nx x ny cells, faces of those cells (x faces
// 1..nx+1, y faces 1..ny+1, z faces of the slab's planes and the one above)
struct ClSlab {
    int nx, ny, pl, k0;   // k0: first (global, 1-based) plane of the slab
    float *y, *x, *f, *d, *sx, *sy, *sz;
    __device__ int cell(int i, int j, int kl) const { return (i - 1) + nx * ((j - 1) + ny * kl); }
    __device__ float fxm(int i, int j, int kl) const { return sx[(i - 1) + (nx + 1) * ((j - 1) + ny * kl)]; }
    __device__ float fxp(int i, int j, int kl) const { return sx[i + (nx + 1) * ((j - 1) + ny * kl)]; }
    __device__ float fym(int i, int j, int kl) const { return sy[(i - 1) + nx * ((j - 1) + (ny + 1) * kl)]; }
    __device__ float fyp(int i, int j, int kl) const { return sy[(i - 1) + nx * (j + (ny + 1) * kl)]; }
    __device__ float fzm(int i, int j, int kl) const { return sz[(i - 1) + nx * ((j - 1) + ny * kl)]; }
    __device__ float fzp(int i, int j, int kl) const { return sz[(i - 1) + nx * ((j - 1) + ny * (kl + 1))]; }
};

__device__ __forceinline__ float* carve(float*& p, int n) {
    float* r = p;
    p += (n + 31) & ~31;
    return r;
}

// A thread's share of a slab array: up to kClLoads elements, all loads issued before the first
// store so that their L2 latencies overlap (a loop with one load and one store per trip would
// wait out each latency in turn).
constexpr int kClLoads = 8;
template <class Idx>
__device__ __forceinline__ void cl_copy(const float* __restrict__ src, float* dst, int n, int tid, Idx gidx) {
    float v[kClLoads];
#pragma unroll
    for (int t = 0; t < kClLoads; ++t) {
        const int q = tid + t * kClThreads;
        v[t] = (q < n) ? src[gidx(q)] : 0.f;
    }
#pragma unroll
    for (int t = 0; t < kClLoads; ++t) {
        const int q = tid + t * kClThreads;
        if (q < n) dst[q] = v[t];
    }
}

__device__ inline void cl_load_slab(const ClLevel& L, ClSlab& S, const float* fglob, int tid) {
    const Geo& G = L.g;
    const int nx = S.nx, ny = S.ny, k0 = S.k0;
    auto cell = [&](int q) { return G.idx(q % nx + 1, (q / nx) % ny + 1, k0 + q / (nx * ny)); };
    cl_copy(L.idg, S.d, nx * ny * S.pl, tid, cell);
    if (fglob) cl_copy(fglob, S.f, nx * ny * S.pl, tid, cell);
    cl_copy(L.sx, S.sx, (nx + 1) * ny * S.pl, tid,
            [&](int q) { return G.idx(q % (nx + 1) + 1, (q / (nx + 1)) % ny + 1, k0 + q / ((nx + 1) * ny)); });
    cl_copy(L.sy, S.sy, nx * (ny + 1) * S.pl, tid,
            [&](int q) { return G.idx(q % nx + 1, (q / nx) % (ny + 1) + 1, k0 + q / (nx * (ny + 1))); });
    cl_copy(L.sz, S.sz, nx * ny * (S.pl + 1), tid, cell);
}

// value of a slab array at global cell (i, j, k) (already ghost-mapped): this CTA's shared
// memory, or the owning CTA's through the cluster
template <class Sel>
__device__ __forceinline__ float cl_at(cg::cluster_group& cl, const ClSlab& S, Sel sel, int i, int j, int k) {
    const int owner = (k - 1) / S.pl, kl = (k - 1) - owner * S.pl;
    const float* base = sel(S);
    if (owner != (int)cl.block_rank()) base = cl.map_shared_rank(base, owner);
    return base[S.cell(i, j, kl)];
}

// A x at local cell (i, j, kl) of slab S for a value source val(i, j, k) (global k, mapped)
template <class Val>
__device__ __forceinline__ float cl_apply(const ClSlab& S, const BC& bc, int nz, int i, int j, int kl, float xc,
                                          Val val) {
    const int k = S.k0 + kl;
    const int im = map_any(i - 1, S.nx, bc.perx), ip = map_any(i + 1, S.nx, bc.perx);
    const int jm = map_any(j - 1, S.ny, bc.pery), jp = map_any(j + 1, S.ny, bc.pery);
    const int km = map_any(k - 1, nz, bc.perz), kp = map_any(k + 1, nz, bc.perz);
    const Faces F{S.fxm(i, j, kl), S.fxp(i, j, kl), S.fym(i, j, kl), S.fyp(i, j, kl), S.fzm(i, j, kl), S.fzp(i, j, kl)};
    return apply_faces(F, xc, val(im, j, k), val(ip, j, k), val(i, jm, k), val(i, jp, k), val(i, j, km),
                       val(i, j, kp));
}

__global__ void __launch_bounds__(kClThreads, 1) k_mg_cluster(const __grid_constant__ ClArgs A, const PCGState* st) {
    pdl_wait();
    if (st->done) return;   // the same value in every CTA of the cluster
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank(), tid = threadIdx.x;
    const BC bc = A.bc;
    const float om = A.omega, om2 = A.omega2, al = A.alpha;
    extern __shared__ __align__(16) float smem[];
    float* p = smem;
    ClSlab M, C;
    M.nx = A.M.g.nx; M.ny = A.M.g.ny; M.pl = 2; M.k0 = rank * 2 + 1;
    C.nx = A.C.g.nx; C.ny = A.C.g.ny; C.pl = 1; C.k0 = rank + 1;
    const int nM = M.nx * M.ny * M.pl, nC = C.nx * C.ny * C.pl;
    M.y = carve(p, nM); M.x = carve(p, nM); M.f = carve(p, nM); M.d = carve(p, nM);
    M.sx = carve(p, (M.nx + 1) * M.ny * M.pl); M.sy = carve(p, M.nx * (M.ny + 1) * M.pl);
    M.sz = carve(p, M.nx * M.ny * (M.pl + 1));
    C.y = carve(p, nC); C.x = carve(p, nC); C.f = carve(p, nC); C.d = carve(p, nC);
    C.sx = carve(p, (C.nx + 1) * C.ny * C.pl); C.sy = carve(p, C.nx * (C.ny + 1) * C.pl);
    C.sz = carve(p, C.nx * C.ny * (C.pl + 1));
    const Geo& GB = A.B.g;
    const int nB = GB.nx * GB.ny * GB.nz, nBp = GB.nx * GB.ny;
    float* xb0 = carve(p, nB);
    float* xb1 = carve(p, nB);
    float* part = carve(p, kClCTAs * nBp);   // CTA 0: half sums of the restriction to B, one row per CTA
    const int nzM = A.M.g.nz, nzC = A.C.g.nz;

    cl_load_slab(A.M, M, A.fM, tid);
    cl_load_slab(A.C, C, nullptr, tid);
    cl.sync();   // every slab loaded: neighbours' f and diagonal readable

    // ---- level M: two Jacobi sweeps from zero, y = x1 + w (f - A x1)/dg with x1 = w f/dg
    auto x1M = [&](int i, int j, int k) {
        return om * cl_at(cl, M, [](const ClSlab& s) { return (const float*)s.f; }, i, j, k) *
               cl_at(cl, M, [](const ClSlab& s) { return (const float*)s.d; }, i, j, k);
    };
    for (int q = tid; q < nM; q += kClThreads) {
        const int i = q % M.nx + 1, j = (q / M.nx) % M.ny + 1, kl = q / (M.nx * M.ny);
        const float xc = om * M.f[q] * M.d[q];
        const float ax = cl_apply(M, bc, nzM, i, j, kl, xc, x1M);
        M.y[q] = xc + om2 * (M.f[q] - ax) * M.d[q];
    }
    cl.sync();
    // ---- restriction M -> C: f_C = (1/8) sum of the 8 children of (f - A y)
    auto yM = [&](int i, int j, int k) { return cl_at(cl, M, [](const ClSlab& s) { return (const float*)s.y; }, i, j, k); };
    for (int q = tid; q < nC; q += kClThreads) {
        const int I = q % C.nx + 1, J = (q / C.nx) % C.ny + 1, Kl = q / (C.nx * C.ny);
        float s = 0.f;
#pragma unroll
        for (int dz = 0; dz < 2; ++dz)
#pragma unroll
            for (int dy = 0; dy < 2; ++dy)
#pragma unroll
                for (int dx = 0; dx < 2; ++dx) {
                    const int i = 2 * I - 1 + dx, j = 2 * J - 1 + dy, kl = 2 * Kl + dz;
                    const int c = M.cell(i, j, kl);
                    s += M.f[c] - cl_apply(M, bc, nzM, i, j, kl, M.y[c], yM);
                }
        C.f[q] = 0.125f * s;
    }
    cl.sync();
    // ---- level C: two sweeps from zero
    auto x1C = [&](int i, int j, int k) {
        return om * cl_at(cl, C, [](const ClSlab& s) { return (const float*)s.f; }, i, j, k) *
               cl_at(cl, C, [](const ClSlab& s) { return (const float*)s.d; }, i, j, k);
    };
    for (int q = tid; q < nC; q += kClThreads) {
        const int i = q % C.nx + 1, j = (q / C.nx) % C.ny + 1, kl = q / (C.nx * C.ny);
        const float xc = om * C.f[q] * C.d[q];
        const float ax = cl_apply(C, bc, nzC, i, j, kl, xc, x1C);
        C.y[q] = xc + om2 * (C.f[q] - ax) * C.d[q];
    }
    cl.sync();
    // ---- restriction C -> B: CTA r holds C plane r + 1, the children dz = r % 2 of B plane r/2 + 1;
    // it sums its 4 children of every B cell of that plane and CTA 0 adds the two halves
    {
        auto yC = [&](int i, int j, int k) { return cl_at(cl, C, [](const ClSlab& s) { return (const float*)s.y; }, i, j, k); };
        float* part0 = cl.map_shared_rank(part, 0);
        for (int q = tid; q < nBp; q += kClThreads) {
            const int I = q % GB.nx + 1, J = q / GB.nx + 1;
            float s = 0.f;
#pragma unroll
            for (int dy = 0; dy < 2; ++dy)
#pragma unroll
                for (int dx = 0; dx < 2; ++dx) {
                    const int i = 2 * I - 1 + dx, j = 2 * J - 1 + dy;
                    const int c = C.cell(i, j, 0);
                    s += C.f[c] - cl_apply(C, bc, nzC, i, j, 0, C.y[c], yC);
                }
            part0[rank * nBp + q] = s;
        }
    }
    cl.sync();
    // ---- coarsest level B in CTA 0: damped Jacobi sweeps from x1 = w f/dg, or the Chebyshev
    //      polynomial (k_mg_coarsest)
    if (rank == 0) {
        float fv = 0.f, idgv = 1.f, s6[6] = {0, 0, 0, 0, 0, 0};
        int nb[6] = {0, 0, 0, 0, 0, 0};
        const int t = tid;
        if (t < nB) {
            const int i = t % GB.nx + 1, j = (t / GB.nx) % GB.ny + 1, k = t / nBp + 1;
            fv = 0.125f * (part[(2 * (k - 1)) * nBp + (t % nBp)] + part[(2 * (k - 1) + 1) * nBp + (t % nBp)]);
            const long long c = GB.idx(i, j, k);
            idgv = A.B.idg[c];
            s6[0] = A.B.sx[c]; s6[1] = A.B.sx[c + 1]; s6[2] = A.B.sy[c]; s6[3] = A.B.sy[c + GB.px];
            s6[4] = A.B.sz[c]; s6[5] = A.B.sz[c + GB.pxy];
            const int im = (i > 1) ? i - 1 : (bc.perx ? GB.nx : i), ip = (i < GB.nx) ? i + 1 : (bc.perx ? 1 : i);
            const int jm = (j > 1) ? j - 1 : (bc.pery ? GB.ny : j), jp = (j < GB.ny) ? j + 1 : (bc.pery ? 1 : j);
            const int km = (k > 1) ? k - 1 : (bc.perz ? GB.nz : k), kp = (k < GB.nz) ? k + 1 : (bc.perz ? 1 : k);
            auto lin = [&](int a, int b, int d) { return (a - 1) + GB.nx * ((b - 1) + GB.ny * (d - 1)); };
            nb[0] = lin(im, j, k); nb[1] = lin(ip, j, k); nb[2] = lin(i, jm, k);
            nb[3] = lin(i, jp, k); nb[4] = lin(i, j, km); nb[5] = lin(i, j, kp);
        }
        const bool cheb = A.cp.lo > 0.f;
        float dv = 0.f;
        if (t < nB) {
            dv = cheb ? A.cp.g0 * fv * idgv : 0.f;
            xb0[t] = cheb ? dv : om * fv * idgv;
        }
        __syncthreads();
        float* cur = xb0;
        float* nxt = xb1;
        for (int sw = 1; sw < A.sweeps; ++sw) {
            const float h = cheb ? A.cp.h[sw - 1] : 0.f, g = cheb ? A.cp.g[sw - 1] : 0.f;
            if (t < nB) {
                const float xc = cur[t];
                float ax = 0.f;
#pragma unroll
                for (int m = 0; m < 6; ++m) ax += s6[m] * (xc - cur[nb[m]]);
                if (cheb) {
                    dv = h * dv + g * (fv - ax) * idgv;
                    nxt[t] = xc + dv;
                } else {
                    nxt[t] = xc + om * (fv - ax) * idgv;
                }
            }
            __syncthreads();
            float* tmp = cur; cur = nxt; nxt = tmp;
        }
        if (t < nB && cur != xb0) xb0[t] = cur[t];   // the solution in xb0
    }
    cl.sync();
    // ---- level C: prolongation x' = y + alpha P x_B, one sweep -> x, one sweep -> result (in y)
    const float* xB = cl.map_shared_rank(xb0, 0);
    auto xpC = [&](int i, int j, int k) {
        return cl_at(cl, C, [](const ClSlab& s) { return (const float*)s.y; }, i, j, k) +
               al * xB[((i + 1) >> 1) - 1 + GB.nx * ((((j + 1) >> 1) - 1) + GB.ny * (((k + 1) >> 1) - 1))];
    };
    for (int q = tid; q < nC; q += kClThreads) {
        const int i = q % C.nx + 1, j = (q / C.nx) % C.ny + 1, kl = q / (C.nx * C.ny);
        const float xv = xpC(i, j, C.k0 + kl);
        const float ax = cl_apply(C, bc, nzC, i, j, kl, xv, xpC);
        C.x[q] = xv + om2 * (C.f[q] - ax) * C.d[q];
    }
    cl.sync();
    auto xC = [&](int i, int j, int k) { return cl_at(cl, C, [](const ClSlab& s) { return (const float*)s.x; }, i, j, k); };
    for (int q = tid; q < nC; q += kClThreads) {
        const int i = q % C.nx + 1, j = (q / C.nx) % C.ny + 1, kl = q / (C.nx * C.ny);
        const float xv = C.x[q];
        const float ax = cl_apply(C, bc, nzC, i, j, kl, xv, xC);
        C.y[q] = xv + om * (C.f[q] - ax) * C.d[q];
    }
    cl.sync();
    // ---- level M: prolongation from C's result, one sweep -> x, one sweep -> result (global)
    auto xpM = [&](int i, int j, int k) {
        return cl_at(cl, M, [](const ClSlab& s) { return (const float*)s.y; }, i, j, k) +
               al * cl_at(cl, C, [](const ClSlab& s) { return (const float*)s.y; }, (i + 1) >> 1, (j + 1) >> 1,
                          (k + 1) >> 1);
    };
    for (int q = tid; q < nM; q += kClThreads) {
        const int i = q % M.nx + 1, j = (q / M.nx) % M.ny + 1, kl = q / (M.nx * M.ny);
        const float xv = xpM(i, j, M.k0 + kl);
        const float ax = cl_apply(M, bc, nzM, i, j, kl, xv, xpM);
        M.x[q] = xv + om2 * (M.f[q] - ax) * M.d[q];
    }
    cl.sync();
    auto xM = [&](int i, int j, int k) { return cl_at(cl, M, [](const ClSlab& s) { return (const float*)s.x; }, i, j, k); };
    for (int q = tid; q < nM; q += kClThreads) {
        const int i = q % M.nx + 1, j = (q / M.nx) % M.ny + 1, kl = q / (M.nx * M.ny);
        const float xv = M.x[q];
        const float ax = cl_apply(M, bc, nzM, i, j, kl, xv, xM);
        A.yM[A.M.g.idx(i, j, M.k0 + kl)] = xv + om * (M.f[q] - ax) * M.d[q];
    }
    cl.sync();   // no CTA leaves while another may still read its shared memory
}

// whether the three coarsest levels fit the cluster kernel's layout
inline bool cl_fits(const Geo& M, const Geo& C, const Geo& B) {
    return M.nz == 2 * kClCTAs && C.nz == kClCTAs && B.nz * 2 == C.nz && C.nx * 2 == M.nx && C.ny * 2 == M.ny &&
           B.nx * 2 == C.nx && B.ny * 2 == C.ny && 2LL * M.nx * M.ny <= kClMaxM && (long long)B.nx * B.ny * B.nz <= kClMaxB &&
           3LL * M.nx * M.ny <= (long long)kClLoads * kClThreads &&                    // z faces of a slab
           2LL * (M.nx + 1) * (M.ny + 1) <= (long long)kClLoads * kClThreads;
}
// shared memory of the cluster kernel
inline size_t cl_smem_bytes(const Geo& M, const Geo& C, const Geo& B) {
    auto r = [](long long n) { return (size_t)((n + 31) & ~31LL); };
    const int pm = 2, pc = 1;
    const long long nM = (long long)M.nx * M.ny * pm, nC = (long long)C.nx * C.ny * pc;
    size_t n = 4 * r(nM) + r((long long)(M.nx + 1) * M.ny * pm) + r((long long)M.nx * (M.ny + 1) * pm) +
               r((long long)M.nx * M.ny * (pm + 1));
    n += 4 * r(nC) + r((long long)(C.nx + 1) * C.ny * pc) + r((long long)C.nx * (C.ny + 1) * pc) +
         r((long long)C.nx * C.ny * (pc + 1));
    const long long nB = (long long)B.nx * B.ny * B.nz;
    n += 2 * r(nB) + r((long long)kClCTAs * B.nx * B.ny);
    return n * sizeof(float);
}

}  // namespace suli
