// k_mg_fused.cuh — one kernel for each leg of the V-cycle on a coarse level (levels 1 .. L-2,
// stored Galerkin faces; included by k_mixed.cu after the vectorised kernels, whose operator
// helpers it uses).
//
// On the coarse levels a kernel has little work (0.3-14 MB) and its time is mostly launch,
// ramp and the latency of its dependent loads, so a level's four kernels (pre-smoothing,
// restriction, prolongation + post-smoothing, last sweep) cost about four times one of them.
// Here a CTA owns a tile of kFTX x kFTY x kFTZ cells and stages in shared memory what its
// neighbours' stages need, recomputing the values of the cells around the tile that other CTAs
// own:
//   down: x1 = w f/dg on the tile and two cells around it, y = x1 + w2 (f - A x1)/dg on the tile
//         and one cell around it, y stored at the tile's cells, the residual f - A y on the tile
//         and its restriction (1/8 of the sum over the 8 children, in the order z, y, x of the
//         children, as k_mgv_restrict sums them) to the coarse right-hand side;
//   up:   x' = y + a P xc on the tile and two cells around it, x'' = x' + w2 (f - A x')/dg on
//         the tile and one cell around it, x_out = x'' + w (f - A x'')/dg on the tile.
// Per cell these are the expressions of k_mgv_pre, k_mgv_restrict, k_mgv_post and k_mgv_jacc;
// the V-cycle is the same operator up to the compiler's choice of fused multiply-adds.  The up
// kernel reads y at cells other CTAs own, so it writes its result into the level's x (the
// per-level path leaves it in y); the level above reads its coarse correction from there.
//
// Cells around the tile follow the operator's ghost map: on a periodic axis a coordinate
// outside 1..n stands for the wrapped cell (its values are computed there from the wrapped
// neighbours), across a Neumann boundary the neighbour of a cell is the cell itself, so values
// outside the domain are never formed or read.
#pragma once

namespace suli {

constexpr int kFTX = 32, kFTY = 8, kFTZ = 4;   // tile (cells); a CTA of kFTX x kFTY threads
constexpr int kFAX = kFTX + 4, kFAY = kFTY + 4, kFAZ = kFTZ + 4;   // tile and two cells around it
constexpr int kFBX = kFTX + 2, kFBY = kFTY + 2, kFBZ = kFTZ + 2;   // tile and one cell around it
constexpr int kFA = kFAX * kFAY * kFAZ, kFB = kFBX * kFBY * kFBZ, kFT = kFTX * kFTY * kFTZ;
constexpr int kFThreads = kFTX * kFTY;

// a coordinate g (1-based cell number, possibly outside 1..n) that stands for a cell
__device__ __forceinline__ bool f_valid(int g, int n, int per) { return per || (g >= 1 && g <= n); }
// the cell a valid coordinate stands for
// (a coordinate lies at most two cells outside 1..n and n >= 2 on every level with a coarser one)
__device__ __forceinline__ int f_cell(int g, int n) { return g < 1 ? g + n : (g > n ? g - n : g); }
// the neighbour coordinate the operator uses: g + d, or g itself across a Neumann boundary
__device__ __forceinline__ int f_nb(int g, int d, int n, int per) {
    const int h = g + d;
    return (per || (h >= 1 && h <= n)) ? h : g;
}

// the tile's first cell and the level's axes
struct FTile {
    int gi0, gj0, gk0;
    int nx, ny, nz, perx, pery, perz;
    __device__ __forceinline__ FTile(const Geo& G, const BC& bc) {
        gi0 = kFTX * blockIdx.x + 1;
        gj0 = kFTY * blockIdx.y + 1;
        gk0 = kFTZ * blockIdx.z + 1;
        nx = G.nx; ny = G.ny; nz = G.nz;
        perx = bc.perx; pery = bc.pery; perz = bc.perz;
    }
    __device__ __forceinline__ bool valid(int gi, int gj, int gk) const {
        return f_valid(gi, nx, perx) && f_valid(gj, ny, pery) && f_valid(gk, nz, perz);
    }
};

// The stencil of a staged array: S holds the values of the coordinates (g0 - h) .. with row
// length SX and plane size SX * SY (h = 2: the region around the tile by two cells, h = 1 by
// one); the value at coordinate (gi, gj, gk) and the operator applied at that cell (faces F)
template <int SX, int SY, int H>
struct FStage {
    const float* s;
    const FTile* t;
    __device__ __forceinline__ int at(int gi, int gj, int gk) const {
        return (gi - t->gi0 + H) + SX * ((gj - t->gj0 + H) + SY * (gk - t->gk0 + H));
    }
    __device__ __forceinline__ float v(int gi, int gj, int gk) const { return s[at(gi, gj, gk)]; }
    __device__ __forceinline__ float apply(const Faces& F, float xc, int gi, int gj, int gk) const {
        const FTile& T = *t;
        return apply_faces(F, xc, v(f_nb(gi, -1, T.nx, T.perx), gj, gk), v(f_nb(gi, 1, T.nx, T.perx), gj, gk),
                           v(gi, f_nb(gj, -1, T.ny, T.pery), gk), v(gi, f_nb(gj, 1, T.ny, T.pery), gk),
                           v(gi, gj, f_nb(gk, -1, T.nz, T.perz)), v(gi, gj, f_nb(gk, 1, T.nz, T.perz)));
    }
};

// the cell index of a valid coordinate
__device__ __forceinline__ int f_index(const Geo& G, const FTile& t, int gi, int gj, int gk, int& ci, int& cj, int& ck) {
    ci = f_cell(gi, t.nx);
    cj = f_cell(gj, t.ny);
    ck = f_cell(gk, t.nz);
    return G.idx32(ci, cj, ck);
}

// A stage's positions: a thread takes positions tid, tid + kFThreads, ...; all its loads are
// issued into registers before any value is combined (the staged arrays are written only after),
// so they are in flight together.
constexpr int kFNA = (kFA + kFThreads - 1) / kFThreads, kFNB = (kFB + kFThreads - 1) / kFThreads;
// position p of the region around the tile by h cells (row sx, rows sy) -> coordinates
template <int SX, int SY, int H>
__device__ __forceinline__ void f_pos(const FTile& T, int p, int& gi, int& gj, int& gk) {
    gi = T.gi0 - H + p % SX;
    gj = T.gj0 - H + (p / SX) % SY;
    gk = T.gk0 - H + p / (SX * SY);
}
// the values a sweep at a cell reads besides the staged ones: faces, f, 1/diag
struct FCell {
    Faces F;
    float f, d;
};
__device__ __forceinline__ FCell f_load(const Geo& G, const OpStored& A, const float* f, int ci, int cj, int ck, int c) {
    return FCell{A.cell(G, ci, cj, ck, c), f[c], A.idg[c]};
}

// ---- down leg of level l: pre-smoothing (weights w, w2) from zero, y stored, restriction of
// f - A y to the coarse right-hand side fc
__global__ void __launch_bounds__(kFThreads) k_mgf_down(Geo G, Geo Gc, BC bc, const float* __restrict__ f,
                                                        OpStored A, float* __restrict__ y, float* __restrict__ fc,
                                                        float omega, float omega2, const PCGState* st) {
    pdl_wait();
    if (st->done) return;
    __shared__ float sx1[kFA];
    __shared__ float sy[kFB];
    __shared__ float sr[kFT];
    const FTile T(G, bc);
    const int tid = threadIdx.x + kFTX * threadIdx.y;
    {   // x1 = w f/dg, two cells around the tile
        float fv[kFNA], dv[kFNA];
        bool ok[kFNA];
#pragma unroll
        for (int q = 0; q < kFNA; ++q) {
            const int p = tid + q * kFThreads;
            int gi, gj, gk;
            f_pos<kFAX, kFAY, 2>(T, p, gi, gj, gk);
            ok[q] = p < kFA && T.valid(gi, gj, gk);
            fv[q] = 0.f;
            dv[q] = 0.f;
            if (ok[q]) {
                int ci, cj, ck;
                const int c = f_index(G, T, gi, gj, gk, ci, cj, ck);
                fv[q] = f[c];
                dv[q] = A.idg[c];
            }
        }
#pragma unroll
        for (int q = 0; q < kFNA; ++q)
            if (ok[q]) sx1[tid + q * kFThreads] = omega * fv[q] * dv[q];
    }
    __syncthreads();
    const FStage<kFAX, kFAY, 2> X1{sx1, &T};
    {   // y = x1 + w2 (f - A x1)/dg, one cell around the tile
        FCell cv[kFNB];
        bool ok[kFNB];
#pragma unroll
        for (int q = 0; q < kFNB; ++q) {
            const int p = tid + q * kFThreads;
            int gi, gj, gk;
            f_pos<kFBX, kFBY, 1>(T, p, gi, gj, gk);
            ok[q] = p < kFB && T.valid(gi, gj, gk);
            if (ok[q]) {
                int ci, cj, ck;
                const int c = f_index(G, T, gi, gj, gk, ci, cj, ck);
                cv[q] = f_load(G, A, f, ci, cj, ck, c);
            }
        }
#pragma unroll
        for (int q = 0; q < kFNB; ++q) {
            if (!ok[q]) continue;
            const int p = tid + q * kFThreads;
            int gi, gj, gk;
            f_pos<kFBX, kFBY, 1>(T, p, gi, gj, gk);
            const float xc = X1.v(gi, gj, gk);
            const float ax = X1.apply(cv[q].F, xc, gi, gj, gk);
            sy[p] = xc + omega2 * (cv[q].f - ax) * cv[q].d;
        }
    }
    __syncthreads();
    const FStage<kFBX, kFBY, 1> Y{sy, &T};
    {   // the residual on the tile (a thread's column of kFTZ cells); y at the tile's cells
        const int gi = T.gi0 + threadIdx.x, gj = T.gj0 + threadIdx.y;
        FCell cv[kFTZ];
        bool ok[kFTZ];
#pragma unroll
        for (int m = 0; m < kFTZ; ++m) {
            const int gk = T.gk0 + m;
            ok[m] = gi <= G.nx && gj <= G.ny && gk <= G.nz;
            if (ok[m]) cv[m] = f_load(G, A, f, gi, gj, gk, G.idx32(gi, gj, gk));
        }
#pragma unroll
        for (int m = 0; m < kFTZ; ++m) {
            const int gk = T.gk0 + m;
            float rv = 0.f;
            if (ok[m]) {
                const float yc = Y.v(gi, gj, gk);
                rv = cv[m].f - Y.apply(cv[m].F, yc, gi, gj, gk);
                y[G.idx32(gi, gj, gk)] = yc;
            }
            sr[threadIdx.x + kFTX * (threadIdx.y + kFTY * m)] = rv;
        }
    }
    __syncthreads();
    // the tile's parents: 1/8 of the sum over their children, in the order z, y, x
    if (tid < kFT / 8) {
        const int pi = tid % (kFTX / 2), pj = (tid / (kFTX / 2)) % (kFTY / 2), pk = tid / ((kFTX / 2) * (kFTY / 2));
        const int I = (T.gi0 + 1) / 2 + pi, J = (T.gj0 + 1) / 2 + pj, K = (T.gk0 + 1) / 2 + pk;
        if (I <= Gc.nx && J <= Gc.ny && K <= Gc.nz) {
            float s = 0.f;
#pragma unroll
            for (int dz = 0; dz < 2; ++dz)
#pragma unroll
                for (int dy = 0; dy < 2; ++dy)
#pragma unroll
                    for (int dx = 0; dx < 2; ++dx) s += sr[(2 * pi + dx) + kFTX * ((2 * pj + dy) + kFTY * (2 * pk + dz))];
            fc[Gc.idx32(I, J, K)] = 0.125f * s;
        }
    }
}

// ---- up leg of level l: x' = y + a P xc (xc the coarse level's correction), the post-smoothing
// sweep (weight w2) and the last sweep (w) into xout
__global__ void __launch_bounds__(kFThreads) k_mgf_up(Geo G, Geo Gc, BC bc, const float* __restrict__ y,
                                                      const float* __restrict__ xc, const float* __restrict__ f,
                                                      OpStored A, float* __restrict__ xout, float omega, float omega2,
                                                      float alpha, const PCGState* st) {
    pdl_wait();
    if (st->done) return;
    __shared__ float sx1[kFA];
    __shared__ float sx2[kFB];
    const FTile T(G, bc);
    const int tid = threadIdx.x + kFTX * threadIdx.y;
    {   // x' = y + a xc(parent), two cells around the tile
        float yv[kFNA], cv[kFNA];
        bool ok[kFNA];
#pragma unroll
        for (int q = 0; q < kFNA; ++q) {
            const int p = tid + q * kFThreads;
            int gi, gj, gk;
            f_pos<kFAX, kFAY, 2>(T, p, gi, gj, gk);
            ok[q] = p < kFA && T.valid(gi, gj, gk);
            yv[q] = 0.f;
            cv[q] = 0.f;
            if (ok[q]) {
                int ci, cj, ck;
                const int c = f_index(G, T, gi, gj, gk, ci, cj, ck);
                yv[q] = y[c];
                cv[q] = xc[Gc.idx32((ci + 1) >> 1, (cj + 1) >> 1, (ck + 1) >> 1)];
            }
        }
#pragma unroll
        for (int q = 0; q < kFNA; ++q)
            if (ok[q]) sx1[tid + q * kFThreads] = yv[q] + alpha * cv[q];
    }
    __syncthreads();
    const FStage<kFAX, kFAY, 2> X1{sx1, &T};
    {   // x'' = x' + w2 (f - A x')/dg, one cell around the tile
        FCell cv[kFNB];
        bool ok[kFNB];
#pragma unroll
        for (int q = 0; q < kFNB; ++q) {
            const int p = tid + q * kFThreads;
            int gi, gj, gk;
            f_pos<kFBX, kFBY, 1>(T, p, gi, gj, gk);
            ok[q] = p < kFB && T.valid(gi, gj, gk);
            if (ok[q]) {
                int ci, cj, ck;
                const int c = f_index(G, T, gi, gj, gk, ci, cj, ck);
                cv[q] = f_load(G, A, f, ci, cj, ck, c);
            }
        }
#pragma unroll
        for (int q = 0; q < kFNB; ++q) {
            if (!ok[q]) continue;
            const int p = tid + q * kFThreads;
            int gi, gj, gk;
            f_pos<kFBX, kFBY, 1>(T, p, gi, gj, gk);
            const float xv = X1.v(gi, gj, gk);
            const float ax = X1.apply(cv[q].F, xv, gi, gj, gk);
            sx2[p] = xv + omega2 * (cv[q].f - ax) * cv[q].d;
        }
    }
    __syncthreads();
    const FStage<kFBX, kFBY, 1> X2{sx2, &T};
    // x_out = x'' + w (f - A x'')/dg on the tile (a thread's column of kFTZ cells)
    const int gi = T.gi0 + threadIdx.x, gj = T.gj0 + threadIdx.y;
    if (gi > G.nx || gj > G.ny) return;
    FCell cv[kFTZ];
#pragma unroll
    for (int m = 0; m < kFTZ; ++m) {
        const int gk = min(T.gk0 + m, G.nz);
        cv[m] = f_load(G, A, f, gi, gj, gk, G.idx32(gi, gj, gk));
    }
#pragma unroll
    for (int m = 0; m < kFTZ; ++m) {
        const int gk = T.gk0 + m;
        if (gk > G.nz) break;
        const float xv = X2.v(gi, gj, gk);
        xout[G.idx32(gi, gj, gk)] = xv + omega * (cv[m].f - X2.apply(cv[m].F, xv, gi, gj, gk)) * cv[m].d;
    }
}

static inline dim3 fgrid(const Geo& g) {
    return dim3((g.nx + kFTX - 1) / kFTX, (g.ny + kFTY - 1) / kFTY, (g.nz + kFTZ - 1) / kFTZ);
}

}  // namespace suli
