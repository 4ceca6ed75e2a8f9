// k_mixed.cu — mixed-precision pressure solve (precision = 1).
//
// The FP64 problem is the reference's scaled system A~ e = b~ (9_grad.f90:118-151).  It is
// solved by iterative refinement: the FP64 residual r~ = A~e - b~ is formed from the FP64
// coefficients, its unscaled form r_u = sqrt(d) r~ = A p - q is rounded to FP32, an FP32
// preconditioned CG solves A dp = r_u on the unscaled operator A (rows sum_f s_f (p_c - p_nb),
// ghost faces folded exactly as the reference's copies), and e <- e - sqrt(d) dp in FP64.  The
// loop stops on the same FP64 test as the plain path: ||r~|| <= tol ||b~||.
//
// Preconditioner: a geometric multigrid V-cycle in FP32 — piecewise-constant prolongation,
// restriction P^T/8 and Galerkin coarse faces (sum of the four fine faces)/8, two damped
// Jacobi sweeps before and after, a one-block Chebyshev polynomial (or damped Jacobi sweeps) on
// the coarsest grid.  Pre- and post-smoothing mirror each other and the coarsest solve is a
// fixed symmetric positive operator, so the V-cycle is one too and plain (not flexible) PCG
// applies.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include "ctx.cuh"
#include "pdl.cuh"
#include "reduce.cuh"

namespace suli {

#define FI(a, i, j, k) (a)[G.idx((i), (j), (k))]



__device__ __forceinline__ int clampi_m(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ------------------------------------------------------------------------------------
// Operators.  Level 0 forms its face conductances on the fly from the FP32 density,
// s = c2/(rho_a + rho_b) with c2 = 2 dt/dx^2 (the reference's c/((rho_a + rho_b)/2),
// 9_grad.f90:46-87), reading one density array instead of three face arrays; the coarser
// levels read their Galerkin faces.  Both keep the inverse Jacobi diagonal.  Boundary faces
// take the first interior face's value (the reference's end-face copy); on a Neumann face the
// neighbour is the cell itself, so that value only matters for periodic faces.
// ------------------------------------------------------------------------------------
struct Faces {
    float xm, xp, ym, yp, zm, zp;
};

// Column kernels: a thread owns kKZ cells of one (i,j) column; z neighbours come from the
// column's registers (with the ghost map on k), x/y neighbours through L1, and all loads of
// the column are independent.
constexpr int kKZ = 4;
struct Col {
    int i, j, k0, c0;
    Nb o;      // x/y offsets (z offsets unused)
    bool in;
};
__device__ __forceinline__ Col column(const Geo& G, const BC& bc) {
    Col q;
    q.i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    q.j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    q.k0 = blockIdx.z * kKZ + 1;
    q.in = (q.i <= G.nx && q.j <= G.ny);
    q.c0 = kBase + (q.i - 1) + G.px * q.j;
    q.o = neighbours(G, bc, q.in ? q.i : 1, q.in ? q.j : 1, 1);
    return q;
}
// load a field along the column, planes k0-1 .. k0+kKZ (ghost-mapped)
template <class F>
__device__ __forceinline__ void load_col(const Geo& G, const BC& bc, const Col& q, F val, float v[kKZ + 2]) {
#pragma unroll
    for (int m = 0; m < kKZ + 2; ++m) v[m] = val(q.c0 + (int)G.pxy * map_any(q.k0 - 1 + m, G.nz, bc.perz));
}
static inline dim3 colgrid(const Geo& g) { return dim3((g.nx + 31) / 32, (g.ny + 7) / 8, (g.nz + kKZ - 1) / kKZ); }

// stored faces: sx[c] is the face between cells c-1 and c (the cell's minus face)
struct OpStored {
    const float *sx, *sy, *sz, *idg;
    struct ColState {};
    __device__ __forceinline__ ColState col(const Geo&, const BC&, const Col&) const { return {}; }
    __device__ __forceinline__ Faces at(const Geo& G, const Col&, const ColState&, int, int c) const {
        return Faces{sx[c], sx[c + 1], sy[c], sy[c + G.px], sz[c], sz[c + (int)G.pxy]};
    }
    __device__ __forceinline__ Faces cell(const Geo& G, int, int, int, int c) const {
        return Faces{sx[c], sx[c + 1], sy[c], sy[c + G.px], sz[c], sz[c + (int)G.pxy]};
    }
    __device__ __forceinline__ float inv_diag(int c) const { return idg[c]; }
};

// c2/(rho_a + rho_b) with the hardware reciprocal (2 ulp): the preconditioner's operator only
// has to be the same everywhere it is formed, and this is the one formula used for it
__device__ __forceinline__ float face_div(float c2, float rsum) { return __fdividef(c2, rsum); }

// faces from the FP32 density (level 0); c2[0..2] = 2 dt/dx^2, 2 dt/dy^2, 2 dt/dz^2 in device
// memory (dt changes per RK stage while the captured graphs stay the same)
struct OpRho {
    const float *rho, *idg, *c2;
    struct ColState {
        float r[kKZ + 2];
        float cx2, cy2, cz2;
    };
    __device__ __forceinline__ ColState col(const Geo& G, const BC& bc, const Col& q) const {
        ColState s;
        load_col(G, bc, q, [&](int cc) { return rho[cc]; }, s.r);
        s.cx2 = c2[0]; s.cy2 = c2[1]; s.cz2 = c2[2];
        return s;
    }
    __device__ __forceinline__ Faces make(const Geo& G, int i, int j, int c, float rc, float rzm, float rzp, float cx2,
                                          float cy2, float cz2) const {
        const int px = G.px;
        const float rxm = rho[(i > 1) ? c - 1 : c + 1], rxp = rho[(i < G.nx) ? c + 1 : c - 1];
        const float rym = rho[(j > 1) ? c - px : c + px], ryp = rho[(j < G.ny) ? c + px : c - px];
        return Faces{face_div(cx2, rc + rxm), face_div(cx2, rc + rxp), face_div(cy2, rc + rym),
                     face_div(cy2, rc + ryp), face_div(cz2, rc + rzm), face_div(cz2, rc + rzp)};
    }
    __device__ __forceinline__ Faces at(const Geo& G, const Col& q, const ColState& s, int m, int c) const {
        const int k = q.k0 + m;
        const float rzm = (k > 1) ? s.r[m] : s.r[m + 2];
        const float rzp = (k < G.nz) ? s.r[m + 2] : s.r[m];
        return make(G, q.i, q.j, c, s.r[m + 1], rzm, rzp, s.cx2, s.cy2, s.cz2);
    }
    __device__ __forceinline__ Faces cell(const Geo& G, int i, int j, int k, int c) const {
        const int pxy = (int)G.pxy;
        const float rzm = rho[(k > 1) ? c - pxy : c + pxy], rzp = rho[(k < G.nz) ? c + pxy : c - pxy];
        return make(G, i, j, c, rho[c], rzm, rzp, c2[0], c2[1], c2[2]);
    }
    __device__ __forceinline__ float inv_diag(int c) const { return idg[c]; }
};

// face conductance of the level-0 operator between two cells (FP32, the formula OpRho uses)
__device__ __forceinline__ float face_rho(float c2, double ra, double rb) {
    return face_div(c2, (float)ra + (float)rb);
}

// ------------------------------------------------------------------------------------
// set-up: FP32 density, the fine faces (for the coarsening) and the inverse diagonal
// ------------------------------------------------------------------------------------
__global__ void k_mx_faces0(Geo G, BC bc, const double* __restrict__ rho, float cx2, float cy2, float cz2,
                            float* rho32, float* sx, float* sy, float* sz, float* idg, float* c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z + 1;
    if (i == 1 && j == 1 && k == 1) { c2[0] = cx2; c2[1] = cy2; c2[2] = cz2; }
    if (i > G.nx || j > G.ny || k > G.nz) return;
    auto fx = [&](int f) { const int fc = clampi_m(f, 2, G.nx); return face_rho(cx2, FI(rho, fc, j, k), FI(rho, fc - 1, j, k)); };
    auto fy = [&](int f) { const int fc = clampi_m(f, 2, G.ny); return face_rho(cy2, FI(rho, i, fc, k), FI(rho, i, fc - 1, k)); };
    auto fz = [&](int f) { const int fc = clampi_m(f, 2, G.nz); return face_rho(cz2, FI(rho, i, j, fc), FI(rho, i, j, fc - 1)); };
    const float xl = fx(i), xh = fx(i + 1), yl = fy(j), yh = fy(j + 1), zl = fz(k), zh = fz(k + 1);
    const long long c = G.idx(i, j, k);
    rho32[c] = (float)rho[c];
    sx[c] = xl; sy[c] = yl; sz[c] = zl;
    if (i == G.nx) FI(sx, i + 1, j, k) = xh;
    if (j == G.ny) FI(sy, i, j + 1, k) = yh;
    if (k == G.nz) FI(sz, i, j, k + 1) = zh;
    float d = 0.f;
    if (i > 1 || bc.perx) d += xl;
    if (i < G.nx || bc.perx) d += xh;
    if (j > 1 || bc.pery) d += yl;
    if (j < G.ny || bc.pery) d += yh;
    if (k > 1 || bc.perz) d += zl;
    if (k < G.nz || bc.perz) d += zh;
    idg[c] = 1.f / (d > 0.f ? d : 1.f);
}

// Galerkin coarse faces: (sum of the 4 fine faces covering a coarse face) / 8
__global__ void k_mg_coarsen(Geo Gf, Geo Gc, BC bc, const float* __restrict__ fx, const float* __restrict__ fy,
                             const float* __restrict__ fz, float* cxs, float* cys, float* czs, float* idg) {
    const int I = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int J = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int K = blockIdx.z + 1;
    if (I > Gc.nx || J > Gc.ny || K > Gc.nz) return;
    auto sumx = [&](int F) {   // coarse x-face F <-> fine x-face 2F-1
        const int f = 2 * F - 1;
        return fx[Gf.idx(f, 2 * J - 1, 2 * K - 1)] + fx[Gf.idx(f, 2 * J, 2 * K - 1)] + fx[Gf.idx(f, 2 * J - 1, 2 * K)] +
               fx[Gf.idx(f, 2 * J, 2 * K)];
    };
    auto sumy = [&](int F) {
        const int f = 2 * F - 1;
        return fy[Gf.idx(2 * I - 1, f, 2 * K - 1)] + fy[Gf.idx(2 * I, f, 2 * K - 1)] + fy[Gf.idx(2 * I - 1, f, 2 * K)] +
               fy[Gf.idx(2 * I, f, 2 * K)];
    };
    auto sumz = [&](int F) {
        const int f = 2 * F - 1;
        return fz[Gf.idx(2 * I - 1, 2 * J - 1, f)] + fz[Gf.idx(2 * I, 2 * J - 1, f)] + fz[Gf.idx(2 * I - 1, 2 * J, f)] +
               fz[Gf.idx(2 * I, 2 * J, f)];
    };
    const float xl = 0.125f * sumx(I), xh = 0.125f * sumx(I + 1);
    const float yl = 0.125f * sumy(J), yh = 0.125f * sumy(J + 1);
    const float zl = 0.125f * sumz(K), zh = 0.125f * sumz(K + 1);
    const long long c = Gc.idx(I, J, K);
    cxs[c] = xl; cys[c] = yl; czs[c] = zl;
    if (I == Gc.nx) cxs[Gc.idx(I + 1, J, K)] = xh;
    if (J == Gc.ny) cys[Gc.idx(I, J + 1, K)] = yh;
    if (K == Gc.nz) czs[Gc.idx(I, J, K + 1)] = zh;
    float d = 0.f;
    if (I > 1 || bc.perx) d += xl;
    if (I < Gc.nx || bc.perx) d += xh;
    if (J > 1 || bc.pery) d += yl;
    if (J < Gc.ny || bc.pery) d += yh;
    if (K > 1 || bc.perz) d += zl;
    if (K < Gc.nz || bc.perz) d += zh;
    idg[c] = 1.f / (d > 0.f ? d : 1.f);
}

// ------------------------------------------------------------------------------------
// V-cycle kernels (all return at once when the inner solve has finished)
// ------------------------------------------------------------------------------------
__device__ __forceinline__ float apply_faces(const Faces& F, float xc, float xm, float xp, float ym, float yp, float zm,
                                             float zp) {
    return F.xm * (xc - xm) + F.xp * (xc - xp) + F.ym * (xc - ym) + F.yp * (xc - yp) + F.zm * (xc - zm) +
           F.zp * (xc - zp);
}

// two damped Jacobi sweeps from zero in one pass: x1 = w f/dg, y = x1 + w (f - A x1)/dg
template <class Op>
__global__ void __launch_bounds__(256) k_mg_pre(Geo G, BC bc, const float* __restrict__ f, Op A,
                                                float* __restrict__ y, float omega, float omega2,
                                                const PCGState* st) {
    pdl_wait();
    if (st->done) return;
    const Col q = column(G, bc);
    if (!q.in) return;
    const int pxy = (int)G.pxy;
    auto x1 = [&](int cc) { return omega * f[cc] * A.inv_diag(cc); };
    float col[kKZ + 2];
    load_col(G, bc, q, x1, col);
    const typename Op::ColState cs = A.col(G, bc, q);
#pragma unroll
    for (int m = 0; m < kKZ; ++m) {
        if (q.k0 + m > G.nz) break;
        const int c = q.c0 + pxy * (q.k0 + m);
        const float xc = col[m + 1];
        const Faces F = A.at(G, q, cs, m, c);
        const float ax = apply_faces(F, xc, x1(c + q.o.xm), x1(c + q.o.xp), x1(c + q.o.ym), x1(c + q.o.yp), col[m],
                                     col[m + 2]);
        y[c] = xc + omega2 * (f[c] - ax) * A.inv_diag(c);
    }
}

// x_out = x_in + w (f - A x_in)/dg; with do_dot (last sweep of level 0) also f.x_out -> rz, beta
template <class Op>
__global__ void __launch_bounds__(256) k_mg_jacc(Geo G, BC bc, const float* __restrict__ xin, const float* __restrict__ f,
                                                 Op A, float* __restrict__ xout, float omega, PCGState* st, int do_dot,
                                                 double* partial, unsigned int* counter) {
    pdl_wait();
    if (st->done) return;
    const Col q = column(G, bc);
    double dot = 0.;
    if (q.in) {
        const int pxy = (int)G.pxy;
        float col[kKZ + 2];
        load_col(G, bc, q, [&](int cc) { return xin[cc]; }, col);
        const typename Op::ColState cs = A.col(G, bc, q);
#pragma unroll
        for (int m = 0; m < kKZ; ++m) {
            if (q.k0 + m > G.nz) break;
            const int c = q.c0 + pxy * (q.k0 + m);
            const float xc = col[m + 1];
            const Faces F = A.at(G, q, cs, m, c);
            const float ax = apply_faces(F, xc, xin[c + q.o.xm], xin[c + q.o.xp], xin[c + q.o.ym], xin[c + q.o.yp],
                                         col[m], col[m + 2]);
            const float fv = f[c];
            const float v = xc + omega * (fv - ax) * A.inv_diag(c);
            xout[c] = v;
            dot += (double)fv * (double)v;
        }
    }
    if (do_dot) {
        double t, u;
        if (reduce2_last(dot, 0.0, partial, counter, t, u) && flat_tid() == 0) {
            const double rz_old = st->rz;
            st->rz = t;
            st->beta = (st->iters == 0) ? 0.0 : t / rz_old;
            if (!isfinite(t)) { st->status = SULI_ERR_NAN; st->done = 1; }
        }
    }
}

// x_out = x' + w (f - A x')/dg with x' = y + a P xc (piecewise-constant prolongation, the
// coarse correction scaled by a)
template <class Op>
__global__ void __launch_bounds__(256) k_mg_post(Geo Gf, Geo Gc, BC bc, const float* __restrict__ y,
                                                 const float* __restrict__ xc, const float* __restrict__ f, Op A,
                                                 float* __restrict__ xout, float omega, float alpha,
                                                 const PCGState* st) {
    pdl_wait();
    if (st->done) return;
    const Col q = column(Gf, bc);
    if (!q.in) return;
    const int pxy = (int)Gf.pxy;
    // parents: coarse (I,J) of this column and of its x/y neighbours (ghost-mapped)
    const int ixm = map_any(q.i - 1, Gf.nx, bc.perx), ixp = map_any(q.i + 1, Gf.nx, bc.perx);
    const int jym = map_any(q.j - 1, Gf.ny, bc.pery), jyp = map_any(q.j + 1, Gf.ny, bc.pery);
    const int I = (q.i + 1) >> 1, J = (q.j + 1) >> 1;
    auto par = [&](int ii, int jj, int kk) { return alpha * xc[Gc.idx((ii + 1) >> 1, (jj + 1) >> 1, (kk + 1) >> 1)]; };
    float col[kKZ + 2];
#pragma unroll
    for (int m = 0; m < kKZ + 2; ++m) {
        const int k = map_any(q.k0 - 1 + m, Gf.nz, bc.perz);
        col[m] = y[q.c0 + pxy * k] + alpha * xc[Gc.idx(I, J, (k + 1) >> 1)];
    }
    const typename Op::ColState cs = A.col(Gf, bc, q);
#pragma unroll
    for (int m = 0; m < kKZ; ++m) {
        const int k = q.k0 + m;
        if (k > Gf.nz) break;
        const int c = q.c0 + pxy * k;
        const float xv = col[m + 1];
        const Faces F = A.at(Gf, q, cs, m, c);
        const float ax = apply_faces(F, xv, y[c + q.o.xm] + par(ixm, q.j, k), y[c + q.o.xp] + par(ixp, q.j, k),
                                     y[c + q.o.ym] + par(q.i, jym, k), y[c + q.o.yp] + par(q.i, jyp, k), col[m],
                                     col[m + 2]);
        xout[c] = xv + omega * (f[c] - ax) * A.inv_diag(c);
    }
}

// x_out = x_in + omega (f - A x_in)/dg; optionally (level 0, last sweep) the dot f.x_out -> rz, beta
__global__ void __launch_bounds__(256) k_mg_jac(Geo G, BC bc, const float* __restrict__ xin, const float* __restrict__ f,
                                                OpStored A, float* __restrict__ xout, float omega, PCGState* st,
                                                int do_dot, double* partial, unsigned int* counter) {
    pdl_wait();
    if (st->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z + 1;
    double dot = 0.;
    if (i <= G.nx && j <= G.ny && k <= G.nz) {
        const int c = (int)G.idx(i, j, k);
        const Nb o = neighbours(G, bc, i, j, k);
        const Faces F = A.cell(G, i, j, k, c);
        const float xc = xin[c];
        const float ax = apply_faces(F, xc, xin[c + o.xm], xin[c + o.xp], xin[c + o.ym], xin[c + o.yp], xin[c + o.zm],
                                     xin[c + o.zp]);
        const float fv = f[c];
        const float v = xc + omega * (fv - ax) * A.inv_diag(c);
        xout[c] = v;
        dot = (double)fv * (double)v;
    }
    if (do_dot) {
        double t, u;
        if (reduce2_last(dot, 0.0, partial, counter, t, u) && flat_tid() == 0) {
            const double rz_old = st->rz;
            st->rz = t;
            st->beta = (st->iters == 0) ? 0.0 : t / rz_old;
            if (!isfinite(t)) { st->status = SULI_ERR_NAN; st->done = 1; }
        }
    }
}

// f_c = (1/8) sum over the 8 children of (f - A x)
template <class Op>
__global__ void __launch_bounds__(256) k_mg_restrict(Geo Gf, Geo Gc, BC bc, const float* __restrict__ x,
                                                     const float* __restrict__ f, Op A, float* fc, const PCGState* st) {
    pdl_wait();
    if (st->done) return;
    const int I = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int J = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int K = blockIdx.z + 1;
    if (I > Gc.nx || J > Gc.ny || K > Gc.nz) return;
    float s = 0.f;
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy)
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                const int i = 2 * I - 1 + dx, j = 2 * J - 1 + dy, k = 2 * K - 1 + dz;
                const int c = (int)Gf.idx(i, j, k);
                const Nb o = neighbours(Gf, bc, i, j, k);
                const Faces F = A.cell(Gf, i, j, k, c);
                const float xv = x[c];
                s += f[c] - apply_faces(F, xv, x[c + o.xm], x[c + o.xp], x[c + o.ym], x[c + o.yp], x[c + o.zm],
                                        x[c + o.zp]);
            }
    fc[Gc.idx(I, J, K)] = 0.125f * s;
}

// The coarsest solve as a Chebyshev polynomial in the Jacobi-scaled operator D^-1 A, whose
// spectrum lies in [0, 2] (Gershgorin: every row's off-diagonal sum is at most its diagonal):
// targeted at [lo, 2], x_1 = g_0 D^-1 f and x_{m+1} = x_m + d_m with
// d_m = h_m d_{m-1} + g_m D^-1 (f - A x_m) (the three-term Chebyshev recurrence: theta and delta
// the interval's centre and half-width, sigma = theta/delta, rho_0 = 1/sigma, g_0 = 1/theta,
// rho_m = 1/(2 sigma - rho_{m-1}), h_m = rho_m rho_{m-1}, g_m = 2 rho_m/delta).  The result is
// q(D^-1 A) D^-1 f with q > 0 on (0, 2], a fixed symmetric positive operator as the damped Jacobi
// sweeps are, but it reduces every mode of [lo, 2] by the Chebyshev factor, where Jacobi leaves
// the smooth modes of the coarsest grid almost untouched.  The coefficients depend only on lo and
// the step count, so the host forms them once (in FP64, rounded to FP32) and the kernels read
// them from their parameters; lo = 0 keeps the damped Jacobi sweeps.
// (CoarsePoly is declared with the solver context)
static CoarsePoly coarse_poly(float lo, int steps) {
    CoarsePoly P = {};
    P.lo = lo;
    if (!(lo > 0.f)) return P;
    const double theta = 1. + 0.5 * lo, delta = 1. - 0.5 * lo, sigma = theta / delta;
    double rho = 1. / sigma;
    P.g0 = (float)(1. / theta);
    for (int m = 1; m < steps && m <= kCoarseMaxCheb; ++m) {
        const double r = 1. / (2. * sigma - rho);
        P.h[m - 1] = (float)(r * rho);
        P.g[m - 1] = (float)(2. * r / delta);
        rho = r;
    }
    return P;
}

// coarsest grid (<= 1024 cells): damped Jacobi sweeps or the Chebyshev polynomial (lo > 0) in
// shared memory, one block
__global__ void __launch_bounds__(1024) k_mg_coarsest(Geo G, BC bc, const float* __restrict__ f, OpStored A,
                                                      float* y, int sweeps, float omega,
                                                      const __grid_constant__ CoarsePoly cp, const PCGState* st) {
    pdl_wait();
    if (st->done) return;
    __shared__ float xs[2][1024];
    const int n = G.nx * G.ny * G.nz;
    const int t = threadIdx.x;
    int c = 0;
    float fv = 0.f, idgv = 1.f, s[6] = {0, 0, 0, 0, 0, 0};
    int nb[6] = {0, 0, 0, 0, 0, 0};
    if (t < n) {
        const int i = t % G.nx + 1, j = (t / G.nx) % G.ny + 1, k = t / (G.nx * G.ny) + 1;
        c = (int)G.idx(i, j, k);
        fv = f[c]; idgv = A.inv_diag(c);
        const Faces F = A.cell(G, i, j, k, c);
        s[0] = F.xm; s[1] = F.xp; s[2] = F.ym; s[3] = F.yp; s[4] = F.zm; s[5] = F.zp;
        const int im = (i > 1) ? i - 1 : (bc.perx ? G.nx : i), ip = (i < G.nx) ? i + 1 : (bc.perx ? 1 : i);
        const int jm = (j > 1) ? j - 1 : (bc.pery ? G.ny : j), jp = (j < G.ny) ? j + 1 : (bc.pery ? 1 : j);
        const int km = (k > 1) ? k - 1 : (bc.perz ? G.nz : k), kp = (k < G.nz) ? k + 1 : (bc.perz ? 1 : k);
        auto lin = [&](int a, int b, int d) { return (a - 1) + G.nx * ((b - 1) + G.ny * (d - 1)); };
        nb[0] = lin(im, j, k); nb[1] = lin(ip, j, k); nb[2] = lin(i, jm, k); nb[3] = lin(i, jp, k); nb[4] = lin(i, j, km); nb[5] = lin(i, j, kp);
    }
    int cur = 0;
    if (cp.lo > 0.f) {
        float d = 0.f;
        if (t < n) {
            d = cp.g0 * fv * idgv;
            xs[0][t] = d;
        }
        __syncthreads();
        for (int sw = 1; sw < sweeps; ++sw) {
            const float h = cp.h[sw - 1], g = cp.g[sw - 1];
            if (t < n) {
                const float xc = xs[cur][t];
                float ax = 0.f;
#pragma unroll
                for (int m = 0; m < 6; ++m) ax += s[m] * (xc - xs[cur][nb[m]]);
                d = h * d + g * (fv - ax) * idgv;
                xs[cur ^ 1][t] = xc + d;
            }
            __syncthreads();
            cur ^= 1;
        }
        if (t < n) y[c] = xs[cur][t];
        return;
    }
    if (t < n) xs[0][t] = omega * fv * idgv;
    __syncthreads();
    for (int sw = 1; sw < sweeps; ++sw) {
        if (t < n) {
            const float xc = xs[cur][t];
            float ax = 0.f;
#pragma unroll
            for (int m = 0; m < 6; ++m) ax += s[m] * (xc - xs[cur][nb[m]]);
            xs[cur ^ 1][t] = xc + omega * (fv - ax) * idgv;
        }
        __syncthreads();
        cur ^= 1;
    }
    if (t < n) y[c] = xs[cur][t];
}

// ------------------------------------------------------------------------------------
// inner PCG on A (FP32 vectors, FP64 reductions)
// ------------------------------------------------------------------------------------
// p = z + beta p_old (also at the neighbours), q = A p, p.q -> alpha
template <class Op>
__global__ void __launch_bounds__(256) k_pcg_spmvc(Geo G, BC bc, const float* __restrict__ z,
                                                   const float* __restrict__ p_old, float* __restrict__ p_new,
                                                   float* __restrict__ q, Op A, PCGState* st, double* partial,
                                                   unsigned int* counter) {
    pdl_wait();
    if (st->done) return;
    const float beta = (float)st->beta;
    const Col cq = column(G, bc);
    double dot = 0.;
    if (cq.in) {
        const int pxy = (int)G.pxy;
        auto pn = [&](int cc) { return z[cc] + beta * p_old[cc]; };
        float col[kKZ + 2];
        load_col(G, bc, cq, pn, col);
        const typename Op::ColState cs = A.col(G, bc, cq);
#pragma unroll
        for (int m = 0; m < kKZ; ++m) {
            if (cq.k0 + m > G.nz) break;
            const int c = cq.c0 + pxy * (cq.k0 + m);
            const float pc = col[m + 1];
            const Faces F = A.at(G, cq, cs, m, c);
            const float qv = apply_faces(F, pc, pn(c + cq.o.xm), pn(c + cq.o.xp), pn(c + cq.o.ym), pn(c + cq.o.yp),
                                         col[m], col[m + 2]);
            p_new[c] = pc;
            q[c] = qv;
            dot += (double)pc * (double)qv;
        }
    }
    double t, u;
    if (reduce2_last(dot, 0.0, partial, counter, t, u) && flat_tid() == 0) {
        st->pq = t;
        st->alpha = st->rz / t;
        if (!isfinite(st->alpha)) { st->status = SULI_ERR_NAN; st->done = 1; }
    }
}

constexpr int kKZU = 8;
__global__ void __launch_bounds__(256) k_pcg_updc(Geo G, float* __restrict__ x, const float* __restrict__ r,
                                                  float* __restrict__ r_out, const float* __restrict__ p,
                                                  const float* __restrict__ q, PCGState* st, double* partial,
                                                  unsigned int* counter, int x_zero) {
    pdl_wait();
    if (st->done) return;
    const float alpha = (float)st->alpha;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k0 = blockIdx.z * kKZU + 1;
    double rr = 0.;
    if (i <= G.nx && j <= G.ny) {
        const int c0 = kBase + (i - 1) + G.px * j, pxy = (int)G.pxy;
        const int k1 = min(k0 + kKZU - 1, G.nz);
        for (int k = k0; k <= k1; ++k) {
            const int c = c0 + pxy * k;
            x[c] = (x_zero ? 0.f : x[c]) + alpha * p[c];
            const float rv = r[c] - alpha * q[c];
            r_out[c] = rv;
            rr += (double)rv * (double)rv;
        }
    }
    double t, u;
    if (reduce2_last(rr, 0.0, partial, counter, t, u) && flat_tid() == 0) {
        st->rr = t;
        st->iters = st->iters + 1;
        bool go = t > st->tol2;
        if (st->iters >= st->maxit) go = false;
        if (!isfinite(t)) { go = false; st->status = SULI_ERR_NAN; }
        st->done = go ? 0 : 1;
    }
}

// ------------------------------------------------------------------------------------
// FP64 refinement: e <- e - sqrt(d) dp, r~ = A~ e - b~, r_u = sqrt(d) r~ (FP32); sqrt(d) is the
// set-up's stored value (sd)
// ------------------------------------------------------------------------------------
// Block partials of the refinement residual: r~.r~, r_u.r_u and max |r_u| (r_u = sqrt(d) r~ is the
// divergence the projection would leave).  The last block sets the stopping test: r~.r~ within
// the threshold and, with div_tol > 0, max |r_u| within div_tol.
__device__ __forceinline__ void mx_outer_finish(double rr, double ru2, double um, int apply, CGState* cg,
                                                PCGState* pst, double* partial, unsigned int* counter) {
    if (isnan(um)) um = INFINITY;
    double t1, t2, tm;
    if (reduce3_last(rr, ru2, um, partial, counter, t1, t2, tm) && flat_tid() == 0) {
        cg->rr = t1;
        cg->rmax = tm;
        if (apply) cg->iters = cg->iters + 1;
        const bool div_ok = !(cg->div_tol > 0.) || tm <= cg->div_tol;
        cg->done = (t1 > cg->thr || !div_ok) ? 0 : 1;
        if (!isfinite(t1)) { cg->status = SULI_ERR_NAN; cg->done = 1; }
        pst->rr0 = t2;
    }
}

__global__ void __launch_bounds__(256) k_mx_outer(Geo G, BC bc, const double* __restrict__ e_in,
                                                  const float* __restrict__ dp, const double* __restrict__ sd,
                                                  const double* __restrict__ ax, const double* __restrict__ ay,
                                                  const double* __restrict__ az, const double* __restrict__ b,
                                                  double* __restrict__ e_out, float* __restrict__ ru, int apply,
                                                  CGState* cg, PCGState* pst, double* partial, unsigned int* counter,
                                                  double* __restrict__ r_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k = blockIdx.z + 1;
    double rr = 0., ru2 = 0., um = 0.;
    if (i <= G.nx && j <= G.ny && k <= G.nz) {
        const int c = (int)G.idx(i, j, k);
        const Nb o = neighbours(G, bc, i, j, k);
        auto en = [&](int cc) { return apply ? e_in[cc] - sd[cc] * (double)dp[cc] : e_in[cc]; };
        const double ec = en(c);
        const double rv = ec - ax[c + 1] * en(c + o.xp) - ax[c] * en(c + o.xm) - ay[c + G.px] * en(c + o.yp) -
                          ay[c] * en(c + o.ym) - az[c + (int)G.pxy] * en(c + o.zp) - az[c] * en(c + o.zm) - b[c];
        e_out[c] = ec;
        if (r_out) r_out[c] = rv;
        const double u = sd[c] * rv;
        ru[c] = (float)u;
        rr = rv * rv;
        ru2 = u * u;
        um = fabs(u);
    }
    mx_outer_finish(rr, ru2, um, apply, cg, pst, partial, counter);
}

// k_mx_outer with two x cells a thread (16-byte row loads; needs nx even) and kOuterZ planes of
// their column (loads from clamped planes, so that the planes' loads are issued together; stores
// and sums only inside the grid): per cell the same expressions, only the two reductions group
// their terms differently.  A quarter of the blocks of one plane a thread; measured at
// 256x128x128 one, two (at 64 registers) and four planes a thread run alike (latency-bound, about
// 80 us a launch).
constexpr int kOuterZ = 4;
__global__ void __launch_bounds__(256) k_mx_outer2(Geo G, BC bc, const double* __restrict__ e_in,
                                                   const float* __restrict__ dp, const double* __restrict__ sd,
                                                   const double* __restrict__ ax, const double* __restrict__ ay,
                                                   const double* __restrict__ az, const double* __restrict__ b,
                                                   double* __restrict__ e_out, float* __restrict__ ru, int apply,
                                                   CGState* cg, PCGState* pst, double* partial, unsigned int* counter,
                                                   double* __restrict__ r_out) {
    const int i0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k0 = blockIdx.z * kOuterZ + 1;
    double rr = 0., ru2 = 0., um = 0.;
    if (i0 <= G.nx && j <= G.ny && k0 <= G.nz) {
        const int px = G.px, pxy = (int)G.pxy;
        auto en = [&](int cc) { return apply ? e_in[cc] - sd[cc] * (double)dp[cc] : e_in[cc]; };
        auto en2 = [&](int cc) {
            const double2 e = *reinterpret_cast<const double2*>(e_in + cc);
            if (!apply) return e;
            const double2 s2 = *reinterpret_cast<const double2*>(sd + cc);
            const float2 d2 = *reinterpret_cast<const float2*>(dp + cc);
            return make_double2(e.x - s2.x * (double)d2.x, e.y - s2.y * (double)d2.y);
        };
        auto ld2 = [](const double* a, int cc) { return *reinterpret_cast<const double2*>(a + cc); };
        // the column's corrected e below, at and above the plane: after the first plane the values
        // at and below are the previous plane's above and at (planes past nz are not stored)
        double2 ec = make_double2(0., 0.), ezp = make_double2(0., 0.);
#pragma unroll
        for (int q = 0; q < kOuterZ; ++q) {
            const int k = min(k0 + q, G.nz);
            const int c = (int)G.idx(i0, j, k);
            const Nb o0 = neighbours(G, bc, i0, j, k), o1 = neighbours(G, bc, i0 + 1, j, k);
            double2 ezm;
            if (q == 0) {
                ec = en2(c);
                ezm = en2(c + o0.zm);
            } else {
                ezm = ec;
                ec = ezp;
            }
            ezp = en2(c + o0.zp);
            const double2 eym = en2(c + o0.ym), eyp = en2(c + o0.yp);
            const double exm = en(c + o0.xm), exp_ = en(c + 1 + o1.xp);
            const double2 axc = ld2(ax, c), ayc = ld2(ay, c), ayp = ld2(ay, c + px), azc = ld2(az, c),
                          azp = ld2(az, c + pxy), bc2 = ld2(b, c), sdc = ld2(sd, c);
            const double ax2 = ax[c + 2];
            const double r0 = ec.x - axc.y * ec.y - axc.x * exm - ayp.x * eyp.x - ayc.x * eym.x - azp.x * ezp.x -
                              azc.x * ezm.x - bc2.x;
            const double r1 = ec.y - ax2 * exp_ - axc.y * ec.x - ayp.y * eyp.y - ayc.y * eym.y - azp.y * ezp.y -
                              azc.y * ezm.y - bc2.y;
            if (k0 + q <= G.nz) {
                *reinterpret_cast<double2*>(e_out + c) = ec;
                if (r_out) *reinterpret_cast<double2*>(r_out + c) = make_double2(r0, r1);
                const double u0 = sdc.x * r0, u1 = sdc.y * r1;
                *reinterpret_cast<float2*>(ru + c) = make_float2((float)u0, (float)u1);
                rr += r0 * r0 + r1 * r1;
                ru2 += u0 * u0 + u1 * u1;
                um = fmax(um, fmax(fabs(u0), fabs(u1)));
            }
        }
    }
    mx_outer_finish(rr, ru2, um, apply, cg, pst, partial, counter);
}

__global__ void k_pcg_init(PCGState* st, double inner_tol, int maxit) {
    st->tol2 = inner_tol * inner_tol * st->rr0;
    st->iters = 0;
    st->done = 0;
    st->status = 0;
    st->maxit = maxit;
    st->beta = 0.;
    st->rz = 0.;
}

__global__ void k_pcg_cond(cudaGraphConditionalHandle h, const PCGState* st) {
    pdl_wait();
    cudaGraphSetConditional(h, st->done ? 0u : 1u);
}

__global__ void k_zero_f(float* a, long long n) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) a[q] = 0.f;
}

}  // namespace suli
#include "k_mg_vec.cuh"
#include "k_mg_fused.cuh"
#include "k_mg_cluster.cuh"
#include "k_mg_stream.cuh"
#include "k_mg_tail.cuh"
namespace suli {

// ------------------------------------------------------------------------------------
// launchers
// ------------------------------------------------------------------------------------
static const dim3 kB2(32, 8, 1);

static inline dim3 cells3(const Geo& g) { return dim3((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz); }
static inline OpStored stored(const MGLevel& L) { return OpStored{L.sx, L.sy, L.sz, L.idg}; }
static inline OpRho from_rho(const MGLevel& L) { return OpRho{L.rho, L.idg, L.c2}; }

void launch_mx_setup(suli_ctx* c) {
    ProfScope ps(c, SULI_K_CG_SETUP, (int)c->mg.size());
    MGLevel& L0 = c->mg[0];
    const float cx2 = (float)(2. * c->dt / (c->P.dx * c->P.dx)), cy2 = (float)(2. * c->dt / (c->P.dy * c->P.dy)),
                cz2 = (float)(2. * c->dt / (c->P.dz * c->P.dz));
    k_mx_faces0<<<cells3(L0.g), kB2, 0, c->stream>>>(L0.g, c->bc, c->f[SULI_F_RHO], cx2, cy2, cz2, L0.rho, L0.sx,
                                                     L0.sy, L0.sz, L0.idg, L0.c2);
    for (size_t l = 1; l < c->mg.size(); ++l) {
        MGLevel& F = c->mg[l - 1];
        MGLevel& C = c->mg[l];
        k_mg_coarsen<<<cells3(C.g), kB2, 0, c->stream>>>(F.g, C.g, c->bc, F.sx, F.sy, F.sz, C.sx, C.sy, C.sz, C.idg);
    }
}

// r_u from the FP64 first residual (no correction applied); also initialises the inner solve.
// With the network as the outer iteration's preconditioner (nn_mode 2) the FP64 scaled residual
// is kept as well, in cg_r, for the network's features and step length.
void launch_mx_residual(suli_ctx* c, const double* e_in, double* e_out, bool apply) {
    double* r_out = (c->nn && c->nn_mode == 2 && !c->rec_in) ? c->cg_r : nullptr;
    ProfScope ps(c, SULI_K_REFINE, 1);
    const Geo& G = c->g;
    if (G.nx % 2 == 0) {
        const dim3 g2((G.nx / 2 + 31) / 32, (G.ny + 7) / 8, (G.nz + kOuterZ - 1) / kOuterZ);
        k_mx_outer2<<<g2, kB2, 0, c->stream>>>(G, c->bc, e_in, c->pc_x, c->cg_sd, c->cg_ax, c->cg_ay, c->cg_az,
                                               c->cg_b, e_out, c->pc_r, apply ? 1 : 0, c->cg, c->pcg,
                                               c->red_partial, c->red_counter, r_out);
    } else {
        k_mx_outer<<<cells3(G), kB2, 0, c->stream>>>(G, c->bc, e_in, c->pc_x, c->cg_sd, c->cg_ax, c->cg_ay, c->cg_az,
                                                     c->cg_b, e_out, c->pc_r, apply ? 1 : 0, c->cg, c->pcg,
                                                     c->red_partial, c->red_counter, r_out);
    }
}

void launch_pcg_cond(suli_ctx* c, cudaGraphConditionalHandle h) { pdl_launch(k_pcg_cond, 1, 1, c->stream, h, c->pcg); }

// The pass's first PCG update writes x = alpha p (launch_pcg_iter with x_zero), so x needs no
// zero fill, except where the update runs inside the pre-smoothing kernel (SULI_FUSED_UPDATE=1).
static bool fused_update(const suli_ctx* c);
void launch_pcg_init(suli_ctx* c, int maxit) {
    k_pcg_init<<<1, 1, 0, c->stream>>>(c->pcg, c->P.inner_tol, maxit);
    if (!fused_update(c)) return;
    const long long n = (long long)c->g.n;
    k_zero_f<<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(c->pc_x, n);
}

static inline OpRho4 from_rho4(const MGLevel& L) { return OpRho4{L.rho, L.idg, L.c2}; }
// launch a column kernel of the vectorised family with the context's column depth (2 or 4)
// (the depth-2 kernels assume an even nz, true of every level that is coarsened further)
#define VLAUNCH(kern, Op, G, ...)                                                                          \
    do {                                                                                                   \
        if (c->mg_kz == 2 && (G).nz % 2 == 0) pdl_launch(kern<2, Op>, vgrid((G), 2), kB2, c->stream, __VA_ARGS__); \
        else pdl_launch(kern<4, Op>, vgrid((G), 4), kB2, c->stream, __VA_ARGS__);                         \
    } while (0)
static inline OpStored4 stored4(const MGLevel& L) { return OpStored4{L.sx, L.sy, L.sz, L.idg}; }
// the 4-cells-a-thread kernels on a level (mg_kernels 0 or 2 and x divisible by 4)
static inline bool vec_level(const suli_ctx* c, const Geo& g) { return c->P.mg_kernels != 1 && g.nx % kVX == 0; }
// the coarse levels 1 .. L-2 run each leg of the V-cycle as one kernel (k_mg_fused.cuh)
static inline bool fused_level(const suli_ctx* c, int l) { return c->mg_fused && l >= 1 && l <= (int)c->mg.size() - 2; }
// where level l leaves its V-cycle result (the coarse correction the level above prolongs):
// the fused up leg writes x, every other path y
static inline const float* mg_corr(const suli_ctx* c, int l) { return fused_level(c, l) ? c->mg[l].x : c->mg[l].y; }

// ---- level-0 kernels streaming z-planes through shared memory (k_mg_stream.cuh)
static PFN_cuTensorMapEncodeTiled_v12000 plane_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    }
    return fn;
}
// a level-0 FP32 array as a 3-D tensor {px, py, nz + 3} (x = kBase + i - 1 within row j of
// plane k), zero fill outside; box {kSBoxX, kSBoxY, 1} (with the halo) or, own = true,
// {kSOBoxX, kSOBoxY, 1} (the tile's own cells)
static bool encode_plane_map(CUtensorMap* m, const Geo& g, const float* a, bool own) {
    auto enc = plane_map_encoder();
    if (!enc || !a || (reinterpret_cast<uintptr_t>(a) & 15)) return false;
    cuuint64_t dims[3] = {(cuuint64_t)g.px, (cuuint64_t)g.py, (cuuint64_t)(g.nz + 3)};
    cuuint64_t strides[2] = {(cuuint64_t)g.px * 4, (cuuint64_t)g.pxy * 4};
    cuuint32_t box[3] = {(cuuint32_t)(own ? kSOBoxX : kSBoxX), (cuuint32_t)(own ? kSOBoxY : kSBoxY), 1};
    cuuint32_t es[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(a), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
static bool add_plane_map(suli_ctx* c, const float* a) {
    if (c->n_smap >= 12) return false;
    const Geo& g = c->mg[0].g;
    if (!encode_plane_map(&c->smap[c->n_smap], g, a, false) || !encode_plane_map(&c->smap_own[c->n_smap], g, a, true))
        return false;
    c->smap_ptr[c->n_smap++] = a;
    return true;
}
// the coarse level-1 correction as the post-smoothing's prolongation source: box {kSCBoxX, kSCBoxY, 1}
static bool set_coarse_map(suli_ctx* c, const float* a) {
    auto enc = plane_map_encoder();
    const Geo& g = c->mg[1].g;
    if (!enc || !a || (reinterpret_cast<uintptr_t>(a) & 15)) return false;
    cuuint64_t dims[3] = {(cuuint64_t)g.px, (cuuint64_t)g.py, (cuuint64_t)(g.nz + 3)};
    cuuint64_t strides[2] = {(cuuint64_t)g.px * 4, (cuuint64_t)g.pxy * 4};
    cuuint32_t box[3] = {(cuuint32_t)kSCBoxX, (cuuint32_t)kSCBoxY, 1};
    cuuint32_t es[3] = {1, 1, 1};
    return enc(&c->smap_c, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(a), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
static const CUtensorMap& plane_map(const suli_ctx* c, const float* a) {
    for (int q = 0; q < c->n_smap; ++q)
        if (c->smap_ptr[q] == a) return c->smap[q];
    return c->smap[0];   // not reached: every array the streaming kernels read has a map
}
static const CUtensorMap& own_map(const suli_ctx* c, const float* a) {
    for (int q = 0; q < c->n_smap; ++q)
        if (c->smap_ptr[q] == a) return c->smap_own[q];
    return c->smap_own[0];
}

// Decide once per context whether level 0 runs the streaming kernels: vectorised kernels on a
// multigrid hierarchy (mg_kernels 0), nx a multiple of 16, no periodic x or y axis, a tensor map
// for every level-0 array they read, and two CTAs' shared memory an SM.  SULI_NO_STREAM=1
// keeps the vectorised level-0 kernels; SULI_STREAM_CHUNK sets the planes a CTA computes.
int stream_ready(suli_ctx* c) {
    c->stream_ok = false;
    c->stream_post_ok = false;
    c->n_smap = 0;
    if (const char* ev = std::getenv("SULI_NO_STREAM"))
        if (std::strcmp(ev, "1") == 0) return SULI_OK;
    if (c->mg.size() < 2 || c->P.mg_kernels != 0) return SULI_OK;
    const Geo& g = c->mg[0].g;
    if (g.nx % 16 != 0 || g.px < g.nx + 16 || c->bc.perx || c->bc.pery) return SULI_OK;
    const MGLevel& M0 = c->mg[0];
    const float* arrays[] = {c->pc_r, c->pc_r2, M0.x, M0.y, c->pc_pa, c->pc_pb, M0.idg, M0.rho};
    for (const float* a : arrays)
        if (!add_plane_map(c, a)) { c->n_smap = 0; return SULI_OK; }
    if (cudaFuncSetAttribute(k_mgs_pre, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stream_smem_bytes(3)) != cudaSuccess ||
        cudaFuncSetAttribute(k_pcgs_spmvc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stream_smem_bytes(3)) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_mgs_jacc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stream_smem_bytes(2, 2)) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_mgs_restrict, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stream_smem_bytes(2, 1)) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_mgs_post, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stream_smem_bytes(2, 2, 1)) !=
            cudaSuccess) {
        cudaGetLastError();
        return SULI_OK;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mgs_post, kSTX * kSTY, stream_smem_bytes(2, 2, 1)) !=
            cudaSuccess ||
        per_sm < 1) {
        cudaGetLastError();
        return SULI_OK;
    }
    // the post-smoothing also needs the level-1 correction's rows to hold its tile's parents
    c->stream_post_ok = (g.nx % 32 == 0) && c->mg[1].g.px >= c->mg[1].g.nx + 16 && set_coarse_map(c, mg_corr(c, 1));
    // planes a CTA computes: as many chunks as fill the SMs' CTA slots once
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
    const int tiles = ((g.nx + kSTileX - 1) / kSTileX) * ((g.ny + kSTY - 1) / kSTY);
    const int chunks = std::max(1, std::min(g.nz, (per_sm * nsm) / std::max(tiles, 1)));
    c->stream_chunk = (g.nz + chunks - 1) / chunks;
    if (const char* ev = std::getenv("SULI_STREAM_CHUNK")) {   // planes a CTA computes, for tests
        const int v = std::atoi(ev);
        if (v >= 1 && v <= g.nz) c->stream_chunk = v;
    }
    c->stream_ok = true;
    return SULI_OK;
}

template <typename... KArgs, typename... Args>
static void stream_launch(suli_ctx* c, void (*kernel)(KArgs...), size_t smem, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = sgrid(c->mg[0].g, c->stream_chunk);
    cfg.blockDim = dim3(kSTX, kSTY, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}
static void launch_stream_pre(suli_ctx* c, const float* f, float om, float om2) {
    const MGLevel& M = c->mg[0];
    stream_launch(c, k_mgs_pre, stream_smem_bytes(3), M.g, c->bc, plane_map(c, f), plane_map(c, M.idg),
                  plane_map(c, M.rho), (const float*)M.c2, M.y, om, om2, c->stream_chunk, c->pcg);
}
static void launch_stream_jacc(suli_ctx* c, const float* f, float om) {
    const MGLevel& M = c->mg[0];
    stream_launch(c, k_mgs_jacc, stream_smem_bytes(2, 2), M.g, c->bc, plane_map(c, M.x), plane_map(c, M.rho),
                  own_map(c, f), own_map(c, M.idg), (const float*)M.c2, M.y, om, c->stream_chunk, c->pcg,
                  c->red_partial, c->red_counter);
}
// the restriction's chunk is even (a coarse plane's two fine planes in one CTA)
static void launch_stream_restrict(suli_ctx* c, const float* f) {
    const MGLevel& M = c->mg[0];
    const MGLevel& C = c->mg[1];
    const int ch = (c->stream_chunk + 1) & ~1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = sgrid(M.g, ch);
    cfg.blockDim = dim3(kSTX, kSTY, 1);
    cfg.dynamicSmemBytes = stream_smem_bytes(2, 1);
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_mgs_restrict, M.g, C.g, c->bc, plane_map(c, M.y), plane_map(c, M.rho), own_map(c, f),
                       (const float*)M.c2, C.f, ch, c->pcg);
}
static void launch_stream_post(suli_ctx* c, const float* f, float om2, float alpha) {
    const MGLevel& M = c->mg[0];
    stream_launch(c, k_mgs_post, stream_smem_bytes(2, 2, 1), M.g, c->bc, plane_map(c, M.y), plane_map(c, M.rho),
                  own_map(c, f), own_map(c, M.idg), c->smap_c, (const float*)M.c2, M.x, om2, alpha, c->stream_chunk,
                  c->pcg);
}
static void launch_stream_spmvc(suli_ctx* c, const float* p_old, float* p_new) {
    const MGLevel& M = c->mg[0];
    stream_launch(c, k_pcgs_spmvc, stream_smem_bytes(3), M.g, c->bc, plane_map(c, M.y), plane_map(c, p_old),
                  plane_map(c, M.rho), (const float*)M.c2, p_new, c->pc_q, c->stream_chunk, c->pcg, c->red_partial,
                  c->red_counter);
}

// pre-smoothing (weights om, then om2) and restriction of level l (level 0 forms its faces from
// the density)
static void vc_down(suli_ctx* c, int l, const float* f, float om, float om2, bool pre_done = false) {
    MGLevel& M = c->mg[l];
    MGLevel& C = c->mg[l + 1];
    const BC bc = c->bc;
    if (fused_level(c, l)) {
        pdl_launch(k_mgf_down, fgrid(M.g), dim3(kFTX, kFTY, 1), c->stream, M.g, C.g, bc, f, stored(M), M.y, C.f, om,
                   om2, c->pcg);
        return;
    }
    if (vec_level(c, M.g)) {
        if (l == 0) {
            if (!pre_done) {
                if (c->stream_ok) launch_stream_pre(c, f, om, om2);
                else VLAUNCH(k_mgv_pre, OpRho4, M.g, M.g, bc, f, from_rho4(M), M.y, om, om2, c->pcg);
            }
            if (c->stream_ok)
                launch_stream_restrict(c, f);
            else
                pdl_launch(k_mgv_restrict<OpRho4>, vgrid_restrict(C.g), kB2, c->stream, M.g, C.g, bc, M.y, f,
                           from_rho4(M), C.f, c->pcg);
        } else {
            VLAUNCH(k_mgv_pre, OpStored4, M.g, M.g, bc, f, stored4(M), M.y, om, om2, c->pcg);
            pdl_launch(k_mgv_restrict<OpStored4>, vgrid_restrict(C.g), kB2, c->stream, M.g, C.g, bc, M.y, f, stored4(M),
                       C.f, c->pcg);
        }
        return;
    }
    if (l == 0) {
        pdl_launch(k_mg_pre<OpRho>, colgrid(M.g), kB2, c->stream, M.g, bc, f, from_rho(M), M.y, om, om2, c->pcg);
        pdl_launch(k_mg_restrict<OpRho>, cells3(C.g), kB2, c->stream, M.g, C.g, bc, M.y, f, from_rho(M), C.f, c->pcg);
    } else {
        pdl_launch(k_mg_pre<OpStored>, colgrid(M.g), kB2, c->stream, M.g, bc, f, stored(M), M.y, om, om2, c->pcg);
        pdl_launch(k_mg_restrict<OpStored>, cells3(C.g), kB2, c->stream, M.g, C.g, bc, M.y, f, stored(M), C.f, c->pcg);
    }
}

// prolongation + post-smoothing of level l (weight om2), then the last sweep (om; level 0: with
// r.z and beta): the pre-smoothing's sweeps in reverse order, so the V-cycle stays symmetric
static void vc_up(suli_ctx* c, int l, const float* f, float om, float om2, float alpha) {
    MGLevel& M = c->mg[l];
    MGLevel& C = c->mg[l + 1];
    const BC bc = c->bc;
    const int dot = (l == 0) ? 1 : 0;
    const float* xc = mg_corr(c, l + 1);
    if (fused_level(c, l)) {
        pdl_launch(k_mgf_up, fgrid(M.g), dim3(kFTX, kFTY, 1), c->stream, M.g, C.g, bc, (const float*)M.y, xc, f,
                   stored(M), M.x, om, om2, alpha, c->pcg);
        return;
    }
    if (vec_level(c, M.g)) {
        if (l == 0) {
            if (c->stream_ok && c->stream_post_ok)
                launch_stream_post(c, f, om2, alpha);
            else
                VLAUNCH(k_mgv_post, OpRho4, M.g, M.g, C.g, bc, M.y, xc, f, from_rho4(M), M.x, om2, alpha, c->pcg);
            if (c->stream_ok) launch_stream_jacc(c, f, om);
            else VLAUNCH(k_mgv_jacc, OpRho4, M.g, M.g, bc, M.x, f, from_rho4(M), M.y, om, c->pcg, dot, c->red_partial,
                         c->red_counter);
        } else {
            VLAUNCH(k_mgv_post, OpStored4, M.g, M.g, C.g, bc, M.y, xc, f, stored4(M), M.x, om2, alpha, c->pcg);
            VLAUNCH(k_mgv_jacc, OpStored4, M.g, M.g, bc, M.x, f, stored4(M), M.y, om, c->pcg, dot, c->red_partial,
                    c->red_counter);
        }
        return;
    }
    if (l == 0) {
        pdl_launch(k_mg_post<OpRho>, colgrid(M.g), kB2, c->stream, M.g, C.g, bc, M.y, xc, f, from_rho(M), M.x, om2,
                   alpha, c->pcg);
        pdl_launch(k_mg_jacc<OpRho>, colgrid(M.g), kB2, c->stream, M.g, bc, M.x, f, from_rho(M), M.y, om, c->pcg, dot,
                   c->red_partial, c->red_counter);
    } else {
        pdl_launch(k_mg_post<OpStored>, colgrid(M.g), kB2, c->stream, M.g, C.g, bc, M.y, xc, f, stored(M), M.x, om2,
                   alpha, c->pcg);
        pdl_launch(k_mg_jacc<OpStored>, colgrid(M.g), kB2, c->stream, M.g, bc, M.x, f, stored(M), M.y, om, c->pcg, dot,
                   c->red_partial, c->red_counter);
    }
}

// The three coarsest levels run as one cluster launch (k_mg_cluster) when selected
// (mg_kernels = 2), their shapes fit it and the device runs a 16-CTA cluster with the kernel's
// shared memory (checked once, cluster_ready).  Measured at 256x128x128 it is slower than the
// per-level kernels it replaces (54 us a launch against about 40 us for the nine kernels), so
// it is not the default.
static bool use_cluster(const suli_ctx* c) {
    const int L = (int)c->mg.size();
    return c->P.mg_kernels == 2 && c->cluster_ok && L >= 4 && vec_level(c, c->mg[L - 4].g) &&
           cl_fits(c->mg[L - 3].g, c->mg[L - 2].g, c->mg[L - 1].g);
}

int cluster_ready(suli_ctx* c) {
    c->cluster_ok = false;
    c->mg_kz = 2;
    if (const char* ev = std::getenv("SULI_MG_KZ"))   // column depth of the vectorised kernels
        if (std::strcmp(ev, "4") == 0) c->mg_kz = 4;
    // The coarsest solve: by default the Chebyshev polynomial over [0.02, 2] with 20 steps
    // (measured at 256x128x128, both stopping tests: 37.7 inner iterations a step against 45.5
    // for the 40 damped Jacobi sweeps, 12.3 against 13.3 ms a step; 30 or 40 steps give the same
    // iterations, lo = 0.05 gives 39.7 and lo = 0.01 49.3).  SULI_COARSE_CHEB sets lo (0: the
    // damped Jacobi sweeps, 40 of them), SULI_COARSE_SWEEPS the number of steps.
    c->coarse_lo = 0.02f;
    if (const char* ev = std::getenv("SULI_COARSE_CHEB")) {
        const double v = std::atof(ev);
        if (v >= 0. && v < 1.) c->coarse_lo = (float)v;
    }
    c->coarse_sweeps = (c->coarse_lo > 0.f) ? 20 : 40;
    if (const char* ev = std::getenv("SULI_COARSE_SWEEPS")) {
        const int v = std::atoi(ev);
        if (v >= 2 && v <= 400) c->coarse_sweeps = v;
    }
    if (c->coarse_lo > 0.f) c->coarse_sweeps = std::min(c->coarse_sweeps, kCoarseMaxCheb + 1);
    c->coarse_poly = coarse_poly(c->coarse_lo, c->coarse_sweeps);
    // one kernel a leg on the coarse levels (k_mg_fused.cuh, SULI_MG_FUSED=1) with the vectorised
    // per-level kernels (mg_kernels 0) and no one-CTA tail.  Measured at 256x128x128 it is slower
    // than the four kernels a level it replaces (228 against 172 us an inner iteration: the cells
    // around a tile triple the first stage's work), so it is not the default.
    c->mg_fused = false;
    if (const char* ev = std::getenv("SULI_MG_FUSED"))
        if (std::strcmp(ev, "1") == 0) c->mg_fused = (c->P.mg_kernels == 0);
    if (const char* ev = std::getenv("SULI_TAIL"))
        if (std::strcmp(ev, "1") == 0) c->mg_fused = false;
    c->fuse_update = false;
    if (const char* ev = std::getenv("SULI_FUSED_UPDATE"))   // the PCG update inside the pre-smoothing
        if (std::strcmp(ev, "1") == 0) c->fuse_update = true;
    if (const char* ev = std::getenv("SULI_NO_CLUSTER"))   // keep the per-level kernels
        if (std::strcmp(ev, "1") == 0) return SULI_OK;
    const int L = (int)c->mg.size();
    if (L < 4 || !cl_fits(c->mg[L - 3].g, c->mg[L - 2].g, c->mg[L - 1].g)) return SULI_OK;
    const size_t smem = cl_smem_bytes(c->mg[L - 3].g, c->mg[L - 2].g, c->mg[L - 1].g);
    if (cudaFuncSetAttribute(k_mg_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaFuncSetAttribute(k_mg_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return SULI_OK;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kClCTAs);
    cfg.blockDim = dim3(kClThreads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClCTAs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_mg_cluster, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return SULI_OK;
    }
    c->cluster_ok = (n > 0);
    return SULI_OK;
}

static void launch_cluster(suli_ctx* c, float om, float alpha) {
    const int L = (int)c->mg.size();
    const MGLevel &M = c->mg[L - 3], &C = c->mg[L - 2], &B = c->mg[L - 1];
    ClArgs a;
    a.M = ClLevel{M.g, M.sx, M.sy, M.sz, M.idg};
    a.C = ClLevel{C.g, C.sx, C.sy, C.sz, C.idg};
    a.B = ClLevel{B.g, B.sx, B.sy, B.sz, B.idg};
    a.bc = c->bc;
    a.fM = M.f;
    a.yM = M.y;
    a.omega = om;
    a.omega2 = (float)c->P.mg_omega2;
    a.alpha = alpha;
    a.sweeps = c->coarse_sweeps;
    a.cp = c->coarse_poly;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(kClCTAs);
    cfg.blockDim = dim3(kClThreads);
    cfg.dynamicSmemBytes = cl_smem_bytes(M.g, C.g, B.g);
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClCTAs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 2;
    cudaLaunchKernelEx(&cfg, k_mg_cluster, a, (const PCGState*)c->pcg);
}

// The last level above the coarsest and the coarsest solve as one CTA (k_mg_tail), selected by
// SULI_TAIL=1, when the vectorised per-level kernels are selected (mg_kernels 0), there are at
// least three levels, the two fit it, and the device grants its shared memory (checked once,
// tail_ready).  Measured at 256x128x128 it is slower than the five launches it replaces (192
// against 168 us an inner iteration: one SM works through 8192 cells a phase), so it is not
// the default.
static bool use_tail(const suli_ctx* c) {
    const int L = (int)c->mg.size();
    if (!c->tail_ok || c->P.mg_kernels != 0 || L < 3) return false;
    const Geo &M = c->mg[L - 2].g, &B = c->mg[L - 1].g;
    return (long long)M.nx * M.ny * M.nz <= kTailM && (long long)B.nx * B.ny * B.nz <= 1024;
}
int tail_ready(suli_ctx* c) {
    c->tail_ok = false;
    const char* ev = std::getenv("SULI_TAIL");
    if (!ev || std::strcmp(ev, "1") != 0) return SULI_OK;
    if (cudaFuncSetAttribute(k_mg_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tail_smem_bytes()) !=
        cudaSuccess) {
        cudaGetLastError();
        return SULI_OK;
    }
    c->tail_ok = true;
    return SULI_OK;
}
static void launch_tail(suli_ctx* c, float om, float om2, float alpha) {
    const int L = (int)c->mg.size();
    const MGLevel &M = c->mg[L - 2], &B = c->mg[L - 1];
    TailArgs a;
    a.gm = M.g;
    a.gb = B.g;
    a.am = stored(M);
    a.ab = stored(B);
    a.fm = M.f;
    a.ym = M.y;
    a.omega = om;
    a.omega2 = om2;
    a.alpha = alpha;
    a.sweeps = c->coarse_sweeps;
    a.cp = c->coarse_poly;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(1);
    cfg.blockDim = dim3(kTailThreads);
    cfg.dynamicSmemBytes = tail_smem_bytes();
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, k_mg_tail, a, c->bc, (const PCGState*)c->pcg);
}

// z = M r for the level-0 right-hand side f0: one V-cycle; the last level-0 sweep also forms r.z
// and beta.  pre_done: the level-0 pre-smoothing already ran (fused with the PCG update).
void launch_vcycle(suli_ctx* c, const float* f0, bool pre_done) {
    const float om = (float)c->P.mg_omega;
    const float om2 = (float)c->P.mg_omega2;
    const float alpha = (float)c->P.mg_alpha;
    const int L = (int)c->mg.size();
    const BC bc = c->bc;
    if (use_cluster(c)) {   // levels 0 .. L-4 as kernels per level, the last three in the cluster
        for (int l = 0; l < L - 3; ++l) vc_down(c, l, l == 0 ? f0 : c->mg[l].f, om, om2, pre_done);
        launch_cluster(c, om, alpha);
        for (int l = L - 4; l >= 0; --l) vc_up(c, l, l == 0 ? f0 : c->mg[l].f, om, om2, alpha);
        return;
    }
    if (use_tail(c)) {   // levels 0 .. L-3 as kernels per level, the last two in one CTA
        for (int l = 0; l < L - 2; ++l) vc_down(c, l, l == 0 ? f0 : c->mg[l].f, om, om2, pre_done);
        launch_tail(c, om, om2, alpha);
        for (int l = L - 3; l >= 0; --l) vc_up(c, l, l == 0 ? f0 : c->mg[l].f, om, om2, alpha);
        return;
    }
    for (int l = 0; l < L - 1; ++l) vc_down(c, l, l == 0 ? f0 : c->mg[l].f, om, om2, pre_done);
    MGLevel& B = c->mg[L - 1];
    if (L == 1) {   // a single level: coarsest sweeps, then one more sweep that forms r.z
        pdl_launch(k_mg_coarsest, 1, 1024, c->stream, B.g, bc, f0, stored(B), B.x, c->coarse_sweeps, om,
                   c->coarse_poly, c->pcg);
        pdl_launch(k_mg_jac, cells3(B.g), kB2, c->stream, B.g, bc, B.x, f0, stored(B), B.y, om, c->pcg, 1,
                   c->red_partial, c->red_counter);
        return;
    }
    pdl_launch(k_mg_coarsest, 1, 1024, c->stream, B.g, bc, B.f, stored(B), B.y, c->coarse_sweeps, om,
               c->coarse_poly, c->pcg);
    for (int l = L - 2; l >= 0; --l) vc_up(c, l, l == 0 ? f0 : c->mg[l].f, om, om2, alpha);
}

// the update fuses into the level-0 pre-smoothing (SULI_FUSED_UPDATE=1) where the level uses
// the vectorised kernels and there is a level below it.  Measured at 256x128x128 the fused
// kernel is slower than the two it replaces (195 against 184 us an inner iteration: it reads r
// and q at the neighbours), so it is not the default.
static bool fused_update(const suli_ctx* c) { return c->fuse_update && c->mg.size() > 1 && vec_level(c, c->g); }

// one inner PCG iteration: p = z + beta p_old, q = A p (p.q -> alpha); x += alpha p,
// r_new = r_old - alpha q (r.r -> stop test); z = M r_new (r.z -> beta)
void launch_pcg_iter(suli_ctx* c, const float* p_old, float* p_new, const float* r_old, float* r_new, bool x_zero) {
    const Geo& G = c->g;
    MGLevel& M0 = c->mg[0];
    const bool vec = vec_level(c, G);
    {
        ProfScope ps(c, SULI_K_CG_SPMV, 1);
        if (c->mg.size() > 1) {
            if (c->stream_ok)
                launch_stream_spmvc(c, p_old, p_new);
            else if (vec)
                VLAUNCH(k_pcgv_spmvc, OpRho4, G, G, c->bc, M0.y, p_old, p_new, c->pc_q, from_rho4(M0), c->pcg,
                        c->red_partial, c->red_counter);
            else
                pdl_launch(k_pcg_spmvc<OpRho>, colgrid(G), kB2, c->stream, G, c->bc, M0.y, p_old, p_new, c->pc_q,
                           from_rho(M0), c->pcg, c->red_partial, c->red_counter);
        } else {
            pdl_launch(k_pcg_spmvc<OpStored>, colgrid(G), kB2, c->stream, G, c->bc, M0.y, p_old, p_new, c->pc_q,
                       stored(M0), c->pcg, c->red_partial, c->red_counter);
        }
    }
    if (fused_update(c)) {
        ProfScope ps(c, SULI_K_MG, vcycle_kernels(c));
        VLAUNCH(k_mgv_preu, OpRho4, G, G, c->bc, c->pc_x, p_new, r_old, c->pc_q, r_new, from_rho4(M0), M0.y,
                (float)c->P.mg_omega, (float)c->P.mg_omega2, c->pcg, c->red_partial, c->red_counter);
        launch_vcycle(c, r_new, true);
        return;
    }
    {
        ProfScope ps(c, SULI_K_CG_UPDATE, 1);
        if (vec) {
            pdl_launch(k_pcgv_updc, vgrid_upd(G), kB2, c->stream, G, c->pc_x, r_old, r_new, p_new, c->pc_q, c->pcg,
                       c->red_partial, c->red_counter, x_zero ? 1 : 0);
        } else {
            const dim3 gu((G.nx + 31) / 32, (G.ny + 7) / 8, (G.nz + kKZU - 1) / kKZU);
            pdl_launch(k_pcg_updc, gu, kB2, c->stream, G, c->pc_x, r_old, r_new, p_new, c->pc_q, c->pcg,
                       c->red_partial, c->red_counter, x_zero ? 1 : 0);
        }
    }
    ProfScope ps(c, SULI_K_MG, vcycle_kernels(c));
    launch_vcycle(c, r_new);
}

int pcg_iter_kernels(const suli_ctx* c) { return fused_update(c) ? 1 + vcycle_kernels(c) : 2 + vcycle_kernels(c); }

int vcycle_kernels(const suli_ctx* c) {
    const int L = (int)c->mg.size();
    if (use_cluster(c)) return 4 * (L - 3) + 1;
    if (use_tail(c)) return 4 * (L - 2) + 1;
    if (L == 1) return 2;
    int n = 1;
    for (int l = 0; l < L - 1; ++l) n += fused_level(c, l) ? 2 : 4;
    return n;
}

}  // namespace suli
