// k_mg_vec.cuh — the inner solve's multigrid and PCG kernels with 4 cells a thread (included by
// k_mixed.cu after the one-cell-a-thread kernels, whose operators and helpers it uses).
//
// A thread owns a quad of 4 consecutive x cells (one float4 of every field: rows start
// 64-byte aligned and the quad's first cell is i = 1 + 4t) of one (j) row, and kKZ cells along z.
// Its z neighbours come from the column it loaded, its y neighbours are float4 loads of the
// neighbouring rows, and only the quad's two outer x neighbours are scalar loads.  One warp-wide
// float4 load moves 512 contiguous bytes, 4x the scalar kernels' 128, so a thread keeps far
// more bytes in flight: the one-cell kernels were latency-bound at 1-1.7 TB/s.
//
// Per cell the arithmetic is the one-cell kernels', in the same order (faces, apply_faces,
// the updates), so the V-cycle and the operator are the same functions; only the FP64 dot
// products sum their terms in another order.  Grids need nx % 4 == 0 (the host falls back to
// the one-cell kernels otherwise).
#pragma once

namespace suli {

constexpr int kVX = 4;

struct V4 {
    float v[kVX];
};
__device__ __forceinline__ V4 ld4(const float* a, int c) {
    const float4 t = *reinterpret_cast<const float4*>(a + c);
    return V4{{t.x, t.y, t.z, t.w}};
}
__device__ __forceinline__ void st4(float* a, int c, const float (&v)[kVX]) {
    *reinterpret_cast<float4*>(a + c) = make_float4(v[0], v[1], v[2], v[3]);
}

// a thread's quad: first cell (i0, j), column k0 .. k0 + kKZ - 1
struct VQ {
    int i0, j, k0;
    int c0;          // index of (i0, j, 0)
    int fxm, fxp;    // ghost-mapped x offsets: minus neighbour of cell i0, plus neighbour of i0 + 3
    int fym, fyp;    // ghost-mapped y offsets of the row
    bool in;
};
__device__ __forceinline__ VQ vquad(const Geo& G, const BC& bc, int kz) {
    VQ q;
    q.i0 = kVX * (blockIdx.x * blockDim.x + threadIdx.x) + 1;
    q.j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    q.k0 = blockIdx.z * kz + 1;
    q.in = (q.i0 <= G.nx && q.j <= G.ny);
    const int i0 = q.in ? q.i0 : 1, j = q.in ? q.j : 1;
    q.c0 = kBase + (i0 - 1) + G.px * j;
    const Nb a = neighbours(G, bc, i0, j, 1), b = neighbours(G, bc, i0 + kVX - 1, j, 1);
    q.fxm = a.xm;
    q.fxp = b.xp;
    q.fym = a.ym;
    q.fyp = a.yp;
    return q;
}
static inline dim3 vgrid(const Geo& g, int kz) {
    return dim3((g.nx / kVX + 31) / 32, (g.ny + 7) / 8, (g.nz + kz - 1) / kz);
}

// ---- operators on a quad: the faces of its 4 cells in plane k (cell index c of the quad's
// first cell), exactly as OpRho::make / OpStored::cell form them per cell
struct OpRho4 {
    const float *rho, *idg, *c2;
    __device__ __forceinline__ void faces(const Geo& G, int i0, int j, int k, int c, Faces (&F)[kVX]) const {
        const int px = G.px, pxy = (int)G.pxy;
        const float cx2 = c2[0], cy2 = c2[1], cz2 = c2[2];
        const V4 rc = ld4(rho, c);
        const V4 rym = ld4(rho, (j > 1) ? c - px : c + px), ryp = ld4(rho, (j < G.ny) ? c + px : c - px);
        const V4 rzm = ld4(rho, (k > 1) ? c - pxy : c + pxy), rzp = ld4(rho, (k < G.nz) ? c + pxy : c - pxy);
        const float rxm0 = rho[(i0 > 1) ? c - 1 : c + 1];
        const float rxp3 = rho[(i0 + kVX - 1 < G.nx) ? c + kVX : c + kVX - 2];
#pragma unroll
        for (int e = 0; e < kVX; ++e) {
            const float r = rc.v[e];
            const float rxm = (e == 0) ? rxm0 : rc.v[e - 1];
            const float rxp = (e == kVX - 1) ? rxp3 : rc.v[e + 1];
            F[e] = Faces{face_div(cx2, r + rxm), face_div(cx2, r + rxp), face_div(cy2, r + rym.v[e]),
                         face_div(cy2, r + ryp.v[e]), face_div(cz2, r + rzm.v[e]), face_div(cz2, r + rzp.v[e])};
        }
    }
    __device__ __forceinline__ V4 inv_diag(int c) const { return ld4(idg, c); }
};
struct OpStored4 {
    const float *sx, *sy, *sz, *idg;
    __device__ __forceinline__ void faces(const Geo& G, int, int, int, int c, Faces (&F)[kVX]) const {
        const V4 x4 = ld4(sx, c), y4 = ld4(sy, c), yp4 = ld4(sy, c + G.px), z4 = ld4(sz, c), zp4 = ld4(sz, c + (int)G.pxy);
        const float xn = sx[c + kVX];   // plus face of the last cell (the ghost face at i = nx + 1)
#pragma unroll
        for (int e = 0; e < kVX; ++e)
            F[e] = Faces{x4.v[e], (e == kVX - 1) ? xn : x4.v[e + 1], y4.v[e], yp4.v[e], z4.v[e], zp4.v[e]};
    }
    __device__ __forceinline__ V4 inv_diag(int c) const { return ld4(idg, c); }
};

// A applied to a quad: x values of the quad (xc), of its rows y-1 / y+1, planes z-1 / z+1 and
// the two outer x neighbours
__device__ __forceinline__ void apply4(const Faces (&F)[kVX], const float (&xc)[kVX], float xm0, float xp3,
                                       const float (&ym)[kVX], const float (&yp)[kVX], const float (&zm)[kVX],
                                       const float (&zp)[kVX], float (&ax)[kVX]) {
#pragma unroll
    for (int e = 0; e < kVX; ++e) {
        const float xm = (e == 0) ? xm0 : xc[e - 1];
        const float xp = (e == kVX - 1) ? xp3 : xc[e + 1];
        ax[e] = apply_faces(F[e], xc[e], xm, xp, ym[e], yp[e], zm[e], zp[e]);
    }
}

// two damped Jacobi sweeps from zero (k_mg_pre): x1 = w f/dg, y = x1 + w2 (f - A x1)/dg
template <int KZ, class Op4>
__global__ void __launch_bounds__(256, KZ == 2 ? 4 : 3) k_mgv_pre(Geo G, BC bc, const float* __restrict__ f, Op4 A,
                                                 float* __restrict__ y, float omega, float omega2,
                                                 const PCGState* st) {
    pdl_wait();
    if (st->done) return;
    const VQ q = vquad(G, bc, KZ);
    if (!q.in) return;
    const int pxy = (int)G.pxy;
    auto x1 = [&](int cc, float (&o)[kVX]) {
        const V4 fv = ld4(f, cc), dv = A.inv_diag(cc);
#pragma unroll
        for (int e = 0; e < kVX; ++e) o[e] = omega * fv.v[e] * dv.v[e];
    };
    auto x1s = [&](int cc) { return omega * f[cc] * A.idg[cc]; };
    float col[KZ + 2][kVX];
#pragma unroll
    for (int m = 0; m < KZ + 2; ++m) x1(q.c0 + pxy * map_any(q.k0 - 1 + m, G.nz, bc.perz), col[m]);
#pragma unroll
    for (int m = 0; m < KZ; ++m) {
        const int k = q.k0 + m;
        if (KZ > 2 && k > G.nz) break;   // KZ = 2 runs only where nz is even
        const int c = q.c0 + pxy * k;
        Faces F[kVX];
        A.faces(G, q.i0, q.j, k, c, F);
        float ym[kVX], yp[kVX], ax[kVX], out[kVX];
        x1(c + q.fym, ym);
        x1(c + q.fyp, yp);
        apply4(F, col[m + 1], x1s(c + q.fxm), x1s(c + kVX - 1 + q.fxp), ym, yp, col[m], col[m + 2], ax);
        const V4 fc = ld4(f, c), dc = A.inv_diag(c);
#pragma unroll
        for (int e = 0; e < kVX; ++e) out[e] = col[m + 1][e] + omega2 * (fc.v[e] - ax[e]) * dc.v[e];
        st4(y, c, out);
    }
}

// The inner PCG's update fused into the V-cycle's first level-0 kernel (k_pcgv_updc followed
// by k_mgv_pre): with alpha from the SpMV's p.q, x += alpha p and r_out = r - alpha q at the
// thread's cells, r.r and the inner stop test; the two pre-smoothing sweeps read the updated
// residual at the neighbours too, formed there again from r and q (the same expression, so the
// same value), which saves the update's own pass over x, p, r and q.  r is read from one buffer
// and written to another, so no thread reads a neighbour's already-updated residual.  When the
// stop test ends the loop, the V-cycle's other kernels return at once.
template <int KZ, class Op4>
__global__ void __launch_bounds__(256, KZ == 2 ? 4 : 3) k_mgv_preu(Geo G, BC bc, float* __restrict__ x,
                                                  const float* __restrict__ p, const float* __restrict__ r,
                                                  const float* __restrict__ qv, float* __restrict__ r_out, Op4 A,
                                                  float* __restrict__ y, float omega, float omega2, PCGState* st,
                                                  double* partial, unsigned int* counter) {
    pdl_wait();
    if (st->done) return;
    const float alpha = (float)st->alpha;
    const VQ q = vquad(G, bc, KZ);
    double rr = 0.;
    if (q.in) {
        const int pxy = (int)G.pxy;
        auto fr = [&](int cc, float (&o)[kVX]) {
            const V4 a = ld4(r, cc), b = ld4(qv, cc);
#pragma unroll
            for (int e = 0; e < kVX; ++e) o[e] = a.v[e] - alpha * b.v[e];
        };
        auto x1 = [&](int cc, float (&o)[kVX]) {
            float fv[kVX];
            fr(cc, fv);
            const V4 dv = A.inv_diag(cc);
#pragma unroll
            for (int e = 0; e < kVX; ++e) o[e] = omega * fv[e] * dv.v[e];
        };
        auto x1s = [&](int cc) {
            const float fv = r[cc] - alpha * qv[cc];
            return omega * fv * A.idg[cc];
        };
        float col[KZ + 2][kVX];
#pragma unroll
        for (int m = 0; m < KZ + 2; ++m) x1(q.c0 + pxy * map_any(q.k0 - 1 + m, G.nz, bc.perz), col[m]);
#pragma unroll
        for (int m = 0; m < KZ; ++m) {
            const int k = q.k0 + m;
            if (KZ > 2 && k > G.nz) break;   // KZ = 2 runs only where nz is even
            const int c = q.c0 + pxy * k;
            Faces F[kVX];
            A.faces(G, q.i0, q.j, k, c, F);
            float ym[kVX], yp[kVX], ax[kVX], out[kVX], fc[kVX];
            x1(c + q.fym, ym);
            x1(c + q.fyp, yp);
            apply4(F, col[m + 1], x1s(c + q.fxm), x1s(c + kVX - 1 + q.fxp), ym, yp, col[m], col[m + 2], ax);
            fr(c, fc);
            const V4 dc = A.inv_diag(c);
#pragma unroll
            for (int e = 0; e < kVX; ++e) {
                out[e] = col[m + 1][e] + omega2 * (fc[e] - ax[e]) * dc.v[e];
                rr += (double)fc[e] * (double)fc[e];
            }
            st4(y, c, out);
            st4(r_out, c, fc);
            const V4 xv = ld4(x, c), pv = ld4(p, c);
            float xo[kVX];
#pragma unroll
            for (int e = 0; e < kVX; ++e) xo[e] = xv.v[e] + alpha * pv.v[e];
            st4(x, c, xo);
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

// x_out = x_in + w (f - A x_in)/dg; with do_dot also f.x_out -> rz, beta (k_mg_jacc)
template <int KZ, class Op4>
__global__ void __launch_bounds__(256, KZ == 2 ? 4 : 3) k_mgv_jacc(Geo G, BC bc, const float* __restrict__ xin,
                                                  const float* __restrict__ f, Op4 A, float* __restrict__ xout,
                                                  float omega, PCGState* st, int do_dot, double* partial,
                                                  unsigned int* counter) {
    pdl_wait();
    if (st->done) return;
    const VQ q = vquad(G, bc, KZ);
    double dot = 0.;
    if (q.in) {
        const int pxy = (int)G.pxy;
        float col[KZ + 2][kVX];
#pragma unroll
        for (int m = 0; m < KZ + 2; ++m) {
            const V4 t = ld4(xin, q.c0 + pxy * map_any(q.k0 - 1 + m, G.nz, bc.perz));
#pragma unroll
            for (int e = 0; e < kVX; ++e) col[m][e] = t.v[e];
        }
#pragma unroll
        for (int m = 0; m < KZ; ++m) {
            const int k = q.k0 + m;
            if (KZ > 2 && k > G.nz) break;   // KZ = 2 runs only where nz is even
            const int c = q.c0 + pxy * k;
            Faces F[kVX];
            A.faces(G, q.i0, q.j, k, c, F);
            const V4 y1 = ld4(xin, c + q.fym), y2 = ld4(xin, c + q.fyp);
            float ax[kVX], out[kVX];
            apply4(F, col[m + 1], xin[c + q.fxm], xin[c + kVX - 1 + q.fxp], y1.v, y2.v, col[m], col[m + 2], ax);
            const V4 fc = ld4(f, c), dc = A.inv_diag(c);
#pragma unroll
            for (int e = 0; e < kVX; ++e) {
                out[e] = col[m + 1][e] + omega * (fc.v[e] - ax[e]) * dc.v[e];
                dot += (double)fc.v[e] * (double)out[e];
            }
            st4(xout, c, out);
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

// x_out = x' + w (f - A x')/dg with x' = y + a P xc (k_mg_post)
template <int KZ, class Op4>
__global__ void __launch_bounds__(256, KZ == 2 ? 4 : 3) k_mgv_post(Geo Gf, Geo Gc, BC bc, const float* __restrict__ y,
                                                  const float* __restrict__ xc, const float* __restrict__ f, Op4 A,
                                                  float* __restrict__ xout, float omega, float alpha,
                                                  const PCGState* st) {
    pdl_wait();
    if (st->done) return;
    const VQ q = vquad(Gf, bc, KZ);
    if (!q.in) return;
    const int pxy = (int)Gf.pxy;
    // x' of the quad in row jj (fine j index, already ghost-mapped) and plane kk (mapped), at
    // fine index cc of the quad's first cell: parents I0 = (i0+1)/2 (cells 0, 1) and I0 + 1 (2, 3)
    const int I0 = (q.i0 + 1) >> 1;
    auto xq = [&](int cc, int jj, int kk, float (&o)[kVX]) {
        const V4 yv = ld4(y, cc);
        const long long pc = Gc.idx(I0, (jj + 1) >> 1, (kk + 1) >> 1);
        const float p0 = alpha * xc[pc], p1 = alpha * xc[pc + 1];
        o[0] = yv.v[0] + p0; o[1] = yv.v[1] + p0; o[2] = yv.v[2] + p1; o[3] = yv.v[3] + p1;
    };
    // x' of a single cell at fine (ii, jj, kk) (mapped), index cc
    auto xs = [&](int cc, int ii, int jj, int kk) {
        return y[cc] + alpha * xc[Gc.idx((ii + 1) >> 1, (jj + 1) >> 1, (kk + 1) >> 1)];
    };
    const int ixm = map_any(q.i0 - 1, Gf.nx, bc.perx), ixp = map_any(q.i0 + kVX, Gf.nx, bc.perx);
    const int jym = map_any(q.j - 1, Gf.ny, bc.pery), jyp = map_any(q.j + 1, Gf.ny, bc.pery);
    float col[KZ + 2][kVX];
#pragma unroll
    for (int m = 0; m < KZ + 2; ++m) {
        const int k = map_any(q.k0 - 1 + m, Gf.nz, bc.perz);
        xq(q.c0 + pxy * k, q.j, k, col[m]);
    }
#pragma unroll
    for (int m = 0; m < KZ; ++m) {
        const int k = q.k0 + m;
        if (KZ > 2 && k > Gf.nz) break;   // KZ = 2 runs only where nz is even
        const int c = q.c0 + pxy * k;
        Faces F[kVX];
        A.faces(Gf, q.i0, q.j, k, c, F);
        float ym[kVX], yp[kVX], ax[kVX], out[kVX];
        xq(c + q.fym, jym, k, ym);
        xq(c + q.fyp, jyp, k, yp);
        apply4(F, col[m + 1], xs(c + q.fxm, ixm, q.j, k), xs(c + kVX - 1 + q.fxp, ixp, q.j, k), ym, yp, col[m],
               col[m + 2], ax);
        const V4 fc = ld4(f, c), dc = A.inv_diag(c);
#pragma unroll
        for (int e = 0; e < kVX; ++e) out[e] = col[m + 1][e] + omega * (fc.v[e] - ax[e]) * dc.v[e];
        st4(xout, c, out);
    }
}

// f_c = (1/8) sum over the 8 children of (f - A x) (k_mg_restrict); a thread makes the two coarse
// cells whose children are one fine quad, in the children order (x, y, z) of the one-cell kernel
template <class Op4>
__global__ void __launch_bounds__(256, 3) k_mgv_restrict(Geo Gf, Geo Gc, BC bc, const float* __restrict__ x,
                                                      const float* __restrict__ f, Op4 A, float* fc,
                                                      const PCGState* st) {
    pdl_wait();
    if (st->done) return;
    const int I0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x) + 1;
    const int J = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int K = blockIdx.z + 1;
    if (I0 > Gc.nx || J > Gc.ny || K > Gc.nz) return;
    const int i0 = 2 * I0 - 1;
    float s0 = 0.f, s1 = 0.f;
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
            const int j = 2 * J - 1 + dy, k = 2 * K - 1 + dz;
            const int c = (int)Gf.idx(i0, j, k);
            const Nb a = neighbours(Gf, bc, i0, j, k), b = neighbours(Gf, bc, i0 + kVX - 1, j, k);
            Faces F[kVX];
            A.faces(Gf, i0, j, k, c, F);
            const V4 xq = ld4(x, c), xym = ld4(x, c + a.ym), xyp = ld4(x, c + a.yp), xzm = ld4(x, c + a.zm),
                     xzp = ld4(x, c + a.zp);
            float ax[kVX];
            apply4(F, xq.v, x[c + a.xm], x[c + kVX - 1 + b.xp], xym.v, xyp.v, xzm.v, xzp.v, ax);
            const V4 fv = ld4(f, c);
            s0 += fv.v[0] - ax[0];
            s0 += fv.v[1] - ax[1];
            s1 += fv.v[2] - ax[2];
            s1 += fv.v[3] - ax[3];
        }
    fc[Gc.idx(I0, J, K)] = 0.125f * s0;
    if (I0 + 1 <= Gc.nx) fc[Gc.idx(I0 + 1, J, K)] = 0.125f * s1;
}
static inline dim3 vgrid_restrict(const Geo& gc) { return dim3((gc.nx / 2 + 31) / 32, (gc.ny + 7) / 8, gc.nz); }

// p = z + beta p_old (also at the neighbours), q = A p, p.q -> alpha (k_pcg_spmvc)
template <int KZ, class Op4>
__global__ void __launch_bounds__(256, KZ == 2 ? 4 : 3) k_pcgv_spmvc(Geo G, BC bc, const float* __restrict__ z,
                                                    const float* __restrict__ p_old, float* __restrict__ p_new,
                                                    float* __restrict__ qv, Op4 A, PCGState* st, double* partial,
                                                    unsigned int* counter) {
    pdl_wait();
    if (st->done) return;
    const float beta = (float)st->beta;
    const VQ q = vquad(G, bc, KZ);
    double dot = 0.;
    if (q.in) {
        const int pxy = (int)G.pxy;
        auto pn = [&](int cc, float (&o)[kVX]) {
            const V4 a = ld4(z, cc), b = ld4(p_old, cc);
#pragma unroll
            for (int e = 0; e < kVX; ++e) o[e] = a.v[e] + beta * b.v[e];
        };
        auto pns = [&](int cc) { return z[cc] + beta * p_old[cc]; };
        float col[KZ + 2][kVX];
#pragma unroll
        for (int m = 0; m < KZ + 2; ++m) pn(q.c0 + pxy * map_any(q.k0 - 1 + m, G.nz, bc.perz), col[m]);
#pragma unroll
        for (int m = 0; m < KZ; ++m) {
            const int k = q.k0 + m;
            if (KZ > 2 && k > G.nz) break;   // KZ = 2 runs only where nz is even
            const int c = q.c0 + pxy * k;
            Faces F[kVX];
            A.faces(G, q.i0, q.j, k, c, F);
            float ym[kVX], yp[kVX], ax[kVX];
            pn(c + q.fym, ym);
            pn(c + q.fyp, yp);
            apply4(F, col[m + 1], pns(c + q.fxm), pns(c + kVX - 1 + q.fxp), ym, yp, col[m], col[m + 2], ax);
            st4(p_new, c, col[m + 1]);
            st4(qv, c, ax);
#pragma unroll
            for (int e = 0; e < kVX; ++e) dot += (double)col[m + 1][e] * (double)ax[e];
        }
    }
    double t, u;
    if (reduce2_last(dot, 0.0, partial, counter, t, u) && flat_tid() == 0) {
        st->pq = t;
        st->alpha = st->rz / t;
        if (!isfinite(st->alpha)) { st->status = SULI_ERR_NAN; st->done = 1; }
    }
}

// x += alpha p (x_zero: x = alpha p, the pass's first update), r -= alpha q, r.r and the inner stop
// test (k_pcg_updc)
__global__ void __launch_bounds__(256) k_pcgv_updc(Geo G, float* __restrict__ x, const float* __restrict__ r,
                                                   float* __restrict__ r_out, const float* __restrict__ p,
                                                   const float* __restrict__ qv, PCGState* st, double* partial,
                                                   unsigned int* counter, int x_zero) {
    pdl_wait();
    if (st->done) return;
    const float alpha = (float)st->alpha;
    const int i0 = kVX * (blockIdx.x * blockDim.x + threadIdx.x) + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int k0 = blockIdx.z * kKZU + 1;
    double rr = 0.;
    if (i0 <= G.nx && j <= G.ny) {
        const int c0 = kBase + (i0 - 1) + G.px * j, pxy = (int)G.pxy;
#pragma unroll
        for (int m = 0; m < kKZU; ++m) {
            const int k = k0 + m;
            if (k > G.nz) break;
            const int c = c0 + pxy * k;
            const V4 xv = x_zero ? V4{{0.f, 0.f, 0.f, 0.f}} : ld4(x, c), pv = ld4(p, c), rv = ld4(r, c), qq = ld4(qv, c);
            float xo[kVX], ro[kVX];
#pragma unroll
            for (int e = 0; e < kVX; ++e) {
                xo[e] = xv.v[e] + alpha * pv.v[e];
                ro[e] = rv.v[e] - alpha * qq.v[e];
                rr += (double)ro[e] * (double)ro[e];
            }
            st4(x, c, xo);
            st4(r_out, c, ro);
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
static inline dim3 vgrid_upd(const Geo& g) { return dim3((g.nx / kVX + 31) / 32, (g.ny + 7) / 8, (g.nz + kKZU - 1) / kKZU); }

}  // namespace suli
