// k_mg_stream.cuh — level-0 kernels of the inner solve that stream z-planes through shared
// memory with TMA (included by k_mixed.cu after the vectorised kernels, whose operator and quad
// helpers they use).
//
// The vectorised kernels (k_mg_vec.cuh) read every value through L1/L2 into registers: a
// thread issues its column's loads, waits out the DRAM latency, computes and exits, and the
// loads it can keep in flight are bounded by its registers, so the level-0 kernels ran
// latency-bound near 40 % of HBM bandwidth.  Here a CTA of 32 x 8 threads owns a tile of 128
// x-cells (one quad of 4 cells a thread) x 8 rows and marches up a chunk of planes.  One thread
// loads each plane the chunk needs (its planes and one on each side, mapped as the operator maps
// them) as one 3-D TMA box per input field (cp.async.bulk.tensor, no multicast): 136 floats x
// 10 rows x 1 plane, starting 4 cells before the tile so that x is 16-byte aligned, and one row
// before it.  The planes land in a ring of kSR slots; while the CTA computes plane k from the
// slots of k-1, k and k+1, the next planes' loads are in flight (tens of KB a CTA, two CTAs an
// SM), decoupled from the threads' registers.  Neighbours are read from shared memory; results
// are stored straight from registers (float4 a thread).
//
// Per cell the arithmetic is the vectorised kernels' (the same operator, faces and update
// expressions in the same order), so the values are the same bits; the FP64 dot products sum
// in another grouping.  Used on level 0 when no x or y axis is periodic (a wrapped neighbour
// would lie outside the tile), nx is a multiple of 16 (the row pitch then holds the tile's
// last x neighbour) and the device grants the shared memory.
//
// Every wait on a slot is bounded: a wait that runs out makes the CTA wait (bounded again) for
// the loads it issued, sets the inner solve's status to SULI_ERR_CUDA and done, and return.
#pragma once
#include <cuda.h>

namespace suli {

constexpr int kSTX = 32, kSTY = 8;                             // threads: quads along x, rows
constexpr int kSTileX = kSTX * kVX;                            // 128 cells along x
constexpr int kSBoxX = kSTileX + 8;                            // 4 cells before the tile .. 4 after
constexpr int kSBoxY = kSTY + 2;                               // one row on each side
constexpr int kSBoxBytes = kSBoxX * kSBoxY * 4;                // 5440
constexpr int kSSlotBytes = (kSBoxBytes + 127) / 128 * 128;    // TMA destinations 128-byte aligned
constexpr int kSR = 5;                                         // ring: planes k-1, k, k+1 + 2 ahead

static inline size_t stream_smem_bytes(int nf) { return (size_t)kSR * nf * kSSlotBytes + kSR * sizeof(uint64_t); }

__device__ __forceinline__ uint32_t s_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ bool s_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait on a phase of a slot's barrier; false if it did not complete
__device__ __forceinline__ bool s_wait(uint32_t bar, uint32_t parity) {
    for (int it = 0; it < (1 << 22); ++it)
        if (s_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void s_tma3(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

// a quad / one value of a slot at tile row ly, tile column lx (lx of a quad a multiple of 4)
__device__ __forceinline__ V4 sq(const float* s, int ly, int lx) {
    const float4 t = *reinterpret_cast<const float4*>(s + ly * kSBoxX + lx);
    return V4{{t.x, t.y, t.z, t.w}};
}
__device__ __forceinline__ float ss(const float* s, int ly, int lx) { return s[ly * kSBoxX + lx]; }

// A thread's quad in the tile and the tile positions of its neighbours: the unknowns' Neumann
// map (a neighbour outside the box is the cell itself) and the faces' clamped end rule (the
// face at the box's end is the next interior face), as vquad and OpRho4::faces take them
struct STile {
    int i0, j, c0;        // first cell of the quad, its index in plane 0
    int qx, ly;           // its tile column and row
    int uxm, uxp, uym, uyp;   // unknowns: x neighbours (scalars), rows
    int fxm, fxp, fym, fyp;   // faces: x neighbours (scalars), rows
    bool in;
};
__device__ __forceinline__ STile s_tile(const Geo& G) {
    STile t;
    const int tx = threadIdx.x, ty = threadIdx.y;
    t.i0 = kSTileX * blockIdx.x + kVX * tx + 1;
    t.j = kSTY * blockIdx.y + ty + 1;
    t.in = (t.i0 <= G.nx && t.j <= G.ny);
    t.c0 = kBase + (t.i0 - 1) + G.px * t.j;
    t.qx = 4 + kVX * tx;
    t.ly = 1 + ty;
    t.uxm = (t.i0 > 1) ? t.qx - 1 : t.qx;
    t.uxp = (t.i0 + kVX - 1 < G.nx) ? t.qx + kVX : t.qx + kVX - 1;
    t.uym = (t.j > 1) ? t.ly - 1 : t.ly;
    t.uyp = (t.j < G.ny) ? t.ly + 1 : t.ly;
    t.fxm = (t.i0 > 1) ? t.qx - 1 : t.qx + 1;
    t.fxp = (t.i0 + kVX - 1 < G.nx) ? t.qx + kVX : t.qx + kVX - 2;
    t.fym = (t.j > 1) ? t.ly - 1 : t.ly + 1;
    t.fyp = (t.j < G.ny) ? t.ly + 1 : t.ly - 1;
    return t;
}

// the quad's faces in plane k from the density slots of planes k-1, k, k+1 (OpRho4::faces)
__device__ __forceinline__ void s_faces(const STile& t, int k, int nz, const float* rm, const float* r0,
                                        const float* rp, float cx2, float cy2, float cz2, Faces (&F)[kVX]) {
    const V4 rc = sq(r0, t.ly, t.qx);
    const V4 rym = sq(r0, t.fym, t.qx), ryp = sq(r0, t.fyp, t.qx);
    const V4 rzm = sq((k > 1) ? rm : rp, t.ly, t.qx), rzp = sq((k < nz) ? rp : rm, t.ly, t.qx);
    const float rxm0 = ss(r0, t.ly, t.fxm), rxp3 = ss(r0, t.ly, t.fxp);
#pragma unroll
    for (int e = 0; e < kVX; ++e) {
        const float r = rc.v[e];
        const float rxm = (e == 0) ? rxm0 : rc.v[e - 1];
        const float rxp = (e == kVX - 1) ? rxp3 : rc.v[e + 1];
        F[e] = Faces{face_div(cx2, r + rxm), face_div(cx2, r + rxp), face_div(cy2, r + rym.v[e]),
                     face_div(cy2, r + ryp.v[e]), face_div(cz2, r + rzm.v[e]), face_div(cz2, r + rzp.v[e])};
    }
}

// The plane engine.  Body::plane(k, sm, s0, sp) computes plane k from the slots (one pointer a
// field) of the planes k-1, k, k+1.  Returns false if a wait ran out.
template <int NF>
struct SSlots {
    const float* f[NF];
};
template <int NF, class Body>
__device__ __forceinline__ bool s_march(const Geo& G, const BC& bc, const CUtensorMap* const (&maps)[NF], int chunk,
                                        Body& body, PCGState* st) {
    extern __shared__ __align__(128) unsigned char s_smem[];
    const int tid = threadIdx.x + kSTX * threadIdx.y;
    const int k0 = 1 + chunk * blockIdx.z;
    const int nplanes = min(chunk, G.nz - k0 + 1);
    const int nseq = nplanes + 2;   // planes k0 - 1 .. k0 + nplanes
    uint64_t* bars = reinterpret_cast<uint64_t*>(s_smem + (size_t)kSR * NF * kSSlotBytes);
    const int x0 = kBase - 1 + kSTileX * blockIdx.x - 3;   // x of cell 128 bx - 3 (4 before the tile): a multiple of 4
    const int y0 = kSTY * blockIdx.y;                       // row j_first - 1
    if (tid == 0) {
        for (int s = 0; s < kSR; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_addr(&bars[s])), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto slot = [&](int q, int f) {
        return reinterpret_cast<const float*>(s_smem + ((size_t)(q % kSR) * NF + f) * kSSlotBytes);
    };
    auto issue = [&](int q) {
        const int s = q % kSR;
        const uint32_t bar = s_addr(&bars[s]);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(NF * kSBoxBytes)
                     : "memory");
        const int z = map_any(k0 - 1 + q, G.nz, bc.perz);
#pragma unroll
        for (int f = 0; f < NF; ++f)
            s_tma3(s_addr(s_smem + ((size_t)s * NF + f) * kSSlotBytes), maps[f], x0, y0, z, bar);
    };
    if (tid == 0)
        for (int q = 0; q < min(kSR, nseq); ++q) issue(q);
    for (int m = 0; m < nplanes; ++m) {
        bool ok = true;
        if (m == 0) ok = s_wait(s_addr(&bars[0]), 0) && s_wait(s_addr(&bars[1]), 0);
        ok = ok && s_wait(s_addr(&bars[(m + 2) % kSR]), ((m + 2) / kSR) & 1);
        if (__syncthreads_or(!ok)) {
            // wait (bounded) for the loads issued and not yet consumed, then give up
            if (tid == 0) {
                const int issued = (m == 0) ? min(kSR, nseq) : min(nseq, m - 1 + kSR);
                for (int q = m; q < issued; ++q) s_wait(s_addr(&bars[q % kSR]), (q / kSR) & 1);
                st->status = SULI_ERR_CUDA;
                st->done = 1;
            }
            __syncthreads();
            return false;
        }
        // every thread is done with plane k0 + m - 2 (sequence m - 1): refill its slot
        if (tid == 0 && m >= 1 && m - 1 + kSR < nseq) issue(m - 1 + kSR);
        SSlots<NF> sm, s0, sp;
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            sm.f[f] = slot(m, f);
            s0.f[f] = slot(m + 1, f);
            sp.f[f] = slot(m + 2, f);
        }
        body.plane(k0 + m, sm, s0, sp);
    }
    return true;
}

// ---- two damped Jacobi sweeps from zero (k_mgv_pre on level 0): fields f, 1/diag, density
struct SPreBody {
    STile t;
    int nz, pxy;
    float omega, omega2, cx2, cy2, cz2;
    float* y;
    __device__ __forceinline__ void x1(const SSlots<3>& s, int ly, int lx, float (&o)[kVX]) const {
        const V4 fv = sq(s.f[0], ly, lx), dv = sq(s.f[1], ly, lx);
#pragma unroll
        for (int e = 0; e < kVX; ++e) o[e] = omega * fv.v[e] * dv.v[e];
    }
    __device__ __forceinline__ float x1s(const SSlots<3>& s, int ly, int lx) const {
        return omega * ss(s.f[0], ly, lx) * ss(s.f[1], ly, lx);
    }
    __device__ __forceinline__ void plane(int k, const SSlots<3>& sm, const SSlots<3>& s0, const SSlots<3>& sp) {
        if (!t.in) return;
        float zm[kVX], xc[kVX], zp[kVX], ym[kVX], yp[kVX], ax[kVX], out[kVX];
        x1(sm, t.ly, t.qx, zm);
        x1(s0, t.ly, t.qx, xc);
        x1(sp, t.ly, t.qx, zp);
        Faces F[kVX];
        s_faces(t, k, nz, sm.f[2], s0.f[2], sp.f[2], cx2, cy2, cz2, F);
        x1(s0, t.uym, t.qx, ym);
        x1(s0, t.uyp, t.qx, yp);
        apply4(F, xc, x1s(s0, t.ly, t.uxm), x1s(s0, t.ly, t.uxp), ym, yp, zm, zp, ax);
        const V4 fc = sq(s0.f[0], t.ly, t.qx), dc = sq(s0.f[1], t.ly, t.qx);
#pragma unroll
        for (int e = 0; e < kVX; ++e) out[e] = xc[e] + omega2 * (fc.v[e] - ax[e]) * dc.v[e];
        st4(y, t.c0 + pxy * k, out);
    }
};
__global__ void __launch_bounds__(kSTX * kSTY, 2) k_mgs_pre(Geo G, BC bc, const __grid_constant__ CUtensorMap mf,
                                                         const __grid_constant__ CUtensorMap md,
                                                         const __grid_constant__ CUtensorMap mr, const float* c2,
                                                         float* y, float omega, float omega2, int chunk,
                                                         PCGState* st) {
    pdl_wait();
    if (st->done) return;
    SPreBody b;
    b.t = s_tile(G);
    b.nz = G.nz;
    b.pxy = (int)G.pxy;
    b.omega = omega;
    b.omega2 = omega2;
    b.cx2 = c2[0]; b.cy2 = c2[1]; b.cz2 = c2[2];
    b.y = y;
    const CUtensorMap* const maps[3] = {&mf, &md, &mr};
    s_march<3>(G, bc, maps, chunk, b, st);
}

// ---- x_out = x_in + w (f - A x_in)/dg, f.x_out -> rz, beta (k_mgv_jacc on level 0, with the
// dot product): fields x_in, f, 1/diag, density
struct SJaccBody {
    STile t;
    int nz, pxy;
    float omega, cx2, cy2, cz2;
    float* xout;
    double dot;
    __device__ __forceinline__ void plane(int k, const SSlots<4>& sm, const SSlots<4>& s0, const SSlots<4>& sp) {
        if (!t.in) return;
        const V4 zm = sq(sm.f[0], t.ly, t.qx), xc = sq(s0.f[0], t.ly, t.qx), zp = sq(sp.f[0], t.ly, t.qx);
        Faces F[kVX];
        s_faces(t, k, nz, sm.f[3], s0.f[3], sp.f[3], cx2, cy2, cz2, F);
        const V4 y1 = sq(s0.f[0], t.uym, t.qx), y2 = sq(s0.f[0], t.uyp, t.qx);
        float ax[kVX], out[kVX];
        apply4(F, xc.v, ss(s0.f[0], t.ly, t.uxm), ss(s0.f[0], t.ly, t.uxp), y1.v, y2.v, zm.v, zp.v, ax);
        const V4 fc = sq(s0.f[1], t.ly, t.qx), dc = sq(s0.f[2], t.ly, t.qx);
#pragma unroll
        for (int e = 0; e < kVX; ++e) {
            out[e] = xc.v[e] + omega * (fc.v[e] - ax[e]) * dc.v[e];
            dot += (double)fc.v[e] * (double)out[e];
        }
        st4(xout, t.c0 + pxy * k, out);
    }
};
__global__ void __launch_bounds__(kSTX * kSTY, 2) k_mgs_jacc(Geo G, BC bc, const __grid_constant__ CUtensorMap mx,
                                                          const __grid_constant__ CUtensorMap mf,
                                                          const __grid_constant__ CUtensorMap md,
                                                          const __grid_constant__ CUtensorMap mr, const float* c2,
                                                          float* xout, float omega, int chunk, PCGState* st,
                                                          double* partial, unsigned int* counter) {
    pdl_wait();
    if (st->done) return;
    SJaccBody b;
    b.t = s_tile(G);
    b.nz = G.nz;
    b.pxy = (int)G.pxy;
    b.omega = omega;
    b.cx2 = c2[0]; b.cy2 = c2[1]; b.cz2 = c2[2];
    b.xout = xout;
    b.dot = 0.;
    const CUtensorMap* const maps[4] = {&mx, &mf, &md, &mr};
    s_march<4>(G, bc, maps, chunk, b, st);   // every CTA joins the reduction, even one that gave up
    double t, u;
    if (reduce2_last(b.dot, 0.0, partial, counter, t, u) && flat_tid() == 0) {
        const double rz_old = st->rz;
        st->rz = t;
        st->beta = (st->iters == 0) ? 0.0 : t / rz_old;
        if (!isfinite(t)) { st->status = SULI_ERR_NAN; st->done = 1; }
    }
}

// ---- p = z + beta p_old (also at the neighbours), q = A p, p.q -> alpha (k_pcgv_spmvc on level
// 0): fields z, p_old, density
struct SSpmvBody {
    STile t;
    int nz, pxy;
    float beta, cx2, cy2, cz2;
    float *p_new, *qv;
    double dot;
    __device__ __forceinline__ void pn(const SSlots<3>& s, int ly, int lx, float (&o)[kVX]) const {
        const V4 a = sq(s.f[0], ly, lx), b = sq(s.f[1], ly, lx);
#pragma unroll
        for (int e = 0; e < kVX; ++e) o[e] = a.v[e] + beta * b.v[e];
    }
    __device__ __forceinline__ float pns(const SSlots<3>& s, int ly, int lx) const {
        return ss(s.f[0], ly, lx) + beta * ss(s.f[1], ly, lx);
    }
    __device__ __forceinline__ void plane(int k, const SSlots<3>& sm, const SSlots<3>& s0, const SSlots<3>& sp) {
        if (!t.in) return;
        float zm[kVX], xc[kVX], zp[kVX], ym[kVX], yp[kVX], ax[kVX];
        pn(sm, t.ly, t.qx, zm);
        pn(s0, t.ly, t.qx, xc);
        pn(sp, t.ly, t.qx, zp);
        Faces F[kVX];
        s_faces(t, k, nz, sm.f[2], s0.f[2], sp.f[2], cx2, cy2, cz2, F);
        pn(s0, t.uym, t.qx, ym);
        pn(s0, t.uyp, t.qx, yp);
        apply4(F, xc, pns(s0, t.ly, t.uxm), pns(s0, t.ly, t.uxp), ym, yp, zm, zp, ax);
        const int c = t.c0 + pxy * k;
        st4(p_new, c, xc);
        st4(qv, c, ax);
#pragma unroll
        for (int e = 0; e < kVX; ++e) dot += (double)xc[e] * (double)ax[e];
    }
};
__global__ void __launch_bounds__(kSTX * kSTY, 2) k_pcgs_spmvc(Geo G, BC bc, const __grid_constant__ CUtensorMap mz,
                                                            const __grid_constant__ CUtensorMap mp,
                                                            const __grid_constant__ CUtensorMap mr, const float* c2,
                                                            float* p_new, float* qv, int chunk, PCGState* st,
                                                            double* partial, unsigned int* counter) {
    pdl_wait();
    if (st->done) return;
    SSpmvBody b;
    b.t = s_tile(G);
    b.nz = G.nz;
    b.pxy = (int)G.pxy;
    b.beta = (float)st->beta;
    b.cx2 = c2[0]; b.cy2 = c2[1]; b.cz2 = c2[2];
    b.p_new = p_new;
    b.qv = qv;
    b.dot = 0.;
    const CUtensorMap* const maps[3] = {&mz, &mp, &mr};
    s_march<3>(G, bc, maps, chunk, b, st);   // every CTA joins the reduction, even one that gave up
    double t, u;
    if (reduce2_last(b.dot, 0.0, partial, counter, t, u) && flat_tid() == 0) {
        st->pq = t;
        st->alpha = st->rz / t;
        if (!isfinite(st->alpha)) { st->status = SULI_ERR_NAN; st->done = 1; }
    }
}

static inline dim3 sgrid(const Geo& g, int chunk) {
    return dim3((g.nx + kSTileX - 1) / kSTileX, (g.ny + kSTY - 1) / kSTY, (g.nz + chunk - 1) / chunk);
}

}  // namespace suli
