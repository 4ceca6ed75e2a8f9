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
// the loads it issued, sets the inner solve's status to SULI_ERR_CUDA and done, and return; the
// host then fails the solve with SULI_ERR_CUDA (a CTA that started after the flag was set skips
// the grid reduction, so the context should be destroyed after that error).  The kernels read
// the level's face constants (c2) before their grid-dependency wait: the multigrid set-up wrote
// them before the inner solve began, never the kernel launched just before.
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
// the coarse level's box (the prolongation source of the post-smoothing): the parents of the
// tile's cells and of their neighbours, 72 floats x 6 rows from coarse cell 64 bx - 3, row 4 by
constexpr int kSCBoxX = 72, kSCBoxY = 6;
constexpr int kSCBoxBytes = kSCBoxX * kSCBoxY * 4;              // 1728
constexpr int kSCSlotBytes = (kSCBoxBytes + 127) / 128 * 128;

// a field read only at the thread's own cells: the tile without halo, 128 floats x 8 rows
constexpr int kSOBoxX = kSTileX, kSOBoxY = kSTY;
constexpr int kSOBoxBytes = kSOBoxX * kSOBoxY * 4;              // 4096
constexpr int kSOSlotBytes = kSOBoxBytes;

static inline size_t stream_stage_bytes(int nf, int no, int nc) {
    return (size_t)nf * kSSlotBytes + (size_t)no * kSOSlotBytes + (size_t)nc * kSCSlotBytes;
}
static inline size_t stream_smem_bytes(int nf, int no = 0, int nc = 0) {
    return kSR * stream_stage_bytes(nf, no, nc) + kSR * sizeof(uint64_t) + 2 * kSTX * kSTY * sizeof(float);
}

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
// the thread's quad in a slot of a field read at its own cells only
__device__ __forceinline__ V4 sqo(const float* s) {
    const float4 t = *reinterpret_cast<const float4*>(s + threadIdx.y * kSOBoxX + kVX * threadIdx.x);
    return V4{{t.x, t.y, t.z, t.w}};
}
// one value of a coarse slot (row pitch kSCBoxX)
__device__ __forceinline__ float ssc(const float* s, int ly, int lx) { return s[ly * kSCBoxX + lx]; }

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

// The quad's faces in plane k from the density slots of planes k-1, k, k+1 (OpRho4::faces).  A
// face shared by two cells is formed once: the three x faces inside the quad (rho_a + rho_b is
// the same sum in either order), and the z face below the plane, which is the face above the
// previous plane of the same march (carried in zc while zk records that plane).
struct SZCarry {
    float f[kVX];
    int k = -1;
};
__device__ __forceinline__ void s_faces(const STile& t, int k, int nz, const float* rm, const float* r0,
                                        const float* rp, float cx2, float cy2, float cz2, Faces (&F)[kVX],
                                        SZCarry& zc) {
    const V4 rc = sq(r0, t.ly, t.qx);
    const V4 rym = sq(r0, t.fym, t.qx), ryp = sq(r0, t.fyp, t.qx);
    const float rxm0 = ss(r0, t.ly, t.fxm), rxp3 = ss(r0, t.ly, t.fxp);
    float fx[kVX + 1];
    fx[0] = face_div(cx2, rc.v[0] + rxm0);
#pragma unroll
    for (int e = 1; e < kVX; ++e) fx[e] = face_div(cx2, rc.v[e - 1] + rc.v[e]);
    fx[kVX] = face_div(cx2, rc.v[kVX - 1] + rxp3);
    float fzm[kVX];
    if (k > 1 && zc.k == k - 1) {
#pragma unroll
        for (int e = 0; e < kVX; ++e) fzm[e] = zc.f[e];
    } else {
        const V4 rzm = sq((k > 1) ? rm : rp, t.ly, t.qx);
#pragma unroll
        for (int e = 0; e < kVX; ++e) fzm[e] = face_div(cz2, rc.v[e] + rzm.v[e]);
    }
    const V4 rzp = sq((k < nz) ? rp : rm, t.ly, t.qx);
#pragma unroll
    for (int e = 0; e < kVX; ++e) {
        const float r = rc.v[e];
        zc.f[e] = face_div(cz2, r + rzp.v[e]);
        F[e] = Faces{fx[e], fx[e + 1], face_div(cy2, r + rym.v[e]), face_div(cy2, r + ryp.v[e]), fzm[e], zc.f[e]};
    }
    zc.k = k;
}

// The plane engine.  NF fine fields with the halo, NO fine fields at the tile's own cells (box
// kSOBox) and NC coarse fields (the parent planes, box kSCBox) are loaded for every plane of the
// sequence.  body.begin() runs before the first wait, body.plane(k,
// sm, s0, sp) computes plane k from the slots (one pointer a field, fine then coarse) of the
// planes k-1, k, k+1, and body.finish() runs after a barrier that follows the last
// plane.  A scratch of 2 floats a thread (body.xbuf) follows the barriers.  The slot barriers
// are set up before the wait for the preceding kernel (griddepcontrol.wait), and the first
// planes' loads are issued before the solve's done flag is read, so neither waits on the
// other; a CTA that finds the solve done waits for those loads and leaves.  Returns -1 when the
// solve was done, 1 if a wait ran out, 0 otherwise.
template <int NF, int NO, int NC>
struct SSlots {
    const float* f[NF + NO + NC];   // fine fields with halo, own-cell fields, coarse fields
};
template <int NF, int NO, int NC, class Body>
__device__ __forceinline__ int s_march(const Geo& G, const BC& bc, const CUtensorMap* const (&maps)[NF + NO + NC],
                                       int chunk, Body& body, PCGState* st) {
    extern __shared__ __align__(128) unsigned char s_smem[];
    constexpr size_t kStage = (size_t)NF * kSSlotBytes + (size_t)NO * kSOSlotBytes + (size_t)NC * kSCSlotBytes;
    const int tid = threadIdx.x + kSTX * threadIdx.y;
    const int k0 = 1 + chunk * blockIdx.z;
    const int nplanes = min(chunk, G.nz - k0 + 1);
    const int nseq = nplanes + 2;   // planes k0 - 1 .. k0 + nplanes
    uint64_t* bars = reinterpret_cast<uint64_t*>(s_smem + kSR * kStage);
    body.xbuf = reinterpret_cast<float*>(bars + kSR);
    const int x0 = kBase - 1 + kSTileX * blockIdx.x - 3;        // x of cell 128 bx - 3: a multiple of 4
    const int y0 = kSTY * blockIdx.y;                            // row j_first - 1
    const int x0c = kBase - 1 + (kSTileX / 2) * blockIdx.x - 3;  // coarse cell 64 bx - 3
    const int y0c = (kSTY / 2) * blockIdx.y;                     // coarse row 4 by
    if (tid == 0) {
        for (int s = 0; s < kSR; ++s)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(s_addr(&bars[s])), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    pdl_wait();
    auto off = [](int f) -> size_t {   // byte offset of field f in a stage
        return f < NF ? (size_t)f * kSSlotBytes
                      : (f < NF + NO ? (size_t)NF * kSSlotBytes + (size_t)(f - NF) * kSOSlotBytes
                                     : (size_t)NF * kSSlotBytes + (size_t)NO * kSOSlotBytes + (size_t)(f - NF - NO) * kSCSlotBytes);
    };
    auto slot_at = [&](int sidx, int f) -> const float* {
        return reinterpret_cast<const float*>(s_smem + (size_t)sidx * kStage + off(f));
    };
    auto issue = [&](int q) {
        const int s = q % kSR;
        const uint32_t bar = s_addr(&bars[s]);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                     "r"(NF * kSBoxBytes + NO * kSOBoxBytes + NC * kSCBoxBytes)
                     : "memory");
        const int z = map_any(k0 - 1 + q, G.nz, bc.perz);
        unsigned char* b = s_smem + (size_t)s * kStage;
#pragma unroll
        for (int f = 0; f < NF; ++f) s_tma3(s_addr(b + off(f)), maps[f], x0, y0, z, bar);
#pragma unroll
        for (int f = NF; f < NF + NO; ++f) s_tma3(s_addr(b + off(f)), maps[f], x0 + 4, y0 + 1, z, bar);
#pragma unroll
        for (int f = NF + NO; f < NF + NO + NC; ++f) s_tma3(s_addr(b + off(f)), maps[f], x0c, y0c, (z + 1) >> 1, bar);
    };
    if (tid == 0)
        for (int q = 0; q < min(kSR, nseq); ++q) issue(q);
    if (st->done) {   // the same for every CTA: wait (bounded) for the issued loads, then leave
        if (tid == 0)
            for (int q = 0; q < min(kSR, nseq); ++q) s_wait(s_addr(&bars[q]), 0);
        __syncthreads();
        return -1;
    }
    body.begin(k0, nplanes);
    int sl0 = 0, sl1 = 1, sl2 = 2;   // ring slots of sequence m, m + 1, m + 2
    for (int m = 0; m < nplanes; ++m) {
        bool ok = true;
        if (m == 0) ok = s_wait(s_addr(&bars[0]), 0) && s_wait(s_addr(&bars[1]), 0);
        ok = ok && s_wait(s_addr(&bars[sl2]), ((m + 2) / kSR) & 1);
        if (__syncthreads_or(!ok)) {
            // wait (bounded) for the loads issued and not yet consumed, then give up
            if (tid == 0) {
                const int issued = (m == 0) ? min(kSR, nseq) : min(nseq, m - 1 + kSR);
                for (int q = m; q < issued; ++q) s_wait(s_addr(&bars[q % kSR]), (q / kSR) & 1);
                st->status = SULI_ERR_CUDA;
                st->done = 1;
            }
            __syncthreads();
            return 1;
        }
        // every thread is done with plane k0 + m - 2 (sequence m - 1): refill its slot
        if (tid == 0 && m >= 1 && m - 1 + kSR < nseq) issue(m - 1 + kSR);
        SSlots<NF, NO, NC> sm, s0, sp;
#pragma unroll
        for (int f = 0; f < NF + NO + NC; ++f) {
            sm.f[f] = slot_at(sl0, f);
            s0.f[f] = slot_at(sl1, f);
            sp.f[f] = slot_at(sl2, f);
        }
        body.plane(k0 + m, sm, s0, sp);
        sl0 = sl1;   // the ring's slots of sequence m + 1, m + 2, m + 3 for the next plane
        sl1 = sl2;
        sl2 = (sl2 + 1 == kSR) ? 0 : sl2 + 1;
    }
    __syncthreads();
    body.finish();
    return 0;
}

// Body members every body has: the thread's tile position and the march's scratch
struct SBase {
    STile t;
    int nz, pxy;
    float cx2, cy2, cz2;
    float* xbuf;
    SZCarry zc;
    __device__ __forceinline__ void init(const Geo& G, const float* c2) {
        t = s_tile(G);
        nz = G.nz;
        pxy = (int)G.pxy;
        cx2 = c2[0]; cy2 = c2[1]; cz2 = c2[2];
    }
    __device__ __forceinline__ void begin(int, int) {}
    __device__ __forceinline__ void finish() {}
};

// ---- two damped Jacobi sweeps from zero (k_mgv_pre on level 0): slots f, 1/diag, density
struct SPreBody : SBase {
    float omega, omega2;
    float* y;
    __device__ __forceinline__ void x1(const SSlots<3, 0, 0>& s, int ly, int lx, float (&o)[kVX]) const {
        const V4 fv = sq(s.f[0], ly, lx), dv = sq(s.f[1], ly, lx);
#pragma unroll
        for (int e = 0; e < kVX; ++e) o[e] = omega * fv.v[e] * dv.v[e];
    }
    __device__ __forceinline__ float x1s(const SSlots<3, 0, 0>& s, int ly, int lx) const {
        return omega * ss(s.f[0], ly, lx) * ss(s.f[1], ly, lx);
    }
    __device__ __forceinline__ void plane(int k, const SSlots<3, 0, 0>& sm, const SSlots<3, 0, 0>& s0, const SSlots<3, 0, 0>& sp) {
        if (!t.in) return;
        float zm[kVX], xc[kVX], zp[kVX], ym[kVX], yp[kVX], ax[kVX], out[kVX];
        x1(sm, t.ly, t.qx, zm);
        x1(s0, t.ly, t.qx, xc);
        x1(sp, t.ly, t.qx, zp);
        Faces F[kVX];
        s_faces(t, k, nz, sm.f[2], s0.f[2], sp.f[2], cx2, cy2, cz2, F, zc);
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
    SPreBody b;
    b.init(G, c2);
    b.omega = omega;
    b.omega2 = omega2;
    b.y = y;
    const CUtensorMap* const maps[3] = {&mf, &md, &mr};
    s_march<3, 0, 0>(G, bc, maps, chunk, b, st);
}

// ---- x_out = x_in + w (f - A x_in)/dg, f.x_out -> rz, beta (k_mgv_jacc on level 0, with the
// dot product): slots x_in, density with the halo; f, 1/diag at the tile's own cells
struct SJaccBody : SBase {
    float omega;
    float* xout;
    double dot;
    __device__ __forceinline__ void plane(int k, const SSlots<2, 2, 0>& sm, const SSlots<2, 2, 0>& s0,
                                          const SSlots<2, 2, 0>& sp) {
        if (!t.in) return;
        const V4 zm = sq(sm.f[0], t.ly, t.qx), xc = sq(s0.f[0], t.ly, t.qx), zp = sq(sp.f[0], t.ly, t.qx);
        Faces F[kVX];
        s_faces(t, k, nz, sm.f[1], s0.f[1], sp.f[1], cx2, cy2, cz2, F, zc);
        const V4 y1 = sq(s0.f[0], t.uym, t.qx), y2 = sq(s0.f[0], t.uyp, t.qx);
        float ax[kVX], out[kVX];
        apply4(F, xc.v, ss(s0.f[0], t.ly, t.uxm), ss(s0.f[0], t.ly, t.uxp), y1.v, y2.v, zm.v, zp.v, ax);
        const V4 fc = sqo(s0.f[2]), dc = sqo(s0.f[3]);
#pragma unroll
        for (int e = 0; e < kVX; ++e) {
            out[e] = xc.v[e] + omega * (fc.v[e] - ax[e]) * dc.v[e];
            dot += (double)fc.v[e] * (double)out[e];
        }
        st4(xout, t.c0 + pxy * k, out);
    }
};
__global__ void __launch_bounds__(kSTX * kSTY, 2) k_mgs_jacc(Geo G, BC bc, const __grid_constant__ CUtensorMap mx,
                                                          const __grid_constant__ CUtensorMap mr,
                                                          const __grid_constant__ CUtensorMap mf,
                                                          const __grid_constant__ CUtensorMap md, const float* c2,
                                                          float* xout, float omega, int chunk, PCGState* st,
                                                          double* partial, unsigned int* counter) {
    SJaccBody b;
    b.init(G, c2);
    b.omega = omega;
    b.xout = xout;
    b.dot = 0.;
    const CUtensorMap* const maps[4] = {&mx, &mr, &mf, &md};
    // every CTA joins the reduction, even one that gave up; none when the solve is done
    if (s_march<2, 2, 0>(G, bc, maps, chunk, b, st) < 0) return;
    double t, u;
    if (reduce2_last(b.dot, 0.0, partial, counter, t, u) && flat_tid() == 0) {
        const double rz_old = st->rz;
        st->rz = t;
        st->beta = (st->iters == 0) ? 0.0 : t / rz_old;
        if (!isfinite(t)) { st->status = SULI_ERR_NAN; st->done = 1; }
    }
}

// ---- p = z + beta p_old (also at the neighbours), q = A p, p.q -> alpha (k_pcgv_spmvc on level
// 0): slots z, p_old, density
struct SSpmvBody : SBase {
    float beta;
    const PCGState* pst;
    float *p_new, *qv;
    double dot;
    // beta comes from the preceding kernel: read after the march's griddepcontrol.wait
    __device__ __forceinline__ void begin(int, int) { beta = (float)pst->beta; }
    __device__ __forceinline__ void pn(const SSlots<3, 0, 0>& s, int ly, int lx, float (&o)[kVX]) const {
        const V4 a = sq(s.f[0], ly, lx), b = sq(s.f[1], ly, lx);
#pragma unroll
        for (int e = 0; e < kVX; ++e) o[e] = a.v[e] + beta * b.v[e];
    }
    __device__ __forceinline__ float pns(const SSlots<3, 0, 0>& s, int ly, int lx) const {
        return ss(s.f[0], ly, lx) + beta * ss(s.f[1], ly, lx);
    }
    __device__ __forceinline__ void plane(int k, const SSlots<3, 0, 0>& sm, const SSlots<3, 0, 0>& s0, const SSlots<3, 0, 0>& sp) {
        if (!t.in) return;
        float zm[kVX], xc[kVX], zp[kVX], ym[kVX], yp[kVX], ax[kVX];
        pn(sm, t.ly, t.qx, zm);
        pn(s0, t.ly, t.qx, xc);
        pn(sp, t.ly, t.qx, zp);
        Faces F[kVX];
        s_faces(t, k, nz, sm.f[2], s0.f[2], sp.f[2], cx2, cy2, cz2, F, zc);
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
    SSpmvBody b;
    b.init(G, c2);
    b.pst = st;
    b.p_new = p_new;
    b.qv = qv;
    b.dot = 0.;
    const CUtensorMap* const maps[3] = {&mz, &mp, &mr};
    // every CTA joins the reduction, even one that gave up; none when the solve is done
    if (s_march<3, 0, 0>(G, bc, maps, chunk, b, st) < 0) return;
    double t, u;
    if (reduce2_last(b.dot, 0.0, partial, counter, t, u) && flat_tid() == 0) {
        st->pq = t;
        st->alpha = st->rz / t;
        if (!isfinite(st->alpha)) { st->status = SULI_ERR_NAN; st->done = 1; }
    }
}

// ---- restriction f_c = (1/8) sum over the 8 children of (f - A x) (k_mgv_restrict on level
// 0): slots x, density with the halo; f at the tile's own cells.  A thread sums its quad's
// residuals over the two planes of a coarse plane (cells 0, 1 -> s0; 2, 3 -> s1, children in
// the order plane, cell); the thread of the odd row adds its row's sums to the even row's
// through the scratch.  The chunk is even and starts on an odd plane, so coarse planes never
// straddle two CTAs.
struct SRestrictBody : SBase {
    Geo Gc;
    float* fc;
    float s0, s1;
    int kpair;   // first fine plane of the pending coarse plane (0: none)
    __device__ __forceinline__ void begin(int, int) {
        s0 = 0.f;
        s1 = 0.f;
        kpair = 0;
    }
    // the pending coarse plane: rows of odd threads in the scratch, the even threads store
    __device__ __forceinline__ void flush() {
        if (kpair == 0) return;
        const int tid = threadIdx.x + kSTX * threadIdx.y;
        if (t.in && (threadIdx.y & 1) == 0) {
            const float a0 = s0 + xbuf[2 * (tid + kSTX)], a1 = s1 + xbuf[2 * (tid + kSTX) + 1];
            const int I0 = (t.i0 + 1) >> 1, J = (t.j + 1) >> 1, K = (kpair + 1) >> 1;
            fc[Gc.idx(I0, J, K)] = 0.125f * a0;
            if (I0 + 1 <= Gc.nx) fc[Gc.idx(I0 + 1, J, K)] = 0.125f * a1;
        }
        kpair = 0;
    }
    __device__ __forceinline__ void plane(int k, const SSlots<2, 1, 0>& sm, const SSlots<2, 1, 0>& s0s,
                                          const SSlots<2, 1, 0>& sp) {
        if ((k & 1) == 1) {   // first plane of a coarse plane: store the previous one (after the barrier)
            flush();
            s0 = 0.f;
            s1 = 0.f;
        }
        if (!t.in) return;
        const V4 zm = sq(sm.f[0], t.ly, t.qx), xc = sq(s0s.f[0], t.ly, t.qx), zp = sq(sp.f[0], t.ly, t.qx);
        Faces F[kVX];
        s_faces(t, k, nz, sm.f[1], s0s.f[1], sp.f[1], cx2, cy2, cz2, F, zc);
        const V4 y1 = sq(s0s.f[0], t.uym, t.qx), y2 = sq(s0s.f[0], t.uyp, t.qx);
        float ax[kVX];
        apply4(F, xc.v, ss(s0s.f[0], t.ly, t.uxm), ss(s0s.f[0], t.ly, t.uxp), y1.v, y2.v, zm.v, zp.v, ax);
        const V4 fv = sqo(s0s.f[2]);
        s0 += fv.v[0] - ax[0];
        s0 += fv.v[1] - ax[1];
        s1 += fv.v[2] - ax[2];
        s1 += fv.v[3] - ax[3];
        if ((k & 1) == 0) {   // second plane: the odd row publishes its sums
            kpair = k - 1;
            if (threadIdx.y & 1) {
                const int tid = threadIdx.x + kSTX * threadIdx.y;
                xbuf[2 * tid] = s0;
                xbuf[2 * tid + 1] = s1;
            }
        }
    }
    __device__ __forceinline__ void finish() { flush(); }
};
__global__ void __launch_bounds__(kSTX * kSTY, 2) k_mgs_restrict(Geo G, Geo Gc, BC bc,
                                                              const __grid_constant__ CUtensorMap mx,
                                                              const __grid_constant__ CUtensorMap mr,
                                                              const __grid_constant__ CUtensorMap mf, const float* c2,
                                                              float* fc, int chunk, PCGState* st) {
    SRestrictBody b;
    b.init(G, c2);
    b.Gc = Gc;
    b.fc = fc;
    const CUtensorMap* const maps[3] = {&mx, &mr, &mf};
    s_march<2, 1, 0>(G, bc, maps, chunk, b, st);
}

// ---- x_out = x' + w (f - A x')/dg with x' = y + a P xc (k_mgv_post on level 0): slots y,
// density with the halo, f and 1/diag at the tile's own cells, the coarse correction xc (parent
// planes).  A fine cell at tile column lx, row ly has its parent at coarse tile
// column lx/2 + 2, row (ly + 1)/2.
struct SPostBody : SBase {
    float omega, alpha;
    float* xout;
    // x' of the quad at tile row ly from the y slot and the coarse slot of its plane
    __device__ __forceinline__ void xq(const float* ys, const float* cs, int ly, float (&o)[kVX]) const {
        const V4 yv = sq(ys, ly, t.qx);
        const int cx = (t.qx >> 1) + 2, cy = (ly + 1) >> 1;
        const float p0 = alpha * ssc(cs, cy, cx), p1 = alpha * ssc(cs, cy, cx + 1);
        o[0] = yv.v[0] + p0; o[1] = yv.v[1] + p0; o[2] = yv.v[2] + p1; o[3] = yv.v[3] + p1;
    }
    __device__ __forceinline__ float xs(const float* ys, const float* cs, int ly, int lx) const {
        return ss(ys, ly, lx) + alpha * ssc(cs, (ly + 1) >> 1, (lx >> 1) + 2);
    }
    __device__ __forceinline__ void plane(int k, const SSlots<2, 2, 1>& sm, const SSlots<2, 2, 1>& s0,
                                          const SSlots<2, 2, 1>& sp) {
        if (!t.in) return;
        float zm[kVX], xc[kVX], zp[kVX], ym[kVX], yp[kVX], ax[kVX], out[kVX];
        xq(sm.f[0], sm.f[4], t.ly, zm);
        xq(s0.f[0], s0.f[4], t.ly, xc);
        xq(sp.f[0], sp.f[4], t.ly, zp);
        Faces F[kVX];
        s_faces(t, k, nz, sm.f[1], s0.f[1], sp.f[1], cx2, cy2, cz2, F, zc);
        xq(s0.f[0], s0.f[4], t.uym, ym);
        xq(s0.f[0], s0.f[4], t.uyp, yp);
        apply4(F, xc, xs(s0.f[0], s0.f[4], t.ly, t.uxm), xs(s0.f[0], s0.f[4], t.ly, t.uxp), ym, yp, zm, zp, ax);
        const V4 fc = sqo(s0.f[2]), dc = sqo(s0.f[3]);
#pragma unroll
        for (int e = 0; e < kVX; ++e) out[e] = xc[e] + omega * (fc.v[e] - ax[e]) * dc.v[e];
        st4(xout, t.c0 + pxy * k, out);
    }
};
__global__ void __launch_bounds__(kSTX * kSTY, 2) k_mgs_post(Geo G, BC bc, const __grid_constant__ CUtensorMap my,
                                                          const __grid_constant__ CUtensorMap mr,
                                                          const __grid_constant__ CUtensorMap mf,
                                                          const __grid_constant__ CUtensorMap md,
                                                          const __grid_constant__ CUtensorMap mc, const float* c2,
                                                          float* xout, float omega, float alpha, int chunk,
                                                          PCGState* st) {
    SPostBody b;
    b.init(G, c2);
    b.omega = omega;
    b.alpha = alpha;
    b.xout = xout;
    const CUtensorMap* const maps[5] = {&my, &mr, &mf, &md, &mc};
    s_march<2, 2, 1>(G, bc, maps, chunk, b, st);
}
static inline dim3 sgrid(const Geo& g, int chunk) {
    return dim3((g.nx + kSTileX - 1) / kSTileX, (g.ny + kSTY - 1) / kSTY, (g.nz + chunk - 1) / chunk);
}

}  // namespace suli
