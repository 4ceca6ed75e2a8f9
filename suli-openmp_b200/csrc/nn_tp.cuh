// nn_tp.cuh — the 3x3x3 convolution of nn_tc.cuh as a persistent, warp-specialised pipeline:
// TMA loads -> tcgen05.mma into tensor memory -> epilogue, each stage running ahead of the next.
//
// Work unit ("tile"): NZ consecutive z-planes of an 8 x 16 voxel column, one MMA tile
// (M = 128 voxels) per plane, exactly as k_conv3_tc.  A CTA runs on every SM (grid = min(tiles,
// SMs)) and walks the tiles t = blockIdx.x, blockIdx.x + gridDim.x, ...; neighbouring CTAs work
// on neighbouring tiles, so halo re-reads hit L2.
//
// Roles (448 threads):
//  * warps 0-3, producer.  For every (tile, 16-channel chunk) it fills one slot of an S-deep ring
//    in shared memory: the (NZ+2) x 18 x 10 input halo as two 8-channel planes, each one
//    cp.async.bulk.tensor 4-D TMA load of a box {8 channels, 10, 18, NZ+2} whose out-of-volume
//    part the TMA unit fills with zeros.  The box lands in exactly the K-major core-matrix layout
//    the MMA descriptors read ([hz][hy][hx] rows of 16 bytes).  The decoder's upsampled input
//    (half resolution, nearest neighbour) cannot be a TMA box; those chunks are gathered with
//    16-byte cp.async by the 128 producer threads, which arrive on the slot's mbarrier when their
//    copies land (cp.async.mbarrier.arrive.noinc).  The weights either stay resident (loaded once
//    per CTA, when the whole layer fits) or travel with each chunk (3-D TMA box {8, Cout, 27}).
//  * warps 4-5, MMA.  One thread of each waits for a full slot, issues the tcgen05.mma (kind::f16,
//    BF16 x BF16 -> FP32) of its half of the tile's z-planes into one of two TMEM accumulator
//    sets, and commits them to the slot's "empty" mbarrier (the producer may refill it once both
//    have) and, after a tile's last chunk, to the accumulator set's "full" mbarrier.  Two issuing
//    threads matter: one thread alone issues an MMA no faster than about every 54 cycles and
//    stalls the tensor pipe at each of its barrier waits; two keep it at the shared-memory bound.
//  * warps 6-13, epilogue: two warps per TMEM lane quadrant (warp w reads lanes 32 (w % 4) ..
//    + 31 with tcgen05.ld), splitting a tile's (plane, 16-channel block) items between them.  A
//    warp releases the accumulator set right after its last TMEM load of the tile, then adds the
//    bias (staged in shared memory), applies the ReLU and stores BF16.
// Every mbarrier wait is bounded; a wait that runs out sets *err and a shared abort flag, after
// which every role leaves its loop (their waits see the flag) and the CTA frees its TMEM.
//
// Tile geometry (template FOLD).  A tcgen05.mma with M = 128, K = 16 reads its whole A tile
// (4 KB) from shared memory, and measured on B200 it costs at least ~46 cycles however small N
// is; with N = Cout = 16 the tensor core would idle most of the time.
//  * FOLD = false: as k_conv3_tc; an 8 x 16 output tile per plane, 27 MMAs of N = Cout per plane
//    and chunk, the x shift dx moving the A start by dx rows.
//  * FOLD = true (Cout 16, 32): the three x taps ride in N.  The MMA rows are 16 x 8 INPUT voxels
//    (x0-1 .. x0+14), B for a (dy, dz) pair is the 3 Cout consecutive weight rows of taps
//    (0..2, dy, dz), so 9 MMAs of N = 3 Cout per plane and chunk produce, per input voxel,
//    P_dx = sum over (dy, dz, ci) of X W(dx).  The epilogue forms
//    out(x) = P_0(x-1) + P_1(x) + P_2(x+1) with two lane shuffles and keeps the 14 interior x of
//    each row (output tile 14 x 8).  Every A and B core matrix starts on a 128-byte boundary.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cstdint>
#include "nn_tc.cuh"

namespace suli {
namespace nn {

constexpr int TP_THREADS = 448;   // 4 producer warps, 2 MMA warps, 8 epilogue warps
constexpr int TP_EPI_WARP0 = 6;
constexpr int TP_TAIL_BYTES = 1280;   // mbarriers, TMEM slot, abort flag (256) + bias (<= 256 floats)
constexpr int TP_MAX_STAGES = 8;
constexpr int TP_HALO_ROW_BYTES = TC_HY * TC_RUN_BYTES;   // one z-plane of one 8-channel halo: 2880

template <bool FOLD>
struct TpGeo;
template <>
struct TpGeo<false> {
    static constexpr int HXR = TC_HX, HYR = TC_HY;   // halo rows of 16 bytes along x, runs along y
    static constexpr int OX = TCX, OY = TCY;         // output tile of one plane
    static constexpr int SBO = TC_RUN_BYTES;         // between core matrices along M (one x-run)
    static constexpr int MMAS = 27;                  // MMAs per plane and chunk
};
template <>
struct TpGeo<true> {
    static constexpr int HXR = 16, HYR = TCY / 2 + 2;
    static constexpr int OX = 14, OY = TCY / 2;
    static constexpr int SBO = 128;
    static constexpr int MMAS = 9;
};

// what the epilogue writes besides (or instead of) the BF16 activation
struct TpEpi {
    __nv_bfloat16* pool;   // 2x2x2 average of the BF16 output at half resolution (null: none)
    const float* head_w;   // 1x1x1 head, 16 weights + bias (null: none; Cout = 16 only)
    float* head_out;       // head output [V] FP32
    int store;             // 1: store the BF16 activation
};

struct TpCfg {
    int cout, tcols, nchunks;
    int ca, a_tma;        // channels of input A; 1: A is full resolution (TMA), 0: half resolution
    int stages, w_resident;
    int kc_bytes;         // one 8-channel halo plane, padded to 128 bytes
    int stage_bytes;      // 2 halo planes (+ the chunk's weights when they are not resident)
    int wchunk_bytes;     // weights of one chunk: 27 x Cout x 16 BF16
    int w_bytes;          // resident weights (0 if streamed)
    int tiles_x, tiles_y, tiles;
    int relu;
};

__device__ __forceinline__ void tp_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tp_arrive_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tp_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tp_cp_async_arrive(uint32_t bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}
// TMA tiled loads (no multicast), completion counted in bytes on an mbarrier
__device__ __forceinline__ void tp_tma4(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                        uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void tp_tma3(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

// bounded wait on a phase parity; gives up when another role has aborted
__device__ __forceinline__ bool tp_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
    for (int it = 0; it < (1 << 22); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 31) == 31 && *abort_flag) return false;
    }
    *abort_flag = 1;
    return false;
}

template <int NZ, bool FOLD>
__global__ void __launch_bounds__(TP_THREADS, 1)
    k_conv3_tp(Vol vol, ConvIn in, const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
               const __grid_constant__ CUtensorMap map_w, const float* __restrict__ bias, TpCfg cfg, TpEpi epi,
               __nv_bfloat16* __restrict__ out, int* err) {
    using G = TpGeo<FOLD>;
    constexpr int RUN = G::HXR * 16;   // bytes of one x-run of the halo
    extern __shared__ __align__(1024) unsigned char smem_tp[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int S = cfg.stages;
    unsigned char* wres = smem_tp;
    unsigned char* ring = smem_tp + cfg.w_bytes;
    uint64_t* bars = reinterpret_cast<uint64_t*>(ring + S * cfg.stage_bytes);
    // bars: full[S] | empty[S] | tfull[2] | tempty[2] | wbar | dbar[2] (each MMA thread's last commit)
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * TP_MAX_STAGES + 7);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    float* sbias = reinterpret_cast<float*>(reinterpret_cast<unsigned char*>(bars) + 256);
    const uint32_t bar0 = smem_u32(bars);
    auto full = [&](int s) { return bar0 + 8u * (uint32_t)s; };
    auto empty = [&](int s) { return bar0 + 8u * (uint32_t)(TP_MAX_STAGES + s); };
    auto tfull = [&](int a) { return bar0 + 8u * (uint32_t)(2 * TP_MAX_STAGES + a); };
    auto tempty = [&](int a) { return bar0 + 8u * (uint32_t)(2 * TP_MAX_STAGES + 2 + a); };
    const uint32_t wbar = bar0 + 8u * (uint32_t)(2 * TP_MAX_STAGES + 4);
    const uint32_t dbar0 = bar0 + 8u * (uint32_t)(2 * TP_MAX_STAGES + 5);
    const int acc_cols = NZ * cfg.tcols;   // one accumulator set
    constexpr int NMMA = NZ >= 2 ? 2 : 1;  // issuing MMA warps (one per half of the planes)

    if (warp == 4) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(2 * acc_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            // slots filled by cp.async gathers need all 128 producer threads; TMA-only layers one
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(full(s)), "r"(cfg.a_tma ? 1 : 128));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(empty(s)), "r"(NMMA));
        }
        for (int a = 0; a < 2; ++a) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tfull(a)), "r"(NMMA));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tempty(a)), "r"(256));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(wbar), "r"(1));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(dbar0), "r"(1));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(dbar0 + 8u), "r"(1));
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_w)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_b)) : "memory");
        if (cfg.a_tma) asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&map_a)) : "memory");
    }
    for (int i = tid; i < cfg.cout; i += TP_THREADS) sbias[i] = bias ? bias[i] : 0.f;
    if (epi.head_w && tid < 17) sbias[cfg.cout + tid] = epi.head_w[tid];
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tmem_slot;
    const int txy = cfg.tiles_x * cfg.tiles_y;
    const int nch = cfg.nchunks;
    const uint32_t ring_u = smem_u32(ring), wres_u = smem_u32(wres);
    const uint32_t wplane = (uint32_t)(27 * cfg.cout * 16);   // one 8-channel plane of a chunk's weights

    if (warp < 4) {
        // ------------------------------------------------------------------ producer
        // (TMA-only layers: thread 0 alone; layers with a half-resolution input: all 128 threads)
        if (tid == 0 && cfg.w_resident) {
            tp_arrive_tx(wbar, (uint32_t)cfg.w_bytes);
            for (int ch = 0; ch < nch; ++ch)
                for (int kc = 0; kc < 2; ++kc)
                    tp_tma3(wres_u + (uint32_t)(ch * cfg.wchunk_bytes) + kc * wplane, &map_w, ch * TC_CC + 8 * kc, 0, 0,
                            wbar);
        }
        const uint32_t halo_tx = 2u * (uint32_t)(RUN * G::HYR * (NZ + 2));
        const int hxn = (vol.nx + 1) / 2, hyn = (vol.ny + 1) / 2;
        int g = 0;
        bool ok = true;
        const bool producing = !cfg.a_tma || tid == 0;
        for (int t = blockIdx.x; t < cfg.tiles && ok && producing; t += gridDim.x) {
            const int bz = t / txy, rem = t - bz * txy, by = rem / cfg.tiles_x, bx = rem - by * cfg.tiles_x;
            const int x0 = bx * G::OX, y0 = by * G::OY, z0 = bz * NZ;
            for (int ch = 0; ch < nch; ++ch, ++g) {
                const int s = g % S, n = g / S;
                if (n > 0 && !tp_wait(empty(s), (uint32_t)((n - 1) & 1), abort_flag)) { ok = false; break; }
                const uint32_t dst = ring_u + (uint32_t)(s * cfg.stage_bytes);
                const uint32_t wdst = dst + 2u * (uint32_t)cfg.kc_bytes;
                const int c0 = ch * TC_CC;
                if (c0 < cfg.ca && !cfg.a_tma) {
                    // half-resolution input: gathered with cp.async (nearest-neighbour upsampling)
                    if (tid == 0 && !cfg.w_resident) {
                        tp_expect_tx(full(s), (uint32_t)cfg.wchunk_bytes);
                        tp_tma3(wdst, &map_w, c0, 0, 0, full(s));
                        tp_tma3(wdst + wplane, &map_w, c0 + 8, 0, 0, full(s));
                    }
                    // a thread copies the rows h = (tid >> 1) + 64 m of 8-channel plane kc = tid & 1;
                    // its (hx, hy, hz) advance by the constant step of 64 rows (no division per row)
                    constexpr int NH = G::HXR * G::HYR * (NZ + 2);
                    constexpr int DX = 64 % G::HXR, DY = (64 / G::HXR) % G::HYR, DZ = 64 / (G::HXR * G::HYR);
                    const int kc = tid & 1, h0 = tid >> 1;
                    int hx = h0 % G::HXR, hy = (h0 / G::HXR) % G::HYR, hz = h0 / (G::HXR * G::HYR);
                    const __nv_bfloat16* abase = in.a + c0 + kc * 8;
                    const uint32_t dbase = dst + (uint32_t)(kc * cfg.kc_bytes);
                    for (int h = h0; h < NH; h += 64) {
                        const int gx = x0 + hx - 1, gy = y0 + hy - 1, gz = z0 + hz - 1;
                        const void* src = in.a;
                        int bytes = 0;
                        if (gx >= 0 && gx < vol.nx && gy >= 0 && gy < vol.ny && gz >= 0 && gz < vol.nz) {
                            const long long vi =
                                (long long)(gx >> 1) + hxn * ((long long)(gy >> 1) + (long long)hyn * (gz >> 1));
                            src = abase + vi * in.ca;
                            bytes = 16;
                        }
                        cp_async16(dbase + (uint32_t)((hz * G::HYR + hy) * RUN + hx * 16), src, bytes);
                        hx += DX;
                        const int cy = (hx >= G::HXR) ? 1 : 0;
                        hx -= cy * G::HXR;
                        hy += DY + cy;
                        const int cz = (hy >= G::HYR) ? 1 : 0;
                        hy -= cz * G::HYR;
                        hz += DZ + cz;
                    }
                    tp_cp_async_arrive(full(s));
                } else if (tid == 0) {
                    const bool fa = c0 < cfg.ca;
                    const CUtensorMap* m = fa ? &map_a : &map_b;
                    const int cl = fa ? c0 : c0 - cfg.ca;
                    tp_arrive_tx(full(s), halo_tx + (cfg.w_resident ? 0u : (uint32_t)cfg.wchunk_bytes));
                    tp_tma4(dst, m, cl, x0 - 1, y0 - 1, z0 - 1, full(s));
                    tp_tma4(dst + (uint32_t)cfg.kc_bytes, m, cl + 8, x0 - 1, y0 - 1, z0 - 1, full(s));
                    if (!cfg.w_resident) {
                        tp_tma3(wdst, &map_w, c0, 0, 0, full(s));
                        tp_tma3(wdst + wplane, &map_w, c0 + 8, 0, 0, full(s));
                    }
                } else {
                    tp_arrive(full(s));
                }
            }
        }
        // drain: the slots' last refills must be consumed before the CTA's shared memory goes away
        asm volatile("cp.async.wait_all;" ::: "memory");
        if (ok && producing) {
            for (int g2 = (g > S ? g - S : 0); g2 < g; ++g2)
                if (!tp_wait(empty(g2 % S), (uint32_t)((g2 / S) & 1), abort_flag)) break;
        }
    } else if (warp < TP_EPI_WARP0) {
        // ------------------------------------------------------------------ MMA issuers
        const int mw = warp - 4;
        if (lane == 0 && mw < NMMA) {
            const uint32_t idesc = tc_idesc(FOLD ? 3 * cfg.cout : cfg.cout);
            const int ng = cfg.cout / 8;
            const uint32_t dbar = dbar0 + 8u * (uint32_t)mw;
            constexpr int NP = NZ / NMMA;   // planes of this issuer
            const int sz0 = mw * NP;
            bool ok = !cfg.w_resident || tp_wait(wbar, 0u, abort_flag);
            int g = 0, it = 0;
            for (int t = blockIdx.x; t < cfg.tiles && ok; t += gridDim.x, ++it) {
                const int a = it & 1;
                if (it >= 2 && !tp_wait(tempty(a), (uint32_t)(((it >> 1) - 1) & 1), abort_flag)) { ok = false; break; }
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t dacc = tmem + (uint32_t)(a * acc_cols);
                for (int ch = 0; ch < nch; ++ch, ++g) {
                    const int s = g % S, n = g / S;
                    if (!tp_wait(full(s), (uint32_t)(n & 1), abort_flag)) { ok = false; break; }
                    // cp.async-filled slots: make the generic-proxy writes visible to the tensor core
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    asm volatile("tcgen05.fence::after_thread_sync;");
                    const uint32_t hb = ring_u + (uint32_t)(s * cfg.stage_bytes);
                    const uint32_t wb = cfg.w_resident ? wres_u + (uint32_t)(ch * cfg.wchunk_bytes)
                                                       : hb + 2u * (uint32_t)cfg.kc_bytes;
                    const uint64_t a0 = tc_desc(hb, (uint32_t)cfg.kc_bytes, G::SBO);
                    const uint64_t b0 = tc_desc(wb, wplane, 128);
#pragma unroll
                    for (int p = 0; p < NP; ++p) {
                        const int sz = sz0 + p;
                        const uint32_t d = dacc + (uint32_t)(sz * cfg.tcols);
#pragma unroll
                        for (int k = 0; k < G::MMAS; ++k) {
                            // FOLD: k = dy + 3 dz, B = taps (0..2, dy, dz); else k = tap = dx + 3 dy + 9 dz
                            const int dx = FOLD ? 0 : k % 3, dy = FOLD ? k % 3 : (k / 3) % 3, dz = FOLD ? k / 3 : k / 9;
                            const int tap0 = FOLD ? 3 * k : k;
                            const uint32_t aoff = (uint32_t)((((sz + dz) * G::HYR + dy) * RUN + dx * 16) >> 4);
                            const uint32_t boff = (uint32_t)((tap0 * ng * 128) >> 4);
                            tc_mma(d, a0 + aoff, b0 + boff, idesc, (ch > 0 || k > 0) ? 1u : 0u);
                        }
                    }
                    tc_commit(empty(s));
                    if (ch == nch - 1) tc_commit(tfull(a));
                }
            }
            // every MMA issued above has completed before the accumulators are freed
            tc_commit(dbar);
            mbar_wait_bounded(dbar, 0u);
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------------------ epilogue
        const int q = warp & 3;                       // TMEM lane quadrant of this warp
        const int half = (warp - TP_EPI_WARP0) >> 2;  // which of the two warps of the quadrant
        const int m = q * 32 + lane;
        // row m of the accumulator: FOLD: input voxel (hx, ty) = (m % 16, m / 16), output x = hx - 1
        // for hx in 1..14; else output voxel (m % 8, m / 8)
        const int rx = FOLD ? (m & 15) - 1 : (m & 7), ry = FOLD ? (m >> 4) : (m >> 3);
        const bool row_ok = !FOLD || (rx >= 0 && rx < G::OX);
        // A warp's work unit is (pair of z-planes, 16-channel block): both planes of a 2x2x2
        // pooling block stay in one warp.  x / y neighbours of the pooling block are lanes +DX, +DY.
        constexpr int ZU = NZ >= 2 ? 2 : 1;
        constexpr int DX = 1, DY = FOLD ? 16 : 8;
        const int ncb = cfg.cout / 16, nunits = (NZ / ZU) * ncb;
        constexpr int LD = FOLD ? 3 : 1;   // 16-column TMEM loads per (plane, block)
        const bool pool_lead = ((FOLD ? rx : (m & 7)) & 1) == 0 && (ry & 1) == 0 && row_ok;
        const int pcx = vol.nx / 2, pcy = vol.ny / 2;
        int it = 0;
        for (int t = blockIdx.x; t < cfg.tiles; t += gridDim.x, ++it) {
            const int a = it & 1;
            // one lane polls, the warp follows (tcgen05.ld is warp-collective)
            bool okw = true;
            if (lane == 0) okw = tp_wait(tfull(a), (uint32_t)((it >> 1) & 1), abort_flag);
            __syncwarp();
            if (!__shfl_sync(0xffffffffu, okw, 0)) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            const int bz = t / txy, rem = t - bz * txy, by = rem / cfg.tiles_x, bx = rem - by * cfg.tiles_x;
            const int ox = bx * G::OX + rx, oy = by * G::OY + ry;
            const bool in_xy = row_ok && ox < vol.nx && oy < vol.ny;
            const uint32_t colq = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(a * acc_cols);
            for (int u = half; u < nunits; u += 2) {
                const int zp = u / ncb, cb = (u - zp * ncb) * 16;
                float pacc[16];   // pooling: the first plane's four values, summed in k_pool's order
#pragma unroll
                for (int zz = 0; zz < ZU; ++zz) {
                    const int sz = zp * ZU + zz;
                    uint32_t r[LD][16];
#pragma unroll
                    for (int l = 0; l < LD; ++l) tc_ld16(colq + (uint32_t)(sz * cfg.tcols + l * cfg.cout + cb), r[l]);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    if (u + 2 >= nunits && zz == ZU - 1) {
                        // last TMEM read of this tile: hand the accumulator set back to the MMA warps
                        asm volatile("tcgen05.fence::before_thread_sync;");
                        tp_arrive(tempty(a));
                    }
                    const int oz = bz * NZ + sz;
                    const bool inside = in_xy && oz < vol.nz;
                    float v[16];
                    if (FOLD) {
#pragma unroll
                        for (int e = 0; e < 16; ++e) {
                            const float pm = __shfl_up_sync(0xffffffffu, __uint_as_float(r[0][e]), 1);
                            const float pp = __shfl_down_sync(0xffffffffu, __uint_as_float(r[LD - 1][e]), 1);
                            v[e] = (pm + __uint_as_float(r[LD > 1 ? 1 : 0][e])) + pp;
                        }
                    } else {
#pragma unroll
                        for (int e = 0; e < 16; ++e) v[e] = __uint_as_float(r[0][e]);
                    }
                    // bias, ReLU, BF16 rounding; rv = the rounded values as the next layer reads them
                    uint32_t packed[8];
                    float rv[16];
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const float2 b2 = reinterpret_cast<const float2*>(sbias + cb)[e];
                        float v0 = v[2 * e] + b2.x, v1 = v[2 * e + 1] + b2.y;
                        if (cfg.relu) { v0 = fmaxf(v0, 0.f); v1 = fmaxf(v1, 0.f); }
                        const __nv_bfloat162 h2 = __floats2bfloat162_rn(v0, v1);
                        packed[e] = *reinterpret_cast<const uint32_t*>(&h2);
                        rv[2 * e] = __low2float(h2);
                        rv[2 * e + 1] = __high2float(h2);
                    }
                    const long long vo = (long long)ox + vol.nx * ((long long)oy + (long long)vol.ny * oz);
                    if (inside && epi.store) {
                        uint4* o = reinterpret_cast<uint4*>(out + vo * cfg.cout + cb);
                        o[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
                        o[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
                    }
                    if (epi.head_out && inside) {
                        // 1x1x1 head on the BF16 activations (Cout = 16), k_head_fwd's order
                        float hs = sbias[cfg.cout + 16];
#pragma unroll
                        for (int e = 0; e < 16; ++e) hs += sbias[cfg.cout + e] * rv[e];
                        epi.head_out[vo] = hs;
                    }
                    if (epi.pool) {
                        // 2x2x2 average: (x0,y0), (x1,y0), (x0,y1), (x1,y1) of plane z0, then of z1
#pragma unroll
                        for (int e = 0; e < 16; ++e) {
                            const float n1 = __shfl_down_sync(0xffffffffu, rv[e], DX);
                            const float n2 = __shfl_down_sync(0xffffffffu, rv[e], DY);
                            const float n3 = __shfl_down_sync(0xffffffffu, rv[e], DX + DY);
                            if (zz == 0) {
                                pacc[e] = ((rv[e] + n1) + n2) + n3;
                            } else {
                                float sum = pacc[e];
                                sum += rv[e];
                                sum += n1;
                                sum += n2;
                                sum += n3;
                                pacc[e] = 0.125f * sum;
                            }
                        }
                        if (zz == ZU - 1 && pool_lead && inside) {
                            const long long pv =
                                (long long)(ox >> 1) + pcx * ((long long)(oy >> 1) + (long long)pcy * (oz >> 1));
                            uint32_t pk[8];
#pragma unroll
                            for (int e = 0; e < 8; ++e) {
                                const __nv_bfloat162 h2 = __floats2bfloat162_rn(pacc[2 * e], pacc[2 * e + 1]);
                                pk[e] = *reinterpret_cast<const uint32_t*>(&h2);
                            }
                            uint4* o = reinterpret_cast<uint4*>(epi.pool + pv * cfg.cout + cb);
                            o[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                            o[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
                        }
                    }
                }
            }
            if (half >= nunits) {
                // no unit in this tile for this warp
                asm volatile("tcgen05.fence::before_thread_sync;");
                tp_arrive(tempty(a));
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (tid == 0 && *abort_flag) atomicExch(err, 1);
    if (warp == 4)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * acc_cols));
}

}  // namespace nn
}  // namespace suli
