// nn_tc.cuh — 3x3x3 convolution of channels-last BF16 volumes on the 5th-generation tensor
// cores: tcgen05.mma (kind::f16, BF16 x BF16 -> FP32) with the accumulator in tensor memory.
//
// GEMM view (as nn_conv.cuh): out[v][co] = sum_{tap, ci} X[v + off(tap)][ci] W[tap][co][ci].
// A CTA (128 threads) owns an 8 x 16 x 1 tile of output voxels: M = 128 rows of the MMA, row
// m = tx + 8 ty, so row group m/8 is one x-run of 8 voxels at height ty.  N = Cout (16..160),
// the accumulator D[128][Cout] FP32 lives in TMEM (lane m, column co).  K runs over channel
// chunks of 16 (one MMA K-step) and the 27 taps.
//
// Shared-memory operands use the canonical K-major layout without swizzle: "core matrices" of
// 8 rows x 16 bytes (8 BF16 of K), 128 contiguous bytes each; the descriptor gives the byte
// distance between core matrices along K (LBO) and along M/N (SBO).
//  * Input halo (10 x 18 x 3 voxels) of the current 16-channel chunk, as [kc][hz][hy][hx] rows
//    of 16 bytes (kc = channels 0-7 / 8-15).  For tap (dx, dy, dz) the core matrix of row
//    group ty is the 8 consecutive rows hx = dx..dx+7 at (hz = dz, hy = ty + dy): it starts
//    dx rows into the x-run, SBO = one x-run (160 bytes), LBO = one kc plane (8640 bytes).
//    So one copy of the halo serves all 27 taps.
//  * Weights of the chunk for all 27 taps: core matrix (tap, co/8, ci/8); SBO = 256 bytes
//    between groups of 8 output channels, LBO = 128 bytes.
// Both are copied global -> shared with cp.async (16 bytes each, zero-filled outside the
// volume), no register staging.
// One thread issues the 27 MMAs of a chunk and commits them to an mbarrier; all threads wait on
// it (bounded) before the buffers are restaged.  The epilogue reads TMEM with tcgen05.ld
// (warp w owns lanes 32w..32w+31), adds the bias, applies the ReLU and stores BF16.
//
// Every wait is bounded: a timed-out wait sets *err and the CTA skips its output.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>
#include "nn_conv.cuh"

namespace suli {
namespace nn {

constexpr int TCX = 8, TCY = 16;                // one MMA tile: 8 x 16 voxels of a z-plane
constexpr int TC_HX = TCX + 2, TC_HY = TCY + 2;
constexpr int TC_CC = 16;                       // channels per K chunk
constexpr int TC_RUN_BYTES = TC_HX * 16;        // one x-run of 10 rows: 160

// A CTA owns NZ consecutive z-planes of an 8 x 16 column (NZ MMA tiles, NZ accumulators):
// the halo has NZ + 2 planes and the weights are staged once for all of them.
template <int NZ>
struct TcTile {
    static constexpr int HZ = NZ + 2;
    static constexpr int KC_BYTES = HZ * TC_HY * TC_RUN_BYTES;   // one 8-channel plane of the halo
    static constexpr int HALO_BYTES = 2 * KC_BYTES;
};
__host__ __device__ constexpr int tc_weight_bytes(int cout) { return 27 * cout * TC_CC * 2; }
template <int NZ>
__host__ __device__ constexpr int tc_smem_bytes(int cout) {
    return TcTile<NZ>::HALO_BYTES + tc_weight_bytes(cout) + 128;
}

__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;    // descriptor version for sm_100
    // base offset 0, LBO mode 0, layout type 0 = no swizzle
    return d;
}

// instruction descriptor, kind::f16: D F32, A and B BF16, both K-major, N, M = 128
__host__ __device__ constexpr uint32_t tc_idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(dtmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(phase)
        : "memory");
    return ok != 0;
}

// bounded wait on an mbarrier phase; false if it did not complete
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mbar, uint32_t phase) {
    for (int it = 0; it < (1 << 24); ++it)
        if (mbar_try_wait(mbar, phase)) return true;
    return false;
}

// 16-byte global -> shared copy; src_bytes = 0 fills zeros
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// Forward 3x3x3 convolution on the tensor cores.  Same operands as k_conv3_fwd; Cout in
// {16, 32, 48, 64, 96, 160}, Cin a multiple of 16.  `tcols` = TMEM columns of one accumulator
// (a power of two >= max(32, Cout)); the CTA allocates NZ of them.  Grid (ceil(nx/8),
// ceil(ny/16), ceil(nz/NZ)), 128 threads.
template <int NZ>
__global__ void __launch_bounds__(128) k_conv3_tc(Vol vol, ConvIn in, const __nv_bfloat16* __restrict__ W,
                                                  const float* __restrict__ bias, int relu, int cout, int tcols,
                                                  __nv_bfloat16* __restrict__ out, int* err) {
    using T = TcTile<NZ>;
    extern __shared__ __align__(1024) unsigned char smem_tc[];
    unsigned char* halo = smem_tc;
    unsigned char* wsm = smem_tc + T::HALO_BYTES;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(wsm + tc_weight_bytes(cout));
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(wsm + tc_weight_bytes(cout) + 64);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int cin = in.ca + in.cb;
    const int x0 = blockIdx.x * TCX, y0 = blockIdx.y * TCY, z0 = blockIdx.z * NZ;
    const uint32_t mbar_a = smem_u32(mbar);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(NZ * tcols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar_a), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tmem_slot;
    const uint32_t idesc = tc_idesc(cout);
    const int hxn = (vol.nx + 1) / 2, hyn = (vol.ny + 1) / 2;
    const int nchunks = cin / TC_CC;
    const int ng = cout / 8;
    const uint32_t hbase = smem_u32(halo), wbase = smem_u32(wsm);
    bool ok = true;
    uint32_t phase = 0;

    for (int ch = 0; ch < nchunks && ok; ++ch) {
        const int c0 = ch * TC_CC;
        // ---- halo of channels c0..c0+15: 10 x 18 x (NZ+2) voxels x 2 rows of 8 channels
        for (int q = tid; q < TC_HX * TC_HY * T::HZ * 2; q += 128) {
            const int kc = q & 1, h = q >> 1;
            const int hx = h % TC_HX, hy = (h / TC_HX) % TC_HY, hz = h / (TC_HX * TC_HY);
            const int gx = x0 + hx - 1, gy = y0 + hy - 1, gz = z0 + hz - 1;
            const void* src = in.a;
            int bytes = 0;
            if (gx >= 0 && gx < vol.nx && gy >= 0 && gy < vol.ny && gz >= 0 && gz < vol.nz) {
                const int c = c0 + kc * 8;
                bytes = 16;
                if (c < in.ca) {
                    const long long vi = in.a_half
                        ? (long long)(gx >> 1) + hxn * ((long long)(gy >> 1) + (long long)hyn * (gz >> 1))
                        : (long long)gx + vol.nx * ((long long)gy + (long long)vol.ny * gz);
                    src = in.a + vi * in.ca + c;
                } else {
                    const long long vi = (long long)gx + vol.nx * ((long long)gy + (long long)vol.ny * gz);
                    src = in.b + vi * in.cb + (c - in.ca);
                }
            }
            cp_async16(hbase + kc * T::KC_BYTES + (hz * TC_HY + hy) * TC_RUN_BYTES + hx * 16, src, bytes);
        }
        // ---- weights of the chunk: core matrix (tap, co/8, kc), row co%8, 16 bytes
        for (int q = tid; q < 27 * cout * 2; q += 128) {
            const int kc = q & 1, row = q >> 1;   // row = tap * cout + co
            const int tap = row / cout, co = row - tap * cout;
            cp_async16(wbase + (((tap * ng + (co >> 3)) * 2 + kc) * 8 + (co & 7)) * 16,
                       W + ((long long)tap * cout + co) * cin + c0 + kc * 8, 16);
        }
        asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
        // completed copies -> visible to the tensor core (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (tid == 0) {
            // descriptors differ per tap only in their start address (field in 16-byte units)
            const uint64_t a0 = tc_desc(hbase, T::KC_BYTES, TC_RUN_BYTES);
            const uint64_t b0 = tc_desc(wbase, 128, 256);
#pragma unroll
            for (int s = 0; s < NZ; ++s) {
                const uint32_t d = tmem + (uint32_t)(s * tcols);
#pragma unroll
                for (int tap = 0; tap < 27; ++tap) {
                    const int dx = tap % 3, dy = (tap / 3) % 3, dz = tap / 9;
                    const uint32_t aoff = (uint32_t)((((s + dz) * TC_HY + dy) * TC_RUN_BYTES + dx * 16) >> 4);
                    const uint32_t boff = (uint32_t)((tap * ng * 256) >> 4);
                    tc_mma(d, a0 + aoff, b0 + boff, idesc, (ch > 0 || tap > 0) ? 1u : 0u);
                }
            }
            tc_commit(mbar_a);
        }
        __syncwarp();
        ok = mbar_wait_bounded(mbar_a, phase);
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        ok = __syncthreads_and(ok);   // uniform; the next chunk overwrites the operands
    }
    if (!ok) {
        if (tid == 0) atomicExch(err, 1);
    } else {
        // ---- epilogue: row m = 32 warp + lane <-> voxel (m % 8, m / 8) of plane z0 + s
        const int m = warp * 32 + lane;
        const int ox = x0 + (m & 7), oy = y0 + (m >> 3);
#pragma unroll
        for (int s = 0; s < NZ; ++s) {
            const int oz = z0 + s;
            const bool store = ox < vol.nx && oy < vol.ny && oz < vol.nz;
            const long long vo = (long long)ox + vol.nx * ((long long)oy + (long long)vol.ny * oz);
            for (int cb = 0; cb < cout; cb += 16) {
                uint32_t r[16];
                tc_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(s * tcols + cb), r);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (store) {
                    uint32_t packed[8];
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        float v0 = __uint_as_float(r[2 * e]), v1 = __uint_as_float(r[2 * e + 1]);
                        if (bias) { v0 += bias[cb + 2 * e]; v1 += bias[cb + 2 * e + 1]; }
                        if (relu) { v0 = fmaxf(v0, 0.f); v1 = fmaxf(v1, 0.f); }
                        const __nv_bfloat162 b2 = __floats2bfloat162_rn(v0, v1);
                        packed[e] = *reinterpret_cast<const uint32_t*>(&b2);
                    }
                    uint4* dst = reinterpret_cast<uint4*>(out + vo * cout + cb);
                    dst[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
                    dst[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NZ * tcols));
}

}  // namespace nn
}  // namespace suli
