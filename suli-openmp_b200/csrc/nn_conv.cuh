// nn_conv.cuh — 3x3x3 convolution of channels-last BF16 volumes as an implicit GEMM on the
// tensor cores (mma.sync m16n8k16, BF16 inputs, FP32 accumulation).
//
// GEMM view: out[v][co] = sum_{tap, ci} X[v + tap][ci] * W[tap][co][ci] (+ bias, ReLU).
//   M = output voxels (a CTA owns an 8 x 4 x 4 tile = 128 voxels, 16 per warp),
//   N = Cout (NF fragments of 8), K = 27 taps x Cin (16 per step).
// The CTA stages its 10 x 6 x 6 input halo in shared memory once; each K step loads the A
// fragment of its 16 voxels at the tap's offset with ldmatrix (rows padded by 16 bytes so the
// 8 row addresses of a phase hit distinct banks) and the B fragments straight from the weight
// array (L1-resident: every CTA reads the same weights).  Zero padding outside the volume.
// The input may be the channel concatenation of a half-resolution tensor A (read with
// nearest-neighbour upsampling) and a full-resolution tensor B: the U-Net decoder's
// "upsample, concatenate the skip" costs no extra pass.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace suli {
namespace nn {

constexpr int TX = 8, TY = 4, TZ = 4;                 // output tile of a CTA (128 voxels)
constexpr int HX = TX + 2, HY = TY + 2, HZ = TZ + 2;   // input halo tile
constexpr int HVOX = HX * HY * HZ;                     // 360

struct Vol {
    int nx, ny, nz;
};
struct ConvIn {
    const __nv_bfloat16* a;   // channels [0, ca)
    int ca;
    int a_half;               // 1: A has half the resolution (nearest upsampling)
    const __nv_bfloat16* b;   // channels [ca, ca + cb), full resolution (may be null if cb = 0)
    int cb;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void ldmatrix_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}

// Conv forward.  W: [27][Cout][Cin] BF16 (tap = dx + 3 dy + 9 dz), bias: [Cout] FP32 (or null).
// out: [V][Cout] BF16 (channels last, V = nx ny nz, x fastest).  Cout = 8 NF, Cin % 16 == 0.
template <int NF>
__global__ void __launch_bounds__(256) k_conv3_fwd(Vol vol, ConvIn in, const __nv_bfloat16* __restrict__ W,
                                                   const float* __restrict__ bias, int relu,
                                                   __nv_bfloat16* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int cin = in.ca + in.cb;
    const int rs = cin * 2 + 16;   // padded row stride in bytes
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY, z0 = blockIdx.z * TZ;
    const int tid = threadIdx.x;
    // ---- stage the halo tile (16-byte vectors; zero outside the volume)
    const int vec_per_vox = cin / 8;
    for (int q = tid; q < HVOX * vec_per_vox; q += 256) {
        const int h = q / vec_per_vox, vq = q - h * vec_per_vox;
        const int hx = h % HX, hy = (h / HX) % HY, hz = h / (HX * HY);
        const int gx = x0 + hx - 1, gy = y0 + hy - 1, gz = z0 + hz - 1;
        uint4 val = make_uint4(0u, 0u, 0u, 0u);
        if (gx >= 0 && gx < vol.nx && gy >= 0 && gy < vol.ny && gz >= 0 && gz < vol.nz) {
            const int ch = vq * 8;
            if (ch < in.ca) {
                long long vi;
                if (in.a_half) {
                    const int hxn = (vol.nx + 1) / 2, hyn = (vol.ny + 1) / 2;
                    vi = (long long)(gx >> 1) + hxn * ((long long)(gy >> 1) + (long long)hyn * (gz >> 1));
                } else {
                    vi = (long long)gx + vol.nx * ((long long)gy + (long long)vol.ny * gz);
                }
                val = *reinterpret_cast<const uint4*>(in.a + vi * in.ca + ch);
            } else {
                const long long vi = (long long)gx + vol.nx * ((long long)gy + (long long)vol.ny * gz);
                val = *reinterpret_cast<const uint4*>(in.b + vi * in.cb + (ch - in.ca));
            }
        }
        *reinterpret_cast<uint4*>(smem + h * rs + vq * 16) = val;
    }
    __syncthreads();
    // ---- implicit GEMM
    const int warp = tid >> 5, lane = tid & 31;
    const int cout = NF * 8;
    float acc[NF][4];
#pragma unroll
    for (int f = 0; f < NF; ++f) acc[f][0] = acc[f][1] = acc[f][2] = acc[f][3] = 0.f;
    // this lane's ldmatrix row: voxel m = lane % 16 of the warp's 16, k offset (lane / 16) * 8
    const int vm = warp * 16 + (lane & 15);
    const int tx = vm % TX, ty = (vm / TX) % TY, tz = vm / (TX * TY);
    const uint32_t sbase = smem_u32(smem) + (uint32_t)((lane >> 4) * 16);
    const int krow = (lane & 3) * 2;   // B fragment: k = krow, krow + 1 (+8)
    const int ncol = lane >> 2;        // B fragment: n = ncol
    for (int tap = 0; tap < 27; ++tap) {
        const int dx = tap % 3, dy = (tap / 3) % 3, dz = tap / 9;
        const int h = (tx + dx) + HX * ((ty + dy) + HY * (tz + dz));
        const uint32_t arow = sbase + (uint32_t)(h * rs);
        const __nv_bfloat16* wt = W + (long long)tap * cout * cin;
        for (int ci0 = 0; ci0 < cin; ci0 += 16) {
            uint32_t a0, a1, a2, a3;
            ldmatrix_x4(arow + (uint32_t)(ci0 * 2), a0, a1, a2, a3);
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                const __nv_bfloat16* wr = wt + (long long)(f * 8 + ncol) * cin + ci0 + krow;
                const uint32_t b0 = *reinterpret_cast<const uint32_t*>(wr);
                const uint32_t b1 = *reinterpret_cast<const uint32_t*>(wr + 8);
                mma_bf16(acc[f], a0, a1, a2, a3, b0, b1);
            }
        }
    }
    // ---- epilogue: rows lane/4 and lane/4 + 8 of the warp's 16 voxels, columns 2 (lane % 4) + {0,1}
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        const int m = warp * 16 + (lane >> 2) + half * 8;
        const int ox = x0 + m % TX, oy = y0 + (m / TX) % TY, oz = z0 + m / (TX * TY);
        if (ox >= vol.nx || oy >= vol.ny || oz >= vol.nz) continue;
        const long long vo = (long long)ox + vol.nx * ((long long)oy + (long long)vol.ny * oz);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            const int co = f * 8 + (lane & 3) * 2;
            float v0 = acc[f][half * 2], v1 = acc[f][half * 2 + 1];
            if (bias) { v0 += bias[co]; v1 += bias[co + 1]; }
            if (relu) { v0 = fmaxf(v0, 0.f); v1 = fmaxf(v1, 0.f); }
            *reinterpret_cast<__nv_bfloat162*>(out + vo * cout + co) = __floats2bfloat162_rn(v0, v1);
        }
    }
}

}  // namespace nn
}  // namespace suli
