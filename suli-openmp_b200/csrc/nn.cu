// nn.cu — the learned initial guess / preconditioner of the pressure solve: a 3-D U-Net
// (4 levels, 16/32/64/96 channels, 3x3x3 convolutions, ReLU, 2x2x2 average pooling, nearest
// upsampling with skip concatenation, 1x1x1 head), BF16 weights and activations, FP32
// accumulation, FP32 master weights trained with Adam.  Forward convolutions and the
// input-gradient (dgrad) convolutions run on the tensor cores: by default the persistent
// TMA + tcgen05 pipeline (nn_tp.cuh), which also computes the encoder's pooling and the head in
// its epilogues; the one-tile tcgen05 kernel (nn_tc.cuh) and mma.sync (nn_conv.cuh) remain
// selectable.  Weight gradients accumulate in FP32 on the CUDA cores.
//
// The network maps (residual r~0/s, density feature, previous pressure e0/s) to the scaled
// correction (e* - e0)/s of the pressure solve, so it is both an initial guess
// (e0 <- e0 + s net(.)) and an approximate inverse of A~ applied to a residual.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include "../../include/suli_gpu.h"
#include "nn_api.cuh"
#include "nn_conv.cuh"
#include "nn_tc.cuh"
#include "nn_tp.cuh"

namespace suli {
namespace nn {

constexpr int kLevels = 4;
constexpr int kCh[kLevels] = {16, 32, 64, 96};
constexpr int kInCh = 3;   // real input channels (padded to 16)

// conv layers in order: enc0a enc0b enc1a enc1b enc2a enc2b enc3a enc3b dec2a dec2b dec1a dec1b dec0a dec0b
struct LayerSpec {
    int cin, cout, level;
};
constexpr int kConv = 14;
constexpr LayerSpec kLayer[kConv] = {
    {16, 16, 0}, {16, 16, 0}, {16, 32, 1}, {32, 32, 1}, {32, 64, 2}, {64, 64, 2}, {64, 96, 3},
    {96, 96, 3}, {160, 64, 2}, {64, 64, 2}, {96, 32, 1}, {32, 32, 1}, {48, 16, 0}, {16, 16, 0},
};

__host__ __device__ inline long long conv_params(const LayerSpec& L) { return 27LL * L.cout * L.cin + L.cout; }

// ------------------------------------------------------------------------------------
// elementwise / small kernels
// ------------------------------------------------------------------------------------
__global__ void k_pack_input(long long V, const float* __restrict__ in3, __nv_bfloat16* __restrict__ out16) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    __nv_bfloat16 t[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) t[c] = __float2bfloat16(c < kInCh ? in3[v * kInCh + c] : 0.f);
    uint4* o = reinterpret_cast<uint4*>(out16 + v * 16);
    o[0] = *reinterpret_cast<uint4*>(&t[0]);
    o[1] = *reinterpret_cast<uint4*>(&t[8]);
}

// 2x2x2 average pooling, channels last
__global__ void k_pool(Vol fine, int C, const __nv_bfloat16* __restrict__ x, __nv_bfloat16* __restrict__ y) {
    const int cx = fine.nx / 2, cy = fine.ny / 2, cz = fine.nz / 2;
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long Vc = (long long)cx * cy * cz;
    if (q >= Vc * C) return;
    const int c = (int)(q % C);
    const long long vc = q / C;
    const int X = (int)(vc % cx), Y = (int)((vc / cx) % cy), Z = (int)(vc / ((long long)cx * cy));
    float s = 0.f;
    for (int d = 0; d < 8; ++d) {
        const int fx = 2 * X + (d & 1), fy = 2 * Y + ((d >> 1) & 1), fz = 2 * Z + (d >> 2);
        s += __bfloat162float(x[((long long)fx + fine.nx * ((long long)fy + (long long)fine.ny * fz)) * C + c]);
    }
    y[q] = __float2bfloat16(0.125f * s);
}

// gradient of the pooling: dx[fine] += dy[parent] / 8
__global__ void k_pool_bwd(Vol fine, int C, const __nv_bfloat16* __restrict__ dy, __nv_bfloat16* dx) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long V = (long long)fine.nx * fine.ny * fine.nz;
    if (q >= V * C) return;
    const int c = (int)(q % C);
    const long long v = q / C;
    const int x = (int)(v % fine.nx), y = (int)((v / fine.nx) % fine.ny), z = (int)(v / ((long long)fine.nx * fine.ny));
    const int cx = fine.nx / 2, cy = fine.ny / 2;
    const long long vc = (long long)(x >> 1) + cx * ((long long)(y >> 1) + (long long)cy * (z >> 1));
    dx[q] = __float2bfloat16(__bfloat162float(dx[q]) + 0.125f * __bfloat162float(dy[vc * C + c]));
}

// dz = dy * (y > 0) in place
__global__ void k_relu_bwd(long long n, const __nv_bfloat16* __restrict__ y, __nv_bfloat16* dy) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n && !(__bfloat162float(y[q]) > 0.f)) dy[q] = __float2bfloat16(0.f);
}

// split the gradient of concat(up(A), B): dA[coarse] = sum of the 8 children (channels < ca);
// dB[fine] += channels >= ca
__global__ void k_concat_bwd(Vol fine, int ca, int cb, const __nv_bfloat16* __restrict__ dcat,
                             __nv_bfloat16* __restrict__ da, __nv_bfloat16* db) {
    const int cx = fine.nx / 2, cy = fine.ny / 2, cz = fine.nz / 2;
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long Vc = (long long)cx * cy * cz, Vf = (long long)fine.nx * fine.ny * fine.nz;
    const int C = ca + cb;
    if (q < Vc * ca) {
        const int c = (int)(q % ca);
        const long long vc = q / ca;
        const int X = (int)(vc % cx), Y = (int)((vc / cx) % cy), Z = (int)(vc / ((long long)cx * cy));
        float s = 0.f;
        for (int d = 0; d < 8; ++d) {
            const int fx = 2 * X + (d & 1), fy = 2 * Y + ((d >> 1) & 1), fz = 2 * Z + (d >> 2);
            s += __bfloat162float(dcat[((long long)fx + fine.nx * ((long long)fy + (long long)fine.ny * fz)) * C + c]);
        }
        da[q] = __float2bfloat16(s);
    }
    if (q < Vf * cb) {
        const int c = (int)(q % cb);
        const long long v = q / cb;
        db[q] = __float2bfloat16(__bfloat162float(db[q]) + __bfloat162float(dcat[v * C + ca + c]));
    }
}

// head: out[v] = sum_c w[c] x[v][c] + b  (FP32 out)
__global__ void k_head_fwd(long long V, const __nv_bfloat16* __restrict__ x, const float* __restrict__ w,
                           float* __restrict__ out) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    float s = w[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) s += w[c] * __bfloat162float(x[v * 16 + c]);
    out[v] = s;
}
// head backward: dx[v][c] = w[c] dout[v]; the block's sums of x[v][c] dout[v] and of dout into
// part[block][0..16] (k_sum_parts adds them to dw, db)
__global__ void k_head_bwd(long long V, const __nv_bfloat16* __restrict__ x, const float* __restrict__ w,
                           const float* __restrict__ dout, __nv_bfloat16* __restrict__ dx, float* part) {
    __shared__ float sh[17][8];
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float g[17];
#pragma unroll
    for (int c = 0; c < 17; ++c) g[c] = 0.f;
    if (v < V) {
        const float d = dout[v];
#pragma unroll
        for (int c = 0; c < 16; ++c) {
            dx[v * 16 + c] = __float2bfloat16(w[c] * d);
            g[c] = __bfloat162float(x[v * 16 + c]) * d;
        }
        g[16] = d;
    }
#pragma unroll
    for (int c = 0; c < 17; ++c)
        for (int o = 16; o > 0; o >>= 1) g[c] += __shfl_xor_sync(0xffffffffu, g[c], o);
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    if (lane == 0)
        for (int c = 0; c < 17; ++c) sh[c][wp] = g[c];
    __syncthreads();
    if (threadIdx.x < 17) {
        float s = 0.f;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += sh[threadIdx.x][q];
        part[(long long)blockIdx.x * 17 + threadIdx.x] = s;   // summed in block order by k_sum_parts
    }
}

// out[q] += sum over the nparts rows of part[row][q], rows in order (a fixed summation order,
// so a gradient is the same from run to run)
__global__ void k_sum_parts(long long nparts, long long width, const float* __restrict__ part, float* out) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= width) return;
    float s = 0.f;
    for (long long r = 0; r < nparts; ++r) s += part[r * width + q];
    out[q] += s;
}

// W'[tap'][ci][co] = W[26 - tap'][co][ci]: weights of the input-gradient convolution
__global__ void k_flip_weights(int cin, int cout, const __nv_bfloat16* __restrict__ w, __nv_bfloat16* __restrict__ wt) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = 27LL * cin * cout;
    if (q >= n) return;
    const int co = (int)(q % cout);
    const int ci = (int)((q / cout) % cin);
    const int tp = (int)(q / ((long long)cout * cin));
    wt[q] = w[((long long)(26 - tp) * cout + co) * cin + ci];
}

// weight gradient of one layer: dW[tap][co][ci] += sum_v X[v + off(tap)][ci] dZ[v][co];
// a CTA owns one tap and a chunk of voxels; threads hold a (CO16 x CI16) register block.  Each
// CTA writes its chunk's sums to its own row of part (row = chunk, 27 COUT CIN weights then COUT
// biases); k_sum_parts adds the rows in chunk order, so there are no float atomics and the
// gradient is reproducible.
constexpr int kWgChunk = 4096, kWgSub = 32;
template <int CO16, int CI16>
__global__ void __launch_bounds__(256) k_wgrad(Vol vol, ConvIn in, const __nv_bfloat16* __restrict__ dz,
                                               float* part) {
    constexpr int COUT = CO16 * 16, CIN = CI16 * 16;
    __shared__ float sx[kWgSub][CIN + 1];
    __shared__ float sz[kWgSub][COUT + 1];
    const int tap = blockIdx.y;
    const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dzz = tap / 9 - 1;
    const long long V = (long long)vol.nx * vol.ny * vol.nz;
    const long long v0 = (long long)blockIdx.x * kWgChunk;
    const int tc = threadIdx.x >> 4, ti = threadIdx.x & 15;
    float acc[CO16][CI16];
#pragma unroll
    for (int a = 0; a < CO16; ++a)
#pragma unroll
        for (int b = 0; b < CI16; ++b) acc[a][b] = 0.f;
    float bacc[CO16];
#pragma unroll
    for (int a = 0; a < CO16; ++a) bacc[a] = 0.f;
    const int hxn = (vol.nx + 1) / 2, hyn = (vol.ny + 1) / 2;
    for (long long vs = v0; vs < v0 + kWgChunk && vs < V; vs += kWgSub) {
        // stage dZ and the shifted input of kWgSub voxels (FP32)
        for (int q = threadIdx.x; q < kWgSub * COUT; q += 256) {
            const int m = q / COUT, c = q % COUT;
            const long long v = vs + m;
            sz[m][c] = (v < V) ? __bfloat162float(dz[v * COUT + c]) : 0.f;
        }
        for (int q = threadIdx.x; q < kWgSub * CIN; q += 256) {
            const int m = q / CIN, c = q % CIN;
            const long long v = vs + m;
            float val = 0.f;
            if (v < V) {
                const int x = (int)(v % vol.nx) + dx, y = (int)((v / vol.nx) % vol.ny) + dy,
                          z = (int)(v / ((long long)vol.nx * vol.ny)) + dzz;
                if (x >= 0 && x < vol.nx && y >= 0 && y < vol.ny && z >= 0 && z < vol.nz) {
                    if (c < in.ca) {
                        const long long vi = in.a_half ? ((long long)(x >> 1) + hxn * ((long long)(y >> 1) + (long long)hyn * (z >> 1)))
                                                       : ((long long)x + vol.nx * ((long long)y + (long long)vol.ny * z));
                        val = __bfloat162float(in.a[vi * in.ca + c]);
                    } else {
                        const long long vi = (long long)x + vol.nx * ((long long)y + (long long)vol.ny * z);
                        val = __bfloat162float(in.b[vi * in.cb + (c - in.ca)]);
                    }
                }
            }
            sx[m][c] = val;
        }
        __syncthreads();
#pragma unroll 4
        for (int m = 0; m < kWgSub; ++m) {
            float zv[CO16], xv[CI16];
#pragma unroll
            for (int a = 0; a < CO16; ++a) zv[a] = sz[m][tc + 16 * a];
#pragma unroll
            for (int b = 0; b < CI16; ++b) xv[b] = sx[m][ti + 16 * b];
#pragma unroll
            for (int a = 0; a < CO16; ++a) {
#pragma unroll
                for (int b = 0; b < CI16; ++b) acc[a][b] += zv[a] * xv[b];
                if (ti == 0 && tap == 13) bacc[a] += zv[a];
            }
        }
        __syncthreads();
    }
    float* row = part + (long long)blockIdx.x * (27LL * COUT * CIN + COUT);
#pragma unroll
    for (int a = 0; a < CO16; ++a) {
#pragma unroll
        for (int b = 0; b < CI16; ++b) row[((long long)tap * COUT + tc + 16 * a) * CIN + ti + 16 * b] = acc[a][b];
        if (ti == 0 && tap == 13) row[27LL * COUT * CIN + tc + 16 * a] = bacc[a];
    }
}

// squared error L = mean(e^2), e = pred - target; dout = 2 e / V.  The sums are block partials
// (fixed warp-shuffle tree) folded in block order by k_loss_fold, so the loss is reproducible.
__global__ void k_loss_sums(long long V, const float* __restrict__ pred, const float* __restrict__ tgt,
                            double* __restrict__ part) {
    __shared__ double sh[2][8];
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0., e2 = 0.;
    if (v < V) {
        e = (double)pred[v] - (double)tgt[v];
        e2 = e * e;
    }
    for (int o = 16; o > 0; o >>= 1) {
        e += __shfl_xor_sync(0xffffffffu, e, o);
        e2 += __shfl_xor_sync(0xffffffffu, e2, o);
    }
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    if (lane == 0) { sh[0][wp] = e; sh[1][wp] = e2; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0., b = 0.;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { a += sh[0][q]; b += sh[1][q]; }
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = b;
    }
}
// one block: thread t folds partials t, t + 256, ... in order, then a fixed tree
__global__ void __launch_bounds__(256) k_loss_fold(int nparts, const double* __restrict__ part, double* sums) {
    __shared__ double sh[2][256];
    double a = 0., b = 0.;
    for (int q = threadIdx.x; q < nparts; q += 256) { a += part[2 * q]; b += part[2 * q + 1]; }
    sh[0][threadIdx.x] = a;
    sh[1][threadIdx.x] = b;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + h];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) { sums[0] = sh[0][0]; sums[1] = sh[1][0]; }
}
__global__ void k_loss_grad(long long V, const float* __restrict__ pred, const float* __restrict__ tgt,
                            float* __restrict__ dout) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    dout[v] = (float)(2.0 / (double)V * ((double)pred[v] - (double)tgt[v]));
}

// Adam on the FP32 master weights, then the BF16 copy the convolutions read
__global__ void k_adam(long long n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, __nv_bfloat16* __restrict__ wb, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    if (lr != 0.f) {
        const float gq = g[q];
        const float mq = b1 * m[q] + (1.f - b1) * gq;
        const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
        m[q] = mq;
        v[q] = vq;
        w[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
    }
    wb[q] = __float2bfloat16(w[q]);
}

__global__ void k_zero_bf(long long n, __nv_bfloat16* a) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) a[q] = __float2bfloat16(0.f);
}

}  // namespace nn
}  // namespace suli

using namespace suli::nn;

// ------------------------------------------------------------------------------------
// host side: network object
// ------------------------------------------------------------------------------------
struct suli_nn {
    int device = 0;
    cudaStream_t stream = nullptr;
    Vol vol[kLevels];
    long long V[kLevels];
    long long nparam = 0;
    long long off[kConv + 1];   // parameter offsets (head at off[kConv])
    float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    __nv_bfloat16* wb = nullptr;     // BF16 copy, same layout
    __nv_bfloat16* wflip = nullptr;  // scratch: flipped weights for dgrad
    unsigned char* frozen = nullptr;
    long long step = 0;
    // activations (BF16, channels last)
    __nv_bfloat16 *in0 = nullptr, *a[kConv] = {nullptr}, *pool[kLevels - 1] = {nullptr};
    // gradients
    __nv_bfloat16 *gact[kConv] = {nullptr}, *gpool[kLevels - 1] = {nullptr}, *gcat = nullptr, *gtmp = nullptr;
    float *out = nullptr, *dout = nullptr;
    double* sums = nullptr;
    double* loss_part = nullptr;     // block partials of the loss sums
    double* host_sums = nullptr;
    int* err_flag = nullptr;         // set by a tensor-core convolution whose wait timed out
    int kernel = 0;                  // convolution kernel: 0 tcgen05 pipeline, 1 mma.sync, 2 tcgen05 one tile per CTA
    float* part = nullptr;           // per-CTA partial sums of the parameter gradient (training)
    long long part_floats = 0;
    bool grad_error = false;         // the partial-sum buffer could not be allocated
    std::string err;
};

namespace {

inline unsigned nb(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

template <int NF>
void conv_launch(suli_nn* N, const Vol& vol, const ConvIn& in, const __nv_bfloat16* W, const float* bias, int relu,
                 __nv_bfloat16* out) {
    const int cin = in.ca + in.cb;
    const size_t smem = (size_t)HVOX * (cin * 2 + 16);
    static bool attr_done[64] = {false};
    if (!attr_done[N->device]) {
        cudaFuncSetAttribute(k_conv3_fwd<NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
        attr_done[N->device] = true;
    }
    const dim3 grid((vol.nx + TX - 1) / TX, (vol.ny + TY - 1) / TY, (vol.nz + TZ - 1) / TZ);
    k_conv3_fwd<NF><<<grid, 256, smem, N->stream>>>(vol, in, W, bias, relu, out);
}

template <int NZ>
void conv_tc_nz(suli_nn* N, const Vol& vol, const ConvIn& in, const __nv_bfloat16* W, const float* bias, int relu,
                int cout, int tcols, __nv_bfloat16* out) {
    static bool attr_done[64] = {false};
    if (!attr_done[N->device]) {
        cudaFuncSetAttribute(k_conv3_tc<NZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        attr_done[N->device] = true;
    }
    const dim3 grid((vol.nx + TCX - 1) / TCX, (vol.ny + TCY - 1) / TCY, (vol.nz + NZ - 1) / NZ);
    k_conv3_tc<NZ><<<grid, 128, tc_smem_bytes<NZ>(cout), N->stream>>>(vol, in, W, bias, relu, cout, tcols, out,
                                                                       N->err_flag);
}

// z-planes per CTA: as many as keep the CTA's accumulators within 128 TMEM columns
int tc_cols(int cout) {
    int tcols = 32;
    while (tcols < cout) tcols *= 2;
    return tcols;
}
void conv_tc(suli_nn* N, const Vol& vol, const ConvIn& in, const __nv_bfloat16* W, const float* bias, int relu,
             int cout, __nv_bfloat16* out) {
    const int tcols = tc_cols(cout);
    if (tcols <= 32) conv_tc_nz<4>(N, vol, in, W, bias, relu, cout, tcols, out);
    else if (tcols <= 64) conv_tc_nz<2>(N, vol, in, W, bias, relu, cout, tcols, out);
    else conv_tc_nz<1>(N, vol, in, W, bias, relu, cout, tcols, out);
}

// ---- the pipelined tcgen05 convolution (nn_tp.cuh): TMA descriptors and launch shape
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
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
// channels-last volume [nz][ny][nx][C]; box {8 channels, hx, hy, hz}, zero fill outside
bool map_volume(CUtensorMap* m, const __nv_bfloat16* p, int C, const Vol& v, int hx, int hy, int hz) {
    auto enc = tensor_map_encoder();
    if (!enc || !p || (reinterpret_cast<uintptr_t>(p) & 15) || C % 8) return false;
    cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)v.nx, (cuuint64_t)v.ny, (cuuint64_t)v.nz};
    cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)C * 2 * v.nx, (cuuint64_t)C * 2 * v.nx * v.ny};
    cuuint32_t box[4] = {8, (cuuint32_t)hx, (cuuint32_t)hy, (cuuint32_t)hz};
    cuuint32_t es[4] = {1, 1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(p), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
// weights [27][cout][cin]; box {8 input channels, cout, 27 taps}
bool map_weights(CUtensorMap* m, const __nv_bfloat16* W, int cin, int cout) {
    auto enc = tensor_map_encoder();
    if (!enc || (reinterpret_cast<uintptr_t>(W) & 15) || cout > 256) return false;
    cuuint64_t dims[3] = {(cuuint64_t)cin, (cuuint64_t)cout, 27};
    cuuint64_t strides[2] = {(cuuint64_t)cin * 2, (cuuint64_t)cin * cout * 2};
    cuuint32_t box[3] = {8, (cuuint32_t)cout, 27};
    cuuint32_t es[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<__nv_bfloat16*>(W), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
int sm_count(int device) {
    static int n[64] = {0};
    if (device < 0 || device >= 64) return 148;
    if (!n[device] && cudaDeviceGetAttribute(&n[device], cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        n[device] = 148;
    }
    return n[device];
}
constexpr int kTpSmemMax = 227 * 1024;

// false: this shape is not supported by the pipeline (the caller uses k_conv3_tc)
template <int NZ, bool FOLD>
bool conv_tp_nz(suli_nn* N, const Vol& vol, const ConvIn& in, const __nv_bfloat16* W, const float* bias, int relu,
                int cout, int tcols, __nv_bfloat16* out, const TpEpi& epi) {
    using G = TpGeo<FOLD>;
    const int cin = in.ca + in.cb;
    if (in.ca % TC_CC || in.cb % TC_CC || 2 * NZ * tcols > 512 || cout > 256) return false;
    if (epi.pool && (NZ < 2 || vol.nx % 2 || vol.ny % 2 || vol.nz % 2)) return false;
    if (epi.head_w && cout != 16) return false;
    TpCfg cfg{};
    cfg.cout = cout;
    cfg.tcols = tcols;
    cfg.nchunks = cin / TC_CC;
    cfg.ca = in.ca;
    cfg.a_tma = in.a_half ? 0 : 1;
    cfg.relu = relu;
    cfg.kc_bytes = (G::HXR * G::HYR * 16 * (NZ + 2) + 127) / 128 * 128;
    cfg.wchunk_bytes = 27 * cout * TC_CC * 2;
    const int wall = cfg.nchunks * cfg.wchunk_bytes;
    const int budget = kTpSmemMax - TP_TAIL_BYTES;
    // the layer's weights stay resident when three halo slots still fit beside them
    cfg.w_resident = (wall + 3 * (2 * cfg.kc_bytes) <= budget) ? 1 : 0;
    cfg.w_bytes = cfg.w_resident ? wall : 0;
    cfg.stage_bytes = 2 * cfg.kc_bytes + (cfg.w_resident ? 0 : cfg.wchunk_bytes);
    cfg.stages = std::min(TP_MAX_STAGES, (budget - cfg.w_bytes) / cfg.stage_bytes);
    if (cfg.stages < 1) return false;
    cfg.tiles_x = (vol.nx + G::OX - 1) / G::OX;
    cfg.tiles_y = (vol.ny + G::OY - 1) / G::OY;
    const long long tiles = (long long)cfg.tiles_x * cfg.tiles_y * ((vol.nz + NZ - 1) / NZ);
    if (tiles > (1LL << 30)) return false;
    cfg.tiles = (int)tiles;
    CUtensorMap ma, mb, mw;
    if (!map_weights(&mw, W, cin, cout)) return false;
    if (in.cb > 0 && !map_volume(&mb, in.b, in.cb, vol, G::HXR, G::HYR, NZ + 2)) return false;
    if (cfg.a_tma) {
        if (!map_volume(&ma, in.a, in.ca, vol, G::HXR, G::HYR, NZ + 2)) return false;
    } else if (reinterpret_cast<uintptr_t>(in.a) & 15) {
        return false;   // 16-byte cp.async sources
    }
    if (in.cb == 0) mb = mw;      // not read
    if (!cfg.a_tma) ma = mw;      // not read
    const size_t smem = (size_t)(cfg.w_bytes + cfg.stages * cfg.stage_bytes + TP_TAIL_BYTES);
    static bool attr_done[64] = {false};
    if (!attr_done[N->device]) {
        cudaFuncSetAttribute(k_conv3_tp<NZ, FOLD>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTpSmemMax);
        attr_done[N->device] = true;
    }
    const int grid = (int)std::min<long long>(tiles, sm_count(N->device));
    k_conv3_tp<NZ, FOLD><<<grid, TP_THREADS, smem, N->stream>>>(vol, in, ma, mb, mw, bias, cfg, epi, out, N->err_flag);
    return true;
}

// Cout 16 and 32 fold the x taps into N (N = 48 -> 64 TMEM columns a plane, 4 planes; N = 96 ->
// 128 columns, 2 planes); wider layers use the 8 x 16 tile.  Two accumulator sets <= 512 columns.
bool conv_tp(suli_nn* N, const Vol& vol, const ConvIn& in, const __nv_bfloat16* W, const float* bias, int relu,
             int cout, __nv_bfloat16* out, const TpEpi& epi) {
    if (cout == 16) return conv_tp_nz<4, true>(N, vol, in, W, bias, relu, cout, 64, out, epi);
    if (cout == 32) return conv_tp_nz<2, true>(N, vol, in, W, bias, relu, cout, 128, out, epi);
    const int tcols = tc_cols(cout);
    if (tcols <= 64) return conv_tp_nz<2, false>(N, vol, in, W, bias, relu, cout, tcols, out, epi);
    return conv_tp_nz<1, false>(N, vol, in, W, bias, relu, cout, tcols, out, epi);
}

void conv(suli_nn* N, const Vol& vol, const ConvIn& in, const __nv_bfloat16* W, const float* bias, int relu, int cout,
          __nv_bfloat16* out) {
    if (N->kernel == 0 && conv_tp(N, vol, in, W, bias, relu, cout, out, TpEpi{nullptr, nullptr, nullptr, 1})) return;
    if (N->kernel == 0 || N->kernel == 2) {
        conv_tc(N, vol, in, W, bias, relu, cout, out);
        return;
    }
    switch (cout) {
    case 16: conv_launch<2>(N, vol, in, W, bias, relu, out); break;
    case 32: conv_launch<4>(N, vol, in, W, bias, relu, out); break;
    case 48: conv_launch<6>(N, vol, in, W, bias, relu, out); break;
    case 64: conv_launch<8>(N, vol, in, W, bias, relu, out); break;
    case 96: conv_launch<12>(N, vol, in, W, bias, relu, out); break;
    case 160: conv_launch<20>(N, vol, in, W, bias, relu, out); break;
    default: break;
    }
}

// The weight gradient on the tensor cores (mma.sync m16n8k16, BF16 x BF16 -> FP32).  Per tap it
// is the GEMM dW_tap (COUT x CIN) += dZ^T (COUT x V) X_tap (V x CIN) over the CTA's chunk of
// voxels: dZ and the shifted input of kWgTcSub voxels are staged as BF16 rows (voxel-major, rows
// padded by 8 elements so that ldmatrix reads are free of bank conflicts), A fragments (COUT rows,
// voxels along K) and B fragments (voxels along K, CIN columns) come from ldmatrix.trans of those
// rows.  The warps split the 16 x 8 output tiles and, where a layer has fewer tiles than warps,
// the voxels; the voxel-split partials are added in warp order through shared memory.  Each CTA
// writes its row of part exactly as k_wgrad does, so the sum over rows is as reproducible.
constexpr int kWgTcSub = 64;
__device__ __forceinline__ void ldmatrix_x4_trans(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2,
                                                  uint32_t& r3) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}
__device__ __forceinline__ void ldmatrix_x2_trans(uint32_t addr, uint32_t& r0, uint32_t& r1) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n" : "=r"(r0), "=r"(r1) : "r"(addr));
}
template <int CO16, int CI16>
__global__ void __launch_bounds__(256) k_wgrad_tc(Vol vol, ConvIn in, const __nv_bfloat16* __restrict__ dz,
                                                  float* part) {
    constexpr int COUT = CO16 * 16, CIN = CI16 * 16;
    constexpr int TN = CIN / 8, TILES = CO16 * TN;
    constexpr int KW = (TILES < 8 && 8 % TILES == 0) ? 8 / TILES : 1;   // warps sharing a tile's voxels
    constexpr int TW = 8 / KW;                                           // warps splitting the tiles
    constexpr int TPW = (TILES + TW - 1) / TW;                           // tiles a warp owns
    constexpr int RZ = COUT + 8, RX = CIN + 8;
    __shared__ __align__(16) __nv_bfloat16 sz[kWgTcSub][RZ];
    __shared__ __align__(16) __nv_bfloat16 sx[kWgTcSub][RX];
    __shared__ float red[KW > 1 ? (KW - 1) * TW * TPW * 128 : 1];
    const int tap = blockIdx.y;
    const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dzz = tap / 9 - 1;
    const long long V = (long long)vol.nx * vol.ny * vol.nz;
    const long long v0 = (long long)blockIdx.x * kWgChunk;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int tw = warp % TW, kw = warp / TW;
    float acc[TPW][4];
#pragma unroll
    for (int i = 0; i < TPW; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
    float bacc = 0.f;   // the bias gradient of channel tid (tap 13)
    const int hxn = (vol.nx + 1) / 2, hyn = (vol.ny + 1) / 2;
    const uint32_t szu = smem_u32(&sz[0][0]), sxu = smem_u32(&sx[0][0]);
    for (long long vs = v0; vs < v0 + kWgChunk && vs < V; vs += kWgTcSub) {
        // stage dZ and the shifted input of kWgTcSub voxels (16-byte vectors, zero outside)
        for (int q = tid; q < kWgTcSub * (COUT / 8); q += 256) {
            const int m = q / (COUT / 8), c = (q % (COUT / 8)) * 8;
            const long long v = vs + m;
            uint4 val = make_uint4(0u, 0u, 0u, 0u);
            if (v < V) val = *reinterpret_cast<const uint4*>(dz + v * COUT + c);
            *reinterpret_cast<uint4*>(&sz[m][c]) = val;
        }
        for (int q = tid; q < kWgTcSub * (CIN / 8); q += 256) {
            const int m = q / (CIN / 8), c = (q % (CIN / 8)) * 8;
            const long long v = vs + m;
            uint4 val = make_uint4(0u, 0u, 0u, 0u);
            if (v < V) {
                const int x = (int)(v % vol.nx) + dx, y = (int)((v / vol.nx) % vol.ny) + dy,
                          z = (int)(v / ((long long)vol.nx * vol.ny)) + dzz;
                if (x >= 0 && x < vol.nx && y >= 0 && y < vol.ny && z >= 0 && z < vol.nz) {
                    if (c < in.ca) {
                        const long long vi = in.a_half ? ((long long)(x >> 1) + hxn * ((long long)(y >> 1) + (long long)hyn * (z >> 1)))
                                                       : ((long long)x + vol.nx * ((long long)y + (long long)vol.ny * z));
                        val = *reinterpret_cast<const uint4*>(in.a + vi * in.ca + c);
                    } else {
                        const long long vi = (long long)x + vol.nx * ((long long)y + (long long)vol.ny * z);
                        val = *reinterpret_cast<const uint4*>(in.b + vi * in.cb + (c - in.ca));
                    }
                }
            }
            *reinterpret_cast<uint4*>(&sx[m][c]) = val;
        }
        __syncthreads();
        if (tap == 13 && tid < COUT)
            for (int m = 0; m < kWgTcSub; ++m) bacc += __bfloat162float(sz[m][tid]);
        // this warp's K steps (16 voxels each) of the staged block
        for (int ks = kw; ks < kWgTcSub / 16; ks += KW) {
            const int vb = ks * 16;
            // A: lane -> matrix mi = lane / 8 (co + 8 (mi & 1), voxels + 8 (mi >> 1)), row lane % 8
            const int ar = vb + (lane & 7) + 8 * (lane >> 4), ac = 8 * ((lane >> 3) & 1);
            // B: lanes 0-15 give the rows of the two 8-voxel halves (x2)
            const int br = vb + (lane & 15);
#pragma unroll
            for (int i = 0; i < TPW; ++i) {
                const int t = tw + TW * i;
                if (t < TILES) {
                    const int co0 = 16 * (t / TN), ci0 = 8 * (t % TN);
                    uint32_t a0, a1, a2, a3, b0, b1;
                    ldmatrix_x4_trans(szu + (uint32_t)((ar * RZ + co0 + ac) * 2), a0, a1, a2, a3);
                    ldmatrix_x2_trans(sxu + (uint32_t)((br * RX + ci0) * 2), b0, b1);
                    mma_bf16(acc[i], a0, a1, a2, a3, b0, b1);
                }
            }
        }
        __syncthreads();
    }
    // voxel-split warps: add the partials in warp order (kw = 1 .. KW - 1 into kw = 0)
    if (KW > 1) {
        if (kw > 0)
#pragma unroll
            for (int i = 0; i < TPW; ++i)
#pragma unroll
                for (int e = 0; e < 4; ++e) red[(((kw - 1) * TW + tw) * TPW + i) * 128 + e * 32 + lane] = acc[i][e];
        __syncthreads();
        if (kw == 0)
            for (int w = 1; w < KW; ++w)
#pragma unroll
                for (int i = 0; i < TPW; ++i)
#pragma unroll
                    for (int e = 0; e < 4; ++e) acc[i][e] += red[(((w - 1) * TW + tw) * TPW + i) * 128 + e * 32 + lane];
    }
    float* row = part + (long long)blockIdx.x * (27LL * COUT * CIN + COUT);
    if (kw == 0) {
#pragma unroll
        for (int i = 0; i < TPW; ++i) {
            const int t = tw + TW * i;
            if (t >= TILES) continue;
            const int co0 = 16 * (t / TN), ci0 = 8 * (t % TN);
            // accumulator: rows lane / 4 (+ 8), columns 2 (lane % 4) + {0, 1}
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                const int co = co0 + (lane >> 2) + 8 * half, ci = ci0 + 2 * (lane & 3);
                row[((long long)tap * COUT + co) * CIN + ci] = acc[i][2 * half];
                row[((long long)tap * COUT + co) * CIN + ci + 1] = acc[i][2 * half + 1];
            }
        }
    }
    if (tap == 13 && tid < COUT) row[27LL * COUT * CIN + tid] = bacc;
}

// per-CTA rows of partial sums (k_wgrad, k_head_bwd), grown on demand (training only)
float* part_buffer(suli_nn* N, long long floats) {
    if (floats > N->part_floats) {
        cudaFree(N->part);
        N->part = nullptr;
        N->part_floats = 0;
        if (cudaMalloc(&N->part, floats * sizeof(float)) != cudaSuccess) return nullptr;
        N->part_floats = floats;
    }
    return N->part;
}

// SULI_WGRAD_CUDA_CORES=1 keeps the CUDA-core weight gradient (k_wgrad), for comparison
static bool wgrad_cuda_cores() {
    const char* ev = std::getenv("SULI_WGRAD_CUDA_CORES");
    return ev && std::strcmp(ev, "1") == 0;
}
template <int CO16, int CI16>
void wgrad_launch(suli_nn* N, const Vol& vol, const ConvIn& in, const __nv_bfloat16* dz, float* dw, float* db) {
    const long long V = (long long)vol.nx * vol.ny * vol.nz;
    const long long chunks = (V + kWgChunk - 1) / kWgChunk;
    const long long width = 27LL * (CO16 * 16) * (CI16 * 16) + CO16 * 16;   // dw then db, contiguous
    float* part = part_buffer(N, chunks * width);
    if (!part) { N->grad_error = true; return; }
    const dim3 grid((unsigned)chunks, 27);
    if (wgrad_cuda_cores())
        k_wgrad<CO16, CI16><<<grid, 256, 0, N->stream>>>(vol, in, dz, part);
    else
        k_wgrad_tc<CO16, CI16><<<grid, 256, 0, N->stream>>>(vol, in, dz, part);
    // the layer's bias follows its weights in the parameter vector (db == dw + 27 COUT CIN)
    if (db != dw + 27LL * (CO16 * 16) * (CI16 * 16)) { N->grad_error = true; return; }
    k_sum_parts<<<nb(width), 256, 0, N->stream>>>(chunks, width, part, dw);
}
void wgrad(suli_nn* N, const Vol& vol, const ConvIn& in, int cout, const __nv_bfloat16* dz, float* dw, float* db) {
    const int cin = in.ca + in.cb;
    const int key = (cout / 16) * 100 + cin / 16;
    switch (key) {
    case 101: wgrad_launch<1, 1>(N, vol, in, dz, dw, db); break;
    case 201: wgrad_launch<2, 1>(N, vol, in, dz, dw, db); break;
    case 202: wgrad_launch<2, 2>(N, vol, in, dz, dw, db); break;
    case 402: wgrad_launch<4, 2>(N, vol, in, dz, dw, db); break;
    case 404: wgrad_launch<4, 4>(N, vol, in, dz, dw, db); break;
    case 604: wgrad_launch<6, 4>(N, vol, in, dz, dw, db); break;
    case 606: wgrad_launch<6, 6>(N, vol, in, dz, dw, db); break;
    case 410: wgrad_launch<4, 10>(N, vol, in, dz, dw, db); break;
    case 206: wgrad_launch<2, 6>(N, vol, in, dz, dw, db); break;
    case 103: wgrad_launch<1, 3>(N, vol, in, dz, dw, db); break;
    default: break;
    }
}

// input of conv layer l (the decoder's first layers read concat(up(coarse), skip))
ConvIn layer_input(suli_nn* N, int l) {
    ConvIn in{nullptr, 0, 0, nullptr, 0};
    switch (l) {
    case 0: in.a = N->in0; in.ca = 16; break;
    case 1: in.a = N->a[0]; in.ca = 16; break;
    case 2: in.a = N->pool[0]; in.ca = 16; break;
    case 3: in.a = N->a[2]; in.ca = 32; break;
    case 4: in.a = N->pool[1]; in.ca = 32; break;
    case 5: in.a = N->a[4]; in.ca = 64; break;
    case 6: in.a = N->pool[2]; in.ca = 64; break;
    case 7: in.a = N->a[6]; in.ca = 96; break;
    case 8: in.a = N->a[7]; in.ca = 96; in.a_half = 1; in.b = N->a[5]; in.cb = 64; break;
    case 9: in.a = N->a[8]; in.ca = 64; break;
    case 10: in.a = N->a[9]; in.ca = 64; in.a_half = 1; in.b = N->a[3]; in.cb = 32; break;
    case 11: in.a = N->a[10]; in.ca = 32; break;
    case 12: in.a = N->a[11]; in.ca = 32; in.a_half = 1; in.b = N->a[1]; in.cb = 16; break;
    case 13: in.a = N->a[12]; in.ca = 16; break;
    }
    return in;
}

// forward pass from N->in0; the head writes `out` [V] FP32.  With the pipelined kernel the
// pooling after each encoder level and the head run in the convolutions' epilogues (same
// arithmetic and order as k_pool / k_head_fwd); `keep` = 0 (inference) also skips storing the last
// layer's activation, which only the backward pass reads.  Returns the kernels launched.
int forward(suli_nn* N, float* out, bool keep) {
    int launches = 0;
    bool head_done = false;
    for (int l = 0; l < kConv; ++l) {
        const LayerSpec& L = kLayer[l];
        const ConvIn in = layer_input(N, l);
        const int lv = L.level;
        const bool pools = (l == 1 || l == 3 || l == 5);   // pooling after each encoder level but the last
        const __nv_bfloat16* W = N->wb + N->off[l];
        const float* b = N->w + N->off[l] + 27LL * L.cout * L.cin;
        TpEpi epi{pools ? N->pool[lv] : nullptr, nullptr, nullptr, 1};
        if (l == kConv - 1) {
            epi.head_w = N->w + N->off[kConv];
            epi.head_out = out;
            epi.store = keep ? 1 : 0;
        }
        ++launches;
        if (N->kernel == 0 && conv_tp(N, N->vol[lv], in, W, b, 1, L.cout, N->a[l], epi)) {
            if (l == kConv - 1) head_done = true;
            continue;
        }
        conv(N, N->vol[lv], in, W, b, 1, L.cout, N->a[l]);
        if (pools) {
            k_pool<<<nb(N->V[lv + 1] * L.cout), 256, 0, N->stream>>>(N->vol[lv], L.cout, N->a[l], N->pool[lv]);
            ++launches;
        }
    }
    if (!head_done) {
        k_head_fwd<<<nb(N->V[0]), 256, 0, N->stream>>>(N->V[0], N->a[13], N->w + N->off[kConv], out);
        ++launches;
    }
    return launches;
}

// backward from N->dout; accumulates parameter gradients into N->g (zeroed by the caller)
void backward(suli_nn* N) {
    // gradients w.r.t. each layer's output, accumulated where a tensor feeds two consumers
    for (int l = 0; l < kConv; ++l)
        k_zero_bf<<<nb(N->V[kLayer[l].level] * kLayer[l].cout), 256, 0, N->stream>>>(N->V[kLayer[l].level] * kLayer[l].cout, N->gact[l]);
    {
        float* part = part_buffer(N, (long long)nb(N->V[0]) * 17);
        if (!part) { N->grad_error = true; return; }
        k_head_bwd<<<nb(N->V[0]), 256, 0, N->stream>>>(N->V[0], N->a[13], N->w + N->off[kConv], N->dout,
                                                      N->gact[13], part);
        k_sum_parts<<<1, 32, 0, N->stream>>>((long long)nb(N->V[0]), 17, part, N->g + N->off[kConv]);
    }
    for (int l = kConv - 1; l >= 0; --l) {
        const LayerSpec& L = kLayer[l];
        const Vol& vol = N->vol[L.level];
        const long long n = N->V[L.level] * L.cout;
        k_relu_bwd<<<nb(n), 256, 0, N->stream>>>(n, N->a[l], N->gact[l]);
        const ConvIn in = layer_input(N, l);
        wgrad(N, vol, in, L.cout, N->gact[l], N->g + N->off[l], N->g + N->off[l] + 27LL * L.cout * L.cin);
        if (l == 0) break;   // no gradient w.r.t. the network input
        // dX = conv(dZ, flipped W) on the tensor cores
        k_flip_weights<<<nb(27LL * L.cin * L.cout), 256, 0, N->stream>>>(L.cin, L.cout, N->wb + N->off[l], N->wflip);
        ConvIn gin{N->gact[l], L.cout, 0, nullptr, 0};
        if (in.cb > 0) {
            // decoder concat(up(coarse), skip): coarse part -> sum over the 8 children (its only
            // consumer), skip part accumulates (the skip also feeds the pooling)
            conv(N, vol, gin, N->wflip, nullptr, 0, L.cin, N->gcat);
            const int coarse = (l == 8) ? 7 : (l == 10 ? 9 : 11);
            const int skip = (l == 8) ? 5 : (l == 10 ? 3 : 1);
            const long long nf = N->V[L.level] * in.cb, nc = N->V[L.level + 1] * in.ca;
            k_concat_bwd<<<nb(nf > nc ? nf : nc), 256, 0, N->stream>>>(vol, in.ca, in.cb, N->gcat, N->gact[coarse],
                                                                       N->gact[skip]);
        } else if (l == 2 || l == 4 || l == 6) {
            // the input was pooled: gradient through the pooling into the encoder output
            conv(N, vol, gin, N->wflip, nullptr, 0, L.cin, N->gtmp);
            const int src = l - 1, lv = kLayer[src].level;
            k_pool_bwd<<<nb(N->V[lv] * kLayer[src].cout), 256, 0, N->stream>>>(N->vol[lv], kLayer[src].cout, N->gtmp,
                                                                             N->gact[src]);
        } else {
            // plain chain: this layer is the only consumer of the previous output
            conv(N, vol, gin, N->wflip, nullptr, 0, L.cin, N->gact[l - 1]);
        }
    }
}

template <class T>
cudaError_t alloc(T** p, long long n) {
    return cudaMalloc(reinterpret_cast<void**>(p), (size_t)n * sizeof(T));
}

int nn_fail(suli_nn* N, int code, const std::string& m) {
    if (N) N->err = m;
    return code;
}

// wait for the network's stream; report a CUDA error or a timed-out tensor-core wait
int nn_sync(suli_nn* N) {
    cudaError_t e = cudaStreamSynchronize(N->stream);
    int flag = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&flag, N->err_flag, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return nn_fail(N, SULI_ERR_CUDA, cudaGetErrorString(e));
    if (flag) {
        cudaMemset(N->err_flag, 0, sizeof(int));
        return nn_fail(N, SULI_ERR_CUDA, "tensor-core convolution: completion wait timed out");
    }
    return SULI_OK;
}

}  // namespace

namespace suli {
namespace nn {
void dims(const suli_nn* N, int* nx, int* ny, int* nz, int* device) {
    *nx = N->vol[0].nx;
    *ny = N->vol[0].ny;
    *nz = N->vol[0].nz;
    *device = N->device;
}
int forward_on(suli_nn* N, cudaStream_t stream, const float* d_in3, float* d_out) {
    const cudaStream_t own = N->stream;
    N->stream = stream;
    k_pack_input<<<nb(N->V[0]), 256, 0, stream>>>(N->V[0], d_in3, N->in0);
    const int n = 1 + forward(N, d_out, false);
    N->stream = own;
    return n;
}
void* input16(suli_nn* N) { return N->in0; }
int forward_packed_on(suli_nn* N, cudaStream_t stream, float* d_out) {
    const cudaStream_t own = N->stream;
    N->stream = stream;
    const int n = forward(N, d_out, false);
    N->stream = own;
    return n;
}
int take_error(suli_nn* N) {
    int flag = 0;
    if (cudaMemcpy(&flag, N->err_flag, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
    if (flag) cudaMemset(N->err_flag, 0, sizeof(int));
    return flag;
}
}  // namespace nn
}  // namespace suli

extern "C" {

long long suli_nn_num_params(void) {
    long long n = 0;
    for (int l = 0; l < kConv; ++l) n += conv_params(kLayer[l]);
    return n + 17;
}

int suli_nn_create(int nx, int ny, int nz, int device, suli_nn** out) {
    if (!out || nx < 8 || ny < 8 || nz < 8 || nx % 8 || ny % 8 || nz % 8) return SULI_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) { cudaGetLastError(); return SULI_ERR_NODEVICE; }
    suli_nn* N = new suli_nn();
    N->device = device;
    // a blocking stream: work the caller queued on the legacy default stream (filling the
    // input buffers) completes before the network's kernels read them
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&N->stream, cudaStreamDefault) != cudaSuccess) {
        delete N;
        return SULI_ERR_CUDA;
    }
    for (int l = 0; l < kLevels; ++l) {
        N->vol[l] = Vol{nx >> l, ny >> l, nz >> l};
        N->V[l] = (long long)(nx >> l) * (ny >> l) * (nz >> l);
    }
    long long o = 0;
    for (int l = 0; l < kConv; ++l) { N->off[l] = o; o += conv_params(kLayer[l]); }
    N->off[kConv] = o;
    N->nparam = o + 17;
    bool ok = true;
    auto A = [&](cudaError_t e) { ok = ok && (e == cudaSuccess); };
    A(alloc(&N->w, N->nparam)); A(alloc(&N->g, N->nparam)); A(alloc(&N->m, N->nparam)); A(alloc(&N->v, N->nparam));
    A(alloc(&N->wb, N->nparam));
    long long wmax = 0;
    for (int l = 0; l < kConv; ++l) wmax = std::max(wmax, 27LL * kLayer[l].cin * kLayer[l].cout);
    A(alloc(&N->wflip, wmax));
    A(alloc(&N->in0, N->V[0] * 16));
    for (int l = 0; l < kConv; ++l) {
        A(alloc(&N->a[l], N->V[kLayer[l].level] * kLayer[l].cout));
        A(alloc(&N->gact[l], N->V[kLayer[l].level] * kLayer[l].cout));
    }
    for (int l = 0; l < kLevels - 1; ++l) A(alloc(&N->pool[l], N->V[l + 1] * kCh[l]));
    A(alloc(&N->gcat, N->V[0] * 48));
    A(alloc(&N->gtmp, N->V[1] * 16));
    A(alloc(&N->out, N->V[0]));
    A(alloc(&N->dout, N->V[0]));
    A(alloc(&N->sums, 4));
    A(alloc(&N->loss_part, 2 * (long long)nb(N->V[0])));
    A(alloc(&N->err_flag, 1));
    A(cudaMallocHost(&N->host_sums, 4 * sizeof(double)));
    if (ok) {
        A(cudaMemsetAsync(N->w, 0, N->nparam * 4, N->stream));
        A(cudaMemsetAsync(N->m, 0, N->nparam * 4, N->stream));
        A(cudaMemsetAsync(N->v, 0, N->nparam * 4, N->stream));
        A(cudaMemsetAsync(N->wb, 0, N->nparam * 2, N->stream));
        A(cudaMemsetAsync(N->err_flag, 0, sizeof(int), N->stream));
        A(cudaStreamSynchronize(N->stream));
    }
    if (!ok) {
        cudaGetLastError();
        suli_nn_destroy(N);
        return SULI_ERR_NOMEM;
    }
    *out = N;
    return SULI_OK;
}

int suli_nn_destroy(suli_nn* N) {
    if (!N) return SULI_OK;
    cudaSetDevice(N->device);
    if (N->stream) cudaStreamSynchronize(N->stream);
    cudaFree(N->w); cudaFree(N->g); cudaFree(N->m); cudaFree(N->v); cudaFree(N->wb); cudaFree(N->wflip);
    cudaFree(N->in0);
    for (int l = 0; l < kConv; ++l) { cudaFree(N->a[l]); cudaFree(N->gact[l]); }
    for (int l = 0; l < kLevels - 1; ++l) cudaFree(N->pool[l]);
    cudaFree(N->gcat); cudaFree(N->gtmp); cudaFree(N->out); cudaFree(N->dout); cudaFree(N->sums); cudaFree(N->loss_part);
    cudaFree(N->part);
    cudaFree(N->err_flag);
    if (N->host_sums) cudaFreeHost(N->host_sums);
    if (N->stream) cudaStreamDestroy(N->stream);
    delete N;
    return SULI_OK;
}

const char* suli_nn_last_error(const suli_nn* N) { return N ? N->err.c_str() : "null network"; }

int suli_nn_set_params(suli_nn* N, const float* host, long long n) {
    if (!N || !host || n != N->nparam) return SULI_ERR_ARG;
    cudaSetDevice(N->device);
    if (cudaMemcpyAsync(N->w, host, n * 4, cudaMemcpyHostToDevice, N->stream) != cudaSuccess) return SULI_ERR_CUDA;
    cudaMemsetAsync(N->m, 0, n * 4, N->stream);
    cudaMemsetAsync(N->v, 0, n * 4, N->stream);
    N->step = 0;
    // the BF16 copy: an Adam pass with learning rate 0 leaves w unchanged
    k_adam<<<nb(n), 256, 0, N->stream>>>(n, N->w, N->g, N->m, N->v, N->wb, 0.f, 0.9f, 0.999f, 1e-8f, 1.f, 1.f);
    const cudaError_t e = cudaStreamSynchronize(N->stream);
    return e == cudaSuccess ? SULI_OK : SULI_ERR_CUDA;
}

int suli_nn_get_params(suli_nn* N, float* host, long long n) {
    if (!N || !host || n != N->nparam) return SULI_ERR_ARG;
    cudaSetDevice(N->device);
    if (cudaMemcpyAsync(host, N->w, n * 4, cudaMemcpyDeviceToHost, N->stream) != cudaSuccess) return SULI_ERR_CUDA;
    return cudaStreamSynchronize(N->stream) == cudaSuccess ? SULI_OK : SULI_ERR_CUDA;
}

// forward on device buffers: in3 [V][3] FP32 (x fastest), out [V] FP32
int suli_nn_forward(suli_nn* N, const float* d_in3, float* d_out) {
    if (!N || !d_in3 || !d_out) return SULI_ERR_ARG;
    cudaSetDevice(N->device);
    k_pack_input<<<nb(N->V[0]), 256, 0, N->stream>>>(N->V[0], d_in3, N->in0);
    forward(N, d_out, false);
    return nn_sync(N);
}

// loss and parameter gradient (host_grad may be null); the gradient stays in the device buffer
int suli_nn_loss_grad(suli_nn* N, const float* d_in3, const float* d_target, double* loss, float* host_grad) {
    if (!N || !d_in3 || !d_target) return SULI_ERR_ARG;
    cudaSetDevice(N->device);
    k_pack_input<<<nb(N->V[0]), 256, 0, N->stream>>>(N->V[0], d_in3, N->in0);
    forward(N, N->out, true);
    k_loss_sums<<<nb(N->V[0]), 256, 0, N->stream>>>(N->V[0], N->out, d_target, N->loss_part);
    k_loss_fold<<<1, 256, 0, N->stream>>>((int)nb(N->V[0]), N->loss_part, N->sums);
    k_loss_grad<<<nb(N->V[0]), 256, 0, N->stream>>>(N->V[0], N->out, d_target, N->dout);
    cudaMemsetAsync(N->g, 0, N->nparam * 4, N->stream);
    N->grad_error = false;
    backward(N);
    if (N->grad_error) return SULI_ERR_NOMEM;
    cudaMemcpyAsync(N->host_sums, N->sums, 2 * sizeof(double), cudaMemcpyDeviceToHost, N->stream);
    if (host_grad) cudaMemcpyAsync(host_grad, N->g, N->nparam * 4, cudaMemcpyDeviceToHost, N->stream);
    if (int r = nn_sync(N)) return r;
    if (loss) *loss = N->host_sums[1] / (double)N->V[0];
    return SULI_OK;
}

// one Adam step on the mean squared error between the prediction and d_target [V]
int suli_nn_train_step(suli_nn* N, const float* d_in3, const float* d_target, float lr, double* loss) {
    int r = suli_nn_loss_grad(N, d_in3, d_target, loss, nullptr);
    if (r != SULI_OK) return r;
    N->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)N->step), c2 = 1.f - powf(b2, (float)N->step);
    k_adam<<<nb(N->nparam), 256, 0, N->stream>>>(N->nparam, N->w, N->g, N->m, N->v, N->wb, lr, b1, b2, 1e-8f, c1, c2);
    return nn_sync(N);
}

int suli_nn_set_kernel(suli_nn* N, int kernel) {
    if (!N || kernel < 0 || kernel > 2) return SULI_ERR_ARG;
    N->kernel = kernel;
    return SULI_OK;
}

// The layer primitive on caller buffers (channels-last BF16), for tests: out = relu?(conv3(x) + b),
// with the pooling and head the network fuses into its convolutions
int suli_nn_conv3d_ex(int nx, int ny, int nz, const void* x, int cin, const void* w, const float* bias, int cout,
                      int relu, void* out, void* pool_out, const float* head_w, float* head_out, int kernel) {
    if (!x || !w || !out || cin % 16 || cout % 8 || nx < 1 || ny < 1 || nz < 1) return SULI_ERR_ARG;
    if (kernel < 0 || kernel > 2) return SULI_ERR_ARG;
    if (cout != 16 && cout != 32 && cout != 48 && cout != 64 && cout != 96 && cout != 160) return SULI_ERR_UNSUPPORTED;
    if (cin > 160) return SULI_ERR_SIZE;
    if (pool_out && (nx % 2 || ny % 2 || nz % 2)) return SULI_ERR_ARG;
    if ((head_w != nullptr) != (head_out != nullptr) || (head_w && cout != 16)) return SULI_ERR_ARG;
    suli_nn tmp;
    int dev = 0;
    cudaGetDevice(&dev);
    tmp.device = dev;
    tmp.stream = nullptr;
    tmp.kernel = kernel;
    if (cudaMalloc(&tmp.err_flag, sizeof(int)) != cudaSuccess) return SULI_ERR_NOMEM;
    cudaMemset(tmp.err_flag, 0, sizeof(int));
    const Vol vol{nx, ny, nz};
    const long long V = (long long)nx * ny * nz;
    ConvIn in{static_cast<const __nv_bfloat16*>(x), cin, 0, nullptr, 0};
    const auto* W = static_cast<const __nv_bfloat16*>(w);
    auto* o = static_cast<__nv_bfloat16*>(out);
    auto* po = static_cast<__nv_bfloat16*>(pool_out);
    const TpEpi epi{po, head_w, head_out, 1};
    if (!(kernel == 0 && conv_tp(&tmp, vol, in, W, bias, relu, cout, o, epi))) {
        conv(&tmp, vol, in, W, bias, relu, cout, o);
        if (po) k_pool<<<nb(V / 8 * cout), 256>>>(vol, cout, o, po);
        if (head_w) k_head_fwd<<<nb(V), 256>>>(V, o, head_w, head_out);
    }
    cudaError_t e = cudaDeviceSynchronize();
    int flag = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&flag, tmp.err_flag, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(tmp.err_flag);
    if (e != cudaSuccess) return SULI_ERR_CUDA;
    return flag ? SULI_ERR_CUDA : SULI_OK;
}
int suli_nn_conv3d(int nx, int ny, int nz, const void* x, int cin, const void* w, const float* bias, int cout,
                   int relu, void* out, int kernel) {
    return suli_nn_conv3d_ex(nx, ny, nz, x, cin, w, bias, cout, relu, out, nullptr, nullptr, nullptr, kernel);
}

}  // extern "C"
