// reduce.cuh — deterministic block and grid reductions shared by the kernel units.
//
// A block reduces with a fixed warp-shuffle tree; each block stores its partial, and the last
// block to arrive (atomic counter) sums all partials in block order.  No floating-point
// atomics, so a launch with the same configuration is bit-reproducible.
#pragma once
#include <cuda_runtime.h>

namespace suli {

__device__ __forceinline__ int flat_tid() {
    return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
}
__device__ __forceinline__ int flat_bid() {
    return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
}

// Sum over the block; the result is valid in thread 0.  Fixed reduction tree.
static __device__ double block_sum(double v) {
    __shared__ double sh[32];
    const int tid = flat_tid();
    const int nt = blockDim.x * blockDim.y * blockDim.z;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((tid & 31) == 0) sh[tid >> 5] = v;
    __syncthreads();
    const int nw = (nt + 31) >> 5;
    v = (tid < nw) ? sh[tid] : 0.0;
    if (tid < 32) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;
}
static __device__ double block_max(double v) {
    __shared__ double sh[32];
    const int tid = flat_tid();
    const int nt = blockDim.x * blockDim.y * blockDim.z;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();
    if ((tid & 31) == 0) sh[tid >> 5] = v;
    __syncthreads();
    const int nw = (nt + 31) >> 5;
    v = (tid < nw) ? sh[tid] : 0.0;
    if (tid < 32) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;
}

// Two block partials per block; the last block to arrive sums all partials in block order
// and returns true (totals valid in thread 0 of that block).  `is_max` selects max.
static __device__ bool reduce2_last(double a, double b, double* partial, unsigned int* counter, double& ta,
                                    double& tb, bool is_max = false) {
    __shared__ bool last;
    const int tid = flat_tid();
    const int nt = blockDim.x * blockDim.y * blockDim.z;
    const int bid = flat_bid();
    const int nb = gridDim.x * gridDim.y * gridDim.z;
    a = is_max ? block_max(a) : block_sum(a);
    b = is_max ? block_max(b) : block_sum(b);
    if (tid == 0) {
        partial[2 * bid] = a;
        partial[2 * bid + 1] = b;
        __threadfence();
        const unsigned int t = atomicAdd(counter, 1u);
        last = (t == (unsigned int)(nb - 1));
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    // each thread folds partials tid, tid + nt, ... in that order; eight loads are issued ahead
    // of the additions (the partials sit in L2, and one dependent load per step would make this
    // single block the kernel's tail)
    constexpr int U = 8;
    double sa = 0.0, sb = 0.0;
    for (int q0 = tid; q0 < nb; q0 += U * nt) {
        double pa[U], pb[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int q = q0 + u * nt;
            pa[u] = (q < nb) ? __ldcg(&partial[2 * q]) : 0.0;
            pb[u] = (q < nb) ? __ldcg(&partial[2 * q + 1]) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (q0 + u * nt >= nb) break;
            if (is_max) { sa = fmax(sa, pa[u]); sb = fmax(sb, pb[u]); }
            else { sa += pa[u]; sb += pb[u]; }
        }
    }
    sa = is_max ? block_max(sa) : block_sum(sa);
    sb = is_max ? block_max(sb) : block_sum(sb);
    if (tid == 0) { ta = sa; tb = sb; *counter = 0u; }
    return true;
}

// Three block partials per block: a and b summed, m maxed; the last block to arrive folds all
// partials in block order and returns true (totals valid in thread 0 of that block).
static __device__ bool reduce3_last(double a, double b, double m, double* partial, unsigned int* counter, double& ta,
                                    double& tb, double& tm) {
    __shared__ bool last;
    const int tid = flat_tid();
    const int nt = blockDim.x * blockDim.y * blockDim.z;
    const int bid = flat_bid();
    const int nb = gridDim.x * gridDim.y * gridDim.z;
    a = block_sum(a);
    b = block_sum(b);
    m = block_max(m);
    if (tid == 0) {
        partial[3 * bid] = a;
        partial[3 * bid + 1] = b;
        partial[3 * bid + 2] = m;
        __threadfence();
        const unsigned int t = atomicAdd(counter, 1u);
        last = (t == (unsigned int)(nb - 1));
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    // partials tid, tid + nt, ... in that order, eight triples loaded ahead of the folds
    constexpr int U = 8;
    double sa = 0.0, sb = 0.0, sm = 0.0;
    for (int q0 = tid; q0 < nb; q0 += U * nt) {
        double pa[U], pb[U], pm[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int q = q0 + u * nt;
            pa[u] = (q < nb) ? __ldcg(&partial[3 * q]) : 0.0;
            pb[u] = (q < nb) ? __ldcg(&partial[3 * q + 1]) : 0.0;
            pm[u] = (q < nb) ? __ldcg(&partial[3 * q + 2]) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (q0 + u * nt >= nb) break;
            sa += pa[u];
            sb += pb[u];
            sm = fmax(sm, pm[u]);
        }
    }
    sa = block_sum(sa);
    sb = block_sum(sb);
    sm = block_max(sm);
    if (tid == 0) { ta = sa; tb = sb; tm = sm; *counter = 0u; }
    return true;
}

}  // namespace suli
