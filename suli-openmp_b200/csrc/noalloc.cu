// noalloc.cu — suli_est_static: the divergence check est() (4_plot.f90:500-525) for callers
// that cannot let a library allocate device memory.
//
// Who needs it: a driver whose device arrays are owned by another runtime (a Fortran program
// whose u, v, w live on the GPU through OpenACC or CUDA Fortran, or a framework whose caching
// allocator has reserved the device memory up front).  Such a caller can hand us device
// pointers, but a cudaMalloc inside the library may fail for lack of unreserved memory, and
// cudaMalloc/cudaFree synchronise the whole device, stalling the caller's other streams.  This
// entry point therefore takes its reduction scratch from a fixed array compiled into the
// library and calls no allocator at all.
//
// The scratch array below is loaded on every GPU that loads this library and stays there
// until the process exits.  All calls share it: two calls that overlap on the GPU (from two
// streams or two threads) race on it and must be ordered by the caller.
#include <cuda_runtime.h>
#include <mutex>
#include "../../include/suli_gpu.h"

namespace {

constexpr int kTX = 32, kTY = 8, kZC = 16;   // tile of one block: 32 x 8 cells, 16 planes in z
constexpr int kCapacityBlocks = SULI_EST_STATIC_MAX_BLOCKS;
constexpr int kScratchDoubles = 32 + kCapacityBlocks;   // 256 bytes of counter slot + partials

// Reduction scratch: [0..31] counter slot (the first 4 bytes), [32..] one partial per block.
static __device__ __align__(256) double g_est_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
void* g_scratch_addr[kMaxDevices] = {nullptr};
cudaError_t g_setup_status[kMaxDevices];
std::once_flag g_setup_once[kMaxDevices];

__device__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// max |div u| over cells, velocities in the reference's Fortran layout:
// u(0:nx+2,0:ny+1,0:nz+1), v(0:nx+1,0:ny+2,0:nz+1), w(0:nx+1,0:ny+1,0:nz+2).
__global__ void __launch_bounds__(kTX * kTY) k_est_static(const double* __restrict__ u, const double* __restrict__ v,
                                                          const double* __restrict__ w, int nx, int ny, int nz,
                                                          double rdx, double rdy, double rdz, double* scratch,
                                                          double* out) {
    __shared__ double sh[kTX * kTY / 32];
    __shared__ bool last;
    const int tid = threadIdx.x + kTX * threadIdx.y;
    const int i = blockIdx.x * kTX + threadIdx.x + 1;
    const int j = blockIdx.y * kTY + threadIdx.y + 1;
    const int k0 = blockIdx.z * kZC + 1;
    const int k1 = min(k0 + kZC - 1, nz);
    const long long su = nx + 3, sv = nx + 2, sw = nx + 2;
    const long long pu = su * (ny + 2), pv = sv * (ny + 3), pw = sw * (ny + 2);
    double m = 0.0;
    if (i <= nx && j <= ny) {
        for (int k = k0; k <= k1; ++k) {
            const long long cu = i + su * j + pu * k;
            const long long cv = i + sv * j + pv * k;
            const long long cw = i + sw * j + pw * k;
            const double dv = (u[cu + 1] - u[cu]) * rdx + (v[cv + sv] - v[cv]) * rdy + (w[cw + pw] - w[cw]) * rdz;
            m = isnan(dv) ? INFINITY : fmax(m, fabs(dv));
        }
    }
    m = warp_max(m);
    if ((tid & 31) == 0) sh[tid >> 5] = m;
    __syncthreads();
    const int nb = gridDim.x * gridDim.y * gridDim.z;
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch);
    double* partial = scratch + 32;
    if (tid < 32) {
        double v2 = (tid < kTX * kTY / 32) ? sh[tid] : 0.0;
        v2 = warp_max(v2);
        if (tid == 0) {
            partial[bid] = v2;
            __threadfence();
            last = (atomicAdd(counter, 1u) == (unsigned int)(nb - 1));
        }
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double r = 0.0;
    for (int q = tid; q < nb; q += kTX * kTY) r = fmax(r, __ldcg(&partial[q]));
    r = warp_max(r);
    __syncthreads();
    if ((tid & 31) == 0) sh[tid >> 5] = r;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int q = 0; q < kTX * kTY / 32; ++q) t = fmax(t, sh[q]);
        *out = t;
        *counter = 0u;
    }
}

}  // namespace

extern "C" int suli_est_static(const double* u, const double* v, const double* w, int nx, int ny, int nz,
                               double dx, double dy, double dz, double* max_div, void* stream) {
    if (!u || !v || !w || !max_div || nx < 1 || ny < 1 || nz < 1 || !(dx > 0) || !(dy > 0) || !(dz > 0))
        return SULI_ERR_ARG;
    const long long gx = (nx + kTX - 1) / kTX, gy = (ny + kTY - 1) / kTY, gz = (nz + kZC - 1) / kZC;
    if (gx * gy * gz > kCapacityBlocks) return SULI_ERR_SIZE;   // grid beyond the static scratch
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return SULI_ERR_NODEVICE;
    // once per device, with that device current: the device address of the static scratch
    std::call_once(g_setup_once[dev], [dev]() {
        g_setup_status[dev] = cudaGetSymbolAddress(&g_scratch_addr[dev], g_est_scratch);
    });
    if (g_setup_status[dev] != cudaSuccess || !g_scratch_addr[dev]) return SULI_ERR_CUDA;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* scratch = static_cast<double*>(g_scratch_addr[dev]);
    // the counter must start at zero even if an earlier call was interrupted
    if (cudaMemsetAsync(scratch, 0, sizeof(unsigned int), s) != cudaSuccess) return SULI_ERR_CUDA;
    // the cell sizes' reciprocals, as k_est multiplies by them
    k_est_static<<<dim3((unsigned)gx, (unsigned)gy, (unsigned)gz), dim3(kTX, kTY), 0, s>>>(
        u, v, w, nx, ny, nz, 1. / dx, 1. / dy, 1. / dz, scratch, max_div);
    return (cudaGetLastError() == cudaSuccess) ? SULI_OK : SULI_ERR_CUDA;
}
