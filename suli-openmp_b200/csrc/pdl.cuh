// pdl.cuh — programmatic dependent launch for the solvers' iteration kernels.
//
// A kernel launched with programmatic stream serialisation may start while its predecessor in
// the stream is still draining; it waits in pdl_wait() (griddepcontrol.wait) before reading
// anything the predecessor wrote, which overlaps the launch and block ramp-up of consecutive
// iteration kernels.  For a plain launch pdl_wait() is a no-op.
#pragma once
#include <cuda_runtime.h>

namespace suli {

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// launch with programmatic stream serialisation (the kernel calls pdl_wait before its loads)
template <typename... KArgs, typename... Args>
static void pdl_launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t stream, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

}  // namespace suli
