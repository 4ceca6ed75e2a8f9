// nn_api.cuh — what the pressure solve needs from the network object (nn.cu), inside the
// library: its grid, its device and a forward pass enqueued on the caller's stream.
#pragma once
#include <cuda_runtime.h>

struct suli_nn;

namespace suli {
namespace nn {

#define SULI_NN_INTERNAL __attribute__((visibility("hidden")))

// Grid (cells) and device the network was created for.
SULI_NN_INTERNAL void dims(const suli_nn* N, int* nx, int* ny, int* nz, int* device);
// Forward pass on `stream` without synchronising: in3 [V][3] FP32 -> out [V] FP32 (device).
// Uses the network's own activation buffers.  Returns the kernels it launched (tracing counters).
SULI_NN_INTERNAL int forward_on(suli_nn* N, cudaStream_t stream, const float* d_in3, float* d_out);
// The network's input buffer, BF16 [V][16] channels last (channels 3-15 zero), and the forward
// pass from it as a caller filled it (no packing); returns the kernels launched.
SULI_NN_INTERNAL void* input16(suli_nn* N);
SULI_NN_INTERNAL int forward_packed_on(suli_nn* N, cudaStream_t stream, float* d_out);
// Nonzero (and cleared) if a tensor-core convolution's completion wait timed out since the
// last call.  Synchronous.
SULI_NN_INTERNAL int take_error(suli_nn* N);

}  // namespace nn
}  // namespace suli
