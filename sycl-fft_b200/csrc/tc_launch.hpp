// Host entry point of the split-precision tensor-core pass kernels (tc_catalog.h ids).
#pragma once

#include <cuda_runtime.h>

#include "tc_kernel.cuh"

namespace sfb {

cudaError_t launch_tc(int id, const TcParams& p, const void* in, void* out, cudaStream_t stream);

}  // namespace sfb
