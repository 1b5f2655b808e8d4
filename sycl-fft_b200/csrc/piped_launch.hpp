// Host entry into the copy-engine-pipelined kernels (piped_variants.cu).
#pragma once

#include <cuda_runtime.h>

#include "piped_catalog.h"
#include "piped_kernel.cuh"

namespace sfb {

// Launches pipelined catalog entry `id` on `grid` persistent CTAs.
cudaError_t launch_piped(int id, const PipedParams& p, int grid, const void* in, void* out, cudaStream_t stream);

}  // namespace sfb
