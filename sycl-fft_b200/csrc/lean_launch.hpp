// Host entry of the runtime-length contiguous pass kernel (lean_kernel.cuh).
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "lean_kernel.cuh"

namespace sfb {

// True if an instantiation exists for (precision, maxv, maxt).
bool has_lean_variant(bool dbl, int maxv, int maxt);

// Launches `grid` tiles of the instantiation (precision, maxv, maxt, layout, feature).
cudaError_t launch_lean(const LeanParams& p, bool dbl, int maxv, int maxt, bool modec, int feat, int threads,
                        size_t smem, int64_t grid, const void* in, void* out, cudaStream_t stream);

}  // namespace sfb
