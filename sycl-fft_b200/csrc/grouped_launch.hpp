// Host entry into the grouped kernels (grouped_variants.cu).
#pragma once

#include <cuda_runtime.h>

#include "grouped_kernel.cuh"

namespace sfb {

// Launches the grouped kernel of plain contiguous-line catalog entry `fixed_id`.
cudaError_t launch_grouped(int fixed_id, const GroupParams& p, int64_t tiles, int threads, size_t smem,
                           cudaStream_t stream);

}  // namespace sfb
