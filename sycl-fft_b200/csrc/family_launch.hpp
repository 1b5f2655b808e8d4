// Host entry into the radix-family kernel (family_variants.cu).
#pragma once

#include <cuda_runtime.h>

#include "family_kernel.cuh"

namespace sfb {

// Launches the family kernel of precision `dbl` over `tiles` tiles (one block each).
cudaError_t launch_family(bool dbl, const FamilyParams& p, int64_t tiles, cudaStream_t stream);

}  // namespace sfb
