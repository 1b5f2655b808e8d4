// Host entry point of the TMA-staged four-step column kernels (tma_cols_kernel.cuh): one per
// size-specialised column-pass entry of fixed_catalog.h with N <= 256.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "tma_cols_kernel.cuh"

namespace sfb {

// Whether catalog entry `fixed_id` has a TMA-staged variant.
bool tma_cols_available(int fixed_id);

// Encodes the input's tensor map (lines x N1 rows x n2 columns, contiguous) and launches the
// persistent kernel. cudaErrorInvalidValue when the map cannot be encoded (the caller then
// runs the plain kernel).
cudaError_t launch_tma_cols(int fixed_id, const void* in, void* out, int64_t lines, const TmaColParams& p,
                            cudaStream_t stream);

}  // namespace sfb
