// Host entry into the size-specialised kernels (fixed_variants.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "fixed_kernel.cuh"

namespace sfb {

cudaError_t launch_fixed_p0(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_fixed_p1(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_fixed_p2(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_fixed_p3(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);

// Launches catalog entry `id` (fixed_catalog.h) of precision `dbl` and mode `modec`.
inline cudaError_t launch_fixed(int id, bool dbl, bool modec, const FixedParams& p, int threads, size_t smem,
                                int64_t grid, const void* in, void* out, cudaStream_t stream) {
    const int part = (dbl ? 2 : 0) + (modec ? 1 : 0);
    switch (part) {
        case 0: return launch_fixed_p0(id, p, threads, smem, grid, in, out, stream);
        case 1: return launch_fixed_p1(id, p, threads, smem, grid, in, out, stream);
        case 2: return launch_fixed_p2(id, p, threads, smem, grid, in, out, stream);
        default: return launch_fixed_p3(id, p, threads, smem, grid, in, out, stream);
    }
}

}  // namespace sfb
