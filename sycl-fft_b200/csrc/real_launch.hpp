// Host entry points of the real-transform post- and pre-process kernels (real_kernel.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace sfb {

// R2C: Z (lines x h complex, the half-length FFT of the real lines) -> X (lines x (h+1)).
cudaError_t launch_r2c_post(bool dbl, const void* z, void* x, int64_t h, int64_t lines, const void* tw, double scale,
                            cudaStream_t stream);
// C2R: X (lines x (h+1) complex) -> Z (lines x h), to be inverse-transformed at length h.
cudaError_t launch_c2r_pre(bool dbl, const void* x, void* z, int64_t h, int64_t lines, const void* tw, double scale,
                           cudaStream_t stream);

}  // namespace sfb
