// Device-side Bluestein table generation (bluestein_init.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace sfb {

// chirp[n] (plan precision, n < L) and the mirrored convolution kernel kern[M] (FP64).
cudaError_t bluestein_chirp(bool dbl, void* chirp, void* kern, int64_t L, int64_t M, int sgn, cudaStream_t s);
// out = K / M in the plan precision, permuted to K'[k1*n2+k2] = K[k1+n1*k2] when `large`.
cudaError_t bluestein_spectrum(bool dbl, void* out, const void* K, int64_t M, int64_t n1, int64_t n2, bool large,
                               cudaStream_t s);

}  // namespace sfb
