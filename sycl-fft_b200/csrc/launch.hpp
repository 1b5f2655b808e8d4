// Host entry into the pass kernels (kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "pass_params.h"

namespace sfb {

// Launches one pass. `maxv`/`maxt` select the kernel instantiation; `threads` is
// blockDim.x and `smem` the dynamic shared memory in bytes. Returns the launch error.
cudaError_t launch_pass(const PassParams& p, bool dbl, int maxv, int maxt, int threads, size_t smem,
                        const void* in, void* out, cudaStream_t stream);

// True if an instantiation exists for (precision, maxv, maxt).
bool has_variant(bool dbl, int maxv, int maxt);

// True if the pass uses a fused extra (tables, zero padding, four-step twiddle, second FFT,
// transposed store) and therefore runs the full kernel flavour.
bool needs_full(const PassParams& p);

}  // namespace sfb
