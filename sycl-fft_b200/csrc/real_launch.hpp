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

// A half length h with a fused single-pass real kernel: the stage radices of its FFT.
struct RealFusedEntry {
    int id, dbl;
    int64_t h;
    int tpl, maxt, nstages;
    int radices[16];
};
const RealFusedEntry* find_real_fused(bool dbl, int64_t h);
// One pass per real transform: R2C reads lines x 2h reals (as h complex) and writes lines x
// (h+1) bins; C2R the reverse. tw_real: W_2h^k, k = 0..h; tw_base: the FFT's base twiddles
// (per stage of radix R after ns points: W_(ns*R)^jm, jm < ns), both in the plan precision.
cudaError_t launch_real_fused(const RealFusedEntry& e, bool r2c, const void* in, void* out, int64_t lines,
                              const void* tw_real, const void* tw_base, double scale, cudaStream_t stream);

}  // namespace sfb
