// Host entry points of the size-specialised Bluestein pass kernels (bluestein_catalog.h).
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "fixed_kernel.cuh"

namespace sfb {

// One compile unit per (Rader, precision, kind): part = 8 * rader + 4 * double + kind. The
// Rader parts instantiate the same catalog entries with the gather / scatter / bin-0
// features in place of the chirp multiplies.
cudaError_t launch_blue_p0(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_blue_p1(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_blue_p2(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_blue_p3(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_blue_p4(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_blue_p5(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_blue_p6(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_blue_p7(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_blue_p8(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_blue_p9(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_blue_p10(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_blue_p11(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_blue_p12(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_blue_p13(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_blue_p14(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);
cudaError_t launch_blue_p15(int id, const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t);

inline cudaError_t launch_blue(int id, bool dbl, int kind, bool rader, const FixedParams& p, int threads, size_t smem,
                               int64_t grid, const void* in, void* out, cudaStream_t stream) {
    switch ((rader ? 8 : 0) + (dbl ? 4 : 0) + kind) {
        case 0: return launch_blue_p0(id, p, threads, smem, grid, in, out, stream);
        case 1: return launch_blue_p1(id, p, threads, smem, grid, in, out, stream);
        case 2: return launch_blue_p2(id, p, threads, smem, grid, in, out, stream);
        case 3: return launch_blue_p3(id, p, threads, smem, grid, in, out, stream);
        case 4: return launch_blue_p4(id, p, threads, smem, grid, in, out, stream);
        case 5: return launch_blue_p5(id, p, threads, smem, grid, in, out, stream);
        case 6: return launch_blue_p6(id, p, threads, smem, grid, in, out, stream);
        case 7: return launch_blue_p7(id, p, threads, smem, grid, in, out, stream);
        case 8: return launch_blue_p8(id, p, threads, smem, grid, in, out, stream);
        case 9: return launch_blue_p9(id, p, threads, smem, grid, in, out, stream);
        case 10: return launch_blue_p10(id, p, threads, smem, grid, in, out, stream);
        case 11: return launch_blue_p11(id, p, threads, smem, grid, in, out, stream);
        case 12: return launch_blue_p12(id, p, threads, smem, grid, in, out, stream);
        case 13: return launch_blue_p13(id, p, threads, smem, grid, in, out, stream);
        case 14: return launch_blue_p14(id, p, threads, smem, grid, in, out, stream);
        case 15: return launch_blue_p15(id, p, threads, smem, grid, in, out, stream);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace sfb
