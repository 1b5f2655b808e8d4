// Host entry into the pipelined 16-CTA cluster kernel for complex<double> 65536-point lines
// (cluster_pipe.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace sfb {

struct ClusterPipeParams {
    int64_t lines = 0;
    int64_t in_pitch = 0, out_pitch = 0;  // complex elements; multiples of 65536 (16-byte rows)
    const void* tw_base = nullptr;        // base twiddles of the 256-point FFT, radices 8, 8, 4
    const void* tw4_hi = nullptr;         // W_65536^m = hi[m >> shift] * lo[m & mask]
    const void* tw4_lo = nullptr;
    int tw4_shift = 0;
    int conj_in = 0, conj_out = 0;
    double scale = 1.0;
    int* status = nullptr;  // set to 1 if a slab copy wait timed out
};

constexpr int64_t kClusterPipeLength = 65536;

// With max_clusters != nullptr nothing is launched: it receives how many clusters fit the GPU.
cudaError_t launch_cluster_pipe(const ClusterPipeParams& prm, const void* in, void* out, cudaStream_t stream,
                                int* max_clusters = nullptr);

}  // namespace sfb
