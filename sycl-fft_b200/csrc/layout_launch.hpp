// Host side of the strided-layout gather / scatter kernels (layout_kernel.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace sfb {

// A batch of `batch` transforms of shape len[0..rank): element (b, i0, .., i_{r-1}) at
// b * dist + sum_k i_k * stride[k] complex elements from the buffer's start.
struct Layout {
    int rank = 1;
    int64_t len[3] = {1, 1, 1};
    int64_t stride[3] = {1, 1, 1};
    int64_t dist = 0;
    int64_t batch = 1;
};

// strided `layout` in src -> contiguous batch-major dst
cudaError_t launch_layout_gather(bool dbl, const void* src, const Layout& layout, void* dst, cudaStream_t stream);
// contiguous batch-major src -> strided `layout` in dst
cudaError_t launch_layout_scatter(bool dbl, const void* src, void* dst, const Layout& layout, cudaStream_t stream);

}  // namespace sfb
