// Host entry into the cluster kernels (cluster_variants.cu).
#pragma once

#include <cuda_runtime.h>

#include "cluster_kernel.cuh"

namespace sfb {

// Launches cluster catalog entry `id` over prm.lines lines. With max_clusters != nullptr
// nothing is launched: it receives how many clusters of this kernel can be resident.
cudaError_t launch_cluster(int id, const ClusterParams& prm, const void* in, void* out, cudaStream_t stream,
                           int* max_clusters = nullptr);

}  // namespace sfb
