// Instantiations and launcher of the cluster kernels listed in cluster_catalog.h.
#include <atomic>
#include <climits>
#include <type_traits>

#include "cluster_catalog.h"
#include "cluster_kernel.cuh"
#include "cluster_launch.hpp"

namespace sfb {
namespace {

constexpr int kMaxDevices = 64;

template <class T, int N1, int N2, int P, int TPL1, int TPL2, int MAXT, int MINB, class R1, class R2>
cudaError_t launch_cluster_t(const ClusterParams& prm, const void* in, void* out, cudaStream_t stream,
                             int* max_clusters) {
    auto kernel = fft_cluster_kernel<T, N1, N2, P, TPL1, TPL2, R1, R2, MAXT, MINB>;
    using C = cplx<T>;
    const size_t smem = sizeof(C) * (size_t)(N1 * N2 / P);
    constexpr int threads = (N2 / P) * TPL1 > (N1 / P) * TPL2 ? (N2 / P) * TPL1 : (N1 / P) * TPL2;
    static_assert(threads <= MAXT, "cluster kernel CTA exceeds its launch bound");
    static std::atomic<int> configured[kMaxDevices];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    if (!configured[dev].load()) {
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        if (P > 8) {
            e = cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            if (e != cudaSuccess) return e;
        }
        configured[dev].store(1);
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(prm.lines * P), 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = P;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (max_clusters) {
        return cudaOccupancyMaxActiveClusters(max_clusters, kernel, &cfg);
    }
    if (prm.lines <= 0 || prm.lines * P > INT_MAX) return cudaErrorInvalidConfiguration;
    e = cudaLaunchKernelEx(&cfg, kernel, prm, static_cast<const C*>(in), static_cast<C*>(out));
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

#define SFB_EXPAND(...) __VA_ARGS__

}  // namespace

cudaError_t launch_cluster(int id, const ClusterParams& prm, const void* in, void* out, cudaStream_t stream,
                           int* max_clusters) {
    switch (id) {
#define SFB_X(ID, DBL, N1, N2, P, TPL1, TPL2, MAXT, MINB, R1, R2)                                           \
    case ID:                                                                                                \
        return launch_cluster_t<std::conditional_t<(DBL) != 0, double, float>, N1, N2, P, TPL1, TPL2, MAXT, MINB, \
                                RadixSeq<SFB_EXPAND R1>, RadixSeq<SFB_EXPAND R2>>(prm, in, out, stream,     \
                                                                                  max_clusters);
        SFB_CLUSTER_CATALOG(SFB_X)
#undef SFB_X
        default:
            return cudaErrorInvalidDeviceFunction;
    }
}

}  // namespace sfb
