// Instantiations of the split-precision tensor-core pass kernels (tc_catalog.h).
#include <atomic>

#include "tc_catalog.h"
#include "tc_launch.hpp"

namespace sfb {
namespace {

template <int R, int S, int L, int COLS, int G>
cudaError_t launch_one(const TcParams& p, const void* in, void* out, cudaStream_t stream) {
    using Sh = TcShape<R, S, L, G>;
    auto kernel = fft_tc_kernel<R, S, L, COLS != 0, G>;
    // CTAs per device: SMs x blocks per SM (one for tensor-memory kernels). Looked up on the
    // first launch on a device and kept only when every query succeeded, so a failed first
    // attempt is retried instead of being remembered.
    static std::atomic<int> resident[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (resident[dev].load() <= 0) {
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(Sh::SMEM));
        int sms = 0, per_sm = 0;
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, Sh::THREADS, Sh::SMEM);
        if (e != cudaSuccess) return e;
        if (per_sm <= 0) return cudaErrorInvalidConfiguration;
        resident[dev].store(sms * per_sm);
    }
    if (p.tiles <= 0) return cudaSuccess;
    const int64_t groups = (p.tiles + G - 1) / G;
    const int64_t res = resident[dev].load();
    const int64_t grid = groups < res ? groups : res;
    kernel<<<dim3(static_cast<unsigned>(grid)), dim3(Sh::THREADS), Sh::SMEM, stream>>>(
        p, static_cast<const float2*>(in), static_cast<float2*>(out));
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_tc(int id, const TcParams& p, const void* in, void* out, cudaStream_t stream) {
    switch (id) {
#define SFB_TC_CASE(ID, R, S, L, COLS, G) \
    case ID:                              \
        return launch_one<R, S, L, COLS, G>(p, in, out, stream);
        SFB_TC_CATALOG(SFB_TC_CASE)
#undef SFB_TC_CASE
        default:
            return cudaErrorInvalidValue;
    }
}

}  // namespace sfb
