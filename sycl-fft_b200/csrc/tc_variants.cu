// Instantiations of the split-precision tensor-core pass kernels (tc_catalog.h).
#include <mutex>

#include "tc_catalog.h"
#include "tc_launch.hpp"

namespace sfb {
namespace {

template <int R, int S, int L, int COLS, int G>
cudaError_t launch_one(const TcParams& p, const void* in, void* out, cudaStream_t stream) {
    using Sh = TcShape<R, S, L, G>;
    auto kernel = fft_tc_kernel<R, S, L, COLS != 0, G>;
    static std::once_flag flags[64];
    static int resident[64];  // CTAs per device: SMs x blocks per SM (one for tensor-memory kernels)
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 64) return cudaErrorInvalidDevice;
    std::call_once(flags[dev], [&] {
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(Sh::SMEM));
        int sms = 0, per_sm = 0;
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, Sh::THREADS, Sh::SMEM);
        resident[dev] = sms * (per_sm > 0 ? per_sm : 1);
    });
    if (e != cudaSuccess) return e;
    if (p.tiles <= 0) return cudaSuccess;
    const int64_t groups = (p.tiles + G - 1) / G;
    const int64_t grid = groups < resident[dev] ? groups : resident[dev];
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
