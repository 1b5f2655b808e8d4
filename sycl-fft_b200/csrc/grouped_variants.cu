// Instantiations of the grouped kernel for every plain contiguous-line entry of
// fixed_catalog.h (one launch per length family), and its launcher.
#include <atomic>
#include <climits>
#include <type_traits>

#include "fixed_catalog.h"
#include "grouped_kernel.cuh"
#include "grouped_launch.hpp"

namespace sfb {
namespace {

constexpr int kMaxDevices = 64;

template <bool ENABLED, class T, int N, int TPL, int MAXT, int... Rs>
struct GroupedLauncher {
    static cudaError_t run(const GroupParams&, int64_t, int, size_t, cudaStream_t) {
        return cudaErrorInvalidDeviceFunction;
    }
};

template <class T, int N, int TPL, int MAXT, int... Rs>
struct GroupedLauncher<true, T, N, TPL, MAXT, Rs...> {
    static cudaError_t run(const GroupParams& p, int64_t tiles, int threads, size_t smem, cudaStream_t stream) {
        auto kernel = fft_grouped_kernel<T, N, TPL, MAXT, Rs...>;
        static std::atomic<int> configured[kMaxDevices];
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
        if (smem > 48 * 1024 && configured[dev].load() < static_cast<int>(smem)) {
            e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
            if (e != cudaSuccess) return e;
            configured[dev].store(static_cast<int>(smem));
        }
        if (threads <= 0 || threads > MAXT || tiles <= 0 || tiles > INT_MAX) return cudaErrorInvalidConfiguration;
        kernel<<<static_cast<unsigned>(tiles), threads, smem, stream>>>(p);
        return cudaGetLastError();
    }
};

}  // namespace

cudaError_t launch_grouped(int fixed_id, const GroupParams& p, int64_t tiles, int threads, size_t smem,
                           cudaStream_t stream) {
    switch (fixed_id) {
#define SFB_X(ID, DBL, MODEC, FEAT, N, TPL, W, MAXT, ...)                                                  \
    case ID:                                                                                               \
        return GroupedLauncher<(MODEC) == 0 && (FEAT) == 0, std::conditional_t<(DBL) != 0, double, float>, N, \
                               TPL, MAXT, __VA_ARGS__>::run(p, tiles, threads, smem, stream);
        SFB_FIXED_CATALOG(SFB_X)
#undef SFB_X
        default:
            return cudaErrorInvalidDeviceFunction;
    }
}

}  // namespace sfb
