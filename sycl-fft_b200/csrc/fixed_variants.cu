// Instantiations of the size-specialised kernels listed in fixed_catalog.h. Compiled
// once per SFB_FIXED_PART (0: float lines, 1: float columns, 2: double lines,
// 3: double columns) so the four groups build in parallel.
#include <atomic>
#include <climits>
#include <type_traits>

#include "fixed_catalog.h"
#include "fixed_kernel.cuh"
#include "fixed_launch.hpp"

#ifndef SFB_FIXED_PART
#error "SFB_FIXED_PART must be defined"
#endif

namespace sfb {
namespace {

constexpr int kMaxDevices = 64;

template <bool ENABLED, class T, int N, int TPL, bool MODEC, int W, int FEAT, int MAXT, int... Rs>
struct FixedLauncher {
    static cudaError_t run(const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t) {
        return cudaErrorInvalidDeviceFunction;
    }
};

template <class T, int N, int TPL, bool MODEC, int W, int FEAT, int MAXT, int... Rs>
struct FixedLauncher<true, T, N, TPL, MODEC, W, FEAT, MAXT, Rs...> {
    static cudaError_t run(const FixedParams& p, int threads, size_t smem, int64_t grid, const void* in, void* out,
                           cudaStream_t stream) {
        auto kernel = fft_fixed_kernel<T, N, TPL, MODEC, W, FEAT, MAXT, 64, Rs...>;
        static std::atomic<int> configured[kMaxDevices];
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (smem > 48 * 1024) {
            if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
            if (configured[dev].load(std::memory_order_relaxed) < static_cast<int>(smem)) {
                e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
                if (e != cudaSuccess) return e;
                int prev = configured[dev].load();
                while (prev < static_cast<int>(smem) &&
                       !configured[dev].compare_exchange_weak(prev, static_cast<int>(smem))) {
                }
            }
        }
        if (threads <= 0 || threads > MAXT || grid <= 0 || grid > INT_MAX) return cudaErrorInvalidConfiguration;
        kernel<<<static_cast<unsigned>(grid), threads, smem, stream>>>(p, static_cast<const cplx<T>*>(in),
                                                                       static_cast<cplx<T>*>(out));
        return cudaGetLastError();
    }
};

}  // namespace

cudaError_t SFB_FIXED_FN(int id, const FixedParams& p, int threads, size_t smem, int64_t grid, const void* in,
                         void* out, cudaStream_t stream) {
    switch (id) {
#define SFB_X(ID, DBL, MODEC, FEAT, N, TPL, W, MAXT, ...)                                                     \
    case ID:                                                                                                  \
        return FixedLauncher<((DBL) * 2 + (MODEC)) == SFB_FIXED_PART, std::conditional_t<(DBL) != 0, double, float>, \
                             N, TPL, (MODEC) != 0, W, FEAT, MAXT, __VA_ARGS__>::run(p, threads, smem, grid, in, out,   \
                                                                                    stream);
        SFB_FIXED_CATALOG(SFB_X)
#undef SFB_X
        default:
            return cudaErrorInvalidDeviceFunction;
    }
}

}  // namespace sfb
