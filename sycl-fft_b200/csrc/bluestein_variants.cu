// Instantiations of the size-specialised Bluestein pass kernels listed in
// bluestein_catalog.h, one compile unit per SFB_BLUE_PART = 8 * rader + 4 * double + kind
// (rader: the Rader features of the same entries).
#include <atomic>
#include <climits>
#include <type_traits>

#include "bluestein_catalog.h"
#include "bluestein_launch.hpp"
#include "fixed_kernel.cuh"

#ifndef SFB_BLUE_PART
#error "SFB_BLUE_PART must be defined"
#endif

namespace sfb {
namespace {

constexpr int kMaxDevices = 64;

// Features of each kind: fused single pass, forward column pass, row convolution pass,
// inverse column pass.
constexpr int kBlueFeat[8] = {kFeatPremul | kFeatConv | kFeatPostmul, kFeatPremul | kFeatTw4,
                              kFeatConv | kFeatTw4 | kFeatTw4Conj, kFeatPostmul,
                              // Rader: gather, convolution with the bin-0 term, scatter
                              kFeatGather | kFeatConv | kFeatScatter | kFeatRaderDC, kFeatGather | kFeatTw4,
                              kFeatConv | kFeatTw4 | kFeatTw4Conj | kFeatRaderDC, kFeatScatter};
constexpr bool kBlueModeC[4] = {false, true, false, true};

constexpr int kRader = SFB_BLUE_PART / 8;

template <bool ENABLED, class T, int KIND, int N, int TPL, int W, int MAXT, int... Rs>
struct BlueLauncher {
    static cudaError_t run(const FixedParams&, int, size_t, int64_t, const void*, void*, cudaStream_t) {
        return cudaErrorInvalidDeviceFunction;
    }
};

template <class T, int KIND, int N, int TPL, int W, int MAXT, int... Rs>
struct BlueLauncher<true, T, KIND, N, TPL, W, MAXT, Rs...> {
    static cudaError_t run(const FixedParams& p, int threads, size_t smem, int64_t grid, const void* in, void* out,
                           cudaStream_t stream) {
        auto kernel = fft_fixed_kernel<T, N, TPL, kBlueModeC[KIND], W, kBlueFeat[kRader * 4 + KIND], MAXT, 64, Rs...>;
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

#define SFB_BLUE_CAT2(a, b) a##b
#define SFB_BLUE_CAT(a, b) SFB_BLUE_CAT2(a, b)
cudaError_t SFB_BLUE_CAT(launch_blue_p, SFB_BLUE_PART)(int id, const FixedParams& p, int threads, size_t smem,
                                                      int64_t grid, const void* in, void* out, cudaStream_t stream) {
    switch (id) {
#define SFB_X(ID, DBL, KIND, N, TPL, W, MAXT, ...)                                                            \
    case ID:                                                                                                  \
        return BlueLauncher<((DBL) * 4 + (KIND)) == SFB_BLUE_PART % 8, std::conditional_t<(DBL) != 0, double, float>, \
                            KIND, N, TPL, W, MAXT, __VA_ARGS__>::run(p, threads, smem, grid, in, out, stream);
        SFB_BLUESTEIN_CATALOG(SFB_X)
#undef SFB_X
        default:
            return cudaErrorInvalidDeviceFunction;
    }
}

}  // namespace sfb
