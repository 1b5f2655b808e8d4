// One compilation unit per (precision, flavour), selected by SFB_VARIANT, so the
// instantiations compile in parallel:
//   0: float  plain FFT   1: float  full (Bluestein / four-step extras)
//   2: double plain FFT   3: double full
#include <atomic>
#include <climits>

#include "launch.hpp"
#include "pass_kernel.cuh"

#ifndef SFB_VARIANT
#error "SFB_VARIANT must be defined"
#endif

namespace sfb {

namespace {

constexpr int kMaxDevices = 64;

template <class T, int MAXV, int MAXT, bool FULL>
cudaError_t launch_t(const PassParams& p, int threads, size_t smem, const void* in, void* out,
                     cudaStream_t stream) {
    auto kernel = fft_pass_kernel<T, MAXV, MAXT, FULL>;
    // Opt-in shared memory above 48 KB is a per-function, per-device attribute.
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
    if (threads <= 0 || threads > MAXT || p.tiles <= 0 || p.tiles > INT_MAX) return cudaErrorInvalidConfiguration;
    kernel<<<static_cast<unsigned>(p.tiles), threads, smem, stream>>>(p, static_cast<const cplx<T>*>(in),
                                                                      static_cast<cplx<T>*>(out));
    return cudaGetLastError();
}

}  // namespace

#if SFB_VARIANT == 0 || SFB_VARIANT == 1
#define SFB_FLAG (SFB_VARIANT == 1)
cudaError_t SFB_VARIANT_FN(const PassParams& p, int maxv, int maxt, int threads, size_t smem, const void* in,
                           void* out, cudaStream_t stream) {
    if (maxv == 16 && maxt == 256) return launch_t<float, 16, 256, SFB_FLAG>(p, threads, smem, in, out, stream);
    if (maxv == 16 && maxt == 512) return launch_t<float, 16, 512, SFB_FLAG>(p, threads, smem, in, out, stream);
    if (maxv == 16 && maxt == 1024) return launch_t<float, 16, 1024, SFB_FLAG>(p, threads, smem, in, out, stream);
    return cudaErrorInvalidDeviceFunction;
}
#else
#define SFB_FLAG (SFB_VARIANT == 3)
cudaError_t SFB_VARIANT_FN(const PassParams& p, int maxv, int maxt, int threads, size_t smem, const void* in,
                           void* out, cudaStream_t stream) {
    if (maxv == 8 && maxt == 256) return launch_t<double, 8, 256, SFB_FLAG>(p, threads, smem, in, out, stream);
    if (maxv == 8 && maxt == 512) return launch_t<double, 8, 512, SFB_FLAG>(p, threads, smem, in, out, stream);
    if (maxv == 8 && maxt == 1024) return launch_t<double, 8, 1024, SFB_FLAG>(p, threads, smem, in, out, stream);
    if (maxv == 16 && maxt == 256) return launch_t<double, 16, 256, SFB_FLAG>(p, threads, smem, in, out, stream);
    if (maxv == 16 && maxt == 512) return launch_t<double, 16, 512, SFB_FLAG>(p, threads, smem, in, out, stream);
    return cudaErrorInvalidDeviceFunction;
}
#endif

}  // namespace sfb
