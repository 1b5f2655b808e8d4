// Instantiations of the runtime-length contiguous pass kernel (lean_kernel.cuh): float with 16
// values per thread, double with 8 or 16, CTA bounds 256 / 512 / 1024, and the three
// (layout, feature) pairs kModeK plain, kModeC four-step twiddle, kModeC plain (four-step rows).
#include <atomic>
#include <climits>

#include "lean_launch.hpp"
#include "planner.hpp"

namespace sfb {
namespace {

constexpr int kMaxDevices = 64;

template <class T, int MAXV, int MAXT, bool MODEC, int FEAT>
cudaError_t run(const LeanParams& p, int threads, size_t smem, int64_t grid, const void* in, void* out,
                cudaStream_t stream) {
    auto kernel = fft_lean_kernel<T, MAXV, MAXT, MODEC, FEAT>;
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
            while (prev < static_cast<int>(smem) && !configured[dev].compare_exchange_weak(prev, static_cast<int>(smem))) {
            }
        }
    }
    if (threads <= 0 || threads > MAXT || grid <= 0 || grid > INT_MAX) return cudaErrorInvalidConfiguration;
    kernel<<<static_cast<unsigned>(grid), threads, smem, stream>>>(p, static_cast<const cplx<T>*>(in),
                                                                   static_cast<cplx<T>*>(out));
    return cudaGetLastError();
}

template <class T, int MAXV, int MAXT>
cudaError_t by_layout(const LeanParams& p, bool modec, int feat, int threads, size_t smem, int64_t grid,
                      const void* in, void* out, cudaStream_t stream) {
    if (!modec && feat == kLeanPlain) return run<T, MAXV, MAXT, false, kLeanPlain>(p, threads, smem, grid, in, out, stream);
    if (modec && feat == kLeanTw4) return run<T, MAXV, MAXT, true, kLeanTw4>(p, threads, smem, grid, in, out, stream);
    if (modec && feat == kLeanPlain) return run<T, MAXV, MAXT, true, kLeanPlain>(p, threads, smem, grid, in, out, stream);
    return cudaErrorInvalidDeviceFunction;
}

}  // namespace

bool has_lean_variant(bool dbl, int maxv, int maxt) { return lean_variant_exists(dbl, maxv, maxt); }

cudaError_t launch_lean(const LeanParams& p, bool dbl, int maxv, int maxt, bool modec, int feat, int threads,
                        size_t smem, int64_t grid, const void* in, void* out, cudaStream_t stream) {
    if (!dbl) {
        if (maxv != 16) return cudaErrorInvalidDeviceFunction;
        if (maxt == 256) return by_layout<float, 16, 256>(p, modec, feat, threads, smem, grid, in, out, stream);
        if (maxt == 512) return by_layout<float, 16, 512>(p, modec, feat, threads, smem, grid, in, out, stream);
        if (maxt == 1024) return by_layout<float, 16, 1024>(p, modec, feat, threads, smem, grid, in, out, stream);
        return cudaErrorInvalidDeviceFunction;
    }
    if (maxv == 8) {
        if (maxt == 256) return by_layout<double, 8, 256>(p, modec, feat, threads, smem, grid, in, out, stream);
        if (maxt == 512) return by_layout<double, 8, 512>(p, modec, feat, threads, smem, grid, in, out, stream);
        if (maxt == 1024) return by_layout<double, 8, 1024>(p, modec, feat, threads, smem, grid, in, out, stream);
    }
    if (maxv == 16) {
        if (maxt == 256) return by_layout<double, 16, 256>(p, modec, feat, threads, smem, grid, in, out, stream);
        if (maxt == 512) return by_layout<double, 16, 512>(p, modec, feat, threads, smem, grid, in, out, stream);
    }
    return cudaErrorInvalidDeviceFunction;
}

}  // namespace sfb
