// Instantiations and launcher of the copy-engine-pipelined kernels (piped_kernel.cuh).
//
// X(ID, DOUBLE, N, TPL, MAXT, RADICES...): one persistent CTA of TPL threads per SM,
// two N-element line buffers in shared memory.
#include <atomic>
#include <climits>
#include <type_traits>

#include "piped_kernel.cuh"
#include "piped_launch.hpp"

namespace sfb {
namespace {

constexpr int kMaxDevices = 64;

template <class T, int N, int TPL, int MAXT, int... Rs>
cudaError_t launch_piped_t(const PipedParams& p, int grid, const void* in, void* out, cudaStream_t stream) {
    auto kernel = fft_piped_kernel<T, N, TPL, MAXT, Rs...>;
    const size_t smem = (N + kpitch<T, N>()) * sizeof(cplx<T>) + 16;
    static std::atomic<int> configured[kMaxDevices];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    if (!configured[dev].load()) {
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        configured[dev].store(1);
    }
    if (grid <= 0) return cudaErrorInvalidConfiguration;
    kernel<<<grid, TPL, smem, stream>>>(p, static_cast<const cplx<T>*>(in), static_cast<cplx<T>*>(out));
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_piped(int id, const PipedParams& p, int grid, const void* in, void* out, cudaStream_t stream) {
    switch (id) {
#define SFB_X(ID, DBL, N, TPL, MAXT, ...) \
    case ID:                               \
        return launch_piped_t<std::conditional_t<(DBL) != 0, double, float>, N, TPL, MAXT, __VA_ARGS__>(p, grid, in, out, stream);
        SFB_PIPED_CATALOG(SFB_X)
#undef SFB_X
        default:
            return cudaErrorInvalidDeviceFunction;
    }
}

}  // namespace sfb
