// Instantiations of the radix-family kernel (family_kernel.cuh) and its launcher.
#include <atomic>
#include <climits>

#include "family_kernel.cuh"
#include "family_launch.hpp"

namespace sfb {
namespace {

constexpr int kMaxDevices = 64;

template <class T>
cudaError_t run_family(const FamilyParams& p, int64_t tiles, cudaStream_t stream) {
    auto kernel = fft_family_kernel<T>;
    constexpr size_t smem = static_cast<size_t>(family_smem_elems<T>()) * sizeof(cplx<T>);
    static std::atomic<int> configured[kMaxDevices];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    if (smem > 48 * 1024 && !configured[dev].load()) {
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        configured[dev].store(1);
    }
    if (tiles <= 0 || tiles > INT_MAX) return cudaErrorInvalidConfiguration;
    kernel<<<static_cast<unsigned>(tiles), kFamilyThreads, smem, stream>>>(p);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_family(bool dbl, const FamilyParams& p, int64_t tiles, cudaStream_t stream) {
    return dbl ? run_family<double>(p, tiles, stream) : run_family<float>(p, tiles, stream);
}

}  // namespace sfb
