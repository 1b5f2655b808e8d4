// Device-side generation of a Bluestein plan's chirp and chirp spectrum.
//
// h_n = exp(-i*sgn*pi*r/L) with r = n^2 mod 2L computed in exact integer arithmetic and the
// angle evaluated in FP64 (sincospi); the convolution kernel is h mirrored into a
// zero-padded line of length M (h[n] and h[M-n] for 1 <= n < L); its spectrum is an FP64
// FFT of length M run by the provider itself, then divided by M, permuted for the
// three-pass form (K'[k1*n2 + k2] = K[k1 + n1*k2]) and stored in the plan precision.
#include <cuda_runtime.h>

#include "bluestein_init.hpp"
#include "butterfly.cuh"

namespace sfb {
namespace {

__device__ __forceinline__ double2 chirp_h(int64_t n, int64_t L, int sgn) {
    const uint64_t r = (static_cast<uint64_t>(n) * static_cast<uint64_t>(n)) % static_cast<uint64_t>(2 * L);
    double s, c;
    sincospi(static_cast<double>(r) / static_cast<double>(L), &s, &c);
    return make_double2(c, -sgn * s);
}

template <class T>
__global__ void chirp_kernel(cplx<T>* chirp, double2* kern, int64_t L, int64_t M, int sgn) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= M) return;
    double2 v = make_double2(0.0, 0.0);
    if (i < L) {
        v = chirp_h(i, L, sgn);
        cplx<T> c;
        c.x = static_cast<T>(v.x);
        c.y = static_cast<T>(-v.y);
        chirp[i] = c;
    } else if (M - i < L) {
        v = chirp_h(M - i, L, sgn);
    }
    kern[i] = v;
}

template <class T>
__global__ void spectrum_kernel(cplx<T>* out, const double2* K, int64_t M, int64_t n1, int64_t n2, int large) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= M) return;
    int64_t src = i;
    if (large) {
        const int64_t k1 = i / n2, k2 = i - k1 * n2;
        src = k1 + n1 * k2;
    }
    const double inv = 1.0 / static_cast<double>(M);
    cplx<T> v;
    v.x = static_cast<T>(K[src].x * inv);
    v.y = static_cast<T>(K[src].y * inv);
    out[i] = v;
}

}  // namespace

cudaError_t bluestein_chirp(bool dbl, void* chirp, void* kern, int64_t L, int64_t M, int sgn, cudaStream_t s) {
    const unsigned blocks = static_cast<unsigned>((M + 255) / 256);
    if (dbl) chirp_kernel<double><<<blocks, 256, 0, s>>>(static_cast<double2*>(chirp), static_cast<double2*>(kern), L, M, sgn);
    else chirp_kernel<float><<<blocks, 256, 0, s>>>(static_cast<float2*>(chirp), static_cast<double2*>(kern), L, M, sgn);
    return cudaGetLastError();
}

cudaError_t bluestein_spectrum(bool dbl, void* out, const void* K, int64_t M, int64_t n1, int64_t n2, bool large,
                               cudaStream_t s) {
    const unsigned blocks = static_cast<unsigned>((M + 255) / 256);
    if (dbl)
        spectrum_kernel<double><<<blocks, 256, 0, s>>>(static_cast<double2*>(out), static_cast<const double2*>(K), M, n1, n2, large);
    else
        spectrum_kernel<float><<<blocks, 256, 0, s>>>(static_cast<float2*>(out), static_cast<const double2*>(K), M, n1, n2, large);
    return cudaGetLastError();
}

}  // namespace sfb
