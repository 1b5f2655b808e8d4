// Real-to-complex and complex-to-real transforms of even length N = 2H over a complex FFT of
// length H (the real line read as H complex values z[m] = x[2m] + i x[2m+1]).
//
//   R2C, after Z = FFT_H(z):  X[k] = 1/2 [ (Z[k] + conj Z[H-k]) - i W_N^k (Z[k] - conj Z[H-k]) ],
//                             k = 0..H (indices of Z mod H), W_N^k = exp(-2 pi i k / N);
//   C2R, before z = IFFT_H(Z) (unnormalized):
//                             Z[k] = (X[k] + conj X[H-k]) + i conj(W_N^k) (X[k] - conj X[H-k]),
//                             k = 0..H-1, with the imaginary parts of X[0] and X[H] ignored;
//                             x[2m] = Re z[m], x[2m+1] = Im z[m].
// Each thread handles the pair (k, H - k), so both of its values are read once; the
// normalization scale is fused.
//
// Where the half length H has a size-specialised single-CTA kernel (the catalog below), the
// pre-/post-process is fused into it instead (kFeatRealPre / kFeatRealPost of
// fixed_kernel.cuh): one HBM pass per real transform.
#include <atomic>
#include <type_traits>

#include <cuda_runtime.h>

#include "butterfly.cuh"
#include "fixed_kernel.cuh"
#include "real_launch.hpp"

namespace sfb {
namespace {

template <class T>
__global__ void r2c_post_kernel(const cplx<T>* __restrict__ Z, cplx<T>* __restrict__ X, int64_t H, int64_t lines,
                                const cplx<T>* __restrict__ tw, T scale) {
    using C = cplx<T>;
    const int64_t pairs = H / 2 + 1;
    const T half = T(0.5) * scale;
    auto post = [&](C a, C c, C w) {
        // Zk = a, Zc = conj(c): E = Zk + Zc, D = Zk - Zc, X = 1/2 (E - i w D)
        const C e = cmake<C>(a.x + c.x, a.y - c.y);
        const C d = cmake<C>(a.x - c.x, a.y + c.y);
        const T p = w.x * d.x - w.y * d.y, q = w.x * d.y + w.y * d.x;  // w * D
        return cmake<C>((e.x + q) * half, (e.y - p) * half);
    };
    for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < lines * pairs;
         idx += int64_t(gridDim.x) * blockDim.x) {
        const int64_t b = idx / pairs, k = idx - b * pairs;
        const C* z = Z + b * H;
        C* x = X + b * (H + 1);
        const int64_t kk = H - k;
        const C a = z[k];
        const C c = z[kk == H ? 0 : kk];
        x[k] = post(a, c, __ldg(tw + k));
        if (kk != k) x[kk] = post(c, a, __ldg(tw + kk));
    }
}

template <class T>
__global__ void c2r_pre_kernel(const cplx<T>* __restrict__ X, cplx<T>* __restrict__ Z, int64_t H, int64_t lines,
                               const cplx<T>* __restrict__ tw, T scale) {
    using C = cplx<T>;
    const int64_t pairs = H / 2 + 1;
    auto pre = [&](C a, C c, C w) {
        // Xk = a, Xc = conj(c): E = Xk + Xc, D = Xk - Xc, Z = E + i conj(w) D
        const C e = cmake<C>(a.x + c.x, a.y - c.y);
        const C d = cmake<C>(a.x - c.x, a.y + c.y);
        const T p = w.x * d.x + w.y * d.y, q = w.x * d.y - w.y * d.x;  // conj(w) * D
        return cmake<C>((e.x - q) * scale, (e.y + p) * scale);
    };
    for (int64_t idx = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; idx < lines * pairs;
         idx += int64_t(gridDim.x) * blockDim.x) {
        const int64_t b = idx / pairs, k = idx - b * pairs;
        const C* x = X + b * (H + 1);
        C* z = Z + b * H;
        const int64_t kk = H - k;
        C a = x[k];
        C c = x[kk];
        if (k == 0) {
            a.y = T(0);  // the DC and Nyquist bins of a real signal are real
            c.y = T(0);
            z[0] = pre(a, c, __ldg(tw));
        } else {
            z[k] = pre(a, c, __ldg(tw + k));
            if (kk != k) z[kk] = pre(c, a, __ldg(tw + kk));
        }
    }
}

// X(ID, DOUBLE, H, TPL, MAXT, RADICES...): the fixed_catalog.h line kernels of these lengths.
#define SFB_REAL_FUSED_CATALOG(X)      \
    X(0, 0, 256, 16, 256, 16, 16)      \
    X(1, 0, 512, 32, 256, 16, 16, 2)   \
    X(2, 0, 1024, 64, 256, 16, 16, 4)  \
    X(3, 0, 2048, 128, 256, 16, 16, 8) \
    X(4, 0, 4096, 256, 256, 16, 16, 16) \
    X(5, 1, 256, 32, 256, 8, 8, 4)     \
    X(6, 1, 512, 64, 256, 8, 8, 8)     \
    X(7, 1, 1024, 128, 256, 8, 8, 8, 2) \
    X(8, 1, 2048, 256, 256, 8, 8, 8, 4)

template <int... Rs>
struct StageCount {
    static constexpr int value = sizeof...(Rs);
};

constexpr int kMaxDevices = 64;

template <class T, int N, int TPL, int MAXT, int FEAT, int... Rs>
cudaError_t launch_fused_t(const FixedParams& p, int64_t lines, const void* in, void* out, cudaStream_t stream) {
    auto kernel = fft_fixed_kernel<T, N, TPL, false, 1, FEAT, MAXT, 64, Rs...>;
    const int w = p.w;
    const size_t smem = static_cast<size_t>(w) * kpitch<T, N>() * sizeof(cplx<T>);
    if (smem > 48 * 1024) {
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
    }
    const int64_t grid = (lines + w - 1) / w;
    if (grid <= 0 || grid > INT32_MAX) return cudaErrorInvalidConfiguration;
    kernel<<<static_cast<unsigned>(grid), w * TPL, smem, stream>>>(p, static_cast<const cplx<T>*>(in),
                                                                   static_cast<cplx<T>*>(out));
    return cudaGetLastError();
}

int grid_for(int64_t work) {
    const int64_t blocks = (work + 255) / 256;
    return static_cast<int>(blocks < 148 * 16 ? blocks : 148 * 16);
}

}  // namespace

const RealFusedEntry* find_real_fused(bool dbl, int64_t h) {
    static const RealFusedEntry entries[] = {
#define SFB_X(ID, DBL, H, TPL, MAXT, ...) {ID, DBL, H, TPL, MAXT, StageCount<__VA_ARGS__>::value, {__VA_ARGS__}},
        SFB_REAL_FUSED_CATALOG(SFB_X)
#undef SFB_X
    };
    for (const auto& e : entries)
        if (e.dbl == (dbl ? 1 : 0) && e.h == h) return &e;
    return nullptr;
}

cudaError_t launch_real_fused(const RealFusedEntry& e, bool r2c, const void* in, void* out, int64_t lines,
                              const void* tw_real, const void* tw_base, double scale, cudaStream_t stream) {
    if (lines <= 0) return cudaSuccess;
    FixedParams p{};
    p.n_cols = lines;
    p.w = e.maxt / e.tpl > 0 ? e.maxt / e.tpl : 1;
    p.col_tiles = (lines + p.w - 1) / p.w;
    p.in_pitch = r2c ? e.h : e.h + 1;
    p.out_pitch = r2c ? e.h + 1 : e.h;
    p.tw = tw_base;
    p.conj_in = p.conj_out = r2c ? 0 : 1;  // C2R: the unnormalized inverse as conj(FFT(conj z))
    p.scale = scale;
    if (r2c) p.postmul = tw_real;
    else p.premul = tw_real;
    switch (e.id) {
#define SFB_X(ID, DBL, H, TPL, MAXT, ...)                                                                    \
    case ID:                                                                                                 \
        return r2c ? launch_fused_t<std::conditional_t<(DBL) != 0, double, float>, H, TPL, MAXT, kFeatRealPost, \
                                    __VA_ARGS__>(p, lines, in, out, stream)                                    \
                   : launch_fused_t<std::conditional_t<(DBL) != 0, double, float>, H, TPL, MAXT, kFeatRealPre,  \
                                    __VA_ARGS__>(p, lines, in, out, stream);
        SFB_REAL_FUSED_CATALOG(SFB_X)
#undef SFB_X
        default:
            return cudaErrorInvalidDeviceFunction;
    }
}

cudaError_t launch_r2c_post(bool dbl, const void* z, void* x, int64_t h, int64_t lines, const void* tw, double scale,
                            cudaStream_t stream) {
    const int64_t work = lines * (h / 2 + 1);
    if (work <= 0) return cudaSuccess;
    if (dbl)
        r2c_post_kernel<double><<<grid_for(work), 256, 0, stream>>>(static_cast<const double2*>(z),
                                                                     static_cast<double2*>(x), h, lines,
                                                                     static_cast<const double2*>(tw), scale);
    else
        r2c_post_kernel<float><<<grid_for(work), 256, 0, stream>>>(static_cast<const float2*>(z),
                                                                   static_cast<float2*>(x), h, lines,
                                                                   static_cast<const float2*>(tw),
                                                                   static_cast<float>(scale));
    return cudaGetLastError();
}

cudaError_t launch_c2r_pre(bool dbl, const void* x, void* z, int64_t h, int64_t lines, const void* tw, double scale,
                           cudaStream_t stream) {
    const int64_t work = lines * (h / 2 + 1);
    if (work <= 0) return cudaSuccess;
    if (dbl)
        c2r_pre_kernel<double><<<grid_for(work), 256, 0, stream>>>(static_cast<const double2*>(x),
                                                                    static_cast<double2*>(z), h, lines,
                                                                    static_cast<const double2*>(tw), scale);
    else
        c2r_pre_kernel<float><<<grid_for(work), 256, 0, stream>>>(static_cast<const float2*>(x),
                                                                  static_cast<float2*>(z), h, lines,
                                                                  static_cast<const float2*>(tw),
                                                                  static_cast<float>(scale));
    return cudaGetLastError();
}

}  // namespace sfb
