// Instantiations of the TMA-staged four-step column kernels: every column-pass entry
// (kModeC, four-step twiddle) of fixed_catalog.h whose length fits one tensor-map box (<= 256).
#include <cudaTypedefs.h>

#include <atomic>
#include <climits>
#include <mutex>
#include <type_traits>

#include "fixed_catalog.h"
#include "tma_launch.hpp"

namespace sfb {
namespace {

constexpr int kMaxDevices = 64;
#ifndef SFB_TMA_BUFFERS
#define SFB_TMA_BUFFERS 1
#endif
constexpr int kTmaBuffers = SFB_TMA_BUFFERS;

PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

template <bool ENABLED, class T, int N, int TPL, int W, int... Rs>
struct TmaLauncher {
    static cudaError_t run(const void*, void*, int64_t, const TmaColParams&, cudaStream_t) {
        return cudaErrorInvalidDeviceFunction;
    }
};

template <class T, int N, int TPL, int W, int... Rs>
struct TmaLauncher<true, T, N, TPL, W, Rs...> {
    static cudaError_t run(const void* in, void* out, int64_t lines, const TmaColParams& p, cudaStream_t stream) {
        constexpr int NBUF = kTmaBuffers;
        auto kernel = fft_tma_cols_kernel<T, N, TPL, W, NBUF, Rs...>;
        constexpr size_t smem = NBUF * size_t(N) * W * sizeof(cplx<T>) + 16;
        static std::once_flag once[kMaxDevices];
        static int resident[kMaxDevices];
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
        std::call_once(once[dev], [&] {
            e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
            int sms = 0, per_sm = 0;
            if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, W * TPL, smem);
            resident[dev] = sms * (per_sm > 0 ? per_sm : 1);
        });
        if (e != cudaSuccess) return e;
        auto encode = encode_tiled();
        if (!encode || p.tiles <= 0 || lines > INT_MAX || (reinterpret_cast<uintptr_t>(in) % 16) != 0)
            return cudaErrorInvalidValue;
        // dims (innermost first): reals of a row (2 * n2), rows (N), lines
        CUtensorMap map;
        const cuuint64_t dims[3] = {cuuint64_t(2) * p.n2, cuuint64_t(N), cuuint64_t(lines)};
        const cuuint64_t strides[2] = {cuuint64_t(2) * p.n2 * sizeof(T), cuuint64_t(2) * p.n2 * N * sizeof(T)};
        const cuuint32_t box[3] = {cuuint32_t(2 * W), cuuint32_t(N), 1};
        const cuuint32_t estr[3] = {1, 1, 1};
        const CUresult r = encode(&map, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                                  3, const_cast<void*>(in), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
        // one buffer: a CTA per tile as far as the GPU holds them (no prefetch, the other CTAs
        // on the SM overlap); two buffers: persistent CTAs prefetching their next tile
        const int64_t grid = NBUF == 1 ? p.tiles : (p.tiles < resident[dev] ? p.tiles : resident[dev]);
        kernel<<<static_cast<unsigned>(grid), W * TPL, smem, stream>>>(map, p, static_cast<cplx<T>*>(out));
        return cudaGetLastError();
    }
};

#define SFB_TMA_ENABLED(MODEC, FEAT, N) ((MODEC) == 1 && (FEAT) == 1 && (N) <= 256)

}  // namespace

bool tma_cols_available(int fixed_id) {
    switch (fixed_id) {
#define SFB_X(ID, DBL, MODEC, FEAT, N, TPL, W, MAXT, ...) \
    case ID:                                             \
        return SFB_TMA_ENABLED(MODEC, FEAT, N);
        SFB_FIXED_CATALOG(SFB_X)
#undef SFB_X
        default:
            return false;
    }
}

cudaError_t launch_tma_cols(int fixed_id, const void* in, void* out, int64_t lines, const TmaColParams& p,
                            cudaStream_t stream) {
    switch (fixed_id) {
#define SFB_X(ID, DBL, MODEC, FEAT, N, TPL, W, MAXT, ...)                                                       \
    case ID:                                                                                                    \
        return TmaLauncher<SFB_TMA_ENABLED(MODEC, FEAT, N), std::conditional_t<(DBL) != 0, double, float>, N, TPL, \
                           W, __VA_ARGS__>::run(in, out, lines, p, stream);
        SFB_FIXED_CATALOG(SFB_X)
#undef SFB_X
        default:
            return cudaErrorInvalidDeviceFunction;
    }
}

}  // namespace sfb
