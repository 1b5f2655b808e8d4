// Instantiations of the fused four-step kernels listed in fused4_catalog.h and their launcher.
#include <atomic>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <type_traits>

#include "fused4_catalog.h"
#include "fused4_launch.hpp"

namespace sfb {
namespace {

constexpr int kMaxDevices = 64;

#define SFB_RADICES(...) Radices<__VA_ARGS__>

template <class T, int N1, int TPL1, int W1, int N2, int TPL2, int W2, int THREADS, int MINB, int PERSIST, class RC,
          class RR>
struct Fused4Launcher {
    static constexpr int64_t smem() {
        constexpr int64_t a = int64_t(N1) * W1;
        constexpr int64_t b = int64_t(W2) * kpitch<T, N2>();
        return (a > b ? a : b) * int64_t(sizeof(cplx<T>));
    }
    // blocks of this kernel that fit one SM (cached per device after the attribute is set)
    static cudaError_t resident(int* per_sm) {
        static std::atomic<int> known[kMaxDevices];
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
        int k = known[dev].load();
        if (k <= 0) {
            auto kernel = fft_fused4_kernel<T, N1, TPL1, W1, N2, TPL2, W2, THREADS, MINB, RC, RR>;
            e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem()));
            if (e != cudaSuccess) return e;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k, kernel, THREADS, static_cast<size_t>(smem()));
            if (e != cudaSuccess) return e;
            if (k <= 0) return cudaErrorInvalidConfiguration;
            known[dev].store(k);
        }
        *per_sm = k;
        return cudaSuccess;
    }
    // persistent claim-ahead kernel or one tile per block: the catalog's choice, unless
    // SYCLFFT_B200_FUSED4_MODE=tile|persistent says otherwise
    static bool persistent() {
        static const bool v = [] {
            const char* m = std::getenv("SYCLFFT_B200_FUSED4_MODE");
            if (m && std::strcmp(m, "tile") == 0) return false;
            if (m && std::strcmp(m, "persistent") == 0) return true;
            return PERSIST != 0;
        }();
        return v;
    }
    static cudaError_t resident_p(int* per_sm) {
        static std::atomic<int> known[kMaxDevices];
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
        int k = known[dev].load();
        if (k <= 0) {
            auto kernel = fft_fused4p_kernel<T, N1, TPL1, W1, N2, TPL2, W2, THREADS, MINB, RC, RR>;
            e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem()));
            if (e != cudaSuccess) return e;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k, kernel, THREADS, static_cast<size_t>(smem()));
            if (e != cudaSuccess) return e;
            if (k <= 0) return cudaErrorInvalidConfiguration;
            known[dev].store(k);
        }
        *per_sm = k;
        return cudaSuccess;
    }
    static cudaError_t run(Fused4Params& p, const void* in, void* out, void* scratch, cudaStream_t stream) {
        using C = cplx<T>;
        constexpr int64_t L = int64_t(N1) * N2;
        constexpr int TILES = N2 / W1 + N1 / W2;  // tickets per line
        if (p.lines < 3) return cudaErrorInvalidValue;
        const bool pers = persistent();
        int per_sm = 0;
        cudaError_t e = pers ? resident_p(&per_sm) : resident(&per_sm);
        if (e != cudaSuccess) return e;
        int dev = 0, sms = 0;
        e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        const int64_t grid = int64_t(sms) * per_sm;
        int lag = 0, ring = 0;
        // persistent blocks hold a claimed-ahead ticket too: twice the tiles in flight
        if (!fused_geometry(pers ? 2 * grid : grid, TILES, p.lines, 2, kFused4MaxRing, &lag, &ring))
            return cudaErrorInvalidValue;
        p.lag = lag;
        p.ring = ring;
        const int64_t tickets = p.lines * TILES;
        if (tickets >= int64_t(INT_MAX)) return cudaErrorInvalidValue;
        auto* ctrl = reinterpret_cast<unsigned*>(static_cast<C*>(scratch) + int64_t(ring) * L);
        e = cudaMemsetAsync(ctrl, 0, kFused4CtrlWords * sizeof(unsigned), stream);
        if (e != cudaSuccess) return e;
        if (pers) {
            const int64_t blocks = grid < tickets ? grid : tickets;
            fft_fused4p_kernel<T, N1, TPL1, W1, N2, TPL2, W2, THREADS, MINB, RC, RR>
                <<<static_cast<unsigned>(blocks), THREADS, static_cast<size_t>(smem()), stream>>>(
                    p, static_cast<const C*>(in), static_cast<C*>(out), static_cast<C*>(scratch), ctrl);
            return cudaGetLastError();
        }
        // one block per tile; the resident blocks (grid) only set the lag
        fft_fused4_kernel<T, N1, TPL1, W1, N2, TPL2, W2, THREADS, MINB, RC, RR>
            <<<static_cast<unsigned>(tickets), THREADS, static_cast<size_t>(smem()), stream>>>(
                p, static_cast<const C*>(in), static_cast<C*>(out), static_cast<C*>(scratch), ctrl);
        return cudaGetLastError();
    }
};

#define SFB_FUSED4_TYPE(ID, DBL, N1, TPL1, W1, COL, N2, TPL2, W2, ROW, THREADS, MINB, PERSIST, RC, RR)              \
    Fused4Launcher<std::conditional_t<(DBL) != 0, double, float>, N1, TPL1, W1, N2, TPL2, W2, THREADS, MINB, PERSIST, \
                   SFB_RADICES RC, SFB_RADICES RR>

const Fused4Entry kEntries[] = {
#define SFB_X(ID, DBL, N1, TPL1, W1, COL, N2, TPL2, W2, ROW, THREADS, MINB, PERSIST, RC, RR) \
    {ID, DBL, N1, W1, COL, N2, W2, ROW, THREADS,                                             \
     SFB_FUSED4_TYPE(ID, DBL, N1, TPL1, W1, COL, N2, TPL2, W2, ROW, THREADS, MINB, PERSIST, RC, RR)::smem()},
    SFB_FUSED4_CATALOG(SFB_X)
#undef SFB_X
};

template <class T, int N1, int TPL1, int W1, int N2, int TPL2, int W2, int THREADS, int MINB, class RC, class RR>
struct FusedBlueLauncher {
    static constexpr int64_t smem() {
        constexpr int64_t a = int64_t(N1) * W1;
        constexpr int64_t b = int64_t(W2) * kpitch<T, N2>();
        return (a > b ? a : b) * int64_t(sizeof(cplx<T>));
    }
    static cudaError_t resident(int* per_sm) {
        static std::atomic<int> known[kMaxDevices];
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
        int k = known[dev].load();
        if (k <= 0) {
            auto kernel = fft_fusedblue_kernel<T, N1, TPL1, W1, N2, TPL2, W2, THREADS, MINB, RC, RR>;
            e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem()));
            if (e != cudaSuccess) return e;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k, kernel, THREADS, static_cast<size_t>(smem()));
            if (e != cudaSuccess) return e;
            if (k <= 0) return cudaErrorInvalidConfiguration;
            known[dev].store(k);
        }
        *per_sm = k;
        return cudaSuccess;
    }
    static cudaError_t run(FusedBlueParams& p, const void* in, void* out, void* scratch, cudaStream_t stream) {
        using C = cplx<T>;
        constexpr int64_t M = int64_t(N1) * N2;
        constexpr int TILES = 2 * (N2 / W1) + N1 / W2;  // tickets per line
        int per_sm = 0;
        cudaError_t e = resident(&per_sm);
        if (e != cudaSuccess) return e;
        int dev = 0, sms = 0;
        e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        const int64_t grid = int64_t(sms) * per_sm;
        int lag = 0, ring = 0;
        if (!fused_geometry(grid, TILES, p.lines, 3, kFused4MaxRing, &lag, &ring)) return cudaErrorInvalidValue;
        p.lag = lag;
        p.ring = ring;
        const int64_t tickets = p.lines * TILES;
        if (tickets >= int64_t(INT_MAX)) return cudaErrorInvalidValue;
        auto* ctrl = reinterpret_cast<unsigned*>(static_cast<C*>(scratch) + int64_t(ring) * M);
        e = cudaMemsetAsync(ctrl, 0, kFused4CtrlWords * sizeof(unsigned), stream);
        if (e != cudaSuccess) return e;
        // one block per tile; the resident blocks (grid) only set the lag
        fft_fusedblue_kernel<T, N1, TPL1, W1, N2, TPL2, W2, THREADS, MINB, RC, RR>
            <<<static_cast<unsigned>(tickets), THREADS, static_cast<size_t>(smem()), stream>>>(
                p, static_cast<const C*>(in), static_cast<C*>(out), static_cast<C*>(scratch), ctrl);
        return cudaGetLastError();
    }
};

#define SFB_FUSEDBLUE_TYPE(ID, DBL, N1, TPL1, W1, CF, N2, TPL2, W2, RW, CI, THREADS, MINB, RC, RR)              \
    FusedBlueLauncher<std::conditional_t<(DBL) != 0, double, float>, N1, TPL1, W1, N2, TPL2, W2, THREADS, MINB, \
                      SFB_RADICES RC, SFB_RADICES RR>

const FusedBlueEntry kBlueEntries[] = {
#define SFB_X(ID, DBL, N1, TPL1, W1, CF, N2, TPL2, W2, RW, CI, THREADS, MINB, RC, RR) \
    {ID, DBL, N1, W1, CF, N2, W2, RW, CI, THREADS,                                    \
     SFB_FUSEDBLUE_TYPE(ID, DBL, N1, TPL1, W1, CF, N2, TPL2, W2, RW, CI, THREADS, MINB, RC, RR)::smem()},
    SFB_FUSEDBLUE_CATALOG(SFB_X)
#undef SFB_X
};

}  // namespace

const FusedBlueEntry* find_fusedblue(bool dbl, int colf_id, int rows_id, int coli_id) {
    for (const auto& e : kBlueEntries)
        if (e.dbl == (dbl ? 1 : 0) && e.colf_id == colf_id && e.rows_id == rows_id && e.coli_id == coli_id) return &e;
    return nullptr;
}

cudaError_t launch_fusedblue(const FusedBlueEntry& entry, FusedBlueParams& p, const void* in, void* out,
                             void* scratch, cudaStream_t stream) {
    switch (entry.id) {
#define SFB_X(ID, DBL, N1, TPL1, W1, CF, N2, TPL2, W2, RW, CI, THREADS, MINB, RC, RR)                             \
    case ID:                                                                                                    \
        return SFB_FUSEDBLUE_TYPE(ID, DBL, N1, TPL1, W1, CF, N2, TPL2, W2, RW, CI, THREADS, MINB, RC, RR)::run( \
            p, in, out, scratch, stream);
        SFB_FUSEDBLUE_CATALOG(SFB_X)
#undef SFB_X
        default:
            return cudaErrorInvalidDeviceFunction;
    }
}

const Fused4Entry* find_fused4(bool dbl, int col_id, int row_id) {
    for (const auto& e : kEntries)
        if (e.dbl == (dbl ? 1 : 0) && e.col_id == col_id && e.row_id == row_id) return &e;
    return nullptr;
}

cudaError_t launch_fused4(const Fused4Entry& entry, Fused4Params& p, const void* in, void* out, void* scratch,
                          cudaStream_t stream) {
    switch (entry.id) {
#define SFB_X(ID, DBL, N1, TPL1, W1, COL, N2, TPL2, W2, ROW, THREADS, MINB, PERSIST, RC, RR)                  \
    case ID:                                                                                                 \
        return SFB_FUSED4_TYPE(ID, DBL, N1, TPL1, W1, COL, N2, TPL2, W2, ROW, THREADS, MINB, PERSIST, RC, RR)::run( \
            p, in, out, scratch, stream);
        SFB_FUSED4_CATALOG(SFB_X)
#undef SFB_X
        default:
            return cudaErrorInvalidDeviceFunction;
    }
}

}  // namespace sfb
