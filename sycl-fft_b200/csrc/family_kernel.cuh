// Radix-family launch: requests of different lengths of one radix family in one kernel.
//
// A family is the power-of-two lengths whose size-specialised single-pass kernels share a
// block shape: complex<float> 64 .. 4096 (16 values per thread, TPL = N / 16) and
// complex<double> 64 .. 2048 (8 values per thread, TPL = N / 8), 256 threads per block, so a
// block holds 256 / TPL lines of any of them in the same ~35 KB of shared memory. Each request
// (its own length, buffers, batch, direction and normalization) contributes ceil(lines / W)
// tiles; a block finds its request by binary search over the first-tile indices and dispatches
// on the request's length to that length's compiled stages (fixed_kernel.cuh), with the radix
// sequences of the single-pass catalog entries. One block per tile: there is no persistent
// loop (the stage code's loop-invariant state would be kept live across tiles and spill).
// The request table travels in the kernel parameters, so a launch needs no device staging and
// can be captured in a CUDA graph.
#pragma once

#include <cuda_runtime.h>

#include "fixed_kernel.cuh"

namespace sfb {

constexpr int kFamilyMaxItems = 256;
constexpr int kFamilyThreads = 256;

struct FamilyItem {
    const void* in;
    void* out;
    const void* tw;      // base twiddles of this length's radix sequence
    int64_t lines;
    int64_t tile_begin;  // first tile of this request in the launch
    double scale;
    int conj;            // 1: inverse transform (conjugate on load and store)
    int log2n;
};

struct FamilyParams {
    int count;
    FamilyItem items[kFamilyMaxItems];
};

template <class T, int N, int... Rs>
__device__ __forceinline__ void family_tile(const FamilyItem& it, int64_t tile, cplx<T>* sm) {
    using C = cplx<T>;
    constexpr int TPL = N / (sizeof(T) == 4 ? 16 : 8);
    constexpr int W = kFamilyThreads / TPL;  // lines per tile
    const int tid = threadIdx.x;
    const int w = tid / TPL;
    FixedCtx<T> X;
    X.t = tid - w * TPL;
    X.active = w < W;
    const int64_t c = (tile - it.tile_begin) * W + w;
    X.line_ok = X.active && c < it.lines;
    X.sm = sm + w * kpitch<T, N>();
    X.gin = static_cast<const C*>(it.in) + c * N;
    X.gout = static_cast<C*>(it.out) + c * N;
    X.twb = static_cast<const C*>(it.tw);
    X.in_ks = 1;
    X.out_ks = 1;
    X.scale = static_cast<T>(it.scale);
    X.conj_in = it.conj != 0;
    X.conj_out = it.conj != 0;
    X.sel = 0;
    fixed_stages<T, N, TPL, false, 1, kFeatPlain, 1, 0, true, Rs...>(X);
}

// Shared memory of a family block: the largest W * kpitch<T, N> over the family's lengths.
template <class T>
__host__ __device__ constexpr int family_smem_elems() {
    constexpr int per = sizeof(T) == 4 ? 16 : 8;
    constexpr int top = sizeof(T) == 4 ? 4096 : 2048;
    int best = 0;
    for (int n = 64; n <= top; n *= 2) {
        const int w = kFamilyThreads / (n / per);
        int p = n + (n >> (sizeof(T) == 4 ? 4 : 3));
        p = (p & 1) ? p : p + 1;
        best = w * p > best ? w * p : best;
    }
    return best;
}

// grid = total tiles of the launch; block = 256; dynamic smem = family_smem_elems<T>() * sizeof(C).
template <class T>
__global__ void __launch_bounds__(kFamilyThreads, 4) fft_family_kernel(const __grid_constant__ FamilyParams P) {
    using C = cplx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* sm = reinterpret_cast<C*>(smem_raw);
    const int64_t tile = blockIdx.x;
    int lo = 0, hi = P.count - 1;  // last item with tile_begin <= tile
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (P.items[mid].tile_begin <= tile) lo = mid;
        else hi = mid - 1;
    }
    const FamilyItem& it = P.items[lo];
    if constexpr (sizeof(T) == 4) {
        switch (it.log2n) {
            case 6: family_tile<T, 64, 16, 4>(it, tile, sm); break;
            case 7: family_tile<T, 128, 16, 8>(it, tile, sm); break;
            case 8: family_tile<T, 256, 16, 16>(it, tile, sm); break;
            case 9: family_tile<T, 512, 16, 16, 2>(it, tile, sm); break;
            case 10: family_tile<T, 1024, 16, 16, 4>(it, tile, sm); break;
            case 11: family_tile<T, 2048, 16, 16, 8>(it, tile, sm); break;
            case 12: family_tile<T, 4096, 16, 16, 16>(it, tile, sm); break;
            default: break;
        }
    } else {
        switch (it.log2n) {
            case 6: family_tile<T, 64, 8, 8>(it, tile, sm); break;
            case 7: family_tile<T, 128, 8, 8, 2>(it, tile, sm); break;
            case 8: family_tile<T, 256, 8, 8, 4>(it, tile, sm); break;
            case 9: family_tile<T, 512, 8, 8, 8>(it, tile, sm); break;
            case 10: family_tile<T, 1024, 8, 8, 8, 2>(it, tile, sm); break;
            case 11: family_tile<T, 2048, 8, 8, 8, 4>(it, tile, sm); break;
            default: break;
        }
    }
}

// Radix sequences of the family's lengths (the single-pass catalog entries'), for the host
// tables: log2n -> stages.
inline int family_radices(bool dbl, int log2n, int* r) {
    static const int f[7][4] = {{16, 4}, {16, 8}, {16, 16}, {16, 16, 2}, {16, 16, 4}, {16, 16, 8}, {16, 16, 16}};
    static const int fn[7] = {2, 2, 2, 3, 3, 3, 3};
    static const int d[6][4] = {{8, 8}, {8, 8, 2}, {8, 8, 4}, {8, 8, 8}, {8, 8, 8, 2}, {8, 8, 8, 4}};
    static const int dn[6] = {2, 3, 3, 3, 4, 4};
    const int k = log2n - 6;
    if (k < 0 || k >= (dbl ? 6 : 7)) return 0;
    const int n = dbl ? dn[k] : fn[k];
    for (int i = 0; i < n; ++i) r[i] = dbl ? d[k][i] : f[k][i];
    return n;
}

}  // namespace sfb
