// Grouped launch: many requests of one length family (same N and precision, contiguous
// lines, any batch count, direction and normalization) in a single kernel launch.
//
// The launch's tiles are the concatenation of every request's tiles (w lines each); a CTA
// finds its request by binary search over the requests' first-tile indices and then runs
// the size-specialised Stockham stages of fixed_kernel.cuh on that request's lines. The
// request table travels in the kernel parameters, so a launch needs no device staging
// memory and can be captured into a CUDA graph and replayed.
#pragma once

#include <cuda_runtime.h>

#include "fixed_kernel.cuh"

namespace sfb {

constexpr int kGroupMaxItems = 192;

struct GroupItem {
    const void* in;
    void* out;
    int64_t lines;
    int64_t tile_begin;  // first tile of this request in the launch
    double scale;
    int conj;            // 1: inverse transform (conjugate on load and store)
    int pad_;
};

struct GroupParams {
    const void* tw;      // base twiddles of the family's radix sequence
    int w;               // lines per tile
    int count;           // requests
    int64_t pitch;       // line pitch (= N)
    GroupItem items[kGroupMaxItems];
};

template <class T, int N, int TPL, int MAXT, int... Rs>
__global__ void __launch_bounds__(MAXT, fixed_min_blocks<T, MAXT, 64>())
    fft_grouped_kernel(const __grid_constant__ GroupParams P) {
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
    const GroupItem& it = P.items[lo];
    const int tid = threadIdx.x;
    const int w = tid / TPL;
    FixedCtx<T> X;
    X.t = tid - w * TPL;
    X.active = w < P.w;
    const int64_t c = (tile - it.tile_begin) * P.w + w;
    X.line_ok = X.active && c < it.lines;
    X.sm = sm + w * kpitch<T, N>();
    X.gin = static_cast<const C*>(it.in) + c * P.pitch;
    X.gout = static_cast<C*>(it.out) + c * P.pitch;
    X.twb = static_cast<const C*>(P.tw);
    X.in_ks = 1;
    X.out_ks = 1;
    X.scale = static_cast<T>(it.scale);
    X.conj_in = it.conj != 0;
    X.conj_out = it.conj != 0;
    X.sel = 0;
    fixed_stages<T, N, TPL, false, 1, kFeatPlain, 1, 0, true, Rs...>(X);
}

}  // namespace sfb
