// TMA-staged column pass of a four-step FFT (contiguous lines of N = n1 * n2 points viewed
// as n1 x n2 matrices; the pass transforms the n2 columns of length n1 and multiplies output
// k1 of column c by W_N^(k1 * c)).
//
// Persistent CTAs. A tile is W adjacent columns of one line: an n1 x W box of the input,
// fetched by the tensor-memory-access engine (cp.async.bulk.tensor, 3-D map: reals of a row,
// rows, lines) into one of two shared buffers while the stages of the previous tile run on
// the other; completion on an mbarrier per buffer. The box lands row-major, which is the
// column-mode layout of the size-specialised stages (element (a, w) at a * W + w), so the
// first stage reads it in place and the last stage stores to HBM with the twiddle fused.
//
// Waits are bounded: after P.wait_polls polls the CTA records a timeout in the status word,
// waits (bounded again, kSpinLimit polls) for its copies in flight and returns.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "async_util.cuh"
#include "fixed_kernel.cuh"

namespace sfb {

struct TmaColParams {
    int64_t tiles = 0;       // lines * col_tiles
    int col_tiles = 1;       // ceil(n2 / W)
    int n2 = 0;              // columns per line
    int64_t out_hi = 0;      // output line pitch (elements)
    int64_t out_ks = 1;      // output stride along a column (= n2)
    const void* tw = nullptr;  // base twiddles of the n1 radices
    const void* tw4_hi = nullptr;
    const void* tw4_lo = nullptr;
    int tw4_shift = 0;
    int conj_in = 0, conj_out = 0;
    double scale = 1.0;
    int* status = nullptr;  // set to 3 if a tile wait timed out
    long long wait_polls = kSpinLimit;  // polls before a tile wait gives up
};

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
            "r"(smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

template <class T, int N1, int TPL, int W, int NBUF, int... Rs>
__global__ void __launch_bounds__(W * TPL)
    fft_tma_cols_kernel(const __grid_constant__ CUtensorMap map, const __grid_constant__ TmaColParams P,
                        cplx<T>* out) {
    using C = cplx<T>;
    constexpr int TILE = N1 * W;  // complex elements per tile
    constexpr uint32_t TILE_BYTES = TILE * sizeof(C);
    extern __shared__ __align__(128) unsigned char smem[];
    C* buf0 = reinterpret_cast<C*>(smem);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + NBUF * TILE_BYTES);
    const int tid = threadIdx.x;
    const int w = tid % W;

    auto issue = [&](int64_t tile, int b) {
        const int64_t line = tile / P.col_tiles;
        const int ct = static_cast<int>(tile - line * P.col_tiles);
        mbar_expect_tx(&bar[b], TILE_BYTES);
        tma_load_3d(buf0 + b * TILE, &map, ct * W * 2, 0, static_cast<int>(line), &bar[b]);
    };
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        if (NBUF > 1) mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        if (blockIdx.x < P.tiles) issue(blockIdx.x, 0);
    }
    __syncthreads();

    FixedCtx<T> X;
    X.t = tid / W;
    X.active = X.t < TPL;
    X.line_ok = X.active;
    X.twb = static_cast<const C*>(P.tw);
    X.tw4_hi = static_cast<const C*>(P.tw4_hi);
    X.tw4_lo = static_cast<const C*>(P.tw4_lo);
    X.tw4_shift = P.tw4_shift;
    X.scale = static_cast<T>(P.scale);
    X.conj_in = P.conj_in != 0;
    X.conj_out = P.conj_out != 0;
    X.in_ks = 1;
    X.out_ks = P.out_ks;
    uint32_t phase[2] = {0u, 0u};
    int it = 0;
    for (int64_t tile = blockIdx.x; tile < P.tiles; tile += gridDim.x, ++it) {
        const int b = NBUF > 1 ? (it & 1) : 0;
        const int64_t next = tile + gridDim.x;
        if (NBUF > 1 && tid == 0 && next < P.tiles) issue(next, b ^ 1);  // the other buffer was released below
        const bool ok = mbar_wait_bounded(&bar[b], phase[b], P.wait_polls);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                report_status(P.status, 3);
                // the tile given up on and the prefetch of the other buffer may still be in
                // flight: let them land (bounded) before the shared memory is released
                mbar_wait_bounded(&bar[b], phase[b], kSpinLimit);
                if (NBUF > 1 && next < P.tiles) mbar_wait_bounded(&bar[b ^ 1], phase[b ^ 1], kSpinLimit);
            }
            __syncthreads();
            return;
        }
        phase[b] ^= 1u;
        const int64_t line = tile / P.col_tiles;
        const int c = static_cast<int>(tile - line * P.col_tiles) * W + w;
        X.sm = buf0 + b * TILE + w;
        X.sel = c;
        X.line_ok = X.active && c < P.n2;
        X.gout = out + line * P.out_hi + c;
        fixed_stages<T, N1, TPL, true, W, kFeatTw4 | kFeatSmemIn, 1, 0, true, Rs...>(X);
        // this buffer's generic reads and writes are done before the copy engine refills it
        fence_proxy_async();
        __syncthreads();
        if (NBUF == 1 && tid == 0 && next < P.tiles) issue(next, 0);
    }
}

}  // namespace sfb
