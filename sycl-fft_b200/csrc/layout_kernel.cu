// Strided ("advanced") layouts: gather a batch of transforms from a user layout into the
// contiguous batch-major order the FFT passes read, and scatter the contiguous result back.
//
// Element (b, i0, .., i_{r-1}) of a layout sits at b * dist + sum_k i_k * stride_k (in complex
// elements). The index space is viewed as a matrix: rows = (b, i0, .., i_{r-2}) with the last
// of them fastest, columns = i_{r-1}. The contiguous side is row-major with C = L_{r-1}
// columns. A 32-row tile goes through shared memory, so both sides are coalesced whichever
// of the two matrix directions the strided side is dense in: "column mode" (warp lanes along
// i_{r-1}) when stride_{r-1} is the smaller step, "row mode" (lanes along the fastest row
// index) otherwise, e.g. transforms down the columns of a row-major matrix.
#include <cuda_runtime.h>

#include "butterfly.cuh"
#include "layout_launch.hpp"

namespace sfb {
namespace {

constexpr int kTile = 32;
constexpr int kRowsPerPass = 8;  // block = 32 x 8 threads

struct RowMap {
    int rank;         // rank - 1 row dimensions after the batch index
    int64_t len[2];   // lengths of i0 .. i_{r-2}
    int64_t stride[2];
    int64_t dist;
    __device__ int64_t offset(int64_t row) const {
        int64_t off = 0;
#pragma unroll
        for (int k = 1; k >= 0; --k) {  // compile-time indices: the arrays stay in registers
            if (k <= rank - 2) {
                const int64_t q = row / len[k];
                off += (row - q * len[k]) * stride[k];
                row = q;
            }
        }
        return off + row * dist;
    }
};

RowMap row_map(const Layout& l) {
    RowMap m{};
    m.rank = l.rank;
    for (int k = 0; k + 1 < l.rank; ++k) {
        m.len[k] = l.len[k];
        m.stride[k] = l.stride[k];
    }
    m.dist = l.dist;
    return m;
}

// Step between consecutive rows' fastest index (the stride of i_{r-2}, or the batch distance).
int64_t row_step(const Layout& l) { return l.rank >= 2 ? l.stride[l.rank - 2] : l.dist; }

// Tile of kTile rows x TC columns (TC = 64 for complex<float>, 32 for complex<double>: 16 KB
// per tile either way), 8 loads or stores per thread per phase.
template <class T>
__host__ __device__ constexpr int tile_cols() {
    return sizeof(T) == 4 ? 64 : 32;
}

template <class T, bool kGather, bool kRowMode>
__global__ void __launch_bounds__(kTile* kRowsPerPass)
    layout_kernel(const cplx<T>* __restrict__ src, cplx<T>* __restrict__ dst, RowMap map, int64_t col_stride,
                  int64_t rows, int64_t cols) {
    using C = cplx<T>;
    constexpr int TC = tile_cols<T>();
    __shared__ C tile[kTile][TC + 1];
    const int64_t col_tiles = (cols + TC - 1) / TC;
    const int64_t tiles = col_tiles * ((rows + kTile - 1) / kTile);
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int64_t r0 = (t / col_tiles) * kTile, c0 = (t % col_tiles) * TC;
        // strided side: read (gather) or write (scatter) through the layout
        // contiguous side: row-major rows x cols, lanes along the columns
        if (kGather) {
            if (kRowMode) {
                const int64_t r = r0 + tx;
                if (r < rows) {
                    const int64_t base = map.offset(r);
#pragma unroll
                    for (int j = ty; j < TC; j += kRowsPerPass)
                        if (c0 + j < cols) tile[tx][j] = src[base + (c0 + j) * col_stride];
                }
            } else {
#pragma unroll
                for (int i = ty; i < kTile; i += kRowsPerPass) {
                    const int64_t r = r0 + i;
                    if (r < rows) {
                        const int64_t base = map.offset(r);
#pragma unroll
                        for (int j = tx; j < TC; j += kTile)
                            if (c0 + j < cols) tile[i][j] = src[base + (c0 + j) * col_stride];
                    }
                }
            }
            __syncthreads();
#pragma unroll
            for (int i = ty; i < kTile; i += kRowsPerPass) {
                const int64_t r = r0 + i;
                if (r < rows) {
#pragma unroll
                    for (int j = tx; j < TC; j += kTile)
                        if (c0 + j < cols) dst[r * cols + c0 + j] = tile[i][j];
                }
            }
        } else {
#pragma unroll
            for (int i = ty; i < kTile; i += kRowsPerPass) {
                const int64_t r = r0 + i;
                if (r < rows) {
#pragma unroll
                    for (int j = tx; j < TC; j += kTile)
                        if (c0 + j < cols) tile[i][j] = src[r * cols + c0 + j];
                }
            }
            __syncthreads();
            if (kRowMode) {
                const int64_t r = r0 + tx;
                if (r < rows) {
                    const int64_t base = map.offset(r);
#pragma unroll
                    for (int j = ty; j < TC; j += kRowsPerPass)
                        if (c0 + j < cols) dst[base + (c0 + j) * col_stride] = tile[tx][j];
                }
            } else {
#pragma unroll
                for (int i = ty; i < kTile; i += kRowsPerPass) {
                    const int64_t r = r0 + i;
                    if (r < rows) {
                        const int64_t base = map.offset(r);
#pragma unroll
                        for (int j = tx; j < TC; j += kTile)
                            if (c0 + j < cols) dst[base + (c0 + j) * col_stride] = tile[i][j];
                    }
                }
            }
        }
        __syncthreads();
    }
}

template <class T, bool kGather>
cudaError_t launch_one(const void* src, void* dst, const Layout& l, cudaStream_t stream) {
    int64_t rows = l.batch;
    for (int k = 0; k + 1 < l.rank; ++k) rows *= l.len[k];
    const int64_t cols = l.len[l.rank - 1];
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    constexpr int TC = tile_cols<T>();
    const int64_t tiles = ((rows + kTile - 1) / kTile) * ((cols + TC - 1) / TC);
    const int grid = static_cast<int>(tiles < 148 * 8 ? tiles : 148 * 8);
    const dim3 block(kTile, kRowsPerPass);
    const RowMap map = row_map(l);
    const int64_t cstride = l.stride[l.rank - 1];
    // row mode when consecutive rows are closer in memory than consecutive columns
    const int64_t rstep = row_step(l);
    const bool row_mode = rows > 1 && rstep < cstride;
    using C = cplx<T>;
    if (row_mode)
        layout_kernel<T, kGather, true><<<grid, block, 0, stream>>>(static_cast<const C*>(src), static_cast<C*>(dst),
                                                                     map, cstride, rows, cols);
    else
        layout_kernel<T, kGather, false><<<grid, block, 0, stream>>>(static_cast<const C*>(src), static_cast<C*>(dst),
                                                                      map, cstride, rows, cols);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_layout_gather(bool dbl, const void* src, const Layout& layout, void* dst, cudaStream_t stream) {
    return dbl ? launch_one<double, true>(src, dst, layout, stream) : launch_one<float, true>(src, dst, layout, stream);
}

cudaError_t launch_layout_scatter(bool dbl, const void* src, void* dst, const Layout& layout, cudaStream_t stream) {
    return dbl ? launch_one<double, false>(src, dst, layout, stream)
               : launch_one<float, false>(src, dst, layout, stream);
}

}  // namespace sfb
