// Single-pass complex<double> FFT of 65536-point lines on 16-CTA thread-block clusters, with
// the next line's load overlapping the current line's work.
//
// A line is the 256 x 256 matrix x[n1][n2] (n = 256*n1 + n2, k = k1 + 256*k2). CTA p of a
// cluster owns the 16 columns n2 in [16p, 16p+16) for the column FFTs and the 16 rows k1 in
// [16p, 16p+16) for the row FFTs. Each CTA is persistent (its cluster walks lines
// cluster, cluster + clusters, ...) and holds three buffers in shared memory:
//   buf[0], buf[1]  the line's 16-column slab, bulk-copied as 256 rows of 256 bytes (next
//                   line's slab into the other buffer while this line runs), transformed in
//                   place by the column stages and then reused for the row stages;
//   Y               the twiddled column spectra Y[k1][n2 - 16p], read by the whole cluster.
// Per line:
//   1. column FFTs (length 256 over n1) of the slab; the last stage multiplies by
//      W_65536^(k1*n2) and writes Y;
//   2. cluster barrier: every CTA's Y is complete;
//   3. row stage 1: row k1 = 16p + w reads its 256 values straight from the owners' Y
//      (lanes along n2: 16 consecutive elements = 256 bytes of one remote CTA);
//   4. cluster barrier: all remote reads are done, Y may be overwritten by the next line;
//   5. the remaining row stages, then a transposed store X[k1 + 256*k2] in 256-byte
//      segments (16 consecutive k1), conjugation and scale fused.
// The size-specialised stage code of fixed_kernel.cuh runs both FFTs (radices 8, 8, 4 with
// base twiddles). Every CTA takes the same barriers in the same order; mbarrier waits are
// bounded (kSpinLimit polls) and a timeout is recorded in the plan's status word without
// leaving the loop, so the cluster barriers stay matched.
#include <atomic>

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "async_util.cuh"
#include "butterfly.cuh"
#include "cluster_pipe.hpp"
#include "fixed_kernel.cuh"

namespace sfb {
namespace {

namespace cg = cooperative_groups;

constexpr int kN1 = 256, kN2 = 256, kP = 16, kW = 16, kTPL = 32, kThreads = kW * kTPL;
using T = double;
using C = cplx<double>;
constexpr int kPitch = kpitch<T, kN2>();  // padded row pitch of the row stages
constexpr uint32_t kSlabElems = kN1 * kW;
constexpr uint32_t kBufElems = (kW * kPitch > (int)kSlabElems) ? kW * kPitch : kSlabElems;
constexpr uint32_t kBufBytes = (kBufElems * sizeof(C) + 15u) / 16u * 16u;
constexpr uint32_t kYBytes = kSlabElems * sizeof(C);
constexpr uint32_t kRowBytes = kW * sizeof(C);  // one n1 row of the slab: 256 bytes
constexpr size_t kSmemBytes = 2 * kBufBytes + kYBytes + 16;
static_assert(kSmemBytes <= 227 * 1024, "cluster pipeline exceeds shared memory");

__device__ __forceinline__ C* buffer(unsigned char* smem, int b) {
    return reinterpret_cast<C*>(smem + b * kBufBytes);
}

__global__ void __launch_bounds__(kThreads, 1)
    fft_cluster_pipe_kernel(const __grid_constant__ ClusterPipeParams P, const C* in, C* out) {
    extern __shared__ __align__(16) unsigned char smem[];
    C* const Y = reinterpret_cast<C*>(smem + 2 * kBufBytes);
    uint64_t* const bars = reinterpret_cast<uint64_t*>(smem + 2 * kBufBytes + kYBytes);
    cg::cluster_group cluster = cg::this_cluster();
    const int p = static_cast<int>(cluster.block_rank());
    const int64_t first = blockIdx.x / kP;
    const int64_t clusters = gridDim.x / kP;
    const int tid = threadIdx.x;
    const C* twb = static_cast<const C*>(P.tw_base);

    // slab of line `line` -> buf[b]: thread n1 < 256 copies row n1 (16 columns, 256 bytes)
    auto load = [&](int b, int64_t line) {
        if (tid == 0) mbar_expect_tx(bars + b, kSlabElems * sizeof(C));
        __syncthreads();
        if (tid < kN1) {
            fence_proxy_async();  // earlier generic accesses of this buffer before the copy
            bulk_g2s(buffer(smem, b) + tid * kW, in + line * P.in_pitch + tid * kN2 + p * kW, kRowBytes, bars + b);
        }
    };

    if (tid == 0) {
        mbar_init(bars, 1);
        mbar_init(bars + 1, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (first < P.lines) load(0, first);

    int it = 0;
    for (int64_t line = first; line < P.lines; line += clusters, ++it) {
        const int b = it & 1;
        const uint32_t parity = static_cast<uint32_t>(it >> 1) & 1u;
        __syncthreads();  // buf[1-b] (the previous line's row scratch) is no longer read
        if (line + clusters < P.lines) load(b ^ 1, line + clusters);
        const bool ok = mbar_wait_bounded(bars + b, parity, kSpinLimit);
        if (__syncthreads_or(!ok) && tid == 0) report_status(P.status, 1);
        C* const slab = buffer(smem, b);

        // 1. column FFTs over n1 (column w = tid % 16, n2 = 16p + w), twiddled into Y
        {
            FixedCtx<T> X;
            const int w = tid % kW;
            X.t = tid / kW;
            X.active = true;
            X.line_ok = true;
            X.sm = slab + w;
            X.gin = nullptr;
            X.gout = Y + w;
            X.twb = twb;
            X.in_ks = kW;
            X.out_ks = kW;
            X.scale = T(1);
            X.conj_in = P.conj_in != 0;
            X.conj_out = false;
            X.sel = p * kW + w;
            X.tw4_hi = static_cast<const C*>(P.tw4_hi);
            X.tw4_lo = static_cast<const C*>(P.tw4_lo);
            X.tw4_shift = P.tw4_shift;
            fixed_stages<T, kN1, kTPL, true, kW, kFeatSmemIn | kFeatTw4, 1, 0, true, 8, 8, 4>(X);
        }
        // 2. every CTA's Y is complete
        cluster.sync();

        // 3. row stage 1 (radix 8, 32 threads per row): row k1 = 16p + w reads n2 = t + 32r
        //    from the owner of column n2 (CTA n2 / 16), then writes the padded row layout
        const int w = tid / kTPL;
        const int t = tid % kTPL;
        C* const row = slab + w * kPitch;
        {
            C u[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const int n2 = t + 32 * r;
                const C* owner = cluster.map_shared_rank(Y, n2 >> 4);
                u[r] = owner[(p * kW + w) * kW + (n2 & 15)];
            }
            dft<8, T>(u);
#pragma unroll
            for (int r = 0; r < 8; ++r) row[pidx<T>(8 * t + r)] = u[r];
        }
        // 4. all remote reads of Y are done (and the rows' first stage is in shared memory)
        cluster.sync();

        // 5. row stages 2-3 (radices 8, 4; natural order back into the row), transposed store
        {
            FixedCtx<T> X;
            X.t = t;
            X.active = true;
            X.line_ok = true;
            X.sm = row;
            X.twb = twb;
            X.in_ks = 1;
            X.out_ks = 1;
            X.scale = T(1);
            X.conj_in = false;
            X.conj_out = false;
            X.sel = 0;
            fixed_stages<T, kN2, kTPL, false, 1, kFeatTStore, 8, 1, false, 8, 4>(X);
        }
        const T sc = static_cast<T>(P.scale);
        const T sy = P.conj_out ? -sc : sc;
        C* dst = out + line * P.out_pitch + p * kW;
#pragma unroll 4
        for (int idx = tid; idx < kW * kN2; idx += kThreads) {
            const int k2 = idx / kW;
            const int ww = idx - k2 * kW;
            const C a = slab[ww * kPitch + pidx<T>(k2)];
            dst[ww + (int64_t)k2 * kN1] = cmake<C>(a.x * sc, a.y * sy);
        }
    }
    // no CTA leaves while another may still read its shared memory
    cluster.sync();
}

constexpr int kMaxDevices = 64;

// Sets the kernel's attributes once per device and returns how many of its clusters fit the
// device at once (cached per device; 0 until known).
cudaError_t configure(int* resident) {
    static std::atomic<int> clusters[kMaxDevices];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    int known = clusters[dev].load();
    if (known <= 0) {
        e = cudaFuncSetAttribute(fft_cluster_pipe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kSmemBytes));
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(fft_cluster_pipe_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(kP, 1, 1);
        cfg.blockDim = dim3(kThreads, 1, 1);
        cfg.dynamicSmemBytes = kSmemBytes;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = kP;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        e = cudaOccupancyMaxActiveClusters(&known, fft_cluster_pipe_kernel, &cfg);
        if (e != cudaSuccess) return e;
        clusters[dev].store(known);
    }
    *resident = known;
    return cudaSuccess;
}

}  // namespace

cudaError_t launch_cluster_pipe(const ClusterPipeParams& prm, const void* in, void* out, cudaStream_t stream,
                                int* max_clusters) {
    int clusters = 0;
    cudaError_t e = configure(&clusters);
    if (e != cudaSuccess) return e;
    if (max_clusters) {
        *max_clusters = clusters;
        return cudaSuccess;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(kThreads, 1, 1);
    cfg.dynamicSmemBytes = kSmemBytes;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kP;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (clusters <= 0) return cudaErrorInvalidConfiguration;
    if (prm.lines <= 0) return cudaSuccess;
    const int64_t use = prm.lines < clusters ? prm.lines : clusters;
    cfg.gridDim = dim3(static_cast<unsigned>(use * kP), 1, 1);
    e = cudaLaunchKernelEx(&cfg, fft_cluster_pipe_kernel, prm, static_cast<const C*>(in), static_cast<C*>(out));
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace sfb
