// Persistent, copy-engine-pipelined pass kernel for long contiguous lines.
//
// For lines so long that one line fills most of a CTA's shared memory (float N=13440 is
// 105 KB), only one CTA fits per SM and a plain kernel alternates load -> exchanges ->
// store with the HBM idle during the exchanges. Here each CTA is persistent (one per SM)
// and owns two buffers: a copy buffer, filled by the bulk-copy engine (cp.async.bulk,
// completion on an mbarrier) with the next line as it is in HBM, and a padded work buffer
// for the exchanges (the conflict-free layout of fixed_kernel.cuh). The first stage reads
// the copy buffer into registers and writes the work buffer; right after it, the copy
// engine is told to fetch the following line into the copy buffer, so that load hides
// behind the remaining stages, and the last stage's stores drain during the next line.
//
// Waits on the copy are bounded: after P.wait_polls polls the CTA records a timeout in the
// plan's status word, lets the copy it gave up on land (bounded again by kSpinLimit, so no
// copy into its shared memory outlives it) and stops (all threads agree through a barrier
// first).
#pragma once

#include <cuda_runtime.h>

#include "async_util.cuh"
#include "butterfly.cuh"
#include "fixed_kernel.cuh"

namespace sfb {

struct PipedParams {
    int64_t lines = 0;
    int64_t in_pitch = 0, out_pitch = 0;  // elements; pitch * sizeof(C) is a multiple of 16
    const void* tw = nullptr;
    int conj_in = 0, conj_out = 0;
    double scale = 1.0;
    int* status = nullptr;  // set to 1 if a copy wait timed out
    long long wait_polls = kSpinLimit;  // polls before a copy wait gives up
};

constexpr int kCopyChunks = 4;

// Stages 2..: the plain padded-layout stages of fixed_kernel.cuh.
template <class T, int N, int TPL, int R0, int... Rest>
__device__ __forceinline__ void piped_rest(FixedCtx<T>& X) {
    if constexpr (sizeof...(Rest) > 0) fixed_stages<T, N, TPL, false, 1, kFeatPlain, R0, 1, false, Rest...>(X);
}

template <class T, int N, int TPL, int R0, int... Rest>
__device__ __forceinline__ void piped_first(FixedCtx<T>& X) {
    fixed_stage<T, N, TPL, false, 1, kFeatPlain, 1, 0, R0, true, sizeof...(Rest) == 0>(X);
}

// grid = min(lines, SMs); block = TPL threads;
// dynamic smem = N * sizeof(C) (copy buffer) + kpitch<T,N>() * sizeof(C) (work buffer) + 16.
template <class T, int N, int TPL, int MAXT, int... Rs>
__global__ void __launch_bounds__(MAXT, 1)
    fft_piped_kernel(const __grid_constant__ PipedParams P, const cplx<T>* in, cplx<T>* out) {
    using C = cplx<T>;
    static_assert((N * sizeof(C)) % (16 * kCopyChunks) == 0, "line must split into 16-byte multiples");
    constexpr uint32_t kLineBytes = N * sizeof(C);
    constexpr uint32_t kChunk = kLineBytes / kCopyChunks;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* const copy = reinterpret_cast<C*>(smem_raw);
    C* const work = copy + N;
    uint64_t* const bar = reinterpret_cast<uint64_t*>(smem_raw + kLineBytes + kpitch<T, N>() * sizeof(C));
    const int t = threadIdx.x;

    FixedCtx<T> X;
    X.sm = work;
    X.gin = copy;
    X.twb = static_cast<const C*>(P.tw);
    X.t = t;
    X.active = t < TPL;
    X.line_ok = true;
    X.in_ks = 1;
    X.out_ks = 1;
    X.scale = static_cast<T>(P.scale);
    X.conj_in = P.conj_in != 0;
    X.conj_out = P.conj_out != 0;
    X.sel = 0;

    auto fetch = [&](int64_t line) {
        mbar_expect_tx(bar, kLineBytes);
        const unsigned char* src = reinterpret_cast<const unsigned char*>(in + line * P.in_pitch);
#pragma unroll
        for (int c = 0; c < kCopyChunks; ++c)
            bulk_g2s(reinterpret_cast<unsigned char*>(copy) + c * kChunk, src + c * kChunk, kChunk, bar);
    };
    if (t == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        if (blockIdx.x < P.lines) fetch(blockIdx.x);
    }
    __syncthreads();

    uint32_t parity = 0;
    for (int64_t line = blockIdx.x; line < P.lines; line += gridDim.x) {
        const bool ok = mbar_wait_bounded(bar, parity, P.wait_polls);
        if (__syncthreads_or(!ok)) {
            if (t == 0) {
                report_status(P.status, 1);
                // the only copy in flight is the one given up on: let it land before the
                // shared memory is released
                mbar_wait_bounded(bar, parity, kSpinLimit);
            }
            __syncthreads();
            return;
        }
        parity ^= 1u;
        X.gout = out + line * P.out_pitch;
        piped_first<T, N, TPL, Rs...>(X);  // ends with a barrier: the copy buffer is consumed
        const int64_t next = line + gridDim.x;
        if (t == 0 && next < P.lines) {
            fence_proxy_async();  // order the generic reads of the copy buffer before the copy
            fetch(next);
        }
        piped_rest<T, N, TPL, Rs...>(X);
        __syncthreads();  // the work buffer is free for the next line's first stage
    }
}

}  // namespace sfb
