// Single-pass FFT of a long line on a thread-block cluster (distributed shared memory).
//
// A line of N = N1 * N2 elements (n = N2*n1 + n2, k = k1 + N1*k2) is split over the P CTAs
// of one cluster; CTA p holds the CW = N2/P columns n2 in [p*CW, (p+1)*CW) in its shared
// memory, so a line that does not fit one SM still makes a single HBM round trip:
//   phase 1  columns: each CTA loads its columns (CW-wide coalesced rows of the line),
//            runs the length-N1 Stockham FFT over n1 per column, multiplies by the
//            four-step twiddle W_N^(n2*k1) and leaves Y[k1][n2] in its shared memory;
//   exchange cluster barrier; CTA p then owns rows k1 in [p*RW, (p+1)*RW), RW = N1/P, and
//            its first row stage reads Y[k1][n2] for all n2 straight from the owning
//            CTAs' shared memory (distributed shared-memory loads, no TMA multicast);
//            a second cluster barrier ends all remote reads before shared memory is reused;
//   phase 2  rows: the length-N2 FFT over n2, stored to X[k1 + N1*k2] with RW consecutive
//            k1 per row of the store (coalesced), conjugation and scale fused.
// Both phases use the column-major shared layout addr = k * W + w (W = CW or RW lines),
// so a warp touches W consecutive elements and stays bank-conflict free.
// Every CTA runs the same barriers unconditionally: no data-dependent waits.
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "butterfly.cuh"

namespace sfb {

namespace cg = cooperative_groups;

struct ClusterParams {
    int64_t lines = 1;
    int64_t in_pitch = 0, out_pitch = 0;  // line pitch in elements
    const void* tw1 = nullptr;            // stage twiddles of the length-N1 FFT
    const void* tw2 = nullptr;            // stage twiddles of the length-N2 FFT
    const void* tw4_hi = nullptr;         // W_N^m = hi[m >> shift] * lo[m & mask]
    const void* tw4_lo = nullptr;
    int tw4_shift = 0;
    int conj_in = 0, conj_out = 0;
    double scale = 1.0;
};

template <int... Rs>
struct RadixSeq {};

// One Stockham stage over W lines of length N held column-major in shared memory.
// SRC: 0 shared, 1 functor `first(k)` (global or remote); DST: 0 shared, 1 functor `last(k, v)`.
template <class T, int N, int TPL, int W, int NS, int TWOFF, int R, int SRC, int DST, class First, class Last>
__device__ __forceinline__ void cl_stage(cplx<T>* smc, int t, bool active, const cplx<T>* twb, First& first,
                                         Last& last) {
    using C = cplx<T>;
    constexpr int NR = N / R;
    constexpr int NB = (NR + TPL - 1) / TPL;
    constexpr bool EXACT = (NR % TPL) == 0;
    C v[NB * R];
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        const int j = t + i * TPL;
        if (active && (EXACT || j < NR)) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if constexpr (SRC == 1) v[i * R + r] = first(j + r * NR);
                else v[i * R + r] = smc[(j + r * NR) * W];
            }
        }
    }
    if constexpr (SRC == 0) __syncthreads();
    else first.after_load();
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        const int j = t + i * TPL;
        if (active && (EXACT || j < NR)) {
            C* u = &v[i * R];
            const int jm = j % NS;
            if constexpr (NS > 1 && R > 1) {
                const C* twp = twb + TWOFF + jm * (R - 1);
#pragma unroll
                for (int r = 1; r < R; ++r) u[r] = cmul(u[r], __ldg(twp + (r - 1)));
            }
            dft<R, T>(u);
            const int base = (j - jm) * R + jm;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if constexpr (DST == 1) last(base + r * NS, u[r]);
                else smc[(base + r * NS) * W] = u[r];
            }
        }
    }
    if constexpr (DST == 0) __syncthreads();
    else last.after_store();
}

template <class T, int N, int TPL, int W, int NS, int TWOFF, bool FIRST, class First, class Last, int R,
          int... Rest>
__device__ __forceinline__ void cl_stages(cplx<T>* smc, int t, bool active, const cplx<T>* twb, First& first,
                                          Last& last) {
    constexpr bool LAST = sizeof...(Rest) == 0;
    cl_stage<T, N, TPL, W, NS, TWOFF, R, FIRST ? 1 : 0, LAST ? 1 : 0>(smc, t, active, twb, first, last);
    if constexpr (!LAST)
        cl_stages<T, N, TPL, W, NS * R, TWOFF + NS * (R - 1), false, First, Last, Rest...>(smc, t, active, twb,
                                                                                           first, last);
}

template <class T, int N, int TPL, int W, class First, class Last, int... Rs>
__device__ __forceinline__ void cl_fft(RadixSeq<Rs...>, cplx<T>* smc, int t, bool active, const cplx<T>* twb,
                                       First& first, Last& last) {
    cl_stages<T, N, TPL, W, 1, 0, true, First, Last, Rs...>(smc, t, active, twb, first, last);
}

template <class T, int N1, int N2, int P, int TPL1, int TPL2, class Rad1, class Rad2, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB)
    fft_cluster_kernel(const __grid_constant__ ClusterParams prm, const cplx<T>* in, cplx<T>* out) {
    using C = cplx<T>;
    constexpr int CW = N2 / P;  // columns per CTA (phase 1)
    constexpr int RW = N1 / P;  // rows per CTA (phase 2)
    constexpr int N = N1 * N2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* sm = reinterpret_cast<C*>(smem_raw);
    cg::cluster_group cluster = cg::this_cluster();
    const int p = static_cast<int>(cluster.block_rank());
    const int64_t line = blockIdx.x / P;
    const int tid = threadIdx.x;
    const T scale = static_cast<T>(prm.scale);
    const bool conj_in = prm.conj_in != 0, conj_out = prm.conj_out != 0;

    // ---- phase 1: columns n2 = p*CW + w, FFT over n1 ----
    {
        const int w = tid % CW;
        const int t = tid / CW;
        const bool active = t < TPL1;
        const C* gcol = in + line * prm.in_pitch + p * CW + w;
        const C* hi = static_cast<const C*>(prm.tw4_hi);
        const C* lo = static_cast<const C*>(prm.tw4_lo);
        const int n2 = p * CW + w;
        const int mask = (1 << prm.tw4_shift) - 1;
        C* smc = sm + w;
        struct {
            const C* g;
            bool cj;
            __device__ C operator()(int k) const {
                C a = g[(int64_t)k * N2];
                if (cj) a.y = -a.y;
                return a;
            }
            __device__ void after_load() const {}
        } first{gcol, conj_in};
        struct {
            C* s;
            const C *hi, *lo;
            int n2, shift, mask;
            __device__ void operator()(int k1, C v) const {
                const int m = k1 * n2;  // < N
                v = cmul(v, cmul(__ldg(hi + (m >> shift)), __ldg(lo + (m & mask))));
                s[k1 * CW] = v;
            }
            __device__ void after_store() const {}
        } last{smc, hi, lo, n2, prm.tw4_shift, mask};
        cl_fft<T, N1, TPL1, CW>(Rad1{}, smc, t, active, static_cast<const C*>(prm.tw1), first, last);
    }
    // Y[k1][n2] of this CTA's columns is in shared memory at k1 * CW + (n2 - p*CW).
    cluster.sync();

    // ---- phase 2: rows k1 = p*RW + w, FFT over n2 ----
    {
        const int w = tid % RW;
        const int t = tid / RW;
        const bool active = t < TPL2;
        const int k1 = p * RW + w;
        C* smc = sm + w;
        struct {
            C* base;
            int k1;
            cg::cluster_group* cl;
            __device__ C operator()(int n2) const {
                const int q = n2 / CW;
                const C* remote = cl->map_shared_rank(base, q);
                return remote[k1 * CW + (n2 - q * CW)];
            }
            // every remote read of this CTA is done before anyone overwrites shared memory
            __device__ void after_load() const { cl->sync(); }
        } first{sm, k1, &cluster};
        C* grow = out + line * prm.out_pitch + k1;
        struct {
            C* g;
            bool cj;
            T sc;
            __device__ void operator()(int k2, C v) const {
                if (cj) v.y = -v.y;
                v.x *= sc;
                v.y *= sc;
                g[(int64_t)k2 * N1] = v;
            }
            __device__ void after_store() const {}
        } last{grow, conj_out, scale};
        cl_fft<T, N2, TPL2, RW>(Rad2{}, smc, t, active, static_cast<const C*>(prm.tw2), first, last);
    }
    (void)N;
}

}  // namespace sfb
