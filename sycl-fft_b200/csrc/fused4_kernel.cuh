// Four-step FFT of long contiguous lines in one launch, with the intermediate kept in L2.
//
// A line of L = N1 * N2 points is an N1 x N2 matrix. The two-pass four-step reads and writes
// every element twice in HBM: columns (input -> scratch, twiddle W_L^(k1*c) fused) and rows
// (scratch -> output, transposed store). Here one persistent launch runs both passes as a
// stream of tiles and keeps the scratch of only a few lines -- a ring of `ring` line slots,
// tens of MB, inside the 126 MB L2 -- so HBM sees the input read once and the output written
// once, as for a single-pass transform.
//
// Work is a sequence of tickets claimed in order with one atomic per tile. Ticket order
// interleaves the column tiles of line l + D with the row tiles of line l (lag D lines), so a
// row tile is claimed long after the column tiles it needs. Dependencies are counters per
// ring slot, monotonic over the launch:
//   - row tiles of line l wait until the slot's column-tile counter reaches TC * (l / ring + 1)
//     (every column tile of line l has stored its part of the slot);
//   - column tiles of line l wait until the slot's row-tile counter reaches TR * (l / ring)
//     (the rows of line l - ring have read the slot before it is overwritten).
// Every wait targets tiles with smaller tickets, which blocks that are already running hold,
// so the launch cannot deadlock whatever the residency (ring > D). Waits are bounded: a wait
// that gives up (P.wait_polls polls) records status 4 in the plan's status word and raises an
// abort flag that makes every block stop at its next ticket; no asynchronous copy is ever in
// flight. The ring is read with ld.global.cg (L1 is not coherent between SMs).
//
// The tile code is the size-specialised stage code of fixed_kernel.cuh: column tiles are the
// kModeC four-step column pass (W1 columns, twiddle on the store), row tiles the kModeK row pass
// (W2 rows, transposed store through shared memory), as the two-pass kernels run them.
#pragma once

#include <cuda_runtime.h>

#include "async_util.cuh"
#include "fixed_kernel.cuh"
#include "fused4_schedule.h"

namespace sfb {

struct Fused4Params {
    int64_t lines = 0;  // transforms of length L = N1 * N2
    const void* tw1 = nullptr;  // base twiddles of the N1-point column FFT
    const void* tw2 = nullptr;  // base twiddles of the N2-point row FFT
    const void* tw4_hi = nullptr;  // W_L^m = hi[m >> shift] * lo[m & mask]
    const void* tw4_lo = nullptr;
    int tw4_shift = 0;
    int conj_in = 0, conj_out = 0;
    double scale = 1.0;
    int ring = 1;  // line slots of the ring (> lag)
    int lag = 0;   // D: column tiles of line l + D are claimed with the row tiles of line l
    long long wait_polls = 1ll << 26;
    int* status = nullptr;  // set to 4 when a dependency wait gave up
};

// Control words of one launch (zeroed before it): [0] ticket (32-bit: launches of fewer than
// 2^32 tiles), [1] abort, [2, 2 + ring) column
// tiles done per slot, [2 + ring, 2 + 2 * ring) row tiles done per slot.
constexpr int kFused4MaxRing = 64;
constexpr int kFused4CtrlWords = 2 + 2 * kFused4MaxRing;

template <int... Rs>
struct Radices {};

// Bounded wait until *word >= target. polls == 0 gives up without looking.
__device__ __forceinline__ bool wait_count(const unsigned* word, unsigned target, long long polls) {
    for (long long spin = 0; spin < polls; ++spin) {
        unsigned v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(word) : "memory");
        if (v >= target) return true;
        __nanosleep(32);
    }
    return false;
}

template <class T, int N1, int TPL1, int W1, int... RC>
__device__ __forceinline__ void fused4_cols(FixedCtx<T>& X, Radices<RC...>) {
    fixed_stages<T, N1, TPL1, true, W1, kFeatTw4, 1, 0, true, RC...>(X);
}

template <class T, int N2, int TPL2, int W2, int... RR>
__device__ __forceinline__ void fused4_rows(FixedCtx<T>& X, Radices<RR...>) {
    fixed_stages<T, N2, TPL2, false, W2, kFeatTStore | kFeatLoadCG, 1, 0, true, RR...>(X);
}

// grid = resident blocks (persistent); block = THREADS >= max(W1 * TPL1, W2 * TPL2);
// dynamic smem = max(N1 * W1, W2 * kpitch<T, N2>) * sizeof(C).
template <class T, int N1, int TPL1, int W1, int N2, int TPL2, int W2, int THREADS, int MINB, class RC, class RR>
__global__ void __launch_bounds__(THREADS, MINB)
    fft_fused4_kernel(const __grid_constant__ Fused4Params P, const cplx<T>* in, cplx<T>* out, cplx<T>* ring,
                      unsigned* ctrl) {
    using C = cplx<T>;
    constexpr int64_t L = int64_t(N1) * N2;
    constexpr int TC = N2 / W1;  // column tiles per line
    constexpr int TR = N1 / W2;  // row tiles per line
    static_assert(N2 % W1 == 0 && N1 % W2 == 0, "tiles must cover a line exactly");
    static_assert(W1 * TPL1 <= THREADS && W2 * TPL2 <= THREADS, "block too small");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* sm = reinterpret_cast<C*>(smem_raw);
    __shared__ long long s_ticket;
    unsigned* const col_done = ctrl + 2;
    unsigned* const row_done = ctrl + 2 + P.ring;
    const int tid = threadIdx.x;
    const int64_t total = fused4_total(P.lines, P.lag, TC, TR);

    for (;;) {
        __syncthreads();  // the previous ticket and tile are done with shared memory
        if (tid == 0) {
            const long long t = atomicAdd(ctrl, 1u);
            unsigned abort;
            asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(abort) : "l"(ctrl + 1) : "memory");
            s_ticket = abort ? total : t;
        }
        __syncthreads();
        const int64_t t = s_ticket;
        if (t >= total) break;
        const Fused4Tile job = fused4_decode(t, P.lines, P.lag, TC, TR);
        const bool col = job.col;
        const int64_t line = job.line;
        const int tile = job.tile;
        const int slot = static_cast<int>(line % P.ring);
        const unsigned gen = static_cast<unsigned>(line / P.ring);
        C* const buf = ring + slot * L;
        // dependency wait (thread 0), then the whole block agrees
        bool ok = true;
        if (tid == 0) {
            if (col) ok = gen == 0 || wait_count(row_done + slot, unsigned(TR) * gen, P.wait_polls);
            else ok = wait_count(col_done + slot, unsigned(TC) * (gen + 1), P.wait_polls);
            if (!ok) {
                report_status(P.status, 4);
                atomicExch(ctrl + 1, 1u);
            }
        }
        if (__syncthreads_or(!ok)) break;
        FixedCtx<T> X;
        X.scale = T(1);
        X.conj_in = false;
        X.conj_out = false;
        if (col) {
            const int w = tid % W1;
            X.t = tid / W1;
            X.active = X.t < TPL1;
            const int c = tile * W1 + w;
            X.line_ok = X.active;
            X.sel = c;
            X.twb = static_cast<const C*>(P.tw1);
            X.tw4_hi = static_cast<const C*>(P.tw4_hi);
            X.tw4_lo = static_cast<const C*>(P.tw4_lo);
            X.tw4_shift = P.tw4_shift;
            X.sm = sm + w;
            X.gin = in + line * L + c;
            X.gout = buf + c;
            X.in_ks = N2;
            X.out_ks = N2;
            X.conj_in = P.conj_in != 0;
            fused4_cols<T, N1, TPL1, W1>(X, RC{});
            __threadfence();  // this thread's ring stores are visible before the count below
            __syncthreads();
            if (tid == 0) atomicAdd(col_done + slot, 1u);
        } else {
            const int w = tid / TPL2;
            X.t = tid - w * TPL2;
            X.active = w < W2;
            const int row = tile * W2 + w;  // k1
            X.line_ok = X.active;
            X.sel = 0;
            X.twb = static_cast<const C*>(P.tw2);
            X.sm = sm + w * kpitch<T, N2>();
            X.gin = buf + static_cast<int64_t>(row) * N2;
            X.gout = nullptr;
            X.in_ks = 1;
            X.out_ks = 1;
            __threadfence();  // acquire side of the column counts read by thread 0
            fused4_rows<T, N2, TPL2, W2>(X, RR{});  // ends with a barrier: the ring slot is read
            if (tid == 0) {
                __threadfence();  // the block's ring reads are ordered before the count
                atomicAdd(row_done + slot, 1u);
            }
            // transposed store: rows k1 = tile*W2 .. +W2-1 of the output line, element k1 + N1 * k2
            C* dst = out + line * L + int64_t(tile) * W2;
            const T sc = static_cast<T>(P.scale);
            const T sy = P.conj_out ? -sc : sc;
#pragma unroll 4
            for (int idx = tid; idx < W2 * N2; idx += THREADS) {
                const int k = idx / W2;
                const int ww = idx - k * W2;
                const C a = sm[ww * kpitch<T, N2>() + pidx<T>(k)];
                dst[ww + int64_t(k) * N1] = cmake<C>(a.x * sc, a.y * sy);
            }
        }
    }
}

}  // namespace sfb
