// Four-step FFT of long contiguous lines in one launch, with the intermediate kept in L2.
//
// A line of L = N1 * N2 points is an N1 x N2 matrix. The two-pass four-step reads and writes
// every element twice in HBM: columns (input -> scratch, twiddle W_L^(k1*c) fused) and rows
// (scratch -> output, transposed store). Here one launch runs both passes as a stream of
// tiles and keeps the scratch of only a few lines -- a ring of `ring` line slots, tens of MB,
// inside the 126 MB L2 -- so HBM sees the input read once and the output written once, as for
// a single-pass transform.
//
// Every block runs one tile. Its ticket comes from one atomic at the block's start, so tickets
// go out in the order blocks start, whatever their index. Ticket order interleaves the column
// tiles of line l + D with the row tiles of line l (lag D lines), so a row tile is claimed
// long after the column tiles it needs. Dependencies are counters per ring slot, monotonic
// over the launch:
//   - row tiles of line l wait until the slot's column-tile counter reaches TC * (l / ring + 1)
//     (every column tile of line l has stored its part of the slot);
//   - column tiles of line l wait until the slot's row-tile counter reaches TR * (l / ring)
//     (the rows of line l - ring have read the slot before it is overwritten).
// Every wait targets tiles with smaller tickets, held by blocks that started earlier and are
// resident or done, so the launch cannot deadlock whatever the residency (ring > D). Waits
// are bounded: a wait that gives up (P.wait_polls polls) records status 4 in the plan's status
// word and raises an abort flag that makes every later block return at once; no asynchronous
// copy is ever in flight. The ring is read with ld.global.cg (L1 is not coherent between SMs).
// (One tile per block rather than a persistent loop: in a loop the compiler keeps the tile
// code's loop-invariant state live across tiles and spills.)
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
// 2^32 tiles), [1] abort, then per phase p the tiles done per ring slot at 2 + p * ring + slot.
constexpr int kFused4MaxRing = 64;
constexpr int kFused4CtrlWords = 2 + kFusedMaxPhases * kFused4MaxRing;

template <int... Rs>
struct Radices {};

// Bounded wait until *word >= target (acquire). polls == 0 gives up without looking.
__device__ __forceinline__ bool wait_count(const unsigned* word, unsigned target, long long polls) {
    for (long long spin = 0; spin < polls; ++spin) {
        unsigned v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(word) : "memory");
        if (v >= target) return true;
        __nanosleep(32);
    }
    return false;
}

// Claims the block's tile (tickets go out in the order blocks start) into *job and waits
// (thread 0, bounded) until the tile's dependency is met: phase p > 0 of a line needs every tile of phase p - 1 of that line; phase
// 0 needs the last phase of the line `ring` lines earlier (the slot's previous user) done.
// Returns false (in every thread) when the launch is finished or was aborted.
template <int PHASES>
__device__ __forceinline__ bool fused_claim(const FusedSched& q, int ring, unsigned* ctrl, long long polls,
                                            int* status, FusedTile* job, long long* s_ticket) {
    const int64_t total = fused_total(q);
    if (threadIdx.x == 0) {
        const long long t = atomicAdd(ctrl, 1u);
        unsigned abort;
        asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(abort) : "l"(ctrl + 1) : "memory");
        *s_ticket = abort ? total : t;
    }
    __syncthreads();
    const int64_t t = *s_ticket;
    if (t >= total) return false;
    *job = fused_decode(q, t);
    const int slot = static_cast<int>(job->line % ring);
    const unsigned gen = static_cast<unsigned>(job->line / ring);
    bool ok = true;
    if (threadIdx.x == 0) {
        if (job->phase == 0)
            ok = gen == 0 || wait_count(ctrl + 2 + (PHASES - 1) * ring + slot, unsigned(q.tiles[PHASES - 1]) * gen,
                                        polls);
        else
            ok = wait_count(ctrl + 2 + (job->phase - 1) * ring + slot, unsigned(q.tiles[job->phase - 1]) * (gen + 1),
                            polls);
        if (!ok) {
            report_status(status, 4);
            atomicExch(ctrl + 1, 1u);
        }
    }
    return !__syncthreads_or(!ok);
}

// Release-add at GPU scope: orders every access that happens before it (the block's, through
// the barrier before it) ahead of the counter update that waiting blocks acquire.
__device__ __forceinline__ void red_release_add(unsigned* word, unsigned v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(word), "r"(v) : "memory");
}

// Counts a finished tile of `phase` for its ring slot once every thread's accesses are done:
// the barrier orders them before thread 0's release (one fence per block, not per thread).
__device__ __forceinline__ void fused_done(unsigned* ctrl, int ring, int phase, int slot) {
    __syncthreads();
    if (threadIdx.x == 0) red_release_add(ctrl + 2 + phase * ring + slot, 1u);
}

template <class T, int N1, int TPL1, int W1, int... RC>
__device__ __forceinline__ void fused4_cols(FixedCtx<T>& X, Radices<RC...>) {
    // the input is read once: streaming loads keep the ring in L2
    fixed_stages<T, N1, TPL1, true, W1, kFeatTw4 | kFeatLoadCS, 1, 0, true, RC...>(X);
}

template <class T, int N2, int TPL2, int W2, int... RR>
__device__ __forceinline__ void fused4_rows(FixedCtx<T>& X, Radices<RR...>) {
    fixed_stages<T, N2, TPL2, false, W2, kFeatTStore | kFeatLoadCG, 1, 0, true, RR...>(X);
}

// grid = lines * (TC + TR) blocks, one tile each; block = THREADS >= max(W1 * TPL1, W2 * TPL2);
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
    const int tid = threadIdx.x;
    FusedSched q;
    q.lines = P.lines;
    q.lag = P.lag;
    q.phases = 2;
    q.tiles[0] = TC;
    q.tiles[1] = TR;
    FusedTile job;
    if (!fused_claim<2>(q, P.ring, ctrl, P.wait_polls, P.status, &job, &s_ticket)) return;
    const int64_t line = job.line;
    const int tile = job.tile;
    const int slot = static_cast<int>(line % P.ring);
    C* const buf = ring + slot * L;
    FixedCtx<T> X;
    X.scale = T(1);
    X.conj_in = false;
    X.conj_out = false;
    if (job.phase == 0) {
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
        fused_done(ctrl, P.ring, 0, slot);
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
        fused4_rows<T, N2, TPL2, W2>(X, RR{});  // ends with a barrier: the ring slot is read
        if (tid == 0) red_release_add(ctrl + 2 + P.ring + slot, 1u);  // the block's ring reads come first
        // transposed store: rows k1 = tile*W2 .. +W2-1 of the output line, element k1 + N1 * k2
        C* dst = out + line * L + int64_t(tile) * W2;
        const T sc = static_cast<T>(P.scale);
        const T sy = P.conj_out ? -sc : sc;
#pragma unroll 4
        for (int idx = tid; idx < W2 * N2; idx += THREADS) {
            const int k = idx / W2;
            const int ww = idx - k * W2;
            const C a = sm[ww * kpitch<T, N2>() + pidx<T>(k)];
            __stcs(dst + ww + int64_t(k) * N1, cmake<C>(a.x * sc, a.y * sy));  // written once: streaming
        }
    }
}

// Persistent form of the same four-step: grid = the resident blocks, each looping over tiles.
// Thread 0 claims the block's next ticket as soon as the current tile starts, so the claim's
// round trip to L2 overlaps the tile's work instead of preceding it (one-tile blocks pay a
// claim, a dependency check and a counter update of latency per tile). A block then holds two
// tickets at once; progress still holds: the smallest unfinished ticket is either some block's
// current tile, whose dependencies are all finished, or some block's claimed-ahead ticket, whose
// block's current tile is smaller and so finished.
template <class T, int N1, int TPL1, int W1, int N2, int TPL2, int W2, int THREADS, int MINB, class RC, class RR>
__global__ void __launch_bounds__(THREADS, MINB)
    fft_fused4p_kernel(const __grid_constant__ Fused4Params P, const cplx<T>* in, cplx<T>* out, cplx<T>* ring,
                       unsigned* ctrl) {
    using C = cplx<T>;
    constexpr int64_t L = int64_t(N1) * N2;
    constexpr int TC = N2 / W1;
    constexpr int TR = N1 / W2;
    static_assert(N2 % W1 == 0 && N1 % W2 == 0, "tiles must cover a line exactly");
    static_assert(W1 * TPL1 <= THREADS && W2 * TPL2 <= THREADS, "block too small");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* sm = reinterpret_cast<C*>(smem_raw);
    __shared__ long long s_ticket;
    const int tid = threadIdx.x;
    FusedSched q;
    q.lines = P.lines;
    q.lag = P.lag;
    q.phases = 2;
    q.tiles[0] = TC;
    q.tiles[1] = TR;
    const int64_t total = fused_total(q);
    long long next = 0;
    if (tid == 0) s_ticket = atomicAdd(ctrl, 1u);
    for (;;) {
        __syncthreads();  // s_ticket is set; the previous tile is done with shared memory
        const int64_t t = s_ticket;
        if (t >= total) break;
        if (tid == 0) next = atomicAdd(ctrl, 1u);  // claimed ahead: used after this tile
        const FusedTile job = fused_decode(q, t);
        const int64_t line = job.line;
        const int tile = job.tile;
        const int slot = static_cast<int>(line % P.ring);
        const unsigned gen = static_cast<unsigned>(line / P.ring);
        bool ok = true;
        if (tid == 0) {
            ok = job.phase == 0 ? (gen == 0 || wait_count(ctrl + 2 + P.ring + slot, unsigned(TR) * gen, P.wait_polls))
                                : wait_count(ctrl + 2 + slot, unsigned(TC) * (gen + 1), P.wait_polls);
            if (!ok) {
                report_status(P.status, 4);
                atomicExch(ctrl + 1, 1u);
            }
        }
        if (__syncthreads_or(!ok)) break;
        C* const buf = ring + slot * L;
        FixedCtx<T> X;
        X.scale = T(1);
        X.conj_in = false;
        X.conj_out = false;
        if (job.phase == 0) {
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
            fused_done(ctrl, P.ring, 0, slot);
        } else {
            const int w = tid / TPL2;
            X.t = tid - w * TPL2;
            X.active = w < W2;
            const int row = tile * W2 + w;
            X.line_ok = X.active;
            X.sel = 0;
            X.twb = static_cast<const C*>(P.tw2);
            X.sm = sm + w * kpitch<T, N2>();
            X.gin = buf + static_cast<int64_t>(row) * N2;
            X.gout = nullptr;
            X.in_ks = 1;
            X.out_ks = 1;
            fused4_rows<T, N2, TPL2, W2>(X, RR{});
            if (tid == 0) red_release_add(ctrl + 2 + P.ring + slot, 1u);
            C* dst = out + line * L + int64_t(tile) * W2;
            const T sc = static_cast<T>(P.scale);
            const T sy = P.conj_out ? -sc : sc;
#pragma unroll 4
            for (int idx = tid; idx < W2 * N2; idx += THREADS) {
                const int k = idx / W2;
                const int ww = idx - k * W2;
                const C a = sm[ww * kpitch<T, N2>() + pidx<T>(k)];
                __stcs(dst + ww + int64_t(k) * N1, cmake<C>(a.x * sc, a.y * sy));
            }
        }
        if (tid == 0) {
            unsigned abort;
            asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(abort) : "l"(ctrl + 1) : "memory");
            s_ticket = abort ? total : next;
        }
    }
}

// ---------------------------------------------------------------- Bluestein, three phases
//
// A Bluestein axis of length L on a convolution of length M = N1 * N2 runs three passes over
// an M-point intermediate per line: forward columns (chirp pre-multiply of the zero-padded
// line, FFT_N1, W_M twiddle), rows (FFT_N2, spectrum multiply, inverse FFT_N2, inverse twiddle,
// in place), inverse columns (inverse FFT_N1, chirp post-multiply, truncation to L). The same
// ticket schedule with three phases keeps the intermediate in the L2-resident ring: HBM sees
// the L-point input once and the L-point output once, not three M-point round trips. Each
// tile runs the stage code of the corresponding size-specialised Bluestein pass with that
// pass's parameters (tables, conjugations, scale, direction flips) as the plan bound them.
struct FusedBlueParams {
    int64_t lines = 0;
    int ring = 1, lag = 0;
    long long wait_polls = 1ll << 26;
    int* status = nullptr;  // set to 4 when a dependency wait gave up
    FixedParams a, b, c;    // forward columns, rows, inverse columns
};

template <class T, int N1, int TPL1, int W1, int FEAT, int... RC>
__device__ __forceinline__ void fusedblue_cols(FixedCtx<T>& X, Radices<RC...>) {
    fixed_stages<T, N1, TPL1, true, W1, FEAT, 1, 0, true, RC...>(X);
}

template <class T, int N2, int TPL2, int W2, int... RR>
__device__ __forceinline__ void fusedblue_rows(FixedCtx<T>& X, Radices<RR...>) {
    // FFT, spectrum multiply into shared memory (conjugated: the inverse FFT runs forward),
    // then the FFT again with the conjugate twiddle on the store
    fixed_stages<T, N2, TPL2, false, W2, kFeatLoadCG | kFeatMid, 1, 0, true, RR...>(X);
    fixed_stages<T, N2, TPL2, false, W2, kFeatTw4 | kFeatTw4Conj, 1, 0, false, RR...>(X);
}

// Column-mode context of a Bluestein column tile from a pass's parameters.
template <class T, int W1, int TPL1>
__device__ __forceinline__ void blue_col_ctx(FixedCtx<T>& X, const FixedParams& P, int tile) {
    using C = cplx<T>;
    const int w = threadIdx.x % W1;
    X.t = threadIdx.x / W1;
    X.active = X.t < TPL1;
    X.line_ok = X.active;
    X.sel = tile * W1 + w;
    X.twb = static_cast<const C*>(P.tw);
    X.scale = static_cast<T>(P.scale);
    X.conj_in = P.conj_in != 0;
    X.conj_out = P.conj_out != 0;
    X.premul = static_cast<const C*>(P.premul);
    X.postmul = static_cast<const C*>(P.postmul);
    X.g_k = P.g_k;
    X.in_len = P.in_len;
    X.out_len = P.out_len;
    X.conj_mid = P.conj_mid != 0;
    X.flip_in = P.flip_in != 0;
    X.flip_out = P.flip_out != 0;
    X.tw4_hi = static_cast<const C*>(P.tw4_hi);
    X.tw4_lo = static_cast<const C*>(P.tw4_lo);
    X.tw4_shift = P.tw4_shift;
    X.in_ks = P.in_ks;
    X.out_ks = P.out_ks;
}

// grid = lines * (2 * TA + TB) blocks, one tile each; block = THREADS >= max(W1 * TPL1, W2 * TPL2);
// dynamic smem = max(N1 * W1, W2 * kpitch<T, N2>) * sizeof(C). `in` / `out` hold lines of
// P.a.in_hi / P.c.out_hi (= L) points; the ring slots hold M = N1 * N2 points.
template <class T, int N1, int TPL1, int W1, int N2, int TPL2, int W2, int THREADS, int MINB, class RC, class RR>
__global__ void __launch_bounds__(THREADS, MINB)
    fft_fusedblue_kernel(const __grid_constant__ FusedBlueParams P, const cplx<T>* in, cplx<T>* out,
                         cplx<T>* ring, unsigned* ctrl) {
    using C = cplx<T>;
    constexpr int64_t M = int64_t(N1) * N2;
    constexpr int TA = N2 / W1;  // column tiles per line (both column phases)
    constexpr int TB = N1 / W2;  // row tiles per line
    static_assert(N2 % W1 == 0 && N1 % W2 == 0, "tiles must cover a line exactly");
    static_assert(W1 * TPL1 <= THREADS && W2 * TPL2 <= THREADS, "block too small");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* sm = reinterpret_cast<C*>(smem_raw);
    __shared__ long long s_ticket;
    FusedSched q;
    q.lines = P.lines;
    q.lag = P.lag;
    q.phases = 3;
    q.tiles[0] = TA;
    q.tiles[1] = TB;
    q.tiles[2] = TA;
    FusedTile job;
    if (fused_claim<3>(q, P.ring, ctrl, P.wait_polls, P.status, &job, &s_ticket)) {
        const int slot = static_cast<int>(job.line % P.ring);
        C* const buf = ring + slot * M;
        FixedCtx<T> X;
        if (job.phase == 0) {
            blue_col_ctx<T, W1, TPL1>(X, P.a, job.tile);
            X.sm = sm + threadIdx.x % W1;
            X.gin = in + job.line * P.a.in_hi + X.sel;
            X.gout = buf + X.sel;
            fusedblue_cols<T, N1, TPL1, W1, kFeatPremul | kFeatTw4 | kFeatLoadCS>(X, RC{});
        } else if (job.phase == 1) {
            const int w = threadIdx.x / TPL2;
            X.t = threadIdx.x - w * TPL2;
            X.active = w < W2;
            X.line_ok = X.active;
            const int row = job.tile * W2 + w;  // k1 of the line
            X.sel = row;
            X.twb = static_cast<const C*>(P.b.tw);
            X.scale = static_cast<T>(P.b.scale);
            X.conj_in = P.b.conj_in != 0;
            X.conj_out = P.b.conj_out != 0;
            X.conj_mid = P.b.conj_mid != 0;
            X.flip_in = X.flip_out = false;
            X.tw4_hi = static_cast<const C*>(P.b.tw4_hi);
            X.tw4_lo = static_cast<const C*>(P.b.tw4_lo);
            X.tw4_shift = P.b.tw4_shift;
            X.pw = static_cast<const C*>(P.b.pointwise) + static_cast<int64_t>(row) * P.b.pw_stride;
            X.sm = sm + w * kpitch<T, N2>();
            X.gin = buf + static_cast<int64_t>(row) * N2;
            X.gout = buf + static_cast<int64_t>(row) * N2;  // in place: the row is read before it is written
            X.in_ks = X.out_ks = 1;
            fusedblue_rows<T, N2, TPL2, W2>(X, RR{});
        } else {
            blue_col_ctx<T, W1, TPL1>(X, P.c, job.tile);
            X.sm = sm + threadIdx.x % W1;
            X.gin = buf + X.sel;
            X.gout = out + job.line * P.c.out_hi + X.sel;
            fusedblue_cols<T, N1, TPL1, W1, kFeatPostmul | kFeatLoadCG | kFeatStoreCS>(X, RC{});
        }
        fused_done(ctrl, P.ring, job.phase, slot);
    }
}

}  // namespace sfb
