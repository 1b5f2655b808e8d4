// Split-precision tensor-core pass for complex<float> lines (optional, per plan).
//
// A line of N = R^S points runs as S radix-R Stockham stages, and each stage is a matrix
// product on the 5th-generation tensor cores (tcgen05.mma, accumulators in tensor memory):
//
//   rows    = the stage's butterflies of all lines in the tile (L * N/R rows);
//   A[row]  = the butterfly's R twiddled inputs, interleaved re/im (K = 2R);
//   B       = the radix-R DFT as a real 2R x 2R matrix ([re; im] of every output);
//   D = A B^T, FP32 in tensor memory: the row's R outputs, interleaved re/im.
//
// BF16 keeps 8 significant bits, so both operands are split, x = hi + lo with hi = bf16(x)
// and lo = bf16(x - hi) (16 bits together), and the product is accumulated in FP32 as
// hi*hi + hi*lo + lo*hi. The dropped lo*lo term is 2^-16 relative; with it, the error of
// random inputs would drop by about 15% (4.3e-6 -> 3.6e-6 relative L2 at 256 points).
// Everything else stays FP32: the twiddles (two-level FP32 tables rounded from FP64, one
// complex product per twiddle, held in shared memory), the
// Stockham exchanges through shared memory, the scale and the conjugations.
//
// A tile is L lines. Per stage every thread of a group owns one row: it gathers and twiddles its
// butterfly's inputs (its staging slots for the first stage, the padded FP32 exchange buffer after),
// writes the hi/lo rows in the UMMA canonical K-major layout (8x16-byte core matrices, no
// swizzle), and after one thread has issued the tile's MMAs and committed them to an
// mbarrier, reads its row back from tensor memory (tcgen05.ld, the thread's own lane) and
// stores the outputs (exchange buffer, or HBM for the last stage).
//
// Waits on the MMA mbarrier are bounded: after P.wait_polls polls the CTA records a timeout
// in the plan's status word, waits (bounded again, kSpinLimit polls) for the commit, frees
// its tensor memory and returns.
#pragma once

#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "async_util.cuh"
#include "pass_params.h"
#include "tc_shape.h"

namespace sfb {

struct TcParams {
    int64_t n_outer = 1, n_cols = 1, col_tiles = 1, tiles = 1;
    LineLayout in, out;      // line (o, c) element k at (o/d)*hi + (o%d)*lo + c*cs + k*ks
    float scale = 1.f;
    int conj_in = 0, conj_out = 0;
    // Twiddles W_N^k = exp(-2 pi i k / N) in two levels, FP32 rounded from FP64:
    // hi[a] = W_N^(64a) for a < ceil(N/64), then lo[b] = W_N^b for b < 64.
    const void* tw = nullptr;
    int* status = nullptr;     // set to 2 if an MMA wait timed out
    long long wait_polls = kSpinLimit;  // polls before an MMA wait gives up
};

// Byte offset of element kk of row `row` in the canonical K-major no-swizzle layout: 8-row x
// 16-byte core matrices, consecutive along K (LBO = 128 B), row groups SBO = K2*16 B apart.
template <int K2>
SFB_TC_HD constexpr uint32_t tc_off(int row, int kk) {
    return uint32_t(((row >> 3) * (K2 / 8) + (kk >> 3)) * 128 + (row & 7) * 16 + (kk & 7) * 2);
}

__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((saddr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);  // descriptor version 1
}

// kind::f16 instruction descriptor: BF16 x BF16 -> F32, both K-major, M x N.
SFB_TC_HD constexpr uint32_t umma_idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive 32-bit columns of this thread's lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&d)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
          "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15]),
          "=r"(d[16]), "=r"(d[17]), "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]), "=r"(d[22]), "=r"(d[23]),
          "=r"(d[24]), "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]), "=r"(d[29]), "=r"(d[30]), "=r"(d[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// x = hi + lo in BF16 for a pair of floats; returns the packed (hi, lo) pairs.
__device__ __forceinline__ void split_bf16x2(float a, float b, uint32_t& hi, uint32_t& lo) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    const float2 hf = __bfloat1622float2(h);
    const __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = *reinterpret_cast<const uint32_t*>(&l);
}

// 8-byte asynchronous global -> shared copy; `valid` false fills zeros and reads nothing.
__device__ __forceinline__ void cp_async8(void* dst, const void* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(valid ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Named barrier over one group's threads; the _or form returns whether any thread passed true.
__device__ __forceinline__ void group_sync(int id, int n) {
    asm volatile("barrier.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}
__device__ __forceinline__ bool group_sync_or(int id, int n, bool v) {
    int r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.b32 p, %1, 0;\n barrier.red.or.pred q, %2, %3, p;\n selp.s32 %0, 1, 0, q;\n}\n"
        : "=r"(r)
        : "r"(int(v)), "r"(id), "r"(n)
        : "memory");
    return r != 0;
}

// Persistent: one CTA per SM, G independent groups. Group g of CTA b runs tiles
// b*G + g, b*G + g + gridDim.x*G, ... Each thread prefetches the next tile's inputs of its
// own row with cp.async into its own staging slots while the current tile computes, so the
// HBM reads overlap the stages and no barrier guards the staging buffer.
template <int R, int S, int L, bool COLS, int G>
__global__ void __launch_bounds__(TcShape<R, S, L, G>::THREADS, 1)
    fft_tc_kernel(const __grid_constant__ TcParams P, const float2* __restrict__ in, float2* __restrict__ out) {
    using Sh = TcShape<R, S, L, G>;
    constexpr int N = Sh::N, NB = Sh::NB, K2 = Sh::K2, PITCH = Sh::PITCH, ROWS = Sh::ROWS;
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char* b_hi = smem;
    unsigned char* b_lo = b_hi + Sh::B_BYTES;
    const int grp = threadIdx.x / ROWS;
    unsigned char* gbase = smem + 2 * Sh::B_BYTES + size_t(grp) * Sh::GROUP_BYTES;
    unsigned char* a_hi = gbase;
    unsigned char* a_lo = gbase + Sh::A_BYTES;
    float2* z = reinterpret_cast<float2*>(gbase + Sh::Z_OFF);
    float2* stage_in = reinterpret_cast<float2*>(gbase + Sh::ST_OFF);  // [R][ROWS]
    uint64_t* bar = reinterpret_cast<uint64_t*>(gbase + Sh::BAR_OFF);
    float2* tw_hi = reinterpret_cast<float2*>(smem + Sh::TW_OFF);
    float2* tw_lo = tw_hi + Sh::TW_HI;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + Sh::TW_OFF + size_t(Sh::TW_HI + 64) * 8);

    const int t = threadIdx.x - grp * ROWS;  // row of this thread within its group
    const int warp = threadIdx.x >> 5;
    const int bar_id = 1 + grp;              // named barrier of the group (0 is __syncthreads)
    // Row -> (line, butterfly): lines fastest when lines are adjacent columns (coalesced
    // across lines), butterflies fastest for contiguous lines (coalesced along the line).
    const int l = COLS ? t % L : t / NB;
    const int j = COLS ? t / L : t % NB;
    for (int e = threadIdx.x; e < Sh::TW_HI + 64; e += Sh::THREADS) tw_hi[e] = static_cast<const float2*>(P.tw)[e];

    // The radix-R DFT as a real matrix, rows = outputs [re, im], columns = inputs [re, im]:
    // B[2m][2n] = cos, B[2m][2n+1] = -sin', B[2m+1][2n] = sin', B[2m+1][2n+1] = cos with
    // exp(-2 pi i m n / R) = cos + i sin'.
    for (int e = threadIdx.x; e < K2 * K2 / 2; e += Sh::THREADS) {
        const int row = e / (K2 / 2);  // output component
        const int kp = e % (K2 / 2);    // input n: columns 2n, 2n+1
        const int m = row >> 1;
        float sv, cv;
        sincospif(-2.f * float((m * kp) % R) / float(R), &sv, &cv);
        const float x0 = (row & 1) ? sv : cv;
        const float x1 = (row & 1) ? cv : -sv;
        uint32_t hi, lo;
        split_bf16x2(x0, x1, hi, lo);
        *reinterpret_cast<uint32_t*>(b_hi + tc_off<K2>(row, 2 * kp)) = hi;
        *reinterpret_cast<uint32_t*>(b_lo + tc_off<K2>(row, 2 * kp)) = lo;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(Sh::TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (t == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }

    const int64_t first = int64_t(blockIdx.x) * G + grp;
    const int64_t stride = int64_t(gridDim.x) * G;
    // This thread's line of a tile, and whether it exists (no 64-bit division in the
    // common layouts: a single outer index, or undivided outer strides).
    auto line_at = [&](int64_t tile, int64_t& o, int64_t& c) {
        if (P.n_outer == 1) {
            o = 0;
            c = tile * L + l;
        } else {
            o = tile / P.col_tiles;
            c = (tile - o * P.col_tiles) * L + l;
        }
        return o < P.n_outer && c < P.n_cols;
    };
    auto base = [&](const LineLayout& y, int64_t o, int64_t c) -> int64_t {
        if (y.d == 1) return o * y.hi + c * y.cs;
        return (o / y.d) * y.hi + (o % y.d) * y.lo + c * y.cs;
    };
    const int64_t in_step = int64_t(NB) * P.in.ks;
    const int64_t out_step = int64_t(NB) * P.out.ks;
    auto prefetch = [&](int64_t tile) {
        if (tile < P.tiles) {
            int64_t o, c;
            const bool ok = line_at(tile, o, c);
            const float2* g = ok ? in + base(P.in, o, c) + int64_t(j) * P.in.ks : in;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                cp_async8(stage_in + r * ROWS + t, g, ok);
                if (ok) g += in_step;
            }
        }
        cp_async_commit();
    };
    prefetch(first);

    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot + uint32_t(grp * Sh::GCOLS);
    constexpr uint32_t idesc = umma_idesc_bf16(128, K2);
    constexpr uint32_t SBO = K2 * 16;
    // descriptors of the first K step; the start address (16-byte units, low bits) advances
    // by 256 bytes per K step and by one 128-row tile per MMA tile
    const uint64_t da_hi = umma_smem_desc(smem_u32(a_hi), 128, SBO), da_lo = umma_smem_desc(smem_u32(a_lo), 128, SBO);
    const uint64_t db_hi = umma_smem_desc(smem_u32(b_hi), 128, SBO), db_lo = umma_smem_desc(smem_u32(b_lo), 128, SBO);
    uint32_t phase = 0;
    bool stuck = false;

    for (int64_t tile = first; tile < P.tiles && !stuck; tile += stride) {
        int64_t o, c;
        const bool line_ok = line_at(tile, o, c);
        float2* gout = out + (line_ok ? base(P.out, o, c) + int64_t(j) * P.out.ks : 0);
        cp_async_wait_all();  // this thread's inputs of this tile are in its staging slots
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int ns = tc_pow(R, s);
            const int jm = j % ns;
            // gather (and twiddle) this row's inputs
            float2 v[R];
            if (s == 0) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    v[r] = stage_in[r * ROWS + t];
                    if (P.conj_in) v[r].y = -v[r].y;
                }
                prefetch(tile + stride);  // own slots consumed: fetch the next tile's
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int idx = j + r * NB;
                    v[r] = z[l * PITCH + idx + idx / R];
                }
                const int step = N / (ns * R);
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    const int e = r * jm * step;
                    const float2 h = tw_hi[e >> 6], q = tw_lo[e & 63];
                    const float2 w = make_float2(h.x * q.x - h.y * q.y, h.x * q.y + h.y * q.x);
                    const float2 a = v[r];
                    v[r] = make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
                }
            }
            // split into the BF16 hi / lo rows (16 bytes = 4 complex per core-matrix row)
#pragma unroll
            for (int q = 0; q < K2 / 8; ++q) {
                uint4 h, lo;
                split_bf16x2(v[4 * q + 0].x, v[4 * q + 0].y, h.x, lo.x);
                split_bf16x2(v[4 * q + 1].x, v[4 * q + 1].y, h.y, lo.y);
                split_bf16x2(v[4 * q + 2].x, v[4 * q + 2].y, h.z, lo.z);
                split_bf16x2(v[4 * q + 3].x, v[4 * q + 3].y, h.w, lo.w);
                *reinterpret_cast<uint4*>(a_hi + tc_off<K2>(t, 8 * q)) = h;
                *reinterpret_cast<uint4*>(a_lo + tc_off<K2>(t, 8 * q)) = lo;
            }
            fence_proxy_async();  // generic-proxy writes of A (and B) -> visible to the tensor core
            tc_fence_before();
            group_sync(bar_id, ROWS);
            if (t == 0) {
                tc_fence_after();
#pragma unroll
                for (int tl = 0; tl < Sh::TILES; ++tl) {
                    const uint32_t d = tmem + uint32_t(tl * K2);
                    const uint64_t a_off = uint64_t(tl) * 128u * Sh::ROWB / 16;
#pragma unroll
                    for (int ks = 0; ks < K2 / 16; ++ks)
                        umma_bf16(d, da_hi + a_off + ks * 16, db_hi + ks * 16, idesc, ks > 0 ? 1u : 0u);
#pragma unroll
                    for (int ks = 0; ks < K2 / 16; ++ks) umma_bf16(d, da_hi + a_off + ks * 16, db_lo + ks * 16, idesc, 1u);
#pragma unroll
                    for (int ks = 0; ks < K2 / 16; ++ks) umma_bf16(d, da_lo + a_off + ks * 16, db_hi + ks * 16, idesc, 1u);
                }
                umma_commit(bar);
            }
            // One thread polls the MMA barrier; the others wait in the named barrier.
            bool done = true;
            if (t == 0) {
                done = mbar_wait_bounded(bar, phase, P.wait_polls);
                tc_fence_before();
            }
            if (group_sync_or(bar_id, ROWS, !done)) {
                stuck = true;
                break;
            }
            phase ^= 1u;
            tc_fence_after();
            // this row of D: the butterfly's R outputs, interleaved re/im
            const uint32_t taddr = tmem + (uint32_t((warp & 3) * 32) << 16) + uint32_t((t >> 7) * K2);
            float y[K2];
#pragma unroll
            for (int h = 0; h < K2 / 32; ++h) {
                uint32_t d[32];
                tmem_ld32(taddr + uint32_t(h * 32), d);
                tmem_wait_ld();
#pragma unroll
                for (int i = 0; i < 32; ++i) y[h * 32 + i] = __uint_as_float(d[i]);
            }
            if (s + 1 < S) {
#pragma unroll
                for (int m = 0; m < R; ++m) {
                    const int idx = (j - jm) * R + jm + m * ns;
                    z[l * PITCH + idx + idx / R] = make_float2(y[2 * m], y[2 * m + 1]);
                }
            } else if (line_ok) {
                const float sy = P.conj_out ? -P.scale : P.scale;
#pragma unroll
                for (int m = 0; m < R; ++m) {
                    *gout = make_float2(y[2 * m] * P.scale, y[2 * m + 1] * sy);
                    gout += out_step;
                }
            }
            tc_fence_before();
            group_sync(bar_id, ROWS);  // exchange buffer complete; tensor-memory reads done before the next MMAs
        }
    }
    cp_async_wait_all();  // no copy into shared memory outlives the CTA
    if (stuck && t == 0) {
        report_status(P.status, 2);
        // let the outstanding MMAs finish (bounded) before their tensor memory is released
        mbar_wait_bounded(bar, phase, kSpinLimit);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmem_slot), "r"(Sh::TCOLS)
                     : "memory");
}

}  // namespace sfb
