// Geometry of the split-precision tensor-core pass kernels (tc_kernel.cuh), shared by the
// host planner (plain C++) and the device code.
#pragma once

#include <cstddef>

#ifdef __CUDACC__
#define SFB_TC_HD __host__ __device__
#else
#define SFB_TC_HD
#endif

namespace sfb {

SFB_TC_HD constexpr int tc_pow(int r, int s) { return s == 0 ? 1 : r * tc_pow(r, s - 1); }
SFB_TC_HD constexpr int tc_tmem_cols(int c) { return c <= 32 ? 32 : c <= 64 ? 64 : c <= 128 ? 128 : c <= 256 ? 256 : 512; }

// One CTA per SM (the occupancy of a kernel that allocates tensor memory is one CTA per
// SM) made of G independent groups; a group of ROWS threads runs its own chain of tiles.
template <int R, int S, int L, int G>
struct TcShape {
    static constexpr int N = tc_pow(R, S);
    static constexpr int NB = N / R;               // butterflies per line and stage
    static constexpr int ROWS = L * NB;            // rows per stage = threads per group
    static constexpr int THREADS = G * ROWS;
    static constexpr int TILES = ROWS / 128;       // M = 128 MMA tiles per stage
    static constexpr int K2 = 2 * R;               // real K of a row, and the MMA's N
    static constexpr int ROWB = K2 * 2;            // bytes of one BF16 row
    static constexpr int PITCH = N + N / R + 1;    // exchange-buffer line pitch (complex)
    static constexpr int GCOLS = TILES * K2;       // tensor-memory columns per group
    static constexpr int TCOLS = tc_tmem_cols(G * GCOLS);
    static constexpr size_t A_BYTES = size_t(ROWS) * ROWB;
    static constexpr size_t B_BYTES = size_t(K2) * ROWB;
    // per group: A hi, A lo, exchange buffer, input staging [R][ROWS], mbarrier
    static constexpr size_t Z_OFF = 2 * A_BYTES;
    static constexpr size_t ST_OFF = Z_OFF + size_t(L) * PITCH * 8;
    static constexpr size_t BAR_OFF = ST_OFF + size_t(R) * ROWS * 8;
    static constexpr size_t GROUP_BYTES = (BAR_OFF + 8 + 127) / 128 * 128;
    // two-level twiddle table W_N^a = hi[a >> 6] * lo[a & 63] (FP32, from FP64)
    static constexpr int TW_HI = (N + 63) / 64;
    static constexpr size_t TW_OFF = 2 * B_BYTES + G * GROUP_BYTES;
    static constexpr size_t SMEM = TW_OFF + size_t(TW_HI + 64) * 8 + 16;
    static_assert(ROWS % 128 == 0, "a stage's rows must fill whole 128-row MMA tiles");
    static_assert(THREADS <= 1024, "one thread per row");
    static_assert(G * GCOLS <= 512, "tensor memory holds 512 columns");
    static_assert(K2 % 32 == 0, "rows are read from tensor memory 32 columns at a time");
    static_assert(G <= 15, "one named barrier per group");
};

}  // namespace sfb
