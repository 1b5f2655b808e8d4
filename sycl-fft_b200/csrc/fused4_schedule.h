// Tile schedule of the fused four-step kernel (fused4_kernel.cuh), shared by the device code,
// its host launcher and the CPU checks of the schedule (tests/native/fused4_check.cpp).
//
// A launch over `lines` lines of TC column tiles and TR row tiles each hands out tickets
// 0 .. total-1 in order. Segment s = 0 .. lines + lag - 1 holds the column tiles of line s
// (s < lines) followed by the row tiles of line s - lag (s >= lag).
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define SFB_F4_HD __host__ __device__
#else
#define SFB_F4_HD
#endif

namespace sfb {

struct Fused4Tile {
    bool col;      // column tile (else row tile)
    int64_t line;  // line index
    int tile;      // tile index within the line's column (0 .. TC-1) or row (0 .. TR-1) tiles
};

SFB_F4_HD inline int64_t fused4_total(int64_t lines, int64_t lag, int tc, int tr) {
    return lag * tc + (lines - lag) * (tc + tr) + lag * tr;
}

// Ticket t (0 <= t < fused4_total) -> tile.
SFB_F4_HD inline Fused4Tile fused4_decode(int64_t t, int64_t lines, int64_t lag, int tc, int tr) {
    Fused4Tile r;
    const int64_t head = lag * tc;
    const int64_t body = (lines - lag) * (tc + tr);
    if (t < head) {
        r.col = true;
        r.line = t / tc;
        r.tile = static_cast<int>(t % tc);
    } else if (t < head + body) {
        const int64_t u = t - head;
        const int64_t s = lag + u / (tc + tr);
        const int k = static_cast<int>(u % (tc + tr));
        r.col = k < tc;
        r.line = r.col ? s : s - lag;
        r.tile = r.col ? k : k - tc;
    } else {
        const int64_t u = t - head - body;
        r.col = false;
        r.line = lines - lag + u / tr;
        r.tile = static_cast<int>(u % tr);
    }
    return r;
}

// Lag and ring size for `blocks` resident blocks: the tiles in flight span fewer lines than
// the lag, so a line's columns are done by the time its rows are claimed, and the ring has
// more slots than the lag (every dependency then points at an earlier ticket). The ring takes
// at most lines - 1 slots of a scratch that holds `lines` lines (the control words follow
// it) and at most `max_ring`. Returns false when lines < 3.
inline bool fused4_geometry(int64_t blocks, int tiles_per_line, int64_t lines, int max_ring, int* lag, int* ring) {
    if (lines < 3 || tiles_per_line <= 0 || max_ring < 2) return false;
    int64_t d = (blocks + tiles_per_line - 1) / tiles_per_line + 2;
    if (d > lines - 2) d = lines - 2;
    int64_t r = 2 * d + 2;
    if (r > lines - 1) r = lines - 1;
    if (r > max_ring) r = max_ring;
    if (d >= r) d = r - 1;
    *lag = static_cast<int>(d);
    *ring = static_cast<int>(r);
    return true;
}

}  // namespace sfb
