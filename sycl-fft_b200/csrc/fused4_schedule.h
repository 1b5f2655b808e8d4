// Tile schedule of the fused multi-pass kernels (fused4_kernel.cuh), shared by the device
// code, its host launcher and the CPU checks of the schedule (tests/native/fused4_check.cpp).
//
// A launch runs P passes (phases) over `lines` lines; phase p has tiles[p] tiles per line and
// needs every tile of phase p - 1 of the same line. Tickets 0 .. total-1 are handed out in
// order. Segment s = 0 .. lines + (P-1) * lag - 1 holds, for p = 0 .. P-1 in turn, the tiles
// of phase p of line s - p * lag (when that line exists), so a tile is claimed about `lag`
// lines of work after the tiles it depends on.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define SFB_F4_HD __host__ __device__
#else
#define SFB_F4_HD
#endif

namespace sfb {

constexpr int kFusedMaxPhases = 3;

struct FusedTile {
    int phase;     // 0 .. P-1
    int64_t line;  // line index
    int tile;      // tile index within the phase's tiles of the line
};

struct FusedSched {
    int64_t lines = 0;
    int64_t lag = 0;
    int phases = 2;
    int tiles[kFusedMaxPhases] = {0, 0, 0};
};

// Tiles of segment s (phases whose line s - p * lag exists).
SFB_F4_HD inline int64_t fused_segment_size(const FusedSched& q, int64_t s) {
    int64_t n = 0;
    for (int p = 0; p < q.phases; ++p) {
        const int64_t l = s - p * q.lag;
        if (l >= 0 && l < q.lines) n += q.tiles[p];
    }
    return n;
}

SFB_F4_HD inline int64_t fused_total(const FusedSched& q) {
    int64_t n = 0;
    for (int p = 0; p < q.phases; ++p) n += q.tiles[p];
    return n * q.lines;
}

// Ticket t (0 <= t < fused_total) -> tile. The segment sizes change only where a phase's line
// range starts or ends (s = p * lag or p * lag + lines), so the decode walks at most
// 2 * phases regions of equal-size segments.
SFB_F4_HD inline FusedTile fused_decode(const FusedSched& q, int64_t t) {
    int64_t edges[2 * kFusedMaxPhases + 1];
    int ne = 0;
    for (int p = 0; p < q.phases; ++p) {
        edges[ne++] = p * q.lag;
        edges[ne++] = p * q.lag + q.lines;
    }
    // sort the region boundaries (at most 6)
    for (int i = 1; i < ne; ++i)
        for (int j = i; j > 0 && edges[j - 1] > edges[j]; --j) {
            const int64_t v = edges[j];
            edges[j] = edges[j - 1];
            edges[j - 1] = v;
        }
    FusedTile r{0, 0, 0};
    int64_t a = 0;
    for (int i = 0; i < ne; ++i) {
        const int64_t b = edges[i];
        if (b <= a) continue;
        const int64_t size = fused_segment_size(q, a);
        const int64_t span = (b - a) * size;
        if (t < span) {
            const int64_t s = a + t / size;
            int64_t k = t % size;
            for (int p = 0; p < q.phases; ++p) {
                const int64_t l = s - p * q.lag;
                if (l < 0 || l >= q.lines) continue;
                if (k < q.tiles[p]) {
                    r.phase = p;
                    r.line = l;
                    r.tile = static_cast<int>(k);
                    return r;
                }
                k -= q.tiles[p];
            }
        }
        t -= span;
        a = b;
    }
    r.phase = -1;  // t out of range
    return r;
}

// Lag and ring size for `blocks` resident blocks: the tiles in flight span fewer lines than
// the lag, so a line's earlier phase is done by the time its next phase is claimed, and the
// ring has more slots than (phases - 1) * lag, so every dependency points at an earlier
// ticket. The ring takes at most lines - 1 slots of a scratch that holds `lines` lines (the
// control words follow it) and at most `max_ring`. Returns false when lines < phases + 1.
inline bool fused_geometry(int64_t blocks, int tiles_per_line, int64_t lines, int phases, int max_ring, int* lag,
                           int* ring) {
    if (phases < 2 || lines < phases + 1 || tiles_per_line <= 0 || max_ring < phases) return false;
    const int64_t span = phases - 1;
    int64_t d = (blocks + tiles_per_line - 1) / tiles_per_line + 2;
    int64_t r = span * d + d + 2;
    const int64_t cap = lines - 1 < max_ring ? lines - 1 : max_ring;
    if (r > cap) {
        // a smaller ring: split it evenly between the phases' lags and the gap before a slot is
        // reused (phase 0 of line l waits for the last phase of line l - ring, claimed
        // ring - span * d segments earlier), so neither wait is claimed right behind its target
        r = cap;
        d = r / phases;
        if (span * d >= r) d = (r - 1) / span;
    }
    if (d < 1) return false;
    *lag = static_cast<int>(d);
    *ring = static_cast<int>(r);
    return true;
}

}  // namespace sfb
