// CPU checks of the fused multi-pass kernels' tile schedule (sycl-fft_b200/csrc/fused4_schedule.h,
// the same code the kernels run): every tile of every phase handed out exactly once, every
// dependency wait pointing at an earlier ticket, the ring and control words inside the scratch,
// and a simulation of `blocks` resident blocks claiming tickets in order with the kernels'
// counter targets, which must finish. Built by tests/native/Makefile, called from
// tests/test_fused4_cpu.py.
#include <algorithm>
#include <climits>
#include <cstdint>
#include <vector>

#include "../../sycl-fft_b200/csrc/fused4_schedule.h"

extern "C" {

// tiles: `phases` tile counts per line. Returns 0 when every check passes, else a code naming
// the first failure; waits_out receives how many claimed tiles found their dependency unmet
// at claim time in the simulation.
int f4_check(int64_t lines, int64_t blocks, int phases, const int* tiles, int max_ring, int64_t ctrl_bytes,
             int64_t line_bytes, int* lag_out, int* ring_out, int64_t* waits_out) {
    int tiles_per_line = 0;
    for (int p = 0; p < phases; ++p) tiles_per_line += tiles[p];
    int lag = 0, ring = 0;
    if (!sfb::fused_geometry(blocks, tiles_per_line, lines, phases, max_ring, &lag, &ring))
        return lines < phases + 1 ? 0 : 1;
    *lag_out = lag;
    *ring_out = ring;
    if (!(lag >= 1 && int64_t(phases - 1) * lag < ring && ring <= lines - 1 && ring <= max_ring)) return 2;
    // a slot's reuse is claimed at least as many segments after its last use as a phase lag
    // minus one (an even split when the ring is capped)
    if (lines > 2 * phases && ring - int64_t(phases - 1) * lag < lag - 1) return 11;
    if (int64_t(ring) * line_bytes + ctrl_bytes > lines * line_bytes) return 3;  // ring + control in scratch
    sfb::FusedSched q;
    q.lines = lines;
    q.lag = lag;
    q.phases = phases;
    for (int p = 0; p < phases; ++p) q.tiles[p] = tiles[p];
    const int64_t total = sfb::fused_total(q);
    if (total != lines * tiles_per_line) return 4;
    // ticket of every (phase, line, tile)
    std::vector<std::vector<int64_t>> ticket(phases);
    for (int p = 0; p < phases; ++p) ticket[p].assign(lines * tiles[p], -1);
    for (int64_t t = 0; t < total; ++t) {
        const sfb::FusedTile j = sfb::fused_decode(q, t);
        if (j.phase < 0 || j.phase >= phases || j.line < 0 || j.line >= lines || j.tile < 0 || j.tile >= tiles[j.phase])
            return 5;
        int64_t& slot = ticket[j.phase][j.line * tiles[j.phase] + j.tile];
        if (slot != -1) return 6;  // handed out twice
        slot = t;
    }
    for (const auto& v : ticket)
        for (int64_t x : v)
            if (x < 0) return 7;
    auto first = [&](int p, int64_t l) {
        int64_t m = INT64_MAX;
        for (int k = 0; k < tiles[p]; ++k) m = std::min(m, ticket[p][l * tiles[p] + k]);
        return m;
    };
    auto last = [&](int p, int64_t l) {
        int64_t m = 0;
        for (int k = 0; k < tiles[p]; ++k) m = std::max(m, ticket[p][l * tiles[p] + k]);
        return m;
    };
    // dependencies point backwards: phase p of l after all of phase p-1 of l; phase 0 of l
    // after all of the last phase of l - ring
    for (int64_t l = 0; l < lines; ++l) {
        for (int p = 1; p < phases; ++p)
            if (last(p - 1, l) >= first(p, l)) return 8;
        if (l >= ring && last(phases - 1, l - ring) >= first(0, l)) return 9;
    }
    // simulation: `blocks` workers, tickets claimed in order, a tile takes 3 steps once its
    // counter target (the kernels') is met; counters per phase and ring slot as in the kernels
    std::vector<std::vector<uint64_t>> done(phases, std::vector<uint64_t>(ring, 0));
    struct Worker {
        int64_t t = -1;
        int left = 0;
        bool waited = false;
    };
    std::vector<Worker> w(static_cast<size_t>(std::min<int64_t>(blocks, total)));
    int64_t next = 0, finished = 0, waits = 0, steps = 0;
    for (auto& x : w) x.t = next < total ? next++ : -1;
    while (finished < total) {
        if (++steps > 100 * (total + 10)) return 10;  // no progress: a deadlock
        for (auto& x : w) {
            if (x.t < 0) continue;
            const sfb::FusedTile j = sfb::fused_decode(q, x.t);
            const int slot = static_cast<int>(j.line % ring);
            const uint64_t gen = static_cast<uint64_t>(j.line / ring);
            if (x.left == 0) {
                const bool ready = j.phase == 0
                                       ? (gen == 0 || done[phases - 1][slot] >= uint64_t(tiles[phases - 1]) * gen)
                                       : done[j.phase - 1][slot] >= uint64_t(tiles[j.phase - 1]) * (gen + 1);
                if (!ready) {
                    if (!x.waited) ++waits;
                    x.waited = true;
                    continue;
                }
                x.left = 3;
            }
            if (--x.left == 0) {
                done[j.phase][slot] += 1;
                ++finished;
                x.waited = false;
                x.t = next < total ? next++ : -1;
            }
        }
    }
    *waits_out = waits;
    return 0;
}

}  // extern "C"
