// CPU checks of the fused four-step kernel's tile schedule (sycl-fft_b200/csrc/fused4_schedule.h,
// the same code the kernel runs): every tile handed out exactly once, every dependency wait
// pointing at an earlier ticket, the ring and control words inside the scratch, and a
// simulation of `blocks` resident blocks claiming tickets in order with the kernel's counter
// targets, which must finish. Built by tests/native/Makefile, called from tests/test_fused4_cpu.py.
#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <climits>
#include <vector>

#include "../../sycl-fft_b200/csrc/fused4_schedule.h"

extern "C" {

// Returns 0 when every check passes, else a code naming the first failure; waits_out receives
// how many claimed tiles found their dependency unmet at claim time in the simulation.
int f4_check(int64_t lines, int64_t blocks, int tc, int tr, int max_ring, int64_t ctrl_bytes, int64_t line_bytes,
             int* lag_out, int* ring_out, int64_t* waits_out) {
    int lag = 0, ring = 0;
    if (!sfb::fused4_geometry(blocks, tc + tr, lines, max_ring, &lag, &ring)) return lines < 3 ? 0 : 1;
    *lag_out = lag;
    *ring_out = ring;
    if (!(lag >= 0 && lag < ring && ring <= lines - 1 && ring <= max_ring)) return 2;
    if (int64_t(ring) * line_bytes + ctrl_bytes > lines * line_bytes) return 3;  // ring + control in scratch
    const int64_t total = sfb::fused4_total(lines, lag, tc, tr);
    if (total != lines * (tc + tr)) return 4;
    std::vector<int64_t> col_ticket(lines * tc, -1), row_ticket(lines * tr, -1);
    for (int64_t t = 0; t < total; ++t) {
        const sfb::Fused4Tile j = sfb::fused4_decode(t, lines, lag, tc, tr);
        if (j.line < 0 || j.line >= lines || j.tile < 0 || j.tile >= (j.col ? tc : tr)) return 5;
        int64_t& slot = j.col ? col_ticket[j.line * tc + j.tile] : row_ticket[j.line * tr + j.tile];
        if (slot != -1) return 6;  // handed out twice
        slot = t;
    }
    for (int64_t v : col_ticket)
        if (v < 0) return 7;
    for (int64_t v : row_ticket)
        if (v < 0) return 7;
    // dependencies point backwards: rows of l after all columns of l; columns of l after all
    // rows of l - ring
    for (int64_t l = 0; l < lines; ++l) {
        int64_t last_col = 0, first_row = INT64_MAX, first_col = INT64_MAX;
        for (int k = 0; k < tc; ++k) {
            last_col = std::max(last_col, col_ticket[l * tc + k]);
            first_col = std::min(first_col, col_ticket[l * tc + k]);
        }
        for (int k = 0; k < tr; ++k) first_row = std::min(first_row, row_ticket[l * tr + k]);
        if (last_col >= first_row) return 8;
        if (l >= ring) {
            int64_t last_prev_row = 0;
            for (int k = 0; k < tr; ++k) last_prev_row = std::max(last_prev_row, row_ticket[(l - ring) * tr + k]);
            if (last_prev_row >= first_col) return 9;
        }
    }
    // simulation: `blocks` workers, tickets claimed in order, a tile takes 3 steps once its
    // counter target (the kernel's) is met; counters per ring slot as in the kernel
    std::vector<uint64_t> col_done(ring, 0), row_done(ring, 0);
    struct Worker {
        int64_t t = -1;
        int left = 0;
        bool waited = false;
    };
    std::vector<Worker> w(static_cast<size_t>(std::min<int64_t>(blocks, total)));
    int64_t next = 0, done = 0, waits = 0, steps = 0;
    for (auto& x : w) x.t = next < total ? next++ : -1;
    while (done < total) {
        if (++steps > 100 * (total + 10)) return 10;  // no progress: a deadlock
        for (auto& x : w) {
            if (x.t < 0) continue;
            const sfb::Fused4Tile j = sfb::fused4_decode(x.t, lines, lag, tc, tr);
            const int slot = static_cast<int>(j.line % ring);
            const uint64_t gen = static_cast<uint64_t>(j.line / ring);
            if (x.left == 0) {
                const bool ready = j.col ? (gen == 0 || row_done[slot] >= uint64_t(tr) * gen)
                                         : col_done[slot] >= uint64_t(tc) * (gen + 1);
                if (!ready) {
                    if (!x.waited) ++waits;
                    x.waited = true;
                    continue;
                }
                x.left = 3;
            }
            if (--x.left == 0) {
                (j.col ? col_done : row_done)[slot] += 1;
                ++done;
                x.waited = false;
                x.t = next < total ? next++ : -1;
            }
        }
    }
    *waits_out = waits;
    return 0;
}

}  // extern "C"
