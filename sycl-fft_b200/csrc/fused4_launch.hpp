// Host entry into the fused four-step kernels (fused4_variants.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "fused4_kernel.cuh"

namespace sfb {

struct Fused4Entry {
    int id, dbl, n1, w1, col_id, n2, w2, row_id, threads;
    int64_t smem;  // dynamic shared memory per block
};

// The fused kernel for a four-step of precision `dbl` whose column and row passes run the
// size-specialised entries col_id / row_id; nullptr if there is none.
const Fused4Entry* find_fused4(bool dbl, int col_id, int row_id);

// Launches entry `e` over `p.lines` lines: zeroes the control words, sizes the grid to the
// resident blocks of the device and picks the lag and ring (p.ring / p.lag are outputs). The
// ring takes p.ring lines of `scratch`, the control words follow it; scratch must hold
// `lines` lines (lines >= 3). Returns cudaErrorInvalidValue when lines < 3.
cudaError_t launch_fused4(const Fused4Entry& e, Fused4Params& p, const void* in, void* out, void* scratch,
                          cudaStream_t stream);

struct FusedBlueEntry {
    int id, dbl, n1, w1, colf_id, n2, w2, rows_id, coli_id, threads;
    int64_t smem;
};

// The fused Bluestein kernel for the three size-specialised Bluestein passes colf_id, rows_id,
// coli_id (bluestein_catalog.h), or nullptr.
const FusedBlueEntry* find_fusedblue(bool dbl, int colf_id, int rows_id, int coli_id);

// Launches entry `e` over `p.lines` lines (ring and lag chosen as for launch_fused4; the ring
// holds M-point slots of `scratch`, which must hold `lines` of them, lines >= 4).
cudaError_t launch_fusedblue(const FusedBlueEntry& e, FusedBlueParams& p, const void* in, void* out, void* scratch,
                             cudaStream_t stream);

}  // namespace sfb
