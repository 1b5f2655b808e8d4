// Catalog of the fused four-step kernels (fused4_kernel.cuh): one persistent launch running
// the column and row passes of a four-step line with an L2-resident ring in between.
//
// X(ID, DOUBLE, N1, TPL1, W1, COL_ID, N2, TPL2, W2, ROW_ID, THREADS, MINB, PERSIST, (RC...), (RR...))
//   N1 / N2: column / row FFT lengths (line L = N1 * N2); TPL, W: threads per column or row and
//   columns or rows per tile, as in the size-specialised two-pass entries COL_ID (four-step
//   column pass) and ROW_ID (four-step row pass) of fixed_catalog.h, whose stage code the tiles
//   run; THREADS the block size, MINB the blocks per SM the registers are budgeted for; RC / RR
//   the radix sequences of the column and row FFTs. PERSIST 1: the persistent claim-ahead kernel
//   by default (0 where its loop spills registers: one tile per block).
#pragma once

#define SFB_FUSED4_CATALOG(X)                                                   \
    X(0, 1, 256, 32, 8, 49, 256, 32, 8, 57, 256, 4, 1, (8, 8, 4), (8, 8, 4))       \
    X(1, 0, 256, 16, 16, 44, 256, 16, 16, 53, 256, 4, 1, (16, 16), (16, 16))         \
    X(2, 0, 112, 8, 24, 61, 120, 8, 16, 62, 192, 5, 0, (16, 7), (8, 15))

#define SFB_FUSED4_COUNT 3

// Fused Bluestein kernels (fft_fusedblue_kernel): the three size-specialised Bluestein passes of
// a convolution of length M = N1 * N2 (forward columns COLF_ID, rows ROWS_ID, inverse columns
// COLI_ID of bluestein_catalog.h) in one launch with the M-point intermediate in the ring.
// X(ID, DOUBLE, N1, TPL1, W1, COLF_ID, N2, TPL2, W2, ROWS_ID, COLI_ID, THREADS, MINB, (RC...), (RR...))
#define SFB_FUSEDBLUE_CATALOG(X)                                                                  \
    X(0, 0, 256, 16, 16, 54, 512, 32, 16, 45, 55, 512, 2, (16, 16), (16, 16, 2))                 \
    X(1, 1, 256, 32, 8, 110, 512, 64, 8, 101, 111, 512, 2, (8, 8, 4), (8, 8, 8))                 \
    X(2, 1, 128, 16, 8, 108, 80, 16, 8, 90, 109, 128, 8, (8, 8, 2), (8, 2, 5))
