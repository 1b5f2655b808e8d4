// Catalog of the copy-engine-pipelined pass kernels (piped_kernel.cuh).
// Kept only where measured faster than the plain size-specialised kernel on B200
// (c64 13440: 3424 vs 2638 GB/s; c64 8192: 4695 vs 4499; c128 4096 lost: 4523 vs 4849).
// For 13440 the stages [16, 8, 3, 5, 7] beat [16, 8, 15, 7] with the prime-factor radix-15
// butterfly (2612 GB/s piped, 3010 plain): its 15 values and 14 twiddle powers spill.
//
// X(ID, DOUBLE, N, TPL, MAXT, RADICES...): contiguous lines of length N, TPL threads per
// (persistent) CTA, two N-element line buffers in shared memory. Listed lengths are those
// whose single line fills most of an SM's shared memory, where the plain kernel cannot
// overlap HBM traffic with the exchanges.
#pragma once

#define SFB_PIPED_CATALOG(X)                 \
    X(0, 0, 13440, 896, 896, 16, 8, 15, 7) \
    X(1, 0, 8192, 512, 512, 16, 16, 16, 2)
