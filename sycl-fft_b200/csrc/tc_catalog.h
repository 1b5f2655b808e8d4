// Catalog of the split-precision tensor-core pass kernels (tc_kernel.cuh).
//
// X(ID, R, S, L, COLS, G): lines of N = R^S complex<float> points as S radix-R stages on
// the tensor cores, L lines per tile (L * N/R threads per group, one per butterfly row), G
// independent groups per CTA (one CTA per SM), COLS = 1 when the lines are adjacent columns
// of a strided axis (coalesced across lines), 0 when each line is contiguous (coalesced
// along the line).
#pragma once

#define SFB_TC_CATALOG(X)   \
    X(0, 16, 2, 8, 0, 4)    \
    X(1, 16, 2, 16, 1, 2)   \
    X(2, 16, 3, 1, 0, 2)
