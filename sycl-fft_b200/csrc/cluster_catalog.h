// Catalog of the thread-block-cluster kernels (cluster_kernel.cuh).
//
// X(ID, DOUBLE, N1, N2, P, TPL1, TPL2, MAXT, MINB, (RADICES1), (RADICES2))
//   line length N = N1 * N2 split over a cluster of P CTAs; TPL1/TPL2 threads per column
//   (length-N1 FFT) and per row (length-N2 FFT); MAXT/MINB the launch bounds;
//   RADICES the Stockham stages of the two FFTs. Shared memory per CTA: N/P elements.
#pragma once

#define SFB_CLUSTER_CATALOG(X)                                         \
    X(0, 1, 256, 256, 8, 32, 32, 1024, 1, (8, 8, 4), (8, 8, 4))         \
    X(1, 1, 256, 256, 16, 32, 32, 512, 2, (8, 8, 4), (8, 8, 4))         \
    X(2, 0, 256, 256, 8, 16, 16, 512, 2, (16, 16), (16, 16))            \
    X(3, 0, 256, 512, 8, 16, 32, 1024, 1, (16, 16), (16, 16, 2))        \
    X(4, 1, 128, 256, 8, 16, 32, 512, 2, (8, 8, 2), (8, 8, 4))          \
    X(5, 0, 128, 256, 8, 8, 16, 512, 2, (16, 8), (16, 16))

#define SFB_CLUSTER_COUNT 6
