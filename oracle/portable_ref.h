/* CPU restatement of the syclfft portable provider -- TEST INFRASTRUCTURE ONLY.
 *
 * Used by tests/ as the parity checker and by bench.py's CPU-baseline leg.
 * Not part of the product library. Semantics follow src/sycl/sycl.cpp of
 * Vaskozlov/sycl-fft (see portable_ref.cpp for the per-function citations).
 */
#ifndef SYCLFFT_ORACLE_PORTABLE_REF_H
#define SYCLFFT_ORACLE_PORTABLE_REF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* direction: -1 forward, +1 backward. normalization: 0 none, 1 forward,
 * 2 backward, 3 orthogonal. lengths in C order (last dimension contiguous).
 * Returns NULL and fills err on failure. */
void *oracle_plan_create(int double_precision, int direction, int normalization, unsigned rank,
                         const uint64_t *lengths, uint64_t batch, char *err, size_t cap);
/* in/out: interleaved complex host arrays of batch*prod(lengths) elements.
 * Returns 0 on success. The input is never modified. */
int oracle_plan_execute(void *plan, const void *in, void *out, char *err, size_t cap);
void oracle_plan_destroy(void *plan);
uint64_t oracle_plan_scratch_bytes(const void *plan);
void oracle_set_threads(int n);
int oracle_max_threads(void);

#ifdef __cplusplus
}
#endif

#endif
