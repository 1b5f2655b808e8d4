/* syclfft B200 device provider: C ABI v1.
 *
 * This is the drop-in boundary of the B200-native FFT provider for syclfft. It is
 * modelled on the reference's provider ABIs:
 *   - include/syclfft/detail/provider_abi.h:23-54 (C ABI v1 of the host/FFTW module:
 *     plan config struct, provider table {abi_version, name, create, destroy,
 *     execute}, exported getter) -- same shape, same error-buffer convention;
 *   - include/syclfft/detail/cufft_provider_abi.hpp:14-47 (C++ ABI v2 of the device
 *     module: config {double_precision, direction, placement, rank, lengths[3] in
 *     C order, batch_count}, table {supports, create, destroy, execute}) -- the
 *     device-provider semantics this module replaces, with the SYCL queue replaced
 *     by a CUDA device ordinal and the event list by a cudaStream_t.
 * Differences from cufft_provider_abi.hpp v2: the config also carries the
 * normalization (fused into the last kernel instead of the front end's extra
 * scaling pass, src/sycl/sycl.cpp:677-683) and the planning mode (measure runs the
 * autotuner, matching plan_options::planning, include/syclfft/common.hpp:66-72).
 *
 * Errors never cross the boundary as exceptions: functions write a NUL-terminated
 * message into `err` (capacity `cap`, 1024 bytes is what the front end passes, as
 * in include/syclfft/detail/provider_error_buffer.hpp:10-18) and return NULL / a
 * non-zero status. All pointers passed to execute are device (or managed)
 * allocations of interleaved complex<float> or complex<double> values.
 */
#ifndef SYCLFFT_B200_PROVIDER_H
#define SYCLFFT_B200_PROVIDER_H

#include <stddef.h>
#include <stdint.h>

#if defined(__cplusplus)
#define SYCLFFT_B200_EXTERN_C extern "C"
#else
#define SYCLFFT_B200_EXTERN_C
#endif
#define SYCLFFT_B200_EXPORT SYCLFFT_B200_EXTERN_C __attribute__((visibility("default")))

#define SYCLFFT_B200_PROVIDER_ABI_VERSION 1u

/* Same values as SYCLFFT_SCALAR_*_V1 and SYCLFFT_DIRECTION_*_V1 (provider_abi.h:41-46). */
#define SYCLFFT_B200_SCALAR_FLOAT 1u
#define SYCLFFT_B200_SCALAR_DOUBLE 2u
#define SYCLFFT_B200_DIRECTION_FORWARD (-1)
#define SYCLFFT_B200_DIRECTION_BACKWARD 1
/* syclfft::normalization order (common.hpp:44-50). */
#define SYCLFFT_B200_NORM_NONE 0u
#define SYCLFFT_B200_NORM_FORWARD 1u
#define SYCLFFT_B200_NORM_BACKWARD 2u
#define SYCLFFT_B200_NORM_ORTHOGONAL 3u

typedef struct syclfft_b200_plan_config_v1 {
    uint32_t abi_version;   /* SYCLFFT_B200_PROVIDER_ABI_VERSION */
    uint32_t scalar;        /* SYCLFFT_B200_SCALAR_FLOAT / _DOUBLE */
    int32_t direction;      /* -1 forward, +1 backward */
    uint32_t rank;          /* 1..3 */
    uint64_t lengths[3];    /* C order, last dimension contiguous */
    uint64_t batch_count;   /* contiguous batches of prod(lengths) elements */
    uint32_t in_place;      /* placement::in_place */
    uint32_t normalization; /* SYCLFFT_B200_NORM_* */
    uint32_t measure;       /* planning_mode::measure: autotune the kernel shapes */
    int32_t device;         /* CUDA device ordinal; -1 = the calling thread's current device */
} syclfft_b200_plan_config_v1;

typedef struct syclfft_b200_provider_v1 {
    uint32_t abi_version;
    const char *name;
    /* cufft_provider_v2::supports: 1 if the device can run this provider. */
    int (*supports)(int32_t device, char *err, size_t cap);
    /* cufft_provider_v2::create: builds tables and scratch on the device; NULL on failure. */
    void *(*create)(const syclfft_b200_plan_config_v1 *config, char *err, size_t cap);
    /* cufft_provider_v2::destroy: frees tables and scratch (waits for the plan's work). */
    void (*destroy)(void *plan);
    /* cufft_provider_v2::execute: enqueues the transform on `stream` (a cudaStream_t,
     * NULL = legacy default stream) and returns 0, or writes err and returns non-zero.
     * For in-place plans pass in == out. The input of an out-of-place plan is not
     * modified. Work is stream-ordered; the caller orders dependencies on the stream. */
    int (*execute)(void *plan, const void *in, void *out, void *stream, char *err, size_t cap);
    /* Plan-owned device scratch in bytes (plan<Scalar>::scratch_size_bytes). */
    uint64_t (*scratch_bytes)(const void *plan);
} syclfft_b200_provider_v1;

typedef const syclfft_b200_provider_v1 *(*syclfft_b200_get_provider_v1_fn)(void);

/* Module entry point, resolved with dlsym like syclfft_get_host_provider_v1
 * (provider_abi.h:54) and syclfft_get_cufft_provider_v2 (cufft_provider_abi.hpp:46-47). */
SYCLFFT_B200_EXPORT const syclfft_b200_provider_v1 *syclfft_b200_get_provider_v1(void);

/* ---- Diagnostics and measurement helpers (no reference counterpart; used by tests,
 *      the benchmark and the autotuner). ---- */

/* JSON description of the plan's passes (kernel kind, FFT length, radices, tile
 * shape, bytes moved). Returns the string length, or -1 if it did not fit. */
SYCLFFT_B200_EXPORT int syclfft_b200_describe_plan(const void *plan, char *buf, size_t cap);
/* Device memory the plan holds: its tables (twiddles, chirps, chirp spectra) and any scratch
 * it owns (plans made with SYCLFFT_B200_CREATE_STREAM_SCRATCH own none). 0 for a null plan. */
SYCLFFT_B200_EXPORT uint64_t syclfft_b200_plan_device_bytes(const void *plan);
/* Number of kernel launches one execute performs. */
SYCLFFT_B200_EXPORT int syclfft_b200_plan_launches(const void *plan);
/* Library version string. */
SYCLFFT_B200_EXPORT const char *syclfft_b200_version(void);
/* create with options (serving): SYCLFFT_B200_CREATE_STREAM_SCRATCH -- the plan owns no
 * scratch; each execute borrows a scratch arena of the executing stream (stream-ordered,
 * grown on demand), so many resident plans cost only their tables.
 * SYCLFFT_B200_CREATE_SYNC -- return only when the tables are on the device (create()
 * does this); without it, executes wait for the tables on the device and the host does not.
 * SYCLFFT_B200_CREATE_SPLIT_BF16 -- complex<float> plans only (ignored for double): axes whose
 * length has a tensor-core kernel (256 and 4096 points, contiguous lines; 256 on strided
 * axes) run their radix-16 butterflies as BF16 hi/lo matrix products with FP32 accumulation
 * on the tensor cores; all other passes, the twiddles and the exchanges stay FP32. Results
 * are within about 1e-5 relative L2 of the exact transform (see the error reports of the
 * tests); the reference has no counterpart (an extension of this provider). */
#define SYCLFFT_B200_CREATE_STREAM_SCRATCH 1u
#define SYCLFFT_B200_CREATE_SYNC 2u
#define SYCLFFT_B200_CREATE_SPLIT_BF16 4u
SYCLFFT_B200_EXPORT void *syclfft_b200_create_ex(const syclfft_b200_plan_config_v1 *config, uint32_t flags, char *err,
                                                 size_t cap);
/* Real transforms (no counterpart in the reference, whose v0.1 scope is complex-to-complex):
 * rank 1-3, batched, out of place, even last length N = lengths[rank-1] (numpy's rfftn /
 * irfftn layouts). R2C (direction -1): prod(lengths) reals per transform in,
 * prod(lengths[0..rank-2]) x (N/2 + 1) complex out; C2R (direction +1) the reverse, the
 * imaginary parts of bins 0 and N/2 of every last-axis line ignored. The last axis is a
 * complex FFT of length N/2 plus a pre- / post-process (fused into one pass where N/2 has a
 * size-specialised kernel); the outer axes are complex FFTs of the spectrum. Normalization as
 * for complex plans, relative to prod(lengths). The handle is used with the provider's
 * execute/destroy, execute_batch and execute_ex (normalization only), describe_plan and
 * plan_launches. */
#define SYCLFFT_B200_REAL_R2C 1
#define SYCLFFT_B200_REAL_C2R 2
SYCLFFT_B200_EXPORT void *syclfft_b200_create_real(const syclfft_b200_plan_config_v1 *config, int32_t kind,
                                                   uint32_t flags, char *err, size_t cap);
/* Strided ("advanced") layouts (no counterpart in the reference, whose v0.1 scope is contiguous
 * batches): element (b, i0, .., i_{rank-1}) of the input is read at
 * b * in_distance + sum_k i_k * in_strides[k] complex elements from the input pointer, and the
 * output written at the same formula with the out_ fields. Strides >= 1; distances >= 1 when
 * batch_count > 1; the output layout must not overlap itself; an in-place plan needs equal
 * input and output layouts. A side that is already contiguous and batch-major is read or
 * written directly; a strided side is gathered into / scattered from the plan's scratch by a
 * tiled pass. When both sides hold the batch as the innermost index of a dense array
 * (distance 1, stride of the last axis = batch_count: transforms down the columns of a
 * row-major matrix), the axis passes run on that array directly and execute_batch must run
 * the whole batch. Used with execute/destroy, execute_batch, execute_ex, describe_plan and
 * plan_launches like any plan. */
typedef struct syclfft_b200_layout_v1 {
    int64_t in_strides[3];
    int64_t in_distance;
    int64_t out_strides[3];
    int64_t out_distance;
} syclfft_b200_layout_v1;
SYCLFFT_B200_EXPORT void *syclfft_b200_create_strided(const syclfft_b200_plan_config_v1 *config,
                                                      const syclfft_b200_layout_v1 *layout, uint32_t flags,
                                                      char *err, size_t cap);
/* Like execute, for the first `batch` transforms only (1 <= batch <= the plan's
 * batch_count): a plan made for up to B transforms serves any smaller batch with the same
 * resident tables and scratch. */
SYCLFFT_B200_EXPORT int syclfft_b200_execute_batch(void *plan, const void *in, void *out, uint64_t batch,
                                                   void *stream, char *err, size_t cap);
/* Like execute_batch (batch 0 = the plan's batch count), in another direction and/or
 * normalization than the plan was made for: direction 0 = the plan's, -1 / +1;
 * normalization -1 = the plan's, else SYCLFFT_B200_NORM_*. The inverse is formed as
 * conj(F(conj x)), so one resident plan (tables, chirps, scratch) serves both directions. */
SYCLFFT_B200_EXPORT int syclfft_b200_execute_ex(void *plan, const void *in, void *out, uint64_t batch,
                                                int32_t direction, int32_t normalization, void *stream, char *err,
                                                size_t cap);
/* Status word of the plan's device work (no reference counterpart; the reference reports a
 * provider failure as a non-empty error buffer, turned into execution_failed by
 * src/sycl/sycl.cpp:671-676): 0 = healthy; 1 / 2 / 3 = a bounded wait in one of the plan's
 * kernels gave up (on a bulk copy, a tensor-core product or a tile copy), so the output of
 * that execution is incomplete. The word lives in page-locked host memory that the kernels
 * store to; read it once the execution has completed (event or stream synchronisation).
 * Reading does not synchronise the device. -1 for a null plan. */
SYCLFFT_B200_EXPORT int syclfft_b200_plan_status(const void *plan);
/* Like plan_status, and resets the word to 0: the front ends call it when an execution's
 * event completes and raise execution_failed for a non-zero value, once per failure. */
SYCLFFT_B200_EXPORT int syclfft_b200_plan_take_status(void *plan);
/* Failure-detection testing (no reference counterpart): the bounded waits in this plan's
 * kernels give up after `polls` polls -- 0 gives up at once, so every such wait of the next
 * execution fails and is reported in the status word; polls < 0 restores the default (2^26
 * polls, about a second). The environment variable SYCLFFT_B200_WAIT_POLLS, when set to a
 * number >= 0, is the limit of plans created while it is set. A copy or tensor-core product still in flight when a wait gives up
 * is waited for (bounded) before the block exits, so nothing writes its shared or tensor
 * memory afterwards. Returns 0, or -1 for a null plan. */
SYCLFFT_B200_EXPORT int syclfft_b200_plan_set_wait_limit(void *plan, int64_t polls);

/* ---- Page-locked host buffers (the reference accepts host USM in execute,
 *      src/sycl/sycl.cpp:72-85; here such buffers are streamed through the device). ----
 *
 * Runs `count` stages -- each a complex plan of contiguous layout, with a direction
 * (0 = the plan's, -1 / +1) and a normalization (-1 = the plan's, else SYCLFFT_B200_NORM_*) --
 * one after the other on `batch` transforms (0 = the first plan's batch count) read from the
 * page-locked host buffer `in` and written to the page-locked host buffer `out` (in == out
 * allowed). All stages have the same precision, transform size and device, and at least
 * `batch` transforms. The batch is cut into chunks (SYCLFFT_B200_HOST_CHUNK_MB, 64 by
 * default) that pass through device staging slots: copy in on an internal stream, the
 * stages on `stream`, copy out on another internal stream, so both copy directions and the
 * kernels overlap. Stream-ordered: the copies start after earlier work on `stream`, and
 * `stream` completes after the last copy out. Not capturable in a CUDA graph (refused).
 * Returns 0, or writes err and returns non-zero. Pageable (not page-locked) host memory is
 * refused. */
typedef struct syclfft_b200_host_stage_v1 {
    void *plan;
    int32_t direction;
    int32_t normalization;
} syclfft_b200_host_stage_v1;
SYCLFFT_B200_EXPORT int syclfft_b200_execute_host(const syclfft_b200_host_stage_v1 *stages, uint32_t count,
                                                  const void *in, void *out, uint64_t batch, void *stream, char *err,
                                                  size_t cap);

/* ---- Grouped execution (no reference counterpart): the serving path's batched launch. ----
 *
 * A group serves one length family: 1-D C2C transforms of length n and one precision over
 * contiguous lines. One execute runs many requests -- each with its own buffers, batch
 * count, direction and normalization -- in a single kernel launch (up to 192 requests per
 * launch; more are split). The request table is passed as kernel parameters, so executes
 * are stream-ordered, need no device staging and can be captured in a CUDA graph.
 * Available for the lengths of the size-specialised single-pass kernels
 * (syclfft_b200_group_supports). in == out is allowed per request. */
typedef struct syclfft_b200_group_item_v1 {
    const void *in;
    void *out;
    uint64_t batch;          /* lines of length n */
    int32_t direction;       /* -1 / +1 */
    uint32_t normalization;  /* SYCLFFT_B200_NORM_* */
} syclfft_b200_group_item_v1;

SYCLFFT_B200_EXPORT int syclfft_b200_group_supports(uint32_t scalar, uint64_t n);
SYCLFFT_B200_EXPORT void *syclfft_b200_group_create(uint32_t scalar, uint64_t n, int32_t device, char *err,
                                                    size_t cap);
SYCLFFT_B200_EXPORT int syclfft_b200_group_execute(void *group, const syclfft_b200_group_item_v1 *items,
                                                   uint32_t count, void *stream, char *err, size_t cap);
SYCLFFT_B200_EXPORT void syclfft_b200_group_destroy(void *group);

/* ---- Radix-family execution (no reference counterpart): one launch for requests of
 *      different lengths. ----
 *
 * A family is the power-of-two lengths whose single-pass kernels share one block shape:
 * complex<float> 64 .. 4096 and complex<double> 64 .. 2048 (syclfft_b200_family_supports).
 * One execute runs up to 256 requests per launch (more are split), each with its own length
 * of the family, buffers, batch, direction and normalization; requests are tiles of one kernel
 * launch that dispatches on each request's length. The request table is passed as kernel
 * parameters, so executes are stream-ordered, need no device staging and can be captured in a
 * CUDA graph. in == out is allowed per request; buffers aligned to the complex element. */
typedef struct syclfft_b200_family_item_v1 {
    const void *in;
    void *out;
    uint64_t n;              /* length: a power of two of the family */
    uint64_t batch;          /* lines of length n */
    int32_t direction;       /* -1 / +1 */
    uint32_t normalization;  /* SYCLFFT_B200_NORM_* */
} syclfft_b200_family_item_v1;

SYCLFFT_B200_EXPORT int syclfft_b200_family_supports(uint32_t scalar, uint64_t n);
SYCLFFT_B200_EXPORT void *syclfft_b200_family_create(uint32_t scalar, int32_t device, char *err, size_t cap);
SYCLFFT_B200_EXPORT int syclfft_b200_family_execute(void *family, const syclfft_b200_family_item_v1 *items,
                                                    uint32_t count, void *stream, char *err, size_t cap);
SYCLFFT_B200_EXPORT void syclfft_b200_family_destroy(void *family);

/* ---- Serving helpers (no reference counterpart): one call per admission round. ----
 *
 * syclfft_b200_execute_many runs `count` executes on `stream` in order, each like
 * syclfft_b200_execute_ex (plan, buffers, batch 0 = the plan's, direction 0 = the plan's,
 * normalization -1 = the plan's); it stops at the first failure and names its index in err.
 * syclfft_b200_fill_uniform writes `count` reals uniform in [-1, 1) into each item's buffer,
 * value i a function of (seed, i) only (SplitMix64 output function), in one launch per 256
 * items. Both return 0, or write err and return non-zero. */
typedef struct syclfft_b200_exec_item_v1 {
    void *plan;
    const void *in;
    void *out;
    uint64_t batch;
    int32_t direction;
    int32_t normalization;
} syclfft_b200_exec_item_v1;

typedef struct syclfft_b200_fill_item_v1 {
    void *data;
    uint64_t count;  /* reals */
    uint64_t seed;
    uint32_t scalar; /* SYCLFFT_B200_SCALAR_FLOAT / _DOUBLE */
    uint32_t reserved;
} syclfft_b200_fill_item_v1;

SYCLFFT_B200_EXPORT int syclfft_b200_execute_many(const syclfft_b200_exec_item_v1 *items, uint32_t count, void *stream,
                                                  char *err, size_t cap);
/* Release the scratch arena that plans made with SYCLFFT_B200_CREATE_STREAM_SCRATCH borrowed
 * on `stream` of `device` (freed in stream order, after the work already on the stream); the
 * next such execute on the stream allocates a new one. Call before destroying a stream that ran
 * stream-scratch plans: arenas are kept per stream and are otherwise held until exit. */
SYCLFFT_B200_EXPORT void syclfft_b200_release_stream_scratch(void *stream, int32_t device);
SYCLFFT_B200_EXPORT int syclfft_b200_fill_uniform(const syclfft_b200_fill_item_v1 *items, uint32_t count,
                                                  void *stream, char *err, size_t cap);

/* ---- Transform without device allocation (no counterpart in the reference). ----
 *
 * For callers that cannot allocate device memory at the point they need a transform:
 * a framework whose memory planner owns the device and hands out only planned buffers,
 * a real-time loop that must not call cudaMalloc (it may synchronize the device), or a
 * process whose free memory already belongs to its own pool. Plans allocate their
 * twiddle tables and four-step scratch; this call instead uses two fixed arrays in the
 * library's device memory (a 32 MiB scratch and a small twiddle table, held by every
 * GPU that loads the library until the process exits) and calls no allocator.
 *
 * Batched 1-D complex<float> C2C of power-of-two length n in [2^15, 2^20] over `batch`
 * contiguous lines, n * batch <= 4194304 (4 Mi) elements; larger sizes are rejected with
 * an error message. in == out (in place) is allowed; both must be 8-byte aligned (a
 * misaligned pointer is refused before anything is launched). direction -1 / +1,
 * normalization SYCLFFT_B200_NORM_*. Enqueued on `stream` (cudaStream_t, NULL = legacy
 * default stream); returns 0, or writes err and returns non-zero.
 * All calls share the arrays: calls that overlap on the GPU race and must be ordered by
 * the caller. The first call on a device looks up the arrays' device addresses and
 * should come before any stream capture (made during a capture it is refused, and a
 * later call retries). */
SYCLFFT_B200_EXPORT int syclfft_b200_execute_noalloc_c2c_f32(const void *in, void *out, uint64_t n, uint64_t batch,
                                                             int32_t direction, uint32_t normalization,
                                                             void *stream, char *err, size_t cap);

#endif /* SYCLFFT_B200_PROVIDER_H */
