/*
 * onefft_b200 — entry points added beside OneFFT's API (include/onefft.h) for device memory,
 * batches, uneven batches and error reporting. OneFFT has no counterpart for these: it is a
 * single-threaded CPU library whose callers parallelise over transforms themselves
 * (OneFFT include/onefft.h:36-44, tests/test_onefft.c:207-259); on the GPU the batch is the unit
 * of work, so it becomes part of the interface.
 *
 * Return codes: 0 success; -1 invalid size or allocation failure (as OneFFT); -2 invalid
 * argument (NULL, misaligned or overlapping device pointers, zero/huge counts); -(1000 + e) for a
 * CUDA runtime error e. On any error the output is left untouched unless the error came from the
 * device after the kernels started. onefft_last_error() describes the last error of the
 * calling thread.
 *
 * Streams are passed as `void *` holding a cudaStream_t (NULL = the legacy default stream), so
 * the header needs no CUDA include. Device entry points only enqueue work; they do not
 * synchronise. They use the CUDA device current in the calling thread, which must be the
 * device the plan was created on.
 */
#ifndef ONEFFT_CUDA_H
#define ONEFFT_CUDA_H

#include <stddef.h>
#include <stdint.h>

#include "onefft.h"

#ifdef __cplusplus
extern "C" {
#endif

#define ONEFFT_ERR_SIZE (-1)
#define ONEFFT_ERR_ARG (-2)
#define ONEFFT_ERR_CUDA_BASE (-1000)

/* ---- batched transforms on device memory ------------------------------------------------------
 * Counterpart of calling OneFFT's onefft_plan_forward/_inverse (src/onefft.c:1138-1140) `batch`
 * times on consecutive transforms: transform b reads d_in + 2 n b and writes d_out + 2 n b.
 * d_in and d_out are device pointers aligned to 8 bytes (one complex64) that do not overlap. */
ONEFFT_API int onefft_dev_forward_batched(const onefft_plan *plan, const float *d_in, float *d_out, size_t batch, void *stream);
ONEFFT_API int onefft_dev_inverse_batched(const onefft_plan *plan, const float *d_in, float *d_out, size_t batch, void *stream);

/* The adjoint of the unnormalised forward transform, F^H = conj(F)^T, applied to `batch`
 * gradients: d_grad_in = F^H d_grad_out. Equal to the unnormalised inverse transform; used by
 * the torch autograd wrapper. Same pointer rules as above. */
ONEFFT_API int onefft_dev_adjoint_batched(const onefft_plan *plan, const float *d_grad_out, float *d_grad_in, size_t batch,
                               void *stream);

/* Transforms with pointwise complex weights applied inside the kernels that read the input and
 * write the output, so the weighting costs no extra pass over the data:
 *   d_out_b = d_post * T(d_pre * d_in_b)      for each of the `batch` transforms b,
 * T the plan's unnormalised forward (or inverse) transform, `*` elementwise complex products.
 * d_pre and d_post are device arrays of n interleaved complex values shared by the whole batch
 * (8-byte aligned, not overlapping d_out); either may be NULL (no weights on that side). Typical
 * uses: windows and phase ramps before the transform, filters or normalisation after it. Same
 * rules as onefft_dev_forward_batched otherwise; split-BF16 plans return ONEFFT_ERR_ARG. OneFFT
 * has no counterpart (its callers multiply in separate loops). */
ONEFFT_API int onefft_dev_forward_weighted(const onefft_plan *plan, const float *d_in, float *d_out, size_t batch,
                                           const float *d_pre, const float *d_post, void *stream);
ONEFFT_API int onefft_dev_inverse_weighted(const onefft_plan *plan, const float *d_in, float *d_out, size_t batch,
                                           const float *d_pre, const float *d_post, void *stream);

/* Loss and gradient of a weighted power spectrum in one pass over the data:
 *   *d_loss = sum over the batch and k of w[k]^2 |(F x_b)[k]|^2          (double, on the device)
 *   d_grad  = F^H (2 w^2 * F x_b) per transform (d loss / d conj(x), torch's convention; NULL =
 *             loss only)
 * with F the unnormalised forward transform of `plan` (FP32, 16 .. 2^14 points) and w a real
 * weight vector of n floats shared by the batch. Each block keeps its transforms on chip from
 * load to store: one read of x and one write of the gradient. The gradient equals the unfused
 * computation (forward, elementwise 2 w^2 y, onefft_dev_adjoint_batched) bit for bit; d_loss is
 * zeroed and accumulated by the call. OneFFT has no counterpart (it has no batch or loss API). */
ONEFFT_API int onefft_dev_weighted_power_loss(const onefft_plan *plan, const float *d_x, const float *d_w,
                                              float *d_grad, size_t batch, double *d_loss, void *stream);

/* ---- batched transforms on host memory ---------------------------------------------------------
 * Same as calling onefft_plan_forward/_inverse on `batch` consecutive transforms of host (or
 * device) buffers, but pipelined: chunks are copied in, transformed and copied out on several
 * streams so that both copy directions overlap the kernels. Pinned host memory gives full
 * overlap; pageable memory works but copies synchronously. Blocks until done. */
ONEFFT_API int onefft_plan_forward_batched(const onefft_plan *plan, const float *in, float *out, size_t batch);
ONEFFT_API int onefft_plan_inverse_batched(const onefft_plan *plan, const float *in, float *out, size_t batch);

/* ---- plans with an explicit pass split ---------------------------------------------------------
 * Creates a plan whose transform runs as `npass` kernels of lengths 2^log2_len[0..npass-1]
 * (product n). npass = 1 allows n <= 2^14; npass = 2 or 3 allow passes of 2^4 .. 2^12 each.
 * onefft_plan_create() picks the split from the tuned table; this form exists for tuning and for
 * tests that exercise every pass kernel at small sizes. NULL on an invalid split. */
ONEFFT_API onefft_plan *onefft_plan_create_split(size_t n, int npass, const int *log2_len);

/* As onefft_plan_create_split, also choosing each pass's tile width: 2^log2_cols[p] adjacent
 * columns per thread block (1 .. 4, at most 16384 values per tile; NULL = default widths). For
 * npass = 1 (n = 2^4 .. 2^14), log2_cols[0] is instead the number of whole transforms per block
 * (log2; the default 4096 / n, or half or twice that up to 8192 values; -1 or NULL = the tuned
 * choice); results are the same bit for bit whatever the choice.
 * `options` (ONEFFT_OPT_L2_KEEP: store the array between passes with L2 evict-last priority;
 * ONEFFT_OPT_TMA: stage each pass tile through one bulk tensor copy where the tile shape has
 * such a kernel and the buffers are 16-byte aligned), and, for three passes, log2_chunk > 0 to
 * run the first two passes chunk by chunk over 2^log2_chunk columns of the last digit so that
 * each chunk's intermediate values stay in L2 (0 = whole passes). */
/* npass = 1 at n = 2^12 or 2^13, log2_cols[0] = ONEFFT_COLS_PIPELINED: a persistent kernel with one
 * transform per block that brings the next transform in by one bulk copy while computing the
 * current one (for 16-byte aligned buffers; results equal the other widths bit for bit). */
#define ONEFFT_COLS_PIPELINED 15
#define ONEFFT_OPT_L2_KEEP 1
#define ONEFFT_OPT_TMA 2
/* ONEFFT_OPT_FUSED (three passes, log2_chunk > 0, with ONEFFT_OPT_TMA): the first two passes run
 * as ONE persistent kernel that takes their tiles chunk by chunk, pass 1 of a chunk as soon as
 * pass 0 of it is done, so the values between them are re-read from L2 rather than HBM; pass 1
 * trails pass 0 by ONEFFT_OPT_LAG(k) chunks (1 .. 15; default 1). Results equal the separate
 * passes bit for bit. */
#define ONEFFT_OPT_FUSED 4
#define ONEFFT_OPT_LAG(k) ((k) << 8)
ONEFFT_API onefft_plan *onefft_plan_create_tiles(size_t n, int npass, const int *log2_len, const int *log2_cols,
                                                 int options, int log2_chunk);

/* ---- split-BF16 tensor-core variant --------------------------------------------------------------
 * A plan whose radix-16 stages run as dense complex 16x16 matrix products on the tensor cores:
 * BF16 operands split into hi + lo parts, three-term products (hi hi + hi lo + lo hi) accumulated
 * in FP32; twiddles and the last radix-2/4/8 stage stay FP32. Same transforms, layouts, entry
 * points and batching as an FP32 plan. Its error is ~2^-17 per stage (about 100x the FP32
 * path's), so it is accepted only at sizes where it meets the FP32 path's error bound: with
 * require_accepted != 0 other sizes return NULL ("does not meet the FP32 error bound"); with 0
 * the plan is built anyway, for measurement. n must be a power of two in [16, 2^30]. No
 * counterpart in OneFFT. */
ONEFFT_API onefft_plan *onefft_plan_create_bf16x3(size_t n, int require_accepted);

/* As onefft_plan_create_bf16x3 with each FP32 value (data and DFT-16 constants) split into THREE
 * bf16 parts hi + mid + lo (24 significant bits) and the six product terms down to 2^-16
 * relative kept (hi hi; hi mid, mid hi; hi lo, lo hi, mid mid), twice the tensor-core products of
 * the three-term form; the terms dropped are ~2^-24, FP32's own rounding. Accepted (with
 * require_accepted != 0) only at sizes where it meets the FP32 path's error bound. No
 * counterpart in OneFFT. */
ONEFFT_API onefft_plan *onefft_plan_create_bf16x6(size_t n, int require_accepted);

/* Number of passes of a plan and their log2 lengths (up to 3 are written to log2_len). */
ONEFFT_API int onefft_plan_passes(const onefft_plan *plan, int *log2_len);

/* ---- uneven batches ----------------------------------------------------------------------------
 * Counterpart of a caller looping over OneFFT's onefft_plan_forward/_inverse with a different
 * plan per size (src/onefft.c:1138-1140): many transforms of different power-of-two sizes packed
 * in one buffer, run by ONE persistent kernel launch that pulls work from a device queue. The
 * counter reset and the launch form a CUDA graph built by onefft_uneven_create() and replayed by
 * each execute. Transform i has size 2^log2n (0 <= log2n <= 16), starts at complex offset
 * `offset` of both buffers, and runs forward (inverse = 0) or inverse (inverse = 1). Transforms
 * must not overlap each other. */
typedef struct onefft_desc {
    int32_t log2n;
    int32_t inverse;
    int64_t offset;
} onefft_desc;

typedef struct onefft_uneven onefft_uneven;

/* Validates the descriptors (host memory), copies them to the device sorted largest first,
 * builds the tables of every size used on the current device and the launch graph. Returns
 * NULL on invalid descriptors (reason in onefft_last_error()) or on allocation failure. */
ONEFFT_API onefft_uneven *onefft_uneven_create(const onefft_desc *desc, size_t count);
/* As onefft_uneven_create, with the in-block split of each size 2^13 .. 2^16 given explicitly:
 * split_choice[m] in 0 .. 2 for 13 <= m <= 16 (other entries ignored; the array has 17 entries;
 * NULL = the tuned choices onefft_uneven_create uses). Choice 0 is the plain path's split where it
 * has one. For the autotuner and tests. No counterpart in OneFFT. */
ONEFFT_API onefft_uneven *onefft_uneven_create_split(const onefft_desc *desc, size_t count, const int *split_choice);
/* NULL is allowed. */
ONEFFT_API void onefft_uneven_destroy(onefft_uneven *batch);
/* Complex values the descriptors span: max over i of offset + 2^log2n. */
ONEFFT_API size_t onefft_uneven_span(const onefft_uneven *batch);
/* Runs the whole batch from d_in to d_out (device buffers of at least onefft_uneven_span()
 * complex values, 8-byte aligned, not overlapping) on `stream`. The batch object holds the work
 * queue counters, so one batch object must not execute on two streams at once. */
ONEFFT_API int onefft_uneven_execute(onefft_uneven *batch, const float *d_in, float *d_out, void *stream);
/* As onefft_plan_status for a batch: the second pass of a transform of 2^13 .. 2^16 waits
 * (bounded) for its first pass, which other blocks run; if that wait ran out, the batch's output
 * is not valid. Returns 0, or ONEFFT_ERR_CUDA_BASE with the reason in onefft_last_error();
 * reading clears it. Call after synchronising the stream of the execute calls. */
ONEFFT_API int onefft_uneven_status(onefft_uneven *batch);

/* The same uneven batch with no device allocation at all, for callers that cannot let a library
 * call cudaMalloc: real-time threads that must not block in the allocator or hit out-of-memory
 * after start-up, and applications whose device memory all belongs to their own arena or
 * budget. It has no counterpart in OneFFT. Instead of a batch object it uses one fixed
 * 384 KiB __device__ array per GPU (held by every GPU that loads the library until the process
 * exits) for the twiddle tables of sizes 2^4 .. 2^16, the sorted descriptors and the work
 * queue. Limits: at most 4096 descriptors per call (more is rejected with -2 and a message in
 * onefft_last_error()), log2n <= 16, same buffer rules as onefft_uneven_execute(). The first
 * call on a device builds the tables there (a few small kernels, then a stream synchronize),
 * and so does the first call after that device's context was reset (cudaDeviceReset); make
 * such a call before any stream capture. Later calls only copy the descriptors in,
 * zero the queue counter and launch. Every call shares the array and overwrites it: calls
 * whose GPU work overlaps race, so issue them in order (for example on one stream). */
ONEFFT_API int onefft_uneven_execute_noalloc(const onefft_desc *desc, size_t count, const float *d_in, float *d_out,
                                             void *stream);

/* ---- column transforms (the local steps of a transform distributed over several GPUs) -------
 *
 * The transforms down the `cols` columns of a row-major n x cols matrix,
 *     Y_b[k] = sum_j in[j cols + b] w_n^(j k)          (0 <= b < cols, 0 <= k < n),
 * optionally multiplied by the four-step twiddle of a larger transform of N = big_n values,
 *     Y_b[k] *= w_N^((col0 + b) k),
 * and written row-wise, split into `blocks` blocks of n / blocks consecutive outputs:
 *     out[((k / r) cols + b) r + k mod r] = Y_b[k],    r = n / blocks.
 * With blocks = 1 column b's results are row b of a cols x n matrix. OneFFT has no counterpart:
 * these are the two local steps of the four-step transform of N = n1 n2 values over P ranks
 * (onefft_b200/distributed.py): (1) each rank's n1 x (n2 / P) column block with n = n1,
 * blocks = P, big_n = N, col0 = rank n2 / P writes the all-to-all send buffer directly; (2) the
 * received n2 x (n1 / P) matrix with n = n2 gives the rank's n1 / P rows of the result. The
 * twiddles follow OneFFT's rule (FP64, rounded once); swap flags give the inverse as
 * swap(F(swap(x))) across the two steps.
 *
 * Sizes: n a power of two in [16, 2^24] (one kernel up to 2^12, two beyond, with an n x cols
 * work buffer held by the object); cols a power of two >= 16 with n cols <= 2^31; blocks a power
 * of two <= n; big_n 0 (no factor) or a power of two in [n, 2^40] with col0 + cols <= big_n / n.
 * NULL / -1 for invalid sizes, as onefft_plan_create. */
typedef struct onefft_columns onefft_columns;
ONEFFT_API onefft_columns *onefft_columns_create(size_t n, size_t cols, size_t blocks, unsigned long long big_n,
                                                 unsigned long long col0);
ONEFFT_API void onefft_columns_destroy(onefft_columns *columns);
/* flags: ONEFFT_SWAP_IN exchanges re/im of the input as it is read, ONEFFT_SWAP_OUT of the
 * result as it is written (after the twiddle). d_in / d_out: n cols complex values each, 8-byte
 * aligned device pointers, not overlapping (16-byte aligned input lets the first pass stage its
 * tiles by bulk tensor copies; the results are the same bits either way). Enqueue only, like the
 * other device entry points. For n > 2^12 the object's work buffer holds the values between the
 * two passes: calls on one object whose GPU work overlaps (other streams, other threads) race on
 * it, so issue them in order on one stream or give each stream its own object. */
#define ONEFFT_SWAP_IN 1
#define ONEFFT_SWAP_OUT 2
ONEFFT_API int onefft_columns_execute(const onefft_columns *columns, const float *d_in, float *d_out, int flags,
                                      void *stream);
/* As onefft_plan_status, for a column transform: 0, or the error of a tile copy whose bounded
 * wait ran out since the last call (reading clears it); call after synchronising the stream. */
ONEFFT_API int onefft_columns_status(const onefft_columns *columns);

/* ---- information and testing hooks -------------------------------------------------------------*/

/* Message of the last error in the calling thread ("" if none). */
ONEFFT_API const char *onefft_last_error(void);

/* Errors that kernels of `plan` found while running, for callers of the device-pointer entry
 * points (which return as soon as the work is enqueued). The multi-pass kernels wait on their
 * tile copies with a bounded wait; a wait that runs out makes the kernel record it in the plan's
 * error word, leave its tile unwritten and return, so the output of that call is not valid.
 * Returns 0 if no such failure was recorded since the last call, else ONEFFT_ERR_CUDA_BASE with
 * the reason in onefft_last_error(); reading clears the word. Call it after synchronising the
 * streams the plan's transforms ran on. The host-pointer calls check the word themselves and
 * return the error (or leave `out` untouched) instead. Counterpart of OneFFT's error return
 * (include/onefft.h:73-75) for work that completes after the call returned. */
ONEFFT_API int onefft_plan_status(const onefft_plan *plan);

/* Test hook: make the k-th device allocation from now on fail (k >= 1), as if the device were
 * out of memory; 0 disarms. Used by the tests of the -1 / untouched-output contract. */
ONEFFT_API void onefft_debug_fail_alloc(int k);

/* Test hook: evaluates the library's FP64 twiddle rule on the current device and copies the
 * FP32-rounded values w_(2^log2n)^k, k = 0 .. count-1, to host memory `out` (2 count floats).
 * This is the rule every device table is built with (OneFFT src/onefft.c:112-141). */
ONEFFT_API int onefft_debug_twiddles(unsigned log2n, size_t count, float *out);

/* Number of kernel launches this process has issued through the library (all threads). */
ONEFFT_API unsigned long long onefft_debug_launch_count(void);

/* Test hook of the failure path above: while `on` is non-zero, the first bounded wait of every
 * tile of the multi-pass kernels on the current device counts as expired, without a real device
 * failure. Each tile then lets its copy land, records the failure and returns unwritten, so
 * host-pointer calls return an error with `out` untouched and onefft_plan_status() reports it.
 * Returns 0, or a CUDA error code. Device state: set it back to 0 before other work. */
ONEFFT_API int onefft_debug_expire_waits(int on);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* ONEFFT_CUDA_H */
