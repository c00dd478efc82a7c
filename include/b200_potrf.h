/*
 * b200_potrf.h -- C ABI of the B200 batched Cholesky (potrf) library.
 *
 * The library factors SPD matrices A = L L^T on an NVIDIA B200 (sm_100a).
 * All buffers are device pointers owned by the caller (b2p_potrf_batched_host
 * alone takes host matrices); the library allocates no device memory on its
 * own and keeps no state between calls except read-only tables and its own
 * streams and events.  Every entry point returns an int status (B2P_OK on
 * success) and never aborts; b2p_status_string() and b2p_last_error()
 * describe failures.  Work is enqueued on the caller's stream (a cudaStream_t
 * passed as void*; NULL means the legacy default stream) and nothing
 * synchronises the host, so every device-buffer call can be captured in a
 * CUDA graph.
 *
 * Layout: a batch of `batch` matrices, each n x n, FP32, row-major and
 * contiguous (matrix b starts at element b*n*n).  The output holds L in the
 * lower triangle, a strictly positive diagonal and exact zeros above it.
 * The input is never written.
 *
 * Reference interface replaced (binga/gpumode_cholesky):
 *   custom_kernel(data) -> output   submission.py:4101-4268
 *   ref_kernel / output contract    reference/reference.py:129-188
 */
#ifndef B200_POTRF_H_
#define B200_POTRF_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define B2P_API __attribute__((visibility("default")))
#else
#define B2P_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define B2P_OK 0
#define B2P_ERR_INVALID_ARG 1   /* bad size, null pointer, misaligned buffer  */
#define B2P_ERR_UNSUPPORTED 2   /* mode/size combination not implemented      */
#define B2P_ERR_WORKSPACE 3     /* workspace missing or smaller than required */
#define B2P_ERR_CUDA 4          /* a CUDA runtime call or launch failed       */
#define B2P_ERR_TIMEOUT 5       /* a bounded device-side wait gave up         */

/* ---- precision modes ------------------------------------------------------ *
 * The diagonal tiles and the panel solves are FP32 in every mode (unless
 * B2P_FLAG_FP64_DIAG); the mode selects the arithmetic of the trailing
 * (Schur complement) updates.                                              */
#define B2P_MODE_FP32 0    /* plain FP32 end to end (SIMT FMA)                 */
#define B2P_MODE_TF32 1    /* trailing update on tcgen05 kind::tf32            */
#define B2P_MODE_BF16X3 2  /* trailing update as hi*hi+hi*lo+lo*hi BF16 on tcgen05 */
#define B2P_MODE_FP8 3     /* trailing update in per-tile scaled E4M3 (n>=16384) */
#define B2P_MODE_MASK 0xff
/* Flag OR-ed into the mode: for n > 128, factor and invert every 64 x 64
 * diagonal tile in FP64 (rounded to FP32 on store).  Flagged calls take the
 * blocked path (the fused, warp-specialized and split paths keep FP32
 * diagonal tiles); orders <= 128 ignore the flag.  No counterpart exists in
 * the reference.                                                             */
#define B2P_FLAG_FP64_DIAG 0x100
/* Flag OR-ed into a tensor mode: the pivot guard.  After the 64 x 64
 * diagonal block of each block column is factored, every pivot is checked
 * against the error the mixed update can carry:
 *     L_jj^2 > 2 (delta + s 2^-23) A_jj,
 * delta = 2^-16 for BF16x3 and 2^-10 for TF32 (operand rounding), s the
 * tensor-core accumulation steps so far (one FP32 ulp each).  A column with
 * a failing (or non-positive, or non-finite) pivot is recomputed with its
 * update in FP32 on the SIMT cores, from the FP32 factor already written, and
 * so is every later column of that matrix, so that from there on the matrix
 * is factored as by B2P_MODE_FP32.  No host synchronisation is involved.
 * The fused, warp-specialized and split paths (n % 64 == 0) honour it; the
 * blocked path ignores it.  The reference's analogue is the accurate retry
 * of its 256-order kernel when a pivot falls under 1e-2 of the input's
 * diagonal (submission.py:866-886, 1004-1031), which refactors the whole
 * matrix.                                                                    */
#define B2P_FLAG_GUARD 0x200

/* Library version as major*10000 + minor*100 + patch. */
B2P_API int b2p_version(void);

/* Static description of a status code. */
B2P_API const char* b2p_status_string(int status);

/* Detail message of the last failing call on this host thread ("" if none). */
B2P_API const char* b2p_last_error(void);

/* Bytes of device workspace b2p_potrf_batched needs (0 for n <= 128). */
B2P_API size_t b2p_potrf_workspace_size(int64_t batch, int64_t n, int mode);

/*
 * Batched dense factorization.  Replaces custom_kernel(data) -> output
 * (submission.py:4101-4268) for a contiguous FP32 (batch, n, n) CUDA tensor.
 *   a, l       device pointers, batch*n*n floats each, 16-byte aligned; must
 *              not overlap.
 *   mode       B2P_MODE_* optionally OR-ed with B2P_FLAG_FP64_DIAG.
 *   workspace  device scratch of at least b2p_potrf_workspace_size() bytes
 *              (may be NULL when that size is 0), 256-byte aligned.
 *   info       optional device int32[batch]: 0 on success, k+1 when the
 *              k-th pivot was not positive (cuSOLVER potrf convention).  A
 *              non-SPD matrix yields NaN from the failing column on.  -1
 *              marks a matrix whose tensor-core update gave up a bounded
 *              device-side wait (its output is then incomplete).
 *   stream     cudaStream_t (as void*).
 */
B2P_API int b2p_potrf_batched(const float* a, float* l, int64_t batch, int64_t n, int mode,
                      void* workspace, size_t workspace_bytes, int32_t* info,
                      void* stream);

/*
 * Algorithm selection for n > 128.  b2p_potrf_batched picks one from
 * (batch, n, mode) (B2P_PATH_AUTO); the _path variants force one, for tests
 * that cover every kernel family and for tuning:
 *   B2P_PATH_BLOCKED   right-looking, one launch per kernel and block column
 *                      (any n > 128, every mode);
 *   B2P_PATH_FUSED     left-looking, one CTA per matrix, two per SM
 *                      (tensor modes, n % 64 == 0, n <= 1024);
 *   B2P_PATH_FUSED_WS  the same, warp-specialized, one CTA per SM;
 *   B2P_PATH_SPLIT     left-looking over many CTAs per matrix, two launches
 *                      per block column (tensor modes, n % 64 == 0).
 * A path that does not support (n, mode) returns B2P_ERR_UNSUPPORTED, and
 * its workspace query returns 0.  n <= 128 ignores the path.  No
 * counterpart exists in the reference (its dispatcher hard-codes one route
 * per benchmark shape, submission.py:4111-4268).
 */
#define B2P_PATH_AUTO 0
#define B2P_PATH_BLOCKED 1
#define B2P_PATH_FUSED 2
#define B2P_PATH_FUSED_WS 3
#define B2P_PATH_SPLIT 4
B2P_API size_t b2p_potrf_path_workspace_size(int64_t batch, int64_t n, int mode, int path);
B2P_API int b2p_potrf_batched_path(const float* a, float* l, int64_t batch, int64_t n, int mode, int path,
                                   void* workspace, size_t workspace_bytes, int32_t* info, void* stream);

/*
 * b2p_potrf_batched_path with one more optional output: fp32_from, a device
 * int32[batch] receiving per matrix the first block column (0-based, 64
 * columns each) from which B2P_FLAG_GUARD recomputed the update in FP32, or
 * -1 when it recomputed none (always -1 without the flag, on the blocked
 * path and for n <= 128).  The same call as b2p_potrf_batched_path
 * otherwise; the workspace query is b2p_potrf_path_workspace_size.
 */
B2P_API int b2p_potrf_batched_ex(const float* a, float* l, int64_t batch, int64_t n, int mode, int path,
                                 void* workspace, size_t workspace_bytes, int32_t* info, int32_t* fp32_from,
                                 void* stream);

/*
 * Host-resident batches: factors a (batch, n, n) FP32 batch held in HOST
 * memory into host memory.  The batch streams through the current device in
 * chunks of `chunk` matrices (0: the library's choice, about 32 MiB and at
 * least four chunks).  The copy in of chunk i+1 (a library stream), the
 * factorization of chunk i (b2p_potrf_batched on `stream`) and the copy out
 * of chunk i-1 (a second library stream) overlap, so a call costs about one
 * direction's PCIe transfer plus one chunk, not both directions in turn.
 *   host_a, host_l  host pointers, batch*n*n floats each, not overlapping;
 *              page-locked (cudaHostAlloc / cudaHostRegister) for the copies
 *              to overlap (pageable memory works, one copy at a time).
 *   workspace  device scratch of b2p_potrf_host_workspace_size() bytes,
 *              256-byte aligned: two input and two output chunk buffers
 *              plus the factorization's workspace for one chunk.
 *   info       optional DEVICE int32[batch], as for b2p_potrf_batched.
 * The call enqueues and returns: host_l holds L once `stream` has passed the
 * call (cudaStreamSynchronize or an event), and host_a, host_l and the
 * workspace must stay valid until then.  Every copy is ordered after the work
 * already on `stream`, and `stream` waits for every copy before its next
 * work.  Chunks use the same algorithm choice as b2p_potrf_batched for their
 * own batch size.  No counterpart exists in the reference: its inputs are
 * made on the device (reference/reference.py:37-55).
 */
B2P_API size_t b2p_potrf_host_workspace_size(int64_t batch, int64_t n, int mode, int64_t chunk);
B2P_API int b2p_potrf_batched_host(const float* host_a, float* host_l, int64_t batch, int64_t n, int mode,
                                   int64_t chunk, void* workspace, size_t workspace_bytes, int32_t* info,
                                   void* stream);

/*
 * Allocation-free variant of b2p_potrf_batched for callers that cannot
 * allocate device memory (code inside an allocator-free region, a plugin
 * whose host owns every device allocation, a serving process that forbids
 * allocation after start-up).  It takes no workspace: the scratch of the
 * blocked path lives in a 16 MiB device array inside this library, held by
 * every GPU that loads it until the process exits
 * (b2p_noalloc_scratch_bytes() reports the size).  A call whose workspace
 * (b2p_potrf_workspace_size) exceeds it is rejected with B2P_ERR_WORKSPACE,
 * and the message names the largest batch of that order and mode that fits.
 * For orders > 128 that is 1024 matrices in FP32, but the tensor modes keep
 * every panel's operand copy, 8192 (n/64) (n/64 - 1) bytes per matrix:
 * about 36 matrices of order 512, 8 of order 1024, and no single matrix
 * above order 2752.  Calls share the array: calls that overlap on
 * the GPU race, so serialise them on one stream.  The first call on each
 * device looks the array's address up (cudaGetSymbolAddress), and the first
 * call reaching the split or FP32 look-ahead paths creates their streams
 * and events; make those warm-up calls before any stream capture.  The
 * address is cached per device: do not call this again after
 * cudaDeviceReset.  No counterpart exists in the reference.
 */
B2P_API size_t b2p_noalloc_scratch_bytes(void);
B2P_API int b2p_potrf_batched_noalloc(const float* a, float* l, int64_t batch, int64_t n,
                                      int mode, int32_t* info, void* stream);

/*
 * Ragged batches: `count` matrices of individual order n_host[i] packed in
 * one buffer, matrix i starting at element offsets_host[i] (row-major,
 * contiguous n_i*n_i floats; offsets multiples of 4).  The output buffer uses
 * the same offsets.  Usage:
 *   b2p_ragged_plan_create   host-only: buckets the orders and precomputes
 *                            every launch.  tc_min_n (tensor modes; 0 =
 *                            default 129): matrices of at least this order
 *                            (and > 128) are copied into identity-padded
 *                            dense batches (order rounded up to the pad
 *                            step, one batch per padded order) and factored
 *                            on the dense tensor-core paths; smaller ones
 *                            take the blocked ragged schedule;
 *   b2p_ragged_plan_upload   copies the plan's tables (table_bytes, 16-byte
 *                            aligned device buffer) to the device; blocking;
 *   b2p_potrf_ragged         enqueues the factorization; reads only device
 *                            memory, so it can be captured in a CUDA graph;
 *                            workspace: b2p_ragged_plan_workspace_bytes (holds
 *                            the padded copies in tensor modes);
 *   b2p_ragged_plan_destroy.
 * info (optional, device int32[count]) follows b2p_potrf_batched.  No
 * counterpart exists in the reference (its dispatcher routes exact
 * (batch, n) shapes only, submission.py:4111-4268).
 */
typedef struct b2p_ragged_plan b2p_ragged_plan;
B2P_API int b2p_ragged_plan_create(const int64_t* offsets_host, const int32_t* n_host, int64_t count,
                                   int mode, int tc_min_n, b2p_ragged_plan** plan);
/*
 * Tuning knobs of the padded dense groups (tensor modes); zero fields take
 * the defaults.  b2p_ragged_plan_create(..., tc_min_n, ...) is
 * b2p_ragged_plan_create_ex with dense_min_n = tc_min_n and the rest zero.
 *   dense_min_n     as tc_min_n above (default 129)
 *   pad_step        padded-order granularity for orders <= 1024: 64, 128 or
 *                   256 (default 128); coarser steps make fewer, larger
 *                   groups at the cost of padding work
 *   pad_step_large  the same for orders > 1024 (default 128)
 *   large_path      path of the groups with padded order > 1024:
 *                   B2P_PATH_AUTO (= FUSED_WS up to 8192, SPLIT above),
 *                   B2P_PATH_FUSED_WS (clusters of CTAs per matrix, one
 *                   launch per group) or B2P_PATH_SPLIT
 *   streams         groups run on this many streams at once (1..8, default
 *                   4): the caller's stream and library-owned ones, forked
 *                   from and joined back into the caller's stream with
 *                   events (capturable); groups on the split path stay on
 *                   the caller's stream
 */
typedef struct b2p_ragged_options {
  int32_t dense_min_n;
  int32_t pad_step;
  int32_t pad_step_large;
  int32_t large_path;
  int32_t streams;
} b2p_ragged_options;
B2P_API int b2p_ragged_plan_create_ex(const int64_t* offsets_host, const int32_t* n_host, int64_t count,
                                      int mode, const b2p_ragged_options* options, b2p_ragged_plan** plan);
B2P_API void b2p_ragged_plan_destroy(b2p_ragged_plan* plan);
B2P_API size_t b2p_ragged_plan_table_bytes(const b2p_ragged_plan* plan);
B2P_API size_t b2p_ragged_plan_workspace_bytes(const b2p_ragged_plan* plan);
B2P_API int b2p_ragged_plan_upload(const b2p_ragged_plan* plan, void* tables, void* stream);
B2P_API int b2p_potrf_ragged(const b2p_ragged_plan* plan, const void* tables, const float* a, float* l,
                             void* workspace, size_t workspace_bytes, int32_t* info, void* stream);

/*
 * Cholesky adjoint: given L (output of the factorization) and Lbar = dLoss/dL
 * (lower triangle used), writes Abar = dLoss/dA, symmetric:
 *   P = Phi(L^T Lbar)  (lower triangle, diagonal halved)
 *   Abar = 1/2 (S + S^T),  S = L^{-T} P L^{-1}.
 * The products (L^{-1} by blocks, L^T Lbar, P L^{-1}, L^{-T} Z) run on the
 * tensor cores; mode is B2P_MODE_BF16X3 (default accuracy, ~1e-6 relative)
 * or B2P_MODE_TF32.  abar must not overlap l or lbar.
 * No counterpart exists in the reference (forward only); the oracle is
 * torch.linalg.cholesky's autograd and FP64 finite differences.
 */
B2P_API size_t b2p_potrf_backward_workspace_size(int64_t batch, int64_t n);
B2P_API int b2p_potrf_backward(const float* l, const float* lbar, float* abar, int64_t batch,
                               int64_t n, int mode, void* workspace, size_t workspace_bytes,
                               void* stream);

/*
 * Triangular solves with a batch of Cholesky factors (batch x n x n, lower,
 * row-major FP32, as b2p_potrf_batched writes them): x = L^{-1} b
 * (trans = 0) or x = L^{-T} b (trans = 1), b and x batch x n (x may alias b).
 * n <= 32768.  FP32 throughout.  Replaces the reference-side
 * torch.linalg.solve_triangular a Gaussian-process loss would call on the
 * factor; the reference itself stops at the factorization.
 */
B2P_API int b2p_trsv_batched(const float* l, const float* b, float* x, int64_t batch, int64_t n, int trans,
                             void* stream);

/*
 * Gaussian-process negative log-likelihood from the factor L of A = L L^T:
 *   b2p_gp_nll_forward:  alpha = L^{-1} y and
 *                        loss[b] = 1/2 alpha^T alpha + sum_i log L_ii
 *                        (the n/2 log 2pi constant omitted);
 *   b2p_gp_nll_backward: from alpha and gloss[b] = dOut/dloss[b]:
 *                        beta = L^{-T} alpha (= A^{-1} y; dOut/dy = gloss beta)
 *                        and Lbar = gloss (tril(-beta alpha^T) + diag(1/L_ii)),
 *                        the dOut/dL that b2p_potrf_backward maps to dOut/dA.
 * y, alpha, beta: batch x n; loss, gloss: batch; lbar: batch x n x n (written
 * whole, zeros above the diagonal).  n <= 32768.  No counterpart exists in
 * the reference (forward factorization only).
 */
B2P_API int b2p_gp_nll_forward(const float* l, const float* y, float* alpha, float* loss, int64_t batch,
                               int64_t n, void* stream);
B2P_API int b2p_gp_nll_backward(const float* l, const float* alpha, const float* gloss, float* beta,
                                float* lbar, int64_t batch, int64_t n, void* stream);

/*
 * Diagnostic: D[t] = A[t] * B[t]^T for `count` independent pairs of 128x64
 * FP32 tiles (row-major, K contiguous) through the library's tcgen05 staging
 * and MMA path; mode B2P_MODE_TF32 or B2P_MODE_BF16X3; err (device int32,
 * optional) receives B2P_ERR_TIMEOUT if a bounded wait gave up.  Used to
 * test the tensor-core path in isolation; no counterpart in the reference.
 */
B2P_API int b2p_debug_tc_gemm(const float* a, const float* b, float* d, int64_t count, int mode,
                              int32_t* err, void* stream);

/*
 * Diagnostic of the bounded-wait error path: b2p_debug_tc_gemm, where every
 * CTA, after its first pair's product is written, waits `stall_polls` polls
 * on an mbarrier that nothing arrives on.  The wait runs out, the kernel
 * writes B2P_ERR_TIMEOUT to err, releases its tensor memory and returns, and
 * the context stays usable (the pairs after each CTA's first are not
 * computed).  The same path ends every other bounded wait of the library;
 * this makes it testable without a fault.  stall_polls = 0 is
 * b2p_debug_tc_gemm.  No counterpart in the reference.
 */
B2P_API int b2p_debug_tc_gemm_stall(const float* a, const float* b, float* d, int64_t count, int mode,
                                    uint32_t stall_polls, int32_t* err, void* stream);

/*
 * Launch trace: when enabled, every kernel the library launches is bracketed
 * by a pair of CUDA events recorded on its launch stream, so a caller can
 * read per-kernel device time (the counterpart of the reference's in-kernel
 * clock64 phase profiler, submission.py:4711-4716,4991-4996).
 *   b2p_trace_enable(capacity)  start recording up to `capacity` launches
 *                               (0 stops recording and frees the events);
 *   b2p_trace_read(ids, ms, max) synchronises the recorded events and writes
 *                               kernel ids and durations; returns the count;
 *   b2p_trace_read_starts(t, max) each recorded launch's start, in ms after
 *                               the first recorded launch's (the launches'
 *                               own streams: a timeline of concurrent work);
 *   b2p_trace_read_units(u, max) the algorithmic work of each recorded
 *                               launch, in the same order: n^3/3 flops per
 *                               matrix for kernels that factor whole
 *                               matrices, 8 n^2 bytes per matrix for the
 *                               n <= 32 kernel, the product's flops for
 *                               update kernels, 0 where none is defined;
 *   b2p_kernel_name(id)         the kernel's name.
 */
B2P_API int b2p_trace_enable(int capacity);
B2P_API int b2p_trace_read(int32_t* kernel_ids, float* ms, int max_entries);
B2P_API int b2p_trace_read_starts(float* start_ms, int max_entries);
B2P_API int b2p_trace_read_units(double* units, int max_entries);
B2P_API const char* b2p_kernel_name(int id);

#ifdef __cplusplus
}
#endif

#endif /* B200_POTRF_H_ */
