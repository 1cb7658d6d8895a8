/* zs_m31.h — C ABI of the B200 (sm_100a) backend for zig-stark's M31 DEEP-FRI
 * commitment path.
 *
 * Conventions follow zig-capi.h (the reference's only C ABI, for the Binius STARK):
 *   - byte buffers use the canonical wire format of docs/wire.md
 *     (src/core/serialization.zig:58-190): little-endian, QM31 = 16 bytes
 *     (a.c0 | a.c1 | b.c0 | b.c1), slices u64-length prefixed, usize = 8 bytes,
 *     optionals with a 1-byte presence flag;
 *   - buffers returned by the library are allocated with the caller's
 *     zs_host_allocator and released with zs_free (zig-capi.h:15-18);
 *   - input buffers are borrowed for the duration of the call;
 *   - return codes: 0 ok, -1 generic, -2 malformed input, -3 out of memory,
 *     -4 protocol error (zig-capi.h:20-21), and -5 device error.
 *
 * The prover, commitment and transform entry points run on the GPU, with no CPU
 * fallback: without a usable CUDA device they return -5. The verifier entry points
 * (zs_m31_verify, zs_m31_verify_batch) run on the host, as the reference's does.
 */
#ifndef ZS_M31_H
#define ZS_M31_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Host memory callbacks; the same layout as zs_host_allocator in zig-capi.h:35-39. */
typedef struct {
    void *ctx;
    void *(*alloc)(void *ctx, size_t size);
    void (*free)(void *ctx, void *ptr, size_t size);
} zs_host_allocator;

/* Compiled-in AIRs. A comptime Zig AIR type (src/m31/stark.zig:45-74) cannot cross
 * a C ABI, so the AIR is chosen by id; its PublicInputs struct is passed in wire form.
 *   ZS_AIR_FIB             FibAir, stark.zig:877-931            PI {claimed_fib: QM31}
 *   ZS_AIR_SEEDED_FIB      FibAir with public a_0, a_1          PI {a0, a1, claimed: QM31}
 *   ZS_AIR_RANGE_CHECK     RangeCheckAir, stark.zig:964-1041    PI {}
 *   ZS_AIR_AND_TABLE       AndTableAir, stark.zig:1048-1131     PI {}
 *   ZS_AIR_MULTIPLICITY    MultiplicityAir, stark.zig:1139-1216 PI {}
 *   ZS_AIR_RESCUE_EXAMPLE  examples/rescue (8 rows)             PI {initial: [4]QM31, final: [4]QM31}
 *   ZS_AIR_LINEAR_EXAMPLE  examples/ml_linear (8 rows)          PI {x: []QM31, claimed_y: QM31}
 *   ZS_AIR_RESCUE_STACKED  the rescue example's permutation, 8 rows each, stacked to
 *                          any 2^k >= 8 rows with square/cube helper columns (12
 *                          columns, degree 2(n-1) + n/8)    PI {initial: [4]QM31, final: [4]QM31}
 *   ZS_AIR_ML_LINEAR       examples/ml_linear widened to one linear layer y = W x, W
 *                          128 x 128: columns x_0..x_127, y_0..y_127, sel, mult; 128
 *                          preprocessed columns holding the input table; one LogUp
 *                          relation binding every input vector (sel = 1 rows) to a
 *                          table row (sel = 0 rows); sel = 0 on the last row
 *                                                           PI {w: []QM31, 16384 M31 values} */
enum {
    ZS_AIR_FIB = 0,
    ZS_AIR_SEEDED_FIB = 1,
    ZS_AIR_RANGE_CHECK = 2,
    ZS_AIR_AND_TABLE = 3,
    ZS_AIR_MULTIPLICITY = 4,
    ZS_AIR_RESCUE_EXAMPLE = 5,
    ZS_AIR_LINEAR_EXAMPLE = 6,
    ZS_AIR_RESCUE_STACKED = 7,
    ZS_AIR_ML_LINEAR = 8
};

/* ---- prover ------------------------------------------------------------------
 * Replaces GenericStark(Air).proveWithPreprocessed (src/m31/stark.zig:327-658) and
 * prove (stark.zig:303-311); the conventions are zs_binius_prove's (zig-capi.h:41-51).
 *   params         wire StarkParams {u8 trace_log, u8 log_blowup, usize num_queries,
 *                  u8 remainder_log} (stark.zig:75-90)
 *   public_inputs  wire Air.PublicInputs of `air_id`
 *   preprocessed   wire []const []const QM31 (empty buffer or a zero-length slice when
 *                  the AIR has none), trace: wire []const []const QM31
 *   channel_sep    the domain separator passed to Channel.init (channel.zig:16-21)
 * On success *out_proof / *out_len hold the serialized GenericStark(Air).Proof
 * (stark.zig:107-122), allocated with `host` and released with zs_free. The proof is
 * byte-identical to the reference prover's for the same inputs. Parameters the
 * reference asserts on (stark.zig:230-232, fri.zig:228) return -4; a domain above 2^26
 * points (trace_log + log_blowup > 26) or more than 2^24 queries returns -2. */
int32_t zs_m31_prove(zs_host_allocator host, uint32_t air_id, const uint8_t *params, size_t params_len,
                     const uint8_t *public_inputs, size_t public_inputs_len, const uint8_t *preprocessed,
                     size_t preprocessed_len, const uint8_t *trace, size_t trace_len, const uint8_t *channel_sep,
                     size_t channel_sep_len, uint8_t **out_proof, size_t *out_len);

/* ---- device contexts ---------------------------------------------------------
 * An explicit handle instead of process-global device state: a context binds one CUDA
 * device ordinal and a stream of its own. zs_m31_prove_ctx is zs_m31_prove run on the
 * context's device and stream; the caller's current device is restored on return.
 * Calls on one context run one at a time (a mutex); calls on distinct contexts run
 * concurrently, on one device or several. The reference keeps its one GPU context in a
 * lazy process global under a spin mutex (circlefft_gpu.zig:21-39).
 * zs_m31_ctx_create returns -5 when `device` is not a valid ordinal or no device is
 * present. zs_m31_prove (no context) runs on the calling thread's current device. */
typedef struct zs_m31_ctx zs_m31_ctx;
int32_t zs_m31_ctx_create(int32_t device, zs_m31_ctx **out);
void zs_m31_ctx_destroy(zs_m31_ctx *ctx);
int32_t zs_m31_ctx_device(const zs_m31_ctx *ctx);
int32_t zs_m31_prove_ctx(zs_m31_ctx *ctx, zs_host_allocator host, uint32_t air_id, const uint8_t *params,
                         size_t params_len, const uint8_t *public_inputs, size_t public_inputs_len,
                         const uint8_t *preprocessed, size_t preprocessed_len, const uint8_t *trace,
                         size_t trace_len, const uint8_t *channel_sep, size_t channel_sep_len,
                         uint8_t **out_proof, size_t *out_len);

/* ---- batched and served proving ---------------------------------------------
 * One proof job: the arguments of zs_m31_prove. */
typedef struct {
    uint32_t air_id;
    const uint8_t *params;
    size_t params_len;
    const uint8_t *public_inputs;
    size_t public_inputs_len;
    const uint8_t *preprocessed;
    size_t preprocessed_len;
    const uint8_t *trace;
    size_t trace_len;
    const uint8_t *channel_sep;
    size_t channel_sep_len;
} zs_m31_job;

/* A finished job: status 0 and a proof allocated with the caller's allocator
 * (release with zs_free), or a negative code; status 1 = still pending (poll). */
typedef struct {
    uint8_t *proof;
    size_t len;
    int32_t status;
} zs_m31_result;

/* Proves n_jobs independent traces with `concurrency` workers, each with its own
 * CUDA stream and transcript, so the device interleaves the proofs' kernels.
 * Admission keeps the estimated device footprint of the proofs in flight under
 * hbm_budget_bytes (0 = 70 % of the free device memory). results[i] is jobs[i]'s
 * proof, byte-identical to zs_m31_prove on the same job. No counterpart in the
 * reference (its prover is single-threaded and proves one trace per call). */
int32_t zs_m31_prove_batch(zs_host_allocator host, size_t n_jobs, const zs_m31_job *jobs, uint32_t concurrency,
                           uint64_t hbm_budget_bytes, zs_m31_result *results);

/* A proof server: requests are admitted as workers and device memory free up
 * (continuous batching), their device work overlaps, and each request's latency
 * (submit to done) is recorded. submit copies the job's buffers. poll returns the
 * result (status 1 while pending; wait != 0 blocks until done) and the latency in
 * milliseconds; a finished ticket is released by the poll that returns it. */
typedef struct zs_m31_server zs_m31_server;
int32_t zs_m31_server_create(uint32_t workers, uint64_t hbm_budget_bytes, zs_m31_server **out);
void zs_m31_server_destroy(zs_m31_server *server);
int32_t zs_m31_server_submit(zs_m31_server *server, const zs_m31_job *job, uint64_t *ticket);
int32_t zs_m31_server_poll(zs_m31_server *server, uint64_t ticket, int32_t wait, zs_host_allocator host,
                           zs_m31_result *result, double *latency_ms);

/* Replaces GenericStark(Air).verify (src/m31/stark.zig:660-784); conventions of
 * zs_binius_verify (zig-capi.h:53-63). Sets *out_ok to 1 when the proof verifies and
 * 0 otherwise; returns 0, or a negative code when the inputs cannot be parsed. Runs
 * on the host (the reference's verifier is a few hundred hashes per query). One
 * deliberate difference: the reference checks only the query reveals a proof carries
 * (stark.zig:713), so it accepts a proof whose reveal list is cut short; this verifier
 * requires one reveal per FRI query (honest proofs always carry that many). */
int32_t zs_m31_verify(zs_host_allocator host, uint32_t air_id, const uint8_t *params, size_t params_len,
                      const uint8_t *public_inputs, size_t public_inputs_len, const uint8_t *proof, size_t proof_len,
                      const uint8_t *channel_sep, size_t channel_sep_len, int *out_ok);

/* Many independent verifications (serving acceptance checks): jobs[i] is checked as
 * zs_m31_verify would check it, on `threads` host threads (0 = all hardware threads).
 * out_ok[i] = 1 when proof i verifies, 0 otherwise; statuses[i] = 0, or the negative
 * code zs_m31_verify would return for job i. Returns 0 unless the arguments themselves
 * are malformed. No counterpart in the reference (its verify checks one proof). */
typedef struct {
    uint32_t air_id;
    const uint8_t *params;
    size_t params_len;
    const uint8_t *public_inputs;
    size_t public_inputs_len;
    const uint8_t *proof;
    size_t proof_len;
    const uint8_t *channel_sep;
    size_t channel_sep_len;
} zs_m31_verify_job;
int32_t zs_m31_verify_batch(size_t n_jobs, const zs_m31_verify_job *jobs, uint32_t threads, int *out_ok,
                            int32_t *statuses);

/* The commitment path alone (stark.zig:397-414): each column (wire
 * []const []const QM31, 2^trace_log values each) is interpolated on H, evaluated on
 * D = FRI_OFFSET * <w_N> with N = 2^(trace_log + log_blowup) and committed as a
 * Merkle tree of hashQM31 leaves. Output: the roots as wire []Digest (u64 count,
 * then 32 bytes per column), allocated with `host`; the shape of zs_binius_commit
 * (zig-capi.h:65-71). */
int32_t zs_m31_commit_columns(zs_host_allocator host, uint8_t trace_log, uint8_t log_blowup, const uint8_t *columns,
                              size_t columns_len, uint8_t **out_roots, size_t *out_len);

/* ---- circle FFT -------------------------------------------------------------
 * Replaces src/cuda/circlefft_gpu.zig:46-108 circleFFT(allocator, coeffs, half_coset,
 * evals) and :111-175 circleIFFT(...), themselves GPU versions of
 * src/m31/ntt/circle.zig:195-246 / 272-346. The half coset is given by its offset
 * point, step point and log size (CircleCoset, coset.zig:10-14); the domain is
 * half_coset ++ conjugate, coefficients use the A-then-B layout, evaluations are in
 * natural domain order. n = 2^(log_half + 1) words, n_columns transforms in a row
 * (column c at offset c * n). Host buffers. Bit-identical to the CPU transform for
 * every size (the reference falls back to the CPU below 8 points; this does not). */
int32_t zs_m31_circle_fft(const uint32_t *coeffs, uint32_t n_columns, uint32_t offset_x, uint32_t offset_y,
                          uint32_t step_x, uint32_t step_y, uint32_t log_half, uint32_t *evals);
int32_t zs_m31_circle_ifft(const uint32_t *evals, uint32_t n_columns, uint32_t offset_x, uint32_t offset_y,
                           uint32_t step_x, uint32_t step_y, uint32_t log_half, uint32_t *coeffs);

/* ---- circle commit (the 64 x 2^20 LDE + Merkle + fold chain workload) --------
 * Composes reference primitives: per column circleIFFT on canonicHalf(log_rows),
 * zero-padding of A and B, circleFFT on canonicHalf(log_rows + log_blowup)
 * (ntt/circle.zig); row leaves hashM31s over all columns (m31/hash.zig:15-25) and a
 * Merkle tree (core/merkle/merkle.zig:17-45); the combination
 * g[r] = sum_c gamma_c * LDE_c[r]; then n_folds FRI folds of g on the fri.zig domains
 * of size 2^(log_rows + log_blowup) with the given fold challenges, each layer
 * committed with hashQM31 leaves before it is folded (fri.zig:195-220).
 *
 * A plan owns every device buffer of one configuration. Typical use:
 *   create -> set_challenges -> (upload | run_device)* -> results -> destroy. */
typedef struct zs_commit_plan zs_commit_plan;

int32_t zs_m31_commit_plan_create(uint32_t n_columns, uint32_t log_rows, uint32_t log_blowup, uint32_t n_folds,
                                  zs_commit_plan **out);
void zs_m31_commit_plan_destroy(zs_commit_plan *plan);
/* gammas: n_columns QM31 (4 words each); alphas: n_folds QM31. Host buffers. */
int32_t zs_m31_commit_plan_set_challenges(zs_commit_plan *plan, const uint32_t *gammas, const uint32_t *alphas);
/* Device pointer to the plan's own trace buffer (n_columns x 2^log_rows words,
 * column-major), for callers that fill it on the device. */
uint32_t *zs_m31_commit_plan_trace_buffer(zs_commit_plan *plan);
/* Copies a host trace into the plan's trace buffer (pinned or pageable memory) on `stream`. */
int32_t zs_m31_commit_plan_upload(zs_commit_plan *plan, const uint32_t *host_trace, void *stream);
/* Runs the whole workload on `stream` (a cudaStream_t; NULL = default stream) over a
 * device trace (NULL = the plan's own trace buffer). Asynchronous. */
int32_t zs_m31_commit_plan_run_device(zs_commit_plan *plan, const uint32_t *d_trace, void *stream);
/* The whole workload from a trace in pinned host memory (C x 2^log_rows words,
 * column-major): column groups are copied on a copy stream while the LDE of the groups
 * already on the device runs, then the rest of the step, all on `stream`. The trace
 * must stay valid and unchanged until the step has run. Asynchronous. */
int32_t zs_m31_commit_plan_run_host(zs_commit_plan *plan, const uint32_t *host_trace, void *stream);
/* Runs one phase of run_device: 0 = circle LDE of all columns, 1 = row-leaf Merkle
 * tree with the gamma combination and the layer-0 tree, 2 = the fold chain. Running
 * 0, 1, 2 in order equals one run_device call. */
int32_t zs_m31_commit_plan_run_phase(zs_commit_plan *plan, int32_t phase, const uint32_t *d_trace, void *stream);
/* Synchronizes `stream` and copies the LDE root (32 bytes), the n_folds layer roots
 * (32 bytes each) and the final layer (2^(log_rows+log_blowup-n_folds) QM31) to host
 * buffers; any pointer may be NULL. */
int32_t zs_m31_commit_plan_results(zs_commit_plan *plan, void *stream, uint8_t *lde_root, uint8_t *layer_roots,
                                   uint32_t *final_layer);
/* Copies the low-degree extension (n_columns x 2^(log_rows+log_blowup) words), or
 * fold layer `layer` (0 = the combination g; 2^(log_rows+log_blowup-layer) QM31) to host. */
int32_t zs_m31_commit_plan_copy_lde(zs_commit_plan *plan, uint32_t *host_out);
int32_t zs_m31_commit_plan_copy_layer(zs_commit_plan *plan, uint32_t layer, uint32_t *host_out);
/* Number of this library's kernel launches in one run_device call. */
uint32_t zs_m31_commit_plan_launches(const zs_commit_plan *plan);

/* One-shot host-buffer version: creates a plan, uploads, runs, copies the results. */
int32_t zs_m31_circle_commit(const uint32_t *trace, uint32_t n_columns, uint32_t log_rows, uint32_t log_blowup,
                             const uint32_t *gammas, const uint32_t *alphas, uint32_t n_folds, uint8_t *lde_root,
                             uint8_t *layer_roots, uint32_t *final_layer);

/* ---- allocation-free circle LDE --------------------------------------------
 * No counterpart in the reference. For callers that cannot call cudaMalloc (a plugin
 * whose host process reserves all device memory up front in its own arena, or a
 * latency-bound loop where an allocation may synchronize the device): the circle
 * low-degree extension of zs_m31_commit_plan's first phase, with the caller's device
 * buffers for input (n_columns x 2^log_rows words, column-major, natural order on
 * canonicHalf(log_rows)) and output (n_columns x 2^(log_rows+log_blowup) words), and
 * every other word it needs in one fixed 16 MiB device array inside the library.
 * It allocates nothing. Limit: 2*2^L + 2*2^(L+B) + n_columns*(2^L + 2^(L+B)) words
 * <= 2^22 (L = log_rows, B = log_blowup); larger requests return -2. All calls share
 * the array, so calls whose GPU work overlaps race. The first call on a device looks
 * up the array's address and, under CUDA's default lazy module loading, is also when
 * the driver loads this library's device code and backs the array with device memory:
 * make one small call on each device before reserving an arena of all free memory and
 * before any stream capture (or run with CUDA_MODULE_LOADING=EAGER); later calls
 * allocate nothing. The address is kept for the life of the process, so the entry
 * point must not be used after a cudaDeviceReset. Asynchronous on `stream` (a
 * cudaStream_t; NULL = default stream). */
int32_t zs_m31_circle_lde_noalloc(const uint32_t *d_in, uint32_t *d_out, uint32_t n_columns, uint32_t log_rows,
                                  uint32_t log_blowup, void *stream);

/* Release a buffer returned by the ABI (zig-capi.h:73-74). */
void zs_free(zs_host_allocator host, uint8_t *ptr, size_t len);

/* Version / configuration string (zig-capi.h:76-77). */
const char *zs_version(void);

#ifdef __cplusplus
}
#endif

#endif /* ZS_M31_H */
