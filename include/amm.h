/*
 * amm.h — C ABI of libamm: the power method for λ_max of C = A·Aᵀ on one B200 (sm_100a),
 * exact and by approximate matrix multiplication (AMM).
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and returns an int status
 * (AMM_OK = 0).  Device pointers are CUDA device addresses on the context's device; stream is
 * a cudaStream_t passed as void* (NULL = the legacy default stream).  All work is
 * stream-ordered on that stream.  Calls on one context are not thread-safe; distinct contexts
 * are independent.  The caller owns A, x0 and every output buffer; the context owns its
 * scratch (column statistics, CDFs, sampling states, per-CTA partial sums, traces).
 *
 * Matrix layout: A is m x n, column-major, leading dimension ld (elements), FP32 or BF16.
 * Column j is the contiguous run A + j*ld.  For the single-pass TMA kernels the columns must
 * start on 16-byte boundaries (ld*elem_size % 16 == 0, A 16-byte aligned) and m*elem_size
 * must be a multiple of 16; m <= 16384.
 *
 * The reference (Takuya-Okuyama/eigenvalueComputation_by_AMM) keeps everything in one
 * translation unit of C++ headers with no C interface; each function below names the
 * reference function it replaces (file:line in that repository).
 */
#ifndef AMM_H_
#define AMM_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------- */
enum amm_status {
  AMM_OK = 0,
  AMM_ERR_INVALID_ARGUMENT = 1, /* bad size, null pointer, c < 1, unknown method ...      */
  AMM_ERR_ALIGNMENT = 2,        /* A or ld not 16-byte aligned, m*elem_size % 16 != 0      */
  AMM_ERR_UNSUPPORTED = 3,      /* shape outside the kernels' range (m > 16384)            */
  AMM_ERR_NOT_READY = 4,        /* amm_set_matrix has not been called                      */
  AMM_ERR_DEGENERATE = 5,       /* sampling CDF total is 0 or not finite (all-zero A, NaN) */
  AMM_ERR_CUDA = 6,             /* a CUDA runtime call failed (see amm_last_cuda_error)   */
  AMM_ERR_DEVICE_TIMEOUT = 7,   /* a bounded device-side wait gave up                      */
  AMM_ERR_OUT_OF_MEMORY = 8,
  AMM_ERR_NO_DEVICE = 9
};

enum amm_dtype { AMM_F32 = 0, AMM_BF16 = 1 };

/* Sampling CDF precision.  AMM_CDF_F64 (default): FP64 prefix sum and FP64 target.
 * AMM_CDF_F32: FP32 CDF and FP32 target exactly as the reference's pick_index
 * (device_memory.h:516-545); the CDF array is the correctly rounded prefix sum unless the
 * caller imports one with amm_set_cdf (e.g. the reference's own CUB-built d_acc_weight). */
enum amm_cdf_precision { AMM_CDF_F64 = 0, AMM_CDF_F32 = 1 };

/* Power-method variants (the reference's -kernel names, host_memory.h:87-89,132-141). */
enum amm_method {
  AMM_METHOD_EXACT = 0,       /* powerMethod_by_exact       (powerMethod_by_exact.cuh:4-100)      */
  AMM_METHOD_PREVIOUS = 1,    /* powerMethod_by_previous    (powerMethod_by_previous.cuh:100-210) */
  AMM_METHOD_PROPOSED = 2,    /* powerMethod_by_proposed    (powerMethod_by_proposed.cuh:317-447) */
  AMM_METHOD_PROPOSED_V2 = 3  /* powerMethod_by_proposed_v2 (powerMethod_by_proposed_v2.cuh:199-377) */
};

/* Per-step kinds recorded in the trace. */
enum amm_step_kind {
  AMM_STEP_EXACT_MEMO = 0,   /* exact C·x, then [x_memo|y_memo] <- [x|y] (a VR step)      */
  AMM_STEP_EXACT = 1,        /* exact C·x, memo untouched                                  */
  AMM_STEP_PREVIOUS = 2,     /* previous AMM (norm-proportional sampling)                  */
  AMM_STEP_PROPOSED = 3      /* proposed AMM (centred sampling + rank-one correction)      */
};
/* amm_benchmark_product: time the set-up pass (not a step kind). */
#define AMM_PASS_SETUP 16

/* Parameters (the reference's host_memory fields, host_memory.h:26-50, plus n, ld, dtype). */
typedef struct amm_config {
  int64_t m;                     /* rows of A = size of C                                   */
  int64_t n;                     /* columns of A                                            */
  int64_t c;                     /* samples per AMM product (-c); 0 means n                 */
  int64_t step;                  /* iterations per power-method call (-step)                */
  int64_t vr_period;             /* periodic variance reduction (-vr); 0 = off              */
  double vr_adaptive_threshold;  /* adaptive VR when cos > 1 - threshold (-vr_adaptive)    */
  double tol;                    /* stop once |λ_i − λ_{i−1}| <= tol·|λ_i|; 0 = run all     */
  int32_t dtype;                 /* enum amm_dtype                                          */
  int32_t cdf_precision;         /* enum amm_cdf_precision                                  */
  int32_t sanity;                /* -sanity: with c == n, weights 1 and indices 0..n-1      */
  int32_t use_graph;             /* capture the iteration loop in a CUDA graph (default 1) */
} amm_config;

typedef struct amm_ctx amm_ctx;

/* Fill cfg with the reference's defaults (host_memory.h:26-50): step 10, no VR, FP32. */
void amm_config_default(amm_config *cfg);

/* Create a context on CUDA device `device` (replaces the device_memory constructor,
 * device_memory.h:172-276).  Allocates all scratch for the configured sizes. */
int amm_create(amm_ctx **out, const amm_config *cfg, int device);
/* Release a context (device_memory destructor, device_memory.h:278-314). */
int amm_destroy(amm_ctx *ctx);

/* Bind A (borrowed device pointer; it must outlive its use).  The one-pass set-up over A
 * runs on the stream of the first call that needs it (an AMM call or a statistics accessor;
 * exact calls never do): per-column mean α_j, ‖A_j‖, ‖A_j − α_j‖ in FP64 (get_norms,
 * device_memory.h:34-59), ‖α‖² (device_memory.h:335-336), z = A·α and v = z − ‖α‖²
 * (powerMethod_by_proposed.cuh:132-145), both sampling CDFs and the inverse-probability
 * weights (set_weights / InclusiveSum / update_weights, powerMethod_by_previous.cuh:9-44). */
int amm_set_matrix(amm_ctx *ctx, const void *dA, int64_t ld, void *stream);

/* xorshift32 sampling states (the reference's d_rnd).  count >= c. */
int amm_set_rng_state(amm_ctx *ctx, const uint32_t *d_states, int64_t count, void *stream);
int amm_get_rng_state(amm_ctx *ctx, uint32_t *d_states_out, int64_t count, void *stream);
/* States as the reference derives them from -seed: curandGenerate with the default
 * (XORWOW) generator seeded with seed + 1234 (set_internal_randomness,
 * device_memory.h:339-343); count values are generated (the reference uses m). */
int amm_seed_rng(amm_ctx *ctx, uint64_t seed, int64_t count, void *stream);
/* The same from position `offset` of that generator's sequence.  The reference drives ONE
 * generator through the whole run and re-seeding it does not rewind it: the states start
 * after the values write_data consumed (size² for a -matrixType matrix, none for -filepath). */
int amm_seed_rng_at(amm_ctx *ctx, uint64_t seed, uint64_t offset, int64_t count, void *stream);

/* Start vectors as the reference draws them: a context-owned default (XORWOW) cuRAND
 * generator re-seeded with `seed` (the reference seeds with 1234 + -seed, AMM.cu:85), and
 * one curandGenerateNormal(m, mean 0, sd 1) per call, continuing the sequence
 * (powerMethod_by_exact.cuh:32 and the same line in every driver). */
int amm_seed_start_vectors(amm_ctx *ctx, uint64_t seed);
/* The same from position `offset` (in the reference's main, after everything write_data and
 * set_internal_randomness drew from its one generator: size² + m or m values). */
int amm_seed_start_vectors_at(amm_ctx *ctx, uint64_t seed, uint64_t offset);
int amm_draw_start_vector(amm_ctx *ctx, float *d_x0, void *stream);

/* Replace the sampling CDF of one weighting (0 = ‖A_j‖², previous AMM; 1 = ‖A_j − α_j‖²,
 * proposed AMM) with a caller-supplied inclusive prefix sum of length n (FP32 when the
 * context uses AMM_CDF_F32, FP64 otherwise).  The weights w_j = total/(weight_j·c) are
 * rebuilt from it.  Used to feed the reference's own CUB-built CDF for bit-exact sampling. */
int amm_set_cdf(amm_ctx *ctx, int which, const void *d_cdf, void *stream);

/* Exact top eigenvector v* (FP64, length m) for the error column; NULL clears it
 * (the reference reads data/exact_eigenvector, device_memory.h:246-254). */
int amm_set_eigenvector(amm_ctx *ctx, const double *d_vstar, void *stream);

/* Run one power-method call of `method` from the raw start vector d_x0 (length m; it is
 * normalised first, common.h:156-183), cfg->step iterations (fewer if tol stops it).
 * Replaces powerMethod_by_exact / _previous / _proposed / _proposed_v2.  Asynchronous;
 * read the results with amm_get_trace / amm_get_vectors. */
int amm_power_method(amm_ctx *ctx, int method, const float *d_x0, void *stream);
int amm_power_exact(amm_ctx *ctx, const float *d_x0, void *stream);        /* powerMethod_by_exact.cuh:4-100 */
int amm_power_previous(amm_ctx *ctx, const float *d_x0, void *stream);     /* powerMethod_by_previous.cuh:100-210 */
int amm_power_proposed(amm_ctx *ctx, const float *d_x0, void *stream);     /* powerMethod_by_proposed.cuh:317-447 */
int amm_power_proposed_v2(amm_ctx *ctx, const float *d_x0, void *stream);  /* powerMethod_by_proposed_v2.cuh:199-377 */

/* Synchronise `stream` and copy the trace of the last call to HOST arrays of length
 * >= cfg->step (any may be NULL): λ_i = x_i·y_i, err_i = (y_i·v*)/‖y_i‖, cos_i = λ_i/‖y_i‖,
 * the step kind, the number of distinct columns read, and device timestamps in ns relative
 * to the start of the call.  *steps_run receives the number of completed steps. */
int amm_get_trace(amm_ctx *ctx, double *eigs, double *errs, double *coss, int32_t *kinds,
                  int64_t *distinct, double *t_ns, int64_t *steps_run, void *stream);

/* Copy the final iterate x (normalised) and the last product y into device buffers of
 * length m (either may be NULL). */
int amm_get_vectors(amm_ctx *ctx, float *d_x, float *d_y, void *stream);

/* One sampled product, the reference's square_of_A_by_previous / previousAMM_kernel1+2
 * (powerMethod_by_previous.cuh:7-98, core_previousAMM.cuh:4-263):
 *   y = y_memo + Σ_k w_{s_k}·A_{s_k}·(A_{s_k}ᵀ(x − x_memo)),
 * drawing c indices from the current states (which advance).  d_idx_out (optional,
 * length c) receives the sorted sampled indices. */
int amm_core_previousAMM(amm_ctx *ctx, const float *d_x, const float *d_x_memo,
                         const float *d_y_memo, float *d_y, uint32_t *d_idx_out, void *stream);
/* The proposed product (powerMethod_by_proposed.cuh:7-103, core_proposedAMM.cuh:17-313):
 *   y = y_memo + Σdx·v + (z·dx)·1 + Σ_k w_{s_k}·(A_{s_k} − α_{s_k})·((A_{s_k} − α_{s_k})ᵀdx). */
int amm_core_proposedAMM(amm_ctx *ctx, const float *d_x, const float *d_x_memo,
                         const float *d_y_memo, float *d_y, uint32_t *d_idx_out, void *stream);
/* The sampled product over a caller-supplied work list instead of the context's own draw:
 *   y = y_memo + Σ_k wm_k·A_{cols_k}·(A_{cols_k}ᵀ(x − x_memo))            (method previous)
 * and the proposed form with the rank-one terms (method proposed), where cols (count distinct
 * column indices, 1 <= count <= c) and wm (w_j times the multiplicity of column j) are device
 * arrays — the previousAMM_kernel1+2 / proposedAMM_kernel1+2 product
 * (core_previousAMM.cuh:163-174,225-232, core_proposedAMM.cuh:195-277) for picks made
 * elsewhere.  The sampling states are not touched.  An index outside [0, n) contributes
 * nothing and makes the next status read (amm_get_trace) return AMM_ERR_INVALID_ARGUMENT. */
int amm_core_list_product(amm_ctx *ctx, int method, const uint32_t *d_cols, const float *d_wm,
                          int64_t count, const float *d_x, const float *d_x_memo,
                          const float *d_y_memo, float *d_y, void *stream);
/* One rank's part of a previous-AMM product over a column-sharded matrix (the reference runs
 * on one GPU; its sampling and product are pick_index (device_memory.h:506-545) and
 * previousAMM_kernel1+2 (core_previousAMM.cuh:163-174,225-232)).  The context holds this
 * rank's n columns, which are global columns [col0, col0 + n) of a matrix with n_global
 * columns; d_cdf_global is the inclusive FP64 CDF of ‖A_j‖² over all n_global columns (the
 * same on every rank).  The c states d_states_in are advanced once into d_states_out (may
 * alias) and c picks drawn from the global CDF; of those that fall in this rank's columns,
 * column j enters with weight mult_j·total/(c·(cdf[j] − cdf[j−1])), and
 *   d_y = y_memo + Σ_j w_j·A_j·(A_jᵀ(x − x_memo))
 * over them.  Summing d_y over the ranks (all but one passing y_memo = NULL) gives the product
 * of the whole matrix: one all-reduce of m floats per step. */
int amm_shard_product(amm_ctx *ctx, const double *d_cdf_global, int64_t n_global, int64_t col0,
                      const uint32_t *d_states_in, uint32_t *d_states_out, const float *d_x,
                      const float *d_x_memo, const float *d_y_memo, float *d_y, void *stream);
/* Exact product y = A·(Aᵀ·x) (the two cublasSgemv of powerMethod_by_exact.cuh:37-53). */
int amm_exact_product(amm_ctx *ctx, const float *d_x, float *d_y, void *stream);

/* Rayleigh step on [x | y] (dotProduct_and_generate_x, common.h:89-154): writes
 * out3 = {x·y, (y·v*)/‖y‖, (x·y)/‖y‖} (device, FP64) and x <- y/‖y‖. */
int amm_rayleigh_normalize(amm_ctx *ctx, float *d_x, const float *d_y, double *d_out3,
                           void *stream);
/* x <- x/‖x‖ (normalize, common.h:156-183). */
int amm_normalize(amm_ctx *ctx, float *d_x, void *stream);

/* Per-column statistics from the set-up pass (device buffers of length n; any may be NULL),
 * z and v (length m), ‖α‖² (host). */
int amm_get_column_stats(amm_ctx *ctx, float *d_alpha, float *d_norm, float *d_normp,
                         float *d_z, float *d_v, double *alpha2, void *stream);
/* The CDF (length n, FP32 or FP64 per the context) and weights (FP32, length n) of one
 * weighting (0 = previous, 1 = proposed). */
int amm_get_sampling_tables(amm_ctx *ctx, int which, void *d_cdf, float *d_weights,
                            void *stream);
/* Draw c indices from the current states with weighting `which` without advancing them
 * (pick_index, device_memory.h:516-545) into d_idx (length c, in draw order). */
int amm_sample_indices(amm_ctx *ctx, int which, uint32_t *d_idx, void *stream);

/* Allocation-free draw and sort (no amm_ctx): advances the c xorshift32 states d_states_in into
 * d_states_out (may alias), draws one index per state from the inclusive CDF d_cdf (length n,
 * FP64 or FP32 per cdf_precision) as pick_index does (device_memory.h:506-545), and writes the
 * c indices in ascending order, repeats included, to d_idx_sorted (as the CUB SortKeys of
 * powerMethod_by_previous.cuh:63-70) and the number of distinct indices to the device int32
 * *d_distinct.  No counterpart in the reference: it exists for callers that may not allocate
 * device memory (a process whose device memory belongs to its own pool, or a loop where an
 * allocator call is not acceptable); it allocates nothing and works in a fixed 1 MiB static
 * device array, so n is limited to 262144 (larger n returns AMM_ERR_UNSUPPORTED).  The first
 * call on each device resolves that array's address and should come before any stream capture.
 * Calls that overlap in time on one device race on the array: serialise them. */
int amm_pick_sorted_noalloc(const uint32_t *d_states_in, uint32_t *d_states_out, int64_t c,
                            const void *d_cdf, int cdf_precision, int64_t n,
                            uint32_t *d_idx_sorted, int32_t *d_distinct, void *stream);

/* ---- Matrix sources of the reference's driver ----
 * amm_generate_matrix: the -matrixType generators of generate_matrix (device_memory.h:360-433):
 * "gaussian_<mean>_<std>", "lognormal_<mean>_<std>" or "uniform_<lo>_<hi>" values from a cuRAND
 * XORWOW generator seeded with `seed` fill the size x size FP32 matrix d_A (column-major,
 * ld = size, size·size even), the lower triangle is mirrored into the upper one and the
 * reference's diagonal offset is added (returned in *offset; the reported eigenvalue of the
 * driver is sqrt(λ) − offset, powerMethod_by_exact.cuh:83-84).  Same seed, same matrix as the
 * reference.  Synchronises the stream. */
int amm_generate_matrix(const char *type, int64_t size, uint64_t seed, float *d_A, float *offset,
                        void *stream);
/* amm_read_matrix_file: the -filepath loader (host_memory.h:143-159, device_memory.h:369-401):
 * a uint32 size header followed by size x size FP32 values; file row y lands at
 * h_A[y*size + x] of a zero-filled size x size host buffer (the reference's layout, so a
 * symmetric covariance file reads as itself).  With h_A NULL only *original_size is set. */
int amm_read_matrix_file(const char *path, float *h_A, int64_t size, int64_t *original_size);

/* ---- Batched λ_max for many independent FP32 matrices (no counterpart in the reference,
 * which solves one matrix per run, AMM.cu:74-95) ----
 * Block power iteration with nvec orthonormal vectors (1, 4 or 8) and Rayleigh–Ritz, all
 * matrices in one persistent launch (captured in a CUDA graph when use_graph is set).  Each A_b
 * is column-major FP32 with m <= 2048, ld % 4 == 0 and 16-byte alignment; rows m..ld-1 are
 * ignored.  The exact product per step is the one of powerMethod_by_exact.cuh:37-53; the
 * Rayleigh quotient generalises dotProduct_and_generate_x (common.h:103-153) to a block. */
typedef struct amm_batch amm_batch;

typedef struct amm_batch_matrix {
  const void *A;   /* device pointer, borrowed */
  int64_t ld;
  int64_t m;
  int64_t n;
} amm_batch_matrix;

typedef struct amm_batch_config {
  int32_t nvec;       /* block size: 1, 4 or 8                                          */
  int32_t rr_period;  /* Rayleigh–Ritz (and convergence test) every rr_period steps      */
  int64_t max_iter;   /* products per matrix at most                                     */
  double tol;         /* stop when ‖C·v − λ_max·v‖ <= tol·λ_max (v: the top Ritz vector)  */
  uint64_t seed;      /* start block (counter-based hash of seed, matrix, row, vector)    */
  int32_t use_graph;  /* replay the launch from a CUDA graph                             */
  int32_t tile_gc;    /* columns per group; 0 lets the autotuner choose; 8 (nvec = 8,     */
                      /* exact products only) is the tensor-core product: TF32 mma.sync   */
                      /* with a hi/lo split of A, X and AᵀX (about FP32 accuracy)          */
  int32_t c_divisor;  /* 0: exact products; k > 0: previous-AMM products with c = n/k      */
                      /* samples per step (n <= 8192, c <= 1024), drawn as pick_index does */
                      /* from a seeded xorshift32 state per sample, every run from the seed */
  int32_t cluster;    /* CTAs (a thread-block cluster) per matrix: 1, 2, 4, 8; 0 = autotune */
  int32_t wide;       /* two-launch plan for uneven batches (amm_batch_wide_plan): 0 = with */
                      /* an autotuned cluster size, kept if it times faster; 1 = whenever   */
                      /* the batch is uneven enough, untimed; -1 = never                    */
  int32_t vr_period;  /* AMM mode only: variance reduction as the reference's -vr            */
                      /* (powerMethod_by_previous.cuh:135-157) over a block: product p is   */
                      /* exact and memoised when (p + 1) % vr_period == 0, and so is the    */
                      /* last product; the others estimate C·X = Y_memo·S + Ĉ·(X − X_memo·S) */
                      /* with S = X_memoᵀX (for one vector, S = x_memo·x).  Convergence is  */
                      /* tested on exact products only.  0 = off                            */
} amm_batch_config;

void amm_batch_config_default(amm_batch_config *cfg);
/* Descriptors are copied; the matrices stay owned by the caller and must outlive the context. */
int amm_batch_create(amm_batch **out, const amm_batch_matrix *mats, int64_t count,
                     const amm_batch_config *cfg, int device);
int amm_batch_destroy(amm_batch *b);
/* offsets[count + 1]: first row of each matrix's vector in the packed vector output. */
int amm_batch_vector_offsets(amm_batch *b, int64_t *offsets);
/* One persistent launch over all matrices (largest first from a device queue).  d_lambda:
 * count x nvec Ritz values, descending (λ_max first); d_vectors: Σ m, the unit top Ritz vector
 * of each matrix; d_iters: products run per matrix (-1: rank-deficient block).  The first call
 * autotunes the tile shape (columns per group) on this batch. */
int amm_batch_run(amm_batch *b, double *d_lambda, float *d_vectors, int32_t *d_iters,
                  void *stream);
/* Rebind the batch to new matrices of the same shapes (same count, m and n per matrix; A and
 * ld may change), stream-ordered: later runs and gradients use them, while the tile choice,
 * the launch plan and any captured graph are kept.  No counterpart in the reference. */
int amm_batch_set_matrices(amm_batch *b, const amm_batch_matrix *mats, int64_t count,
                           void *stream);
/* The same computation with one launch per matrix (the comparison arm). */
int amm_batch_run_each(amm_batch *b, double *d_lambda, float *d_vectors, int32_t *d_iters,
                       void *stream);
/* Backward of λ_max: grad_b = scale_b · 2·v_b·(v_bᵀA_b), column-major with leading dimension
 * grad_ld[b]; grad_ptrs and grad_ld are host arrays of count entries (read before the call
 * returns), d_scale a device array of count factors or NULL.  Asynchronous on the stream. */
int amm_batch_grad(amm_batch *b, const float *d_vectors, void *const *grad_ptrs,
                   const int64_t *grad_ld, const float *d_scale, void *stream);
/* Parity record of the AMM mode (no counterpart in the reference; test aid): with d_cdf set,
 * each run writes every matrix's FP32 sampling CDF (its n_b entries at the matrix's column
 * offset, Σ n_b floats in all); with d_picks set, the raw picks of AMM product p < products of
 * matrix b, in draw order, at (Σ_{a<b} c_a)·products + p·c_b + k (exact products leave their
 * slots untouched).  NULL pointers stop recording.  The buffers must outlive the runs. */
int amm_batch_record(amm_batch *b, float *d_cdf, uint32_t *d_picks, int64_t products);
/* The tile shape the autotuner picked: block size, columns per group and CTAs per matrix
 * (cluster size; cluster_size may be NULL).  AMM_ERR_NOT_READY before the first run. */
int amm_batch_tile_choice(amm_batch *b, int32_t *nvec, int32_t *cols_per_group,
                          int32_t *cluster_size);
/* The launch plan the autotuner kept for uneven batches (cluster size autotuned only): when a
 * few matrices would each take longer on one cluster than the rest of the batch takes spread
 * over the GPU, a run is two launches.  The first takes those *count heaviest matrices on
 * clusters of *cluster_size CTAs (*ctas in all), the second is queued behind it as a
 * programmatic dependent launch on the SMs left, and both then share the rest of the batch.
 * *count = 0: one launch per run.  *ms: the plan's time in the autotuner (0 if not timed).
 * AMM_ERR_NOT_READY before the first run. */
int amm_batch_wide_plan(amm_batch *b, int32_t *count, int32_t *cluster_size, int32_t *ctas,
                        float *ms);

/* Measurement hook: time `reps` back-to-back launches of the fused product kernel for one
 * step kind (AMM_STEP_EXACT, AMM_STEP_PREVIOUS or AMM_STEP_PROPOSED) on the bound matrix,
 * with CUDA events on `stream`, from the start vector of the last call (ones before any
 * call).  AMM kinds draw one set of picks from the current states without advancing them.
 * AMM_PASS_SETUP times the set-up pass instead (column sums, sums of squares and z = A·α in
 * one read of A; it rewrites the same statistics each time).
 * *ms_per_launch receives the mean time per launch and *distinct the distinct columns read
 * per launch (n for an exact launch or the set-up pass).  Synchronises `stream`.  No counterpart in the
 * reference (its per-step timing is cudaEventElapsedTime around whole steps,
 * powerMethod_by_exact.cuh:60-64). */
int amm_benchmark_product(amm_ctx *ctx, int kind, int reps, float *ms_per_launch,
                          int64_t *distinct, void *stream);

/* ∂λ_max/∂A = 2·v·(vᵀA) for a unit vector v (length m), written to d_grad (m x n,
 * column-major, leading dimension ld_grad, FP32).  No counterpart in the reference. */
int amm_grad_lambda(amm_ctx *ctx, const float *d_v, float *d_grad, int64_t ld_grad,
                    void *stream);

/* Profiling aids (no counterpart in the reference, which has no device timeline):
 * amm_device_clock enqueues on `stream` a one-thread kernel that writes the device clock
 * (%globaltimer, ns) to *d_out; amm_get_step_clocks synchronises `stream` and copies the raw
 * device clock stamps of the last call to the HOST array out (cap >= steps_run + 1): [0] when
 * the call's first kernel finished, [i + 1] when step i finished.  *count receives how many
 * were written. */
int amm_device_clock(uint64_t *d_out, void *stream);
/* Failure-path check of the device-side waits (no counterpart in the reference, which has no
 * device-side error reporting): enqueues on `stream` a one-CTA kernel that waits on an mbarrier
 * that nothing arrives on and on a grid barrier one CTA short, each giving up after the
 * library's wait limit (2 s), and synchronises `stream`.  Returns AMM_ERR_DEVICE_TIMEOUT, the
 * status of a step kernel whose wait gave up, with the HOST array result3 = {mbarrier wait
 * completed, grid barrier completed, µs spent}; the status is cleared and the context stays
 * usable. */
int amm_probe_bounded_waits(amm_ctx *ctx, uint32_t *result3, void *stream);
int amm_get_step_clocks(amm_ctx *ctx, uint64_t *out, int64_t cap, int64_t *count, void *stream);

/* Launch geometry of the fused product kernel chosen for this context, 10 values:
 * {cluster size, rows per CTA, clusters, consumer threads, vector slots per thread,
 *  columns per stage, stages, stage bytes, shared memory bytes, work-list capacity}. */
int amm_get_geometry(amm_ctx *ctx, int32_t *out10);

/* Human-readable name of a status code; the last CUDA error string of this thread. */
const char *amm_status_string(int status);
const char *amm_last_cuda_error(void);
/* Number of this library's kernel launches so far in this process (all contexts). */
int64_t amm_kernel_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* AMM_H_ */
