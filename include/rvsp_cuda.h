/*
 * rvsp_cuda.h -- the C ABI of the B200 SpGEMM backend.
 *
 * This is the boundary the reference's host C calls to reach the GPU: plain
 * pointers, sizes and status codes, no CUDA or C++ types. Each entry point
 * names the reference function or struct it replaces when the reference adds
 * RVSP_BACKEND_CUDA.
 *
 * Conventions
 *   - Return values are rvsp_status_t codes (0 = success).
 *   - Array arguments may be host or device pointers (device memory of the
 *     current CUDA device); residency is detected per pointer.
 *   - Index arrays are int32, values FP32, op counts int64, as in the
 *     reference (rv-sparse include/rv_sparse_types.h:53-67).
 *   - Inputs are canonical CSR, unchecked (rv-sparse
 *     src/kernels/spgemm/rvsp_spgemm.h:12-17), except in rvsp_cuda_csr_check.
 *   - A device-resident A may be a row panel of a larger CSR: row_ptr points
 *     at the panel's first row and need not start at 0; its offsets index
 *     col_idx and values directly (nnz arguments are then the end offset
 *     row_ptr[rows]). This is how products too large for one int32 C run.
 *   - A plan is not thread-safe; different plans are independent.
 */

#ifndef RVSP_CUDA_H
#define RVSP_CUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define RVSP_CUDA_API __attribute__((visibility("default")))
#else
#define RVSP_CUDA_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Opaque device-side state of one SpGEMM descriptor. */
typedef struct rvsp_cuda_plan *rvsp_cuda_plan_t;

/* Plan algorithms (values of rvsp_spgemm_algo_t). */
#define RVSP_CUDA_ALGO_EXACT 4
#define RVSP_CUDA_ALGO_LEARNED 5

/* Number of usable CUDA devices (0 when no driver or device). */
RVSP_CUDA_API int rvsp_cuda_device_count(void);

/* Text of the last CUDA error seen by this library on this thread. */
RVSP_CUDA_API const char *rvsp_cuda_last_error(void);

/* 1 if p is device (or managed) memory, 0 if host memory. */
RVSP_CUDA_API int rvsp_cuda_is_device_pointer(const void *p);

/* Frees arrays the one-shot path allocated on the device
 * (owns_data == RVSP_OWNS_DEVICE; rv-sparse src/core/matrix.c:99-104 frees
 * host arrays with free()). NULL is accepted. */
RVSP_CUDA_API void rvsp_cuda_free(void *device_ptr);

/* Releases a host array the library allocated for a result (owns_data ==
 * RVSP_OWNS_HOST; the counterpart of free() at rv-sparse
 * src/core/matrix.c:99-104). Such arrays may also be released with free();
 * through this call arrays of 64 MiB and more are kept (at most 4, within a
 * sixteenth of host memory, 32 GiB at most) and handed out again to later
 * products, whose copy-back then writes pages already mapped.
 * RVSP_HOST_CACHE=0 in the environment makes it a plain free(). NULL is
 * accepted.
 * Pageable host results of 64 MiB and more (and pageable operands of 16 MiB
 * and more) move through a ring of pinned 32 MiB pieces that host threads
 * fill or empty while the device copies the next ones; the threads are the
 * process's cores, 16 at most, or RVSP_HOST_COPY_THREADS (1: plain copies). */
RVSP_CUDA_API void rvsp_cuda_host_free(void *host_ptr);

/*
 * Plan lifecycle. Replaces the state of struct rvsp_spgemm_descr
 * (rv-sparse src/core/spgemm_descr.c:19-37) and its create/destroy
 * (spgemm_descr.c:66-100). The plan owns a CUDA stream, the analysed
 * structure on the device and the cached numeric CUDA graph.
 */
RVSP_CUDA_API int rvsp_cuda_plan_create(rvsp_cuda_plan_t *plan, int algo);
RVSP_CUDA_API void rvsp_cuda_plan_destroy(rvsp_cuda_plan_t plan);

/* When async is nonzero, calls whose outputs are all device-resident return
 * once the work is enqueued on the plan's stream instead of synchronising. */
RVSP_CUDA_API int rvsp_cuda_plan_set_async(rvsp_cuda_plan_t plan, int async);

/* The plan's cudaStream_t, as an opaque pointer (for event timing). */
RVSP_CUDA_API void *rvsp_cuda_plan_stream(rvsp_cuda_plan_t plan);

/*
 * Runtime bin parameters. The reference fixes its kernel tunables at compile
 * time (RVSP_CONTIG_MIN, rv-sparse src/kernels/spgemm/accum_contig_f32.c:18-19;
 * RVSP_GATHER_MIN, accum_adaptive_f32.c:28-29; RVSP_SORT_INSERTION_LIMIT,
 * rvsp_sort.h:17-18). Here the equivalent choices are per plan, as
 * RVSP_CUDA_BIN_PARAMS int32 values:
 *   [0] tiny_ops      rows with at most this many products run one thread
 *                     per row (0..32); the others get a warp
 *   [1] slack_shift   a warp row's hash table holds at least
 *                     ub + (ub >> slack_shift) slots, ub = min(products, cols(B))
 *                     (1..4: load factor at most 2/3, 4/5, 8/9, 16/17)
 *   [2] warp_cap_max  largest warp hash table, a power of two in 64..4096;
 *                     rows needing more are split into column chunks, a warp each
 *   [3] heavy_cw_log2 log2 of the columns of one chunk (9..13)
 * Defaults: 32, 2, 2048, 11. Results do not depend on the parameters (the
 * pattern and the values are bit-identical under every valid setting); only
 * the time does.
 *
 * set_params takes effect at the plan's next symbolic call and discards the
 * current analysis (numeric fails until symbolic runs again). The default
 * applies to plans created afterwards and to the one-shot and batched entry
 * points; NULL restores the built-in default. Out-of-range values return
 * RVSP_ERROR_INVALID_ARGUMENT.
 */
#define RVSP_CUDA_BIN_PARAMS 4
RVSP_CUDA_API int rvsp_cuda_plan_set_params(rvsp_cuda_plan_t plan, const int32_t *params, int32_t n);
RVSP_CUDA_API int rvsp_cuda_plan_get_params(rvsp_cuda_plan_t plan, int32_t *params, int32_t n);
RVSP_CUDA_API int rvsp_cuda_set_default_params(const int32_t *params, int32_t n);
RVSP_CUDA_API int rvsp_cuda_get_default_params(int32_t *params, int32_t n);

/*
 * Autotuner: symbolic analysis that first picks the plan's bin parameters
 * for this product. Coordinate descent over the candidates of each parameter
 * (warp_cap_max 1024/2048/4096, heavy_cw_log2 10..13 when the product has
 * chunked rows, slack_shift 1/2/3, tiny_ops 16/32), each trial timing
 * symbolic + a structure-filling numeric of the plan's own algorithm into
 * scratch memory, best of `reps` runs (>= 1). The best parameters stay in
 * the plan, which is left analysed with them exactly as after
 * rvsp_cuda_symbolic (same outputs). Operand values are needed for the
 * numeric trials. No reference counterpart (the reference has no runtime
 * tuning; its choice of strategy is rvsp_spgemm_descr_set_algo,
 * src/core/spgemm_descr.c:102-125).
 *   params_out      RVSP_CUDA_BIN_PARAMS values of the choice (may be NULL)
 *   trial_params    max_trials x RVSP_CUDA_BIN_PARAMS values tried (may be NULL)
 *   trial_ms        milliseconds of each trial (may be NULL)
 *   n_trials_out    trials run (may be NULL); at most max_trials are recorded
 */
RVSP_CUDA_API int rvsp_cuda_plan_autotune(rvsp_cuda_plan_t plan,
                       int32_t a_rows, int32_t a_cols, int32_t a_nnz,
                       const int32_t *a_row_ptr, const int32_t *a_col_idx, const float *a_values,
                       int32_t b_rows, int32_t b_cols, int32_t b_nnz,
                       const int32_t *b_row_ptr, const int32_t *b_col_idx, const float *b_values,
                       int32_t reps, int32_t *params_out, int32_t *trial_params,
                       float *trial_ms, int32_t max_trials, int32_t *n_trials_out,
                       int64_t *c_nnz_out, size_t *ws_bytes_out);

/*
 * Structure analysis. Replaces rvsp_symbolic_count
 * (rv-sparse src/kernels/spgemm/rvsp_symbolic.c:13-87) as called by
 * rvsp_spgemm_work_estimation (spgemm_descr.c:162-255): per-row op counts,
 * exact nnz per output row, exclusive prefix into C's row pointer, kept on
 * the device in the plan. Fails with RVSP_ERROR_ALLOCATION_FAILED when
 * nnz(C) exceeds INT32_MAX (rvsp_symbolic.c:69).
 * *ws_bytes_out is the device workspace compute needs.
 */
RVSP_CUDA_API int rvsp_cuda_symbolic(rvsp_cuda_plan_t plan,
                       int32_t a_rows, int32_t a_cols, int32_t a_nnz,
                       const int32_t *a_row_ptr, const int32_t *a_col_idx,
                       int32_t b_rows, int32_t b_cols, int32_t b_nnz,
                       const int32_t *b_row_ptr, const int32_t *b_col_idx,
                       int64_t *c_nnz_out, size_t *ws_bytes_out);

/*
 * Numeric phase on the analysed structure. Replaces, as driven by
 * rvsp_spgemm_compute (spgemm_descr.c:257-355): the row-pointer copy
 * (:325), rvsp_symbolic_fill (rvsp_symbolic.c:91-137) when fill_structure is
 * nonzero, and the numeric function RVSP_NUMERIC_FN
 * (rv-sparse src/kernels/spgemm/gustavson_core_f32.inc:18-64 with
 * accum_scalar_f32.c:20-71). With fill_structure == 0 the column indices in
 * c_col_idx are taken as the structure and only c_values are written.
 * workspace may be NULL or host memory (the plan then uses its own device
 * workspace) or device memory of at least the size symbolic reported.
 */
RVSP_CUDA_API int rvsp_cuda_numeric(rvsp_cuda_plan_t plan,
                      const int32_t *a_row_ptr, const int32_t *a_col_idx, const float *a_values,
                      const int32_t *b_row_ptr, const int32_t *b_col_idx, const float *b_values,
                      int32_t *c_row_ptr, int32_t *c_col_idx, float *c_values,
                      int fill_structure, void *workspace);

/* Per-row intermediate product counts of the last analysis.
 * Replaces rvsp_spgemm_get_op_counts (spgemm_descr.c:357-380). */
RVSP_CUDA_API int rvsp_cuda_op_counts(rvsp_cuda_plan_t plan, int64_t *op_counts_out, int32_t n);

/*
 * One-call product. Replaces the raw kernel rvsp_spgemm_scalar_f32
 * (RVSP_SPGEMM_PARAMS, rv-sparse src/kernels/spgemm/rvsp_spgemm.h:68-82;
 * gustavson_core_f32.inc:66-193): analysis, C allocation, fill, numeric.
 * C's arrays are allocated by the callee where the inputs live (device
 * inputs: device memory, release with rvsp_cuda_free; host inputs: host
 * memory, release with free(); arrays of 64 MiB and more are 2 MiB aligned
 * with transparent huge pages advised). op_counts_out is optional (a_rows
 * entries, host or device). algo is RVSP_CUDA_ALGO_EXACT or
 * RVSP_CUDA_ALGO_LEARNED.
 */
RVSP_CUDA_API int rvsp_cuda_spgemm_f32(int algo, int32_t a_rows, int32_t a_cols, int32_t b_cols,
                         const int32_t *a_row_ptr, const int32_t *a_col_idx,
                         const float *a_values,
                         const int32_t *b_row_ptr, const int32_t *b_col_idx,
                         const float *b_values,
                         int32_t **c_row_ptr_out, int32_t **c_col_idx_out,
                         float **c_values_out, int32_t *c_nnz_out, int64_t *op_counts_out);

/*
 * The reference's other dtypes, one call each. Replace its legacy raw kernels
 * rvsp_spgemm_csr_scalar_f64_raw and rvsp_spgemm_csr_scalar_i8_raw
 * (rv-sparse src/kernels/spgemm/legacy/csr_spgemm_kernels.h:80-94,156-170;
 * csr_scalar_f64.c:49-272, csr_scalar_i8.c:24-196), reached from
 * rvsp_spgemm_csr with FP64/FP64 or INT8/INT32 dtypes (spgemm.c:181-193).
 * Same semantics: per column acc += a * b in A-row order from zero (FP64
 * rounded to nearest without FMA; INT8 products and INT32 sums in two's
 * complement), columns ascending, and entries whose sum is exactly zero are
 * not stored, so *c_nnz_out can be below the symbolic count. Ownership and
 * residency as rvsp_cuda_spgemm_f32.
 */
RVSP_CUDA_API int rvsp_cuda_spgemm_f64(int32_t a_rows, int32_t a_cols, int32_t b_cols,
                         const int32_t *a_row_ptr, const int32_t *a_col_idx, const double *a_values,
                         const int32_t *b_row_ptr, const int32_t *b_col_idx, const double *b_values,
                         int32_t **c_row_ptr, int32_t **c_col_idx, double **c_values,
                         int32_t *c_nnz_out);
RVSP_CUDA_API int rvsp_cuda_spgemm_i8(int32_t a_rows, int32_t a_cols, int32_t b_cols,
                         const int32_t *a_row_ptr, const int32_t *a_col_idx, const int8_t *a_values,
                         const int32_t *b_row_ptr, const int32_t *b_col_idx, const int8_t *b_values,
                         int32_t **c_row_ptr, int32_t **c_col_idx, int32_t **c_values,
                         int32_t *c_nnz_out);

/*
 * COO -> canonical CSR on the device. Replaces the canonicalisation half of
 * the reference's Matrix Market loader assemble_csr_matrix (rv-sparse
 * tools/include/mtx_to_csr_formatter.h:12; tools/src/mtx_to_csr_formatter.c:
 * 219-330 with canonicalise_rows :74-151): with symmetric != 0 every
 * off-diagonal entry's mirror is appended after all stored entries; entries
 * are ordered by (row, column), stably, so repeated (row, column) entries
 * keep their COO order and are summed left to right from the first value;
 * columns ascending within a row. Indices are 0-based; coo_val may be NULL
 * (every value 1.0f, a "pattern" file). Inputs may be host or device memory;
 * outputs are allocated on the device when device_out is nonzero (release
 * with rvsp_cuda_free), with malloc otherwise. An index out of range returns
 * RVSP_ERROR_INVALID_ARGUMENT (the reference does not check).
 */
RVSP_CUDA_API int rvsp_cuda_coo_to_csr(int32_t rows, int32_t cols, int64_t n,
                         const int32_t *coo_row, const int32_t *coo_col, const float *coo_val,
                         int symmetric, int device_out, int32_t **row_ptr, int32_t **col_idx,
                         float **values, int32_t *nnz_out);

/*
 * Matrix Market files. rvsp_cuda_mtx_read is the parsing half of
 * assemble_csr_matrix (mtx_to_csr_formatter.c:153-217: banner "pattern" and
 * "symmetric", comment lines, "M N L", up to L 1-based entries read with the
 * same scanf formats) into malloc'd 0-based COO arrays; rvsp_cuda_mtx_to_csr
 * reads a file and canonicalises it with rvsp_cuda_coo_to_csr.
 */
RVSP_CUDA_API int rvsp_cuda_mtx_read(const char *path, int32_t *rows, int32_t *cols, int64_t *n,
                       int32_t **coo_row, int32_t **coo_col, float **coo_val, int *symmetric);
RVSP_CUDA_API int rvsp_cuda_mtx_to_csr(const char *path, int device_out, int32_t *rows,
                         int32_t *cols, int32_t *nnz, int32_t **row_ptr, int32_t **col_idx,
                         float **values);

/*
 * Canonical-CSR check on the device. Replaces rvsp_csr_check
 * (rv-sparse src/kernels/spgemm/rvsp_support.c:37-127) with the same result
 * codes (0 ok, 1 bad row_ptr, 2 column out of range, 3 unsorted,
 * 4 duplicate) and the lowest offending row in *bad_row_out (or -1).
 */
RVSP_CUDA_API int rvsp_cuda_csr_check(int32_t rows, int32_t cols, int32_t nnz,
                        const int32_t *row_ptr, const int32_t *col_idx,
                        int32_t *bad_row_out);

/*
 * Basic CSR validation of host or device arrays. Replaces the loops of
 * rvsp_csr_validate (rv-sparse src/core/matrix.c:51-90): row_ptr[rows] == nnz,
 * non-decreasing row offsets within [0, nnz], columns in range; sortedness
 * and duplicates are not checked. Returns RVSP_SUCCESS or
 * RVSP_ERROR_INVALID_CSR (or a null-pointer / argument error).
 */
RVSP_CUDA_API int rvsp_cuda_csr_validate(int32_t rows, int32_t cols, int32_t nnz,
                           const int32_t *row_ptr, const int32_t *col_idx);

/*
 * Batched products C_i = A_i * B_i, i < count, in one call (no counterpart
 * in the reference, whose callers loop over rvsp_spgemm_csr: each product is
 * what rv-sparse src/kernels/spgemm/gustavson_core_f32.inc:66-193 computes).
 * Sizes are host arrays [count]; operand arrays are host arrays [count] of
 * device pointers to whole CSR matrices (row_ptr[0] == 0; a row pointer that
 * does not start at 0 returns RVSP_ERROR_INVALID_CSR). The operands are
 * packed on the device into block-stacked matrices (A_i's columns shifted,
 * B_i's kept); consecutive products are grouped so every group's C fits an
 * int32 row pointer, and each group is multiplied as one product, so every
 * row of every product in it is binned and launched together. Each product's
 * own nnz must fit int32; their sum need not.
 * Output (device, callee-allocated, release each with rvsp_cuda_free):
 *   c_row_ptr_out  sum(a_rows[i] + 1) int32: C_i's row pointer (from 0) at
 *                  c_row_ptr + row_offsets_out[i] + i
 *   c_col_idx_out / c_values_out  C_i's entries (its own column indices) at
 *                  offsets [c_offsets_out[i], c_offsets_out[i + 1])
 *   c_nnz_out      total entries (int64)
 * row_offsets_out and c_offsets_out are host arrays [count + 1]: the rows
 * before product i and the entries before product i. algo is
 * RVSP_CUDA_ALGO_EXACT or RVSP_CUDA_ALGO_LEARNED.
 */
RVSP_CUDA_API int rvsp_cuda_spgemm_batched_f32(
    int algo, int32_t count, const int32_t *a_rows, const int32_t *a_cols, const int32_t *b_cols,
    const int32_t *a_nnz, const int32_t *b_nnz, const int32_t *const *a_row_ptr,
    const int32_t *const *a_col_idx, const float *const *a_values,
    const int32_t *const *b_row_ptr, const int32_t *const *b_col_idx,
    const float *const *b_values, int32_t **c_row_ptr_out, int32_t **c_col_idx_out,
    float **c_values_out, int64_t *c_nnz_out, int64_t *row_offsets_out,
    int64_t *c_offsets_out);

/* ------------------------------------------------------------------------
 * Learned row-size predictor (no counterpart in the reference).
 *
 * A 4-32-32-2 MLP over per-row features (A-row nnz, sum and max of the
 * referenced B-row lengths, column span) predicts each output row's nnz; the
 * learned path (RVSP_CUDA_ALGO_LEARNED) sizes hash tables and output slots
 * from it, sweeps the products once, and re-runs rows that outgrow their
 * prediction on the exact kernels, so results stay bit-identical.
 * A model is the float vector [mean(4), inv_std(4), z, params(1282)]
 * (RVSP_CUDA_MLP_FLOATS floats); a checkpoint file holds it with a magic,
 * version and checksum. The default checkpoint is $RVSP_MLP_WEIGHTS or
 * weights/row_mlp_v1.bin beside the library's directory.
 * ------------------------------------------------------------------------ */
#define RVSP_CUDA_MLP_PARAMS 1282
#define RVSP_CUDA_MLP_FLOATS 1291

/* 1 when a model is loaded (the default checkpoint is tried once). */
RVSP_CUDA_API int rvsp_cuda_learned_available(void);
RVSP_CUDA_API int rvsp_cuda_mlp_load(const char *path);
RVSP_CUDA_API int rvsp_cuda_mlp_set(const float *model, int32_t nfloats);
RVSP_CUDA_API int rvsp_cuda_mlp_get(float *model_out, int32_t nfloats);
RVSP_CUDA_API int rvsp_cuda_mlp_save(const char *path, const float *model, int32_t nfloats);

/* Mean loss and its gradient over n samples on the GPU (the training
 * kernel's forward/backward pass, one batch). X is [n][4] normalised
 * features, y = log2(1 + nnz), w optional per-sample weights. */
RVSP_CUDA_API int rvsp_cuda_mlp_grad(const float *params, const float *X, const float *y,
                                     const float *w, int32_t n, float *loss_out,
                                     float *grad_out);

/* Adam training on the GPU, params updated in place (host arrays).
 * epoch_loss_out (optional) gets the mean batch loss of every epoch. */
RVSP_CUDA_API int rvsp_cuda_mlp_train(float *params, const float *X, const float *y,
                                      const float *w, int32_t n, int32_t epochs, int32_t batch,
                                      float lr, uint64_t seed, float *epoch_loss_out);

/* Inference kernel on raw features [n][4]: mu, sigma and the capacity
 * ceil(2^(mu + z sigma) - 1) clamped to [1, ub] (0 when ub <= 0). */
RVSP_CUDA_API int rvsp_cuda_mlp_infer(const float *model, int32_t nfloats, const float *feat,
                                      const int32_t *ub, int32_t n, float *mu_out,
                                      float *sigma_out, int32_t *cap_out);

/* Analysis of this plan also records the per-row model features. */
RVSP_CUDA_API int rvsp_cuda_plan_collect_features(rvsp_cuda_plan_t plan, int on);

/* Per-row features [n][4], exact output counts and upper bounds
 * min(products, cols(B)) of the last analysis (any pointer may be NULL). */
RVSP_CUDA_API int rvsp_cuda_plan_row_stats(rvsp_cuda_plan_t plan, float *feat_out,
                                           int32_t *cnt_out, int32_t *ub_out, int32_t n);

/* Learned-path statistics of the last analysis (n >= 7): [0] rows sized by
 * the prediction (where it gives a smaller table than the upper bound),
 * [1] of those, rows that outgrew it, [2] rows too large for a table (exact
 * path), [3] sum of the counts, [4] sum of the predicted capacities and
 * [6] sum of the upper bounds of predicted rows that fit, [5] rows finished
 * by the exact path, and (n >= 8) [7] rows sized by the prediction whose
 * exact count exceeds the predicted capacity: the misprediction count, and
 * (n >= 10) [8] entries of heavy rows placed in the shared overflow pool
 * and [9] that pool's capacity. In the one-shot product heavy rows are
 * sized by the prediction too; a heavy row counts in [1] only when some of
 * its chunks found room neither in its slot nor in the pool (it is filled
 * again), in [7] whenever its count passes its capacity. In the descriptor's
 * count a row whose hash table still held it needs no re-run.
 * No reference counterpart (the reference has no learned sizing). */
RVSP_CUDA_API int rvsp_cuda_plan_learned_stats(rvsp_cuda_plan_t plan, int64_t *out, int32_t n);

/* The same statistics for the calling thread's last learned one-shot product
 * (rvsp_cuda_spgemm_f32 with RVSP_CUDA_ALGO_LEARNED); RVSP_ERROR_INVALID_ARGUMENT
 * before the first one. No reference counterpart. */
RVSP_CUDA_API int rvsp_cuda_oneshot_learned_stats(int64_t *out, int32_t n);

/*
 * Allocation-free row pointer of C from per-row counts. No counterpart in the
 * reference: this entry point exists for callers that cannot allocate device
 * memory where they need the prefix sum -- code recording a CUDA graph under
 * stream capture, latency-critical loops that cannot take the device-wide
 * synchronisation of cudaFree, hosts whose memory budget another allocator
 * owns. It calls no cudaMalloc/cudaFree: its scratch is a static ~32 KiB
 * device array held by every GPU that loads this library until exit.
 *
 * counts (n int32, device) -> row_ptr (n + 1 int32, device), exclusive prefix
 * sum with row_ptr[n] = total; the same values the plan path writes to C's
 * row pointer. n is limited to 8,388,608 rows (RVSP_ERROR_INVALID_ARGUMENT
 * beyond). counts must be non-negative (a negative count gives an undefined
 * row pointer). stream is a cudaStream_t (NULL: legacy default stream). With
 * total_out non-NULL the call synchronises the stream, stores the total and
 * returns RVSP_ERROR_ALLOCATION_FAILED when it exceeds INT32_MAX; with
 * total_out NULL it returns once the work is enqueued and an overflow is NOT
 * reported (row_ptr then holds wrapped offsets): pass total_out whenever the
 * total may pass INT32_MAX.
 * The first call on a device resolves the scratch array's address (once per
 * device, with that device current; again after cudaDeviceReset, in the new
 * context), so make it before any stream capture.
 * All calls on a device share the scratch: calls that overlap on the GPU race
 * and must be serialised by the caller.
 */
RVSP_CUDA_API int rvsp_cuda_row_ptr_noalloc(const int32_t *counts, int32_t n, int32_t *row_ptr,
                                            int64_t *total_out, void *stream);

/* Number of kernels this library has launched in this process (graph
 * replays count each kernel node), for launch accounting in benchmarks. */
RVSP_CUDA_API int64_t rvsp_cuda_launch_count(void);

/*
 * Device time of this library's kernels by family, for benchmarks and
 * profiling (no counterpart in the reference, whose bench times whole calls,
 * rv-sparse bench/bench.c:856-861). rvsp_cuda_kernel_timing(1) resets the
 * totals and starts timing: every later launch of a family records a CUDA
 * event pair on its plan's stream (graph replays are not timed);
 * rvsp_cuda_kernel_timing(0) stops. rvsp_cuda_kernel_times waits for the
 * recorded pairs and writes each family's total milliseconds (and launch
 * count, when launches_out is non-NULL); n must be at least
 * RVSP_CUDA_KERNEL_FAMILIES. rvsp_cuda_kernel_family(i) names family i
 * (NULL out of range).
 */
#define RVSP_CUDA_KERNEL_FAMILIES 14
RVSP_CUDA_API int rvsp_cuda_kernel_timing(int on);
RVSP_CUDA_API int rvsp_cuda_kernel_times(double *ms_out, int64_t *launches_out, int32_t n);
RVSP_CUDA_API const char *rvsp_cuda_kernel_family(int32_t i);

#ifdef __cplusplus
}
#endif

#endif /* RVSP_CUDA_H */
