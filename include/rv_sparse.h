/*
 * rv-sparse B200 backend: public API.
 *
 * The same entry points, argument meaning and status codes as the reference
 * API (rv-sparse include/rv_sparse.h:27-142). This build implements them on
 * the CUDA backend only:
 *
 *   - rvsp_spgemm_csr accepts RVSP_BACKEND_CUDA and RVSP_BACKEND_CUDA_LEARNED
 *     (options == NULL selects RVSP_BACKEND_CUDA). The reference's scalar
 *     backends (RVSP_BACKEND_SCALAR for FP32, FP64 and INT8 -> INT32,
 *     RVSP_BACKEND_SCALAR_UNROLL4 for FP32; rv-sparse src/core/spgemm.c:160-193)
 *     run on the CUDA exact path, whose results are bit-identical to theirs.
 *     RVSP_BACKEND_RVV_INTRINSICS returns RVSP_ERROR_UNSUPPORTED_BACKEND, as
 *     the reference does on a build without the vector extension.
 *   - the descriptor accepts RVSP_SPGEMM_ALGO_DEFAULT (the strategy a new
 *     descriptor starts with, rv-sparse src/core/spgemm_descr.c:83) and
 *     RVSP_SPGEMM_ALGO_CUDA, both the CUDA exact path, and
 *     RVSP_SPGEMM_ALGO_CUDA_LEARNED; the vector strategies return
 *     RVSP_ERROR_UNSUPPORTED_BACKEND (rv-sparse src/core/spgemm_descr.c:43-64).
 *
 * Residency: every array of A, B and C may live in host memory or in device
 * memory of the current CUDA device; the backend detects which per pointer.
 * Host inputs are staged to the device; host outputs are copied back before
 * the call returns. One-shot outputs are allocated where the inputs live
 * (host memory that free() releases and owns_data = RVSP_OWNS_HOST, or
 * device memory and owns_data = RVSP_OWNS_DEVICE); rvsp_csr_destroy frees
 * either.
 *
 * Results: C's structure (row_ptr, col_idx) is bit-exact against the
 * reference scalar kernel. Values are computed in the reference's order
 * (per output column, products a*b rounded to FP32 and added in A-row order
 * from +0.0f, no FMA contraction), so they are bit-exact too.
 */

#ifndef RV_SPARSE_H
#define RV_SPARSE_H

#include <stddef.h>

#include "rv_sparse_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define RVSP_VERSION_MAJOR 0
#define RVSP_VERSION_MINOR 1
#define RVSP_VERSION_PATCH 0

const char *rvsp_get_version(void);

const char *rvsp_status_to_string(rvsp_status_t status);

/* CSR lifecycle (rv-sparse src/core/matrix.c:18-115). create borrows the
 * arrays, validate checks row_ptr/column range (not sortedness), destroy
 * frees arrays the library allocated. */
rvsp_status_t rvsp_csr_create(rvsp_csr_matrix_t *A, int32_t rows, int32_t cols, int32_t nnz,
                              int32_t *row_ptr, int32_t *col_idx, void *values,
                              rvsp_dtype_t dtype);

rvsp_status_t rvsp_csr_validate(const rvsp_csr_matrix_t *A);

void rvsp_csr_destroy(rvsp_csr_matrix_t *A);

/* One-shot C = A * B (rv-sparse src/core/spgemm.c:135-211). Allocates C.
 * Inputs must be canonical CSR; they are checked once (on the device for
 * device-resident inputs) and RVSP_ERROR_INVALID_CSR is returned otherwise. */
rvsp_status_t rvsp_spgemm_csr(const rvsp_csr_matrix_t *A, const rvsp_csr_matrix_t *B,
                              rvsp_csr_matrix_t *C, const rvsp_spgemm_options_t *options);

/* Two-phase SpGEMM (rv-sparse src/core/spgemm_descr.c). */
rvsp_status_t rvsp_spgemm_descr_create(rvsp_spgemm_descr_t *descr);

void rvsp_spgemm_descr_destroy(rvsp_spgemm_descr_t descr);

rvsp_status_t rvsp_spgemm_set_algo(rvsp_spgemm_descr_t descr, rvsp_spgemm_algo_t algo);

/* Analyses A and B; reports the exact nnz of C and the workspace compute()
 * needs. The workspace may be host memory (the descriptor then keeps its own
 * device workspace) or device memory of at least workspace_bytes. */
rvsp_status_t rvsp_spgemm_work_estimation(rvsp_spgemm_descr_t descr,
                                          const rvsp_csr_matrix_t *A,
                                          const rvsp_csr_matrix_t *B,
                                          size_t *workspace_bytes, int32_t *c_nnz_out);

/* C = A * B on the analysed structure. When C->col_idx is the array the
 * previous compute filled (and invalidate_structure was not called), only the
 * values are recomputed; on device-resident operands that numeric-only pass
 * is replayed from a CUDA graph. */
rvsp_status_t rvsp_spgemm_compute(rvsp_spgemm_descr_t descr, const rvsp_csr_matrix_t *A,
                                  const rvsp_csr_matrix_t *B, rvsp_csr_matrix_t *C,
                                  void *workspace);

rvsp_status_t rvsp_spgemm_get_op_counts(rvsp_spgemm_descr_t descr, int64_t *op_counts_out,
                                        int32_t n);

void rvsp_spgemm_invalidate_structure(rvsp_spgemm_descr_t descr);

#ifdef __cplusplus
}
#endif

#endif /* RV_SPARSE_H */
