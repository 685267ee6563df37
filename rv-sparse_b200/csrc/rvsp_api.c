/*
 * rv-sparse public API (include/rv_sparse.h) on the B200 CUDA backend.
 *
 * Host C11, as in the reference. Matrix lifecycle and status strings follow
 * rv-sparse src/core/matrix.c and src/core/error.c; one-shot dispatch follows
 * src/core/spgemm.c:26-211; the descriptor state machine follows
 * src/core/spgemm_descr.c:19-380 (same argument checks, in the same order,
 * with the same status codes). All arithmetic runs on the GPU through the
 * C ABI in include/rvsp_cuda.h; this file does bookkeeping only.
 */

#include <stdlib.h>
#include <string.h>

#include "rv_sparse.h"
#include "rvsp_cuda.h"

const char *rvsp_get_version(void)
{
    return "0.1.0";
}

const char *rvsp_status_to_string(rvsp_status_t status)
{
    switch (status)
    {
    case RVSP_SUCCESS:
        return "success";
    case RVSP_ERROR_NULL_POINTER:
        return "null pointer";
    case RVSP_ERROR_INVALID_ARGUMENT:
        return "invalid argument";
    case RVSP_ERROR_INVALID_CSR:
        return "invalid CSR matrix";
    case RVSP_ERROR_UNSUPPORTED_DTYPE:
        return "unsupported data type";
    case RVSP_ERROR_UNSUPPORTED_BACKEND:
        return "unsupported backend";
    case RVSP_ERROR_ALLOCATION_FAILED:
        return "allocation failed";
    case RVSP_ERROR_DEVICE_FAILURE:
        return "device failure";
    default:
        return "unknown error";
    }
}

/* ------------------------------------------------------------------------ */
/* CSR lifecycle (rv-sparse src/core/matrix.c:18-115)                        */
/* ------------------------------------------------------------------------ */

rvsp_status_t rvsp_csr_create(rvsp_csr_matrix_t *A, int32_t rows, int32_t cols, int32_t nnz,
                              int32_t *row_ptr, int32_t *col_idx, void *values,
                              rvsp_dtype_t dtype)
{
    if (!A || !row_ptr || !col_idx || !values)
        return RVSP_ERROR_NULL_POINTER;
    if (rows <= 0 || cols <= 0 || nnz < 0)
        return RVSP_ERROR_INVALID_ARGUMENT;
    A->rows = rows;
    A->cols = cols;
    A->nnz = nnz;
    A->row_ptr = row_ptr;
    A->col_idx = col_idx;
    A->values = values;
    A->dtype = dtype;
    A->format = RVSP_FORMAT_CSR;
    A->owns_data = 0;
    return rvsp_csr_validate(A);
}

static int host_resident(const void *p)
{
    return !rvsp_cuda_is_device_pointer(p);
}

rvsp_status_t rvsp_csr_validate(const rvsp_csr_matrix_t *A)
{
    if (!A || !A->row_ptr || !A->col_idx || !A->values)
        return RVSP_ERROR_NULL_POINTER;
    if (A->rows <= 0 || A->cols <= 0 || A->nnz < 0)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (host_resident(A->row_ptr) && host_resident(A->col_idx))
    {
        if (A->row_ptr[0] != 0 || A->row_ptr[A->rows] != A->nnz)
            return RVSP_ERROR_INVALID_CSR;
        for (int32_t i = 0; i < A->rows; i++)
            if (A->row_ptr[i] > A->row_ptr[i + 1])
                return RVSP_ERROR_INVALID_CSR;
        for (int32_t i = 0; i < A->nnz; i++)
            if (A->col_idx[i] < 0 || A->col_idx[i] >= A->cols)
                return RVSP_ERROR_INVALID_CSR;
        return RVSP_SUCCESS;
    }
    return (rvsp_status_t)rvsp_cuda_csr_validate(A->rows, A->cols, A->nnz, A->row_ptr, A->col_idx);
}

void rvsp_csr_destroy(rvsp_csr_matrix_t *A)
{
    if (!A)
        return;
    if (A->owns_data == RVSP_OWNS_HOST)
    {
        rvsp_cuda_host_free(A->row_ptr);
        rvsp_cuda_host_free(A->col_idx);
        rvsp_cuda_host_free(A->values);
    }
    else if (A->owns_data == RVSP_OWNS_DEVICE)
    {
        rvsp_cuda_free(A->row_ptr);
        rvsp_cuda_free(A->col_idx);
        rvsp_cuda_free(A->values);
    }
    A->rows = 0;
    A->cols = 0;
    A->nnz = 0;
    A->row_ptr = NULL;
    A->col_idx = NULL;
    A->values = NULL;
    A->dtype = RVSP_DTYPE_FP32;
    A->format = RVSP_FORMAT_CSR;
    A->owns_data = 0;
}

/* ------------------------------------------------------------------------ */
/* Canonical check of one operand (rv-sparse src/core/spgemm.c:45-51)        */
/* ------------------------------------------------------------------------ */

static int canonical(const rvsp_csr_matrix_t *M)
{
    int32_t bad = -1;
    if (host_resident(M->row_ptr) && host_resident(M->col_idx))
    {
        if (M->row_ptr[0] != 0)
            return 0;
        for (int32_t r = 0; r < M->rows; r++)
        {
            int32_t s = M->row_ptr[r], e = M->row_ptr[r + 1];
            if (e < s)
                return 0;
            int32_t last = -1;
            for (int32_t p = s; p < e; p++)
            {
                int32_t c = M->col_idx[p];
                if (c < 0 || c >= M->cols || c <= last)
                    return 0;
                last = c;
            }
        }
        return 1;
    }
    return rvsp_cuda_csr_check(M->rows, M->cols, M->nnz, M->row_ptr, M->col_idx, &bad) == 0;
}

/* ------------------------------------------------------------------------ */
/* One-shot (rv-sparse src/core/spgemm.c:135-211)                            */
/* ------------------------------------------------------------------------ */

/* FP64 x FP64 -> FP64 and INT8 x INT8 -> INT32 one-shot products with the
 * checks of the reference's legacy wrappers, in their order and with their
 * codes: INT8 validates both operands, then a dtype mismatch is
 * UNSUPPORTED_DTYPE (csr_spgemm_wrappers.c:19-50); FP64 reports a dtype
 * mismatch as INVALID_ARGUMENT (:352-371); both then check the shapes. */
static rvsp_status_t spgemm_typed(const rvsp_csr_matrix_t *A, const rvsp_csr_matrix_t *B,
                                  rvsp_csr_matrix_t *C, rvsp_dtype_t in_dt, rvsp_dtype_t out_dt)
{
    if (rvsp_cuda_device_count() == 0)
        return RVSP_ERROR_UNSUPPORTED_BACKEND;
    if (in_dt == RVSP_DTYPE_INT8)
    {
        rvsp_status_t vs = rvsp_csr_validate(A);
        if (vs == RVSP_SUCCESS)
            vs = rvsp_csr_validate(B);
        if (vs != RVSP_SUCCESS)
            return vs;
        if (A->dtype != RVSP_DTYPE_INT8 || B->dtype != RVSP_DTYPE_INT8)
            return RVSP_ERROR_UNSUPPORTED_DTYPE;
    }
    else if (A->dtype != RVSP_DTYPE_FP64 || B->dtype != RVSP_DTYPE_FP64)
    {
        return RVSP_ERROR_INVALID_ARGUMENT;
    }
    if (A->cols != B->rows)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (!A->row_ptr || !A->col_idx || !A->values || !B->row_ptr || !B->col_idx || !B->values)
        return RVSP_ERROR_NULL_POINTER;
    if (A->rows <= 0 || A->cols <= 0 || B->cols <= 0)
        return RVSP_ERROR_INVALID_ARGUMENT;
    int32_t *rp = NULL, *ci = NULL, nnz = 0;
    void *v = NULL;
    int st;
    if (in_dt == RVSP_DTYPE_FP64)
        st = rvsp_cuda_spgemm_f64(A->rows, A->cols, B->cols, A->row_ptr, A->col_idx,
                                  (const double *)A->values, B->row_ptr, B->col_idx,
                                  (const double *)B->values, &rp, &ci, (double **)&v, &nnz);
    else
        st = rvsp_cuda_spgemm_i8(A->rows, A->cols, B->cols, A->row_ptr, A->col_idx,
                                 (const int8_t *)A->values, B->row_ptr, B->col_idx,
                                 (const int8_t *)B->values, &rp, &ci, (int32_t **)&v, &nnz);
    if (st != RVSP_SUCCESS)
    {
        C->row_ptr = NULL;
        C->col_idx = NULL;
        C->values = NULL;
        C->nnz = 0;
        C->owns_data = 0;
        return (rvsp_status_t)st;
    }
    C->rows = A->rows;
    C->cols = B->cols;
    C->nnz = nnz;
    C->row_ptr = rp;
    C->col_idx = ci;
    C->values = v;
    C->dtype = out_dt;
    C->format = RVSP_FORMAT_CSR;
    C->owns_data = rvsp_cuda_is_device_pointer(rp) ? RVSP_OWNS_DEVICE : RVSP_OWNS_HOST;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_csr(const rvsp_csr_matrix_t *A, const rvsp_csr_matrix_t *B,
                              rvsp_csr_matrix_t *C, const rvsp_spgemm_options_t *options)
{
    rvsp_backend_t backend = RVSP_BACKEND_CUDA;
    rvsp_dtype_t in_dt = RVSP_DTYPE_FP32, out_dt = RVSP_DTYPE_FP32;

    if (!A || !B || !C)
        return RVSP_ERROR_NULL_POINTER;
    if (options)
    {
        backend = options->backend;
        in_dt = options->input_dtype;
        out_dt = options->output_dtype;
    }
    /* The reference's scalar backends (spgemm.c:160-167, :181-193) run on the
     * CUDA exact path, whose results are bit-identical to the scalar kernels'
     * (FP32 and the FP64 / INT8 -> INT32 legacy products alike). */
    if (backend == RVSP_BACKEND_SCALAR ||
        (backend == RVSP_BACKEND_SCALAR_UNROLL4 && in_dt == RVSP_DTYPE_FP32 &&
         out_dt == RVSP_DTYPE_FP32))
        backend = RVSP_BACKEND_CUDA;
    /* the reference's other dtypes (its legacy kernels, spgemm.c:181-193) */
    if (backend == RVSP_BACKEND_CUDA &&
        ((in_dt == RVSP_DTYPE_FP64 && out_dt == RVSP_DTYPE_FP64) ||
         (in_dt == RVSP_DTYPE_INT8 && out_dt == RVSP_DTYPE_INT32)))
        return spgemm_typed(A, B, C, in_dt, out_dt);
    if ((backend != RVSP_BACKEND_CUDA && backend != RVSP_BACKEND_CUDA_LEARNED) ||
        in_dt != RVSP_DTYPE_FP32 || out_dt != RVSP_DTYPE_FP32)
        return RVSP_ERROR_UNSUPPORTED_BACKEND;
    if (rvsp_cuda_device_count() == 0)
        return RVSP_ERROR_UNSUPPORTED_BACKEND;
    if (A->dtype != RVSP_DTYPE_FP32 || B->dtype != RVSP_DTYPE_FP32)
        return RVSP_ERROR_UNSUPPORTED_DTYPE;
    if (A->cols != B->rows)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (!A->row_ptr || !A->col_idx || !A->values || !B->row_ptr || !B->col_idx || !B->values)
        return RVSP_ERROR_NULL_POINTER;
    if (A->rows <= 0 || A->cols <= 0 || B->cols <= 0)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (!canonical(A) || !canonical(B))
        return RVSP_ERROR_INVALID_CSR;

    int32_t *rp = NULL, *ci = NULL, nnz = 0;
    float *v = NULL;
    int st = rvsp_cuda_spgemm_f32(backend == RVSP_BACKEND_CUDA_LEARNED ? RVSP_CUDA_ALGO_LEARNED
                                                                       : RVSP_CUDA_ALGO_EXACT,
                                  A->rows, A->cols, B->cols, A->row_ptr, A->col_idx,
                                  (const float *)A->values, B->row_ptr, B->col_idx,
                                  (const float *)B->values, &rp, &ci, &v, &nnz, NULL);
    if (st != RVSP_SUCCESS)
    {
        C->row_ptr = NULL;
        C->col_idx = NULL;
        C->values = NULL;
        C->nnz = 0;
        C->owns_data = 0;
        return (rvsp_status_t)st;
    }
    C->rows = A->rows;
    C->cols = B->cols;
    C->nnz = nnz;
    C->row_ptr = rp;
    C->col_idx = ci;
    C->values = v;
    C->dtype = RVSP_DTYPE_FP32;
    C->format = RVSP_FORMAT_CSR;
    C->owns_data = rvsp_cuda_is_device_pointer(rp) ? RVSP_OWNS_DEVICE : RVSP_OWNS_HOST;
    return RVSP_SUCCESS;
}

/* ------------------------------------------------------------------------ */
/* Descriptor (rv-sparse src/core/spgemm_descr.c:19-380)                     */
/* ------------------------------------------------------------------------ */

struct rvsp_spgemm_descr
{
    rvsp_spgemm_algo_t algo;
    int estimated;
    rvsp_cuda_plan_t plan;
    int32_t c_nnz;
    /* C->col_idx the most recent fill wrote into, for reuse detection */
    const int32_t *filled_into;
    int32_t a_rows, a_cols, a_nnz;
    int32_t b_rows, b_cols, b_nnz;
    size_t workspace_bytes;
};

/* The reference's default strategy is its scalar kernel
 * (spgemm_descr.c:43-64, :83). The CUDA exact path computes bit-identical
 * results (same structure, same FP32 operation order), so DEFAULT selects it:
 * code written against the reference runs unchanged, on the GPU. The vector
 * strategies are refused as the reference refuses them on a build without
 * the vector extension. */
static int plan_algo(rvsp_spgemm_algo_t algo)
{
    return algo == RVSP_SPGEMM_ALGO_CUDA_LEARNED ? RVSP_CUDA_ALGO_LEARNED : RVSP_CUDA_ALGO_EXACT;
}

static int algo_available(rvsp_spgemm_algo_t algo)
{
    if (algo != RVSP_SPGEMM_ALGO_DEFAULT && algo != RVSP_SPGEMM_ALGO_CUDA &&
        algo != RVSP_SPGEMM_ALGO_CUDA_LEARNED)
        return 0;
    if (rvsp_cuda_device_count() == 0)
        return 0;
    /* the learned strategy needs a row-size model (the shipped checkpoint) */
    return algo != RVSP_SPGEMM_ALGO_CUDA_LEARNED || rvsp_cuda_learned_available();
}

rvsp_status_t rvsp_spgemm_descr_create(rvsp_spgemm_descr_t *descr)
{
    if (descr == NULL)
        return RVSP_ERROR_NULL_POINTER;
    *descr = NULL;
    struct rvsp_spgemm_descr *d = (struct rvsp_spgemm_descr *)calloc(1, sizeof(*d));
    if (d == NULL)
        return RVSP_ERROR_ALLOCATION_FAILED;
    d->algo = RVSP_SPGEMM_ALGO_DEFAULT; /* as the reference (spgemm_descr.c:83) */
    *descr = d;
    return RVSP_SUCCESS;
}

void rvsp_spgemm_descr_destroy(rvsp_spgemm_descr_t descr)
{
    if (descr == NULL)
        return;
    rvsp_cuda_plan_destroy(descr->plan);
    free(descr);
}

rvsp_status_t rvsp_spgemm_set_algo(rvsp_spgemm_descr_t descr, rvsp_spgemm_algo_t algo)
{
    if (descr == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (descr->estimated)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (!algo_available(algo))
        return RVSP_ERROR_UNSUPPORTED_BACKEND;
    descr->algo = algo;
    return RVSP_SUCCESS;
}

void rvsp_spgemm_invalidate_structure(rvsp_spgemm_descr_t descr)
{
    if (descr != NULL)
        descr->filled_into = NULL;
}

static rvsp_status_t check_operand(const rvsp_csr_matrix_t *M)
{
    if (M == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (M->row_ptr == NULL || M->col_idx == NULL || M->values == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (M->dtype != RVSP_DTYPE_FP32)
        return RVSP_ERROR_UNSUPPORTED_DTYPE;
    if (M->rows <= 0 || M->cols <= 0 || M->nnz < 0)
        return RVSP_ERROR_INVALID_ARGUMENT;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_work_estimation(rvsp_spgemm_descr_t descr, const rvsp_csr_matrix_t *A,
                                          const rvsp_csr_matrix_t *B, size_t *workspace_bytes,
                                          int32_t *c_nnz_out)
{
    if (descr == NULL || workspace_bytes == NULL || c_nnz_out == NULL)
        return RVSP_ERROR_NULL_POINTER;
    rvsp_status_t st = check_operand(A);
    if (st != RVSP_SUCCESS)
        return st;
    st = check_operand(B);
    if (st != RVSP_SUCCESS)
        return st;
    if (A->cols != B->rows)
        return RVSP_ERROR_INVALID_ARGUMENT;

    /* re-estimating discards the previous structure */
    descr->filled_into = NULL;
    descr->estimated = 0;
    descr->c_nnz = 0;
    if (descr->plan == NULL)
    {
        int cst = rvsp_cuda_plan_create(&descr->plan, plan_algo(descr->algo));
        if (cst != RVSP_SUCCESS)
            return (rvsp_status_t)cst;
    }
    int64_t nnz = 0;
    size_t ws = 0;
    int cst;
    /* RVSP_AUTOTUNE=1: pick the plan's bin parameters for this product first
     * (the descriptor keeps them for its computes) */
    const char *tune = getenv("RVSP_AUTOTUNE");
    if (tune != NULL && tune[0] == '1' && A->values != NULL && B->values != NULL)
        cst = rvsp_cuda_plan_autotune(descr->plan, A->rows, A->cols, A->nnz, A->row_ptr,
                                      A->col_idx, (const float *)A->values, B->rows, B->cols,
                                      B->nnz, B->row_ptr, B->col_idx, (const float *)B->values,
                                      2, NULL, NULL, NULL, 0, NULL, &nnz, &ws);
    else
        cst = rvsp_cuda_symbolic(descr->plan, A->rows, A->cols, A->nnz, A->row_ptr, A->col_idx,
                                 B->rows, B->cols, B->nnz, B->row_ptr, B->col_idx, &nnz, &ws);
    if (cst != RVSP_SUCCESS)
        return (rvsp_status_t)cst;
    descr->c_nnz = (int32_t)nnz;
    descr->a_rows = A->rows;
    descr->a_cols = A->cols;
    descr->a_nnz = A->nnz;
    descr->b_rows = B->rows;
    descr->b_cols = B->cols;
    descr->b_nnz = B->nnz;
    descr->workspace_bytes = ws;
    descr->estimated = 1;
    *workspace_bytes = ws;
    *c_nnz_out = descr->c_nnz;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_compute(rvsp_spgemm_descr_t descr, const rvsp_csr_matrix_t *A,
                                  const rvsp_csr_matrix_t *B, rvsp_csr_matrix_t *C,
                                  void *workspace)
{
    if (descr == NULL || C == NULL || workspace == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (!descr->estimated)
        return RVSP_ERROR_INVALID_ARGUMENT;
    rvsp_status_t st = check_operand(A);
    if (st != RVSP_SUCCESS)
        return st;
    st = check_operand(B);
    if (st != RVSP_SUCCESS)
        return st;
    if (A->rows != descr->a_rows || A->cols != descr->a_cols || A->nnz != descr->a_nnz ||
        B->rows != descr->b_rows || B->cols != descr->b_cols || B->nnz != descr->b_nnz)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (C->row_ptr == NULL || C->col_idx == NULL || C->values == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (C->dtype != RVSP_DTYPE_FP32)
        return RVSP_ERROR_UNSUPPORTED_DTYPE;
    if (C->rows != descr->a_rows || C->cols != descr->b_cols)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (C->nnz < descr->c_nnz)
        return RVSP_ERROR_INVALID_ARGUMENT;

    const int fill = descr->filled_into != C->col_idx;
    int cst = rvsp_cuda_numeric(descr->plan, A->row_ptr, A->col_idx, (const float *)A->values,
                                B->row_ptr, B->col_idx, (const float *)B->values, C->row_ptr,
                                C->col_idx, (float *)C->values, fill, workspace);
    if (cst != RVSP_SUCCESS)
        return (rvsp_status_t)cst;
    descr->filled_into = C->col_idx;
    C->nnz = descr->c_nnz;
    C->format = RVSP_FORMAT_CSR;
    return RVSP_SUCCESS;
}

rvsp_status_t rvsp_spgemm_get_op_counts(rvsp_spgemm_descr_t descr, int64_t *op_counts_out,
                                        int32_t n)
{
    if (descr == NULL || op_counts_out == NULL)
        return RVSP_ERROR_NULL_POINTER;
    if (!descr->estimated)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (n < descr->a_rows)
        return RVSP_ERROR_INVALID_ARGUMENT;
    return (rvsp_status_t)rvsp_cuda_op_counts(descr->plan, op_counts_out, n);
}
