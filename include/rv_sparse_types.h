/*
 * rv-sparse B200 backend: public types.
 *
 * Same type names, enumerator names and values as the reference's public
 * types (rv-sparse include/rv_sparse_types.h:21-96), so code written against
 * the reference compiles unchanged. The CUDA backend only APPENDS:
 *
 *   RVSP_ERROR_DEVICE_FAILURE      (-7)  a CUDA call or kernel failed
 *   RVSP_BACKEND_CUDA              (3)   one-shot: exact-symbolic CUDA path
 *   RVSP_BACKEND_CUDA_LEARNED      (4)   one-shot: learned-capacity CUDA path
 *   RVSP_SPGEMM_ALGO_CUDA          (4)   descriptor: exact-symbolic CUDA path
 *   RVSP_SPGEMM_ALGO_CUDA_LEARNED  (5)   descriptor: learned-capacity CUDA path
 *   RVSP_OWNS_HOST / RVSP_OWNS_DEVICE    values of owns_data
 *
 * Existing values are never renumbered.
 */

#ifndef RV_SPARSE_TYPES_H
#define RV_SPARSE_TYPES_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum
{
    RVSP_SUCCESS = 0,
    RVSP_ERROR_NULL_POINTER = -1,
    RVSP_ERROR_INVALID_ARGUMENT = -2,
    RVSP_ERROR_INVALID_CSR = -3,
    RVSP_ERROR_UNSUPPORTED_DTYPE = -4,
    RVSP_ERROR_UNSUPPORTED_BACKEND = -5,
    RVSP_ERROR_ALLOCATION_FAILED = -6,
    /* appended: a CUDA runtime call or a kernel reported an error */
    RVSP_ERROR_DEVICE_FAILURE = -7
} rvsp_status_t;

typedef enum
{
    RVSP_DTYPE_INT8,
    RVSP_DTYPE_INT32,
    RVSP_DTYPE_BF16,
    RVSP_DTYPE_FP32,
    RVSP_DTYPE_FP64
} rvsp_dtype_t;

typedef enum
{
    RVSP_FORMAT_CSR
} rvsp_format_t;

typedef enum
{
    RVSP_BACKEND_SCALAR,
    RVSP_BACKEND_SCALAR_UNROLL4,
    RVSP_BACKEND_RVV_INTRINSICS,
    /* appended */
    RVSP_BACKEND_CUDA,
    RVSP_BACKEND_CUDA_LEARNED
} rvsp_backend_t;

/*
 * owns_data: 0 = caller-owned arrays (rvsp_csr_create), RVSP_OWNS_HOST = the
 * library allocated them in host memory that free() releases (the
 * reference's value 1), RVSP_OWNS_DEVICE = the CUDA backend allocated them in
 * device memory because the inputs were device-resident.
 * rvsp_csr_destroy frees each kind with the matching call.
 */
#define RVSP_OWNS_HOST 1
#define RVSP_OWNS_DEVICE 2

typedef struct
{
    int32_t rows;
    int32_t cols;
    int32_t nnz;

    int32_t *row_ptr;
    int32_t *col_idx;
    void *values;

    rvsp_dtype_t dtype;
    rvsp_format_t format;

    int owns_data;
} rvsp_csr_matrix_t;

typedef struct
{
    rvsp_backend_t backend;
    rvsp_dtype_t input_dtype;
    rvsp_dtype_t output_dtype;
} rvsp_spgemm_options_t;

/* Opaque two-phase SpGEMM descriptor. */
typedef struct rvsp_spgemm_descr *rvsp_spgemm_descr_t;

typedef enum
{
    RVSP_SPGEMM_ALGO_DEFAULT = 0, /* the reference's scalar kernel; here the CUDA exact path,
                                     whose results are bit-identical */
    RVSP_SPGEMM_ALGO_RVV,         /* RISC-V vector: not provided by this build */
    RVSP_SPGEMM_ALGO_CONTIG,      /* RISC-V vector: not provided by this build */
    RVSP_SPGEMM_ALGO_ADAPTIVE,    /* RISC-V vector: not provided by this build */
    /* appended */
    RVSP_SPGEMM_ALGO_CUDA,        /* B200: exact symbolic count, binned, order-preserving */
    RVSP_SPGEMM_ALGO_CUDA_LEARNED /* B200: MLP-predicted row capacity, overflow re-run exactly */
} rvsp_spgemm_algo_t;

#ifdef __cplusplus
}
#endif

#endif /* RV_SPARSE_TYPES_H */
