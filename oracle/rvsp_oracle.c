/*
 * CPU oracle for FP32 CSR SpGEMM (C = A * B).
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker that the CUDA backend is
 * compared against. It is loaded by tests/, by __graft_entry__.smoke() and by
 * the cpu_baseline leg of bench.py, never by the library itself.
 *
 * It restates the reference's scalar Gustavson path in plain C:
 *
 *   per-row op count and distinct-column count
 *       rv-sparse src/kernels/spgemm/rvsp_symbolic.c:13-87
 *   distinct columns of a row, sorted ascending
 *       rv-sparse src/kernels/spgemm/rvsp_symbolic.c:91-137, rvsp_sort.h:105-124
 *   numeric pass: for each A entry (k, a) in row order, for each B entry
 *   (j, b) of row k in order, acc[j] += a * b, starting from +0.0f, then the
 *   row is drained in ascending column order
 *       rv-sparse src/kernels/spgemm/gustavson_core_f32.inc:18-64,
 *       src/kernels/spgemm/accum_scalar_f32.c:20-71 (line 69)
 *   canonical CSR validation
 *       rv-sparse src/kernels/spgemm/rvsp_support.c:37-127
 *
 * The reference is built with -std=c11, under which GCC does not contract
 * a * b + c into an FMA. This file is built with -ffp-contract=off for the
 * same reason, so every product is rounded to FP32 before it is added.
 *
 * An FP64 variant of the numeric pass gives the error yardstick for the
 * FP32 results. It has no reference counterpart.
 *
 * The reference's other two dtypes (its legacy one-shot kernels) are
 * restated too: FP64 x FP64 -> FP64
 *       rv-sparse src/kernels/spgemm/legacy/csr_scalar_f64.c:49-272
 * and INT8 x INT8 -> INT32
 *       rv-sparse src/kernels/spgemm/legacy/csr_scalar_i8.c:24-196
 * Both accumulate acc[j] += a * b in A-row order from zero and, unlike the
 * FP32 path, do not store an output entry whose sum is exactly zero.
 *
 * The canonicalisation of the reference's Matrix Market loader (COO ->
 * sorted CSR with repeated entries summed) is restated as oracle_coo_to_csr
 *       rv-sparse tools/src/mtx_to_csr_formatter.c:219-330, :74-151
 *
 * Every entry point works on a half-open row range [row_begin, row_end) so a
 * test can check sampled rows of a product too large to redo in full.
 */

#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_OK 0
#define ORACLE_ERR_ALLOC -6
#define ORACLE_ERR_INVALID -2

/* Canonical CSR check; codes follow rvsp_csr_status_t
 * (rv-sparse src/kernels/spgemm/rvsp_spgemm.h:38-45):
 * 0 ok, 1 bad row_ptr, 2 column out of range, 3 unsorted, 4 duplicate. */
int oracle_csr_check(int32_t rows, int32_t cols, const int32_t *row_ptr,
                     const int32_t *col_idx, int32_t *bad_row_out)
{
    if (bad_row_out)
        *bad_row_out = -1;
    if (rows < 0 || cols < 0 || !row_ptr || row_ptr[0] != 0)
        return 1;
    for (int32_t r = 0; r < rows; r++)
    {
        int32_t s = row_ptr[r], e = row_ptr[r + 1];
        if (e < s)
        {
            if (bad_row_out)
                *bad_row_out = r;
            return 1;
        }
        int32_t last = -1;
        for (int32_t p = s; p < e; p++)
        {
            int32_t c = col_idx[p];
            int code = 0;
            if (c < 0 || c >= cols)
                code = 2;
            else if (c == last)
                code = 4;
            else if (c < last)
                code = 3;
            if (code)
            {
                if (bad_row_out)
                    *bad_row_out = r;
                return code;
            }
            last = c;
        }
    }
    return 0;
}

/* Per-row intermediate products and distinct output columns for rows
 * [row_begin, row_end). ops_out and cnt_out are indexed from row_begin.
 * Returns the sum of cnt_out. */
int64_t oracle_symbolic(int32_t row_begin, int32_t row_end, int32_t n_cols,
                        const int32_t *a_rp, const int32_t *a_ci,
                        const int32_t *b_rp, const int32_t *b_ci,
                        int64_t *ops_out, int64_t *cnt_out)
{
    uint8_t *seen = (uint8_t *)calloc((size_t)(n_cols > 0 ? n_cols : 1), 1);
    int32_t *list = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n_cols > 0 ? n_cols : 1));
    if (!seen || !list)
    {
        free(seen);
        free(list);
        return -1;
    }
    int64_t total = 0;
    for (int32_t r = row_begin; r < row_end; r++)
    {
        int64_t ops = 0;
        int64_t cnt = 0;
        for (int32_t p = a_rp[r]; p < a_rp[r + 1]; p++)
        {
            int32_t k = a_ci[p];
            ops += b_rp[k + 1] - b_rp[k];
            for (int32_t q = b_rp[k]; q < b_rp[k + 1]; q++)
            {
                int32_t j = b_ci[q];
                if (!seen[j])
                {
                    seen[j] = 1;
                    list[cnt++] = j;
                }
            }
        }
        for (int64_t t = 0; t < cnt; t++)
            seen[list[t]] = 0;
        if (ops_out)
            ops_out[r - row_begin] = ops;
        if (cnt_out)
            cnt_out[r - row_begin] = cnt;
        total += cnt;
    }
    free(seen);
    free(list);
    return total;
}

static int cmp_i32(const void *x, const void *y)
{
    int32_t a = *(const int32_t *)x, b = *(const int32_t *)y;
    return (a > b) - (a < b);
}

/*
 * Full product for rows [row_begin, row_end): writes the row offsets
 * (relative, c_rp[0] = 0, row_end - row_begin + 1 entries), the sorted column
 * indices and the FP32 values. c_ci / c_v must hold the total returned by
 * oracle_symbolic for the same range. Values follow the reference's order of
 * operations exactly.
 */
int oracle_spgemm_f32(int32_t row_begin, int32_t row_end, int32_t n_cols,
                      const int32_t *a_rp, const int32_t *a_ci, const float *a_v,
                      const int32_t *b_rp, const int32_t *b_ci, const float *b_v,
                      int64_t *c_rp, int32_t *c_ci, float *c_v)
{
    size_t n = (size_t)(n_cols > 0 ? n_cols : 1);
    uint8_t *seen = (uint8_t *)calloc(n, 1);
    float *acc = (float *)calloc(n, sizeof(float));
    if (!seen || !acc)
    {
        free(seen);
        free(acc);
        return ORACLE_ERR_ALLOC;
    }
    int64_t pos = 0;
    c_rp[0] = 0;
    for (int32_t r = row_begin; r < row_end; r++)
    {
        int64_t start = pos;
        /* structure: distinct columns, then ascending order */
        for (int32_t p = a_rp[r]; p < a_rp[r + 1]; p++)
        {
            int32_t k = a_ci[p];
            for (int32_t q = b_rp[k]; q < b_rp[k + 1]; q++)
            {
                int32_t j = b_ci[q];
                if (!seen[j])
                {
                    seen[j] = 1;
                    c_ci[pos++] = j;
                }
            }
        }
        qsort(c_ci + start, (size_t)(pos - start), sizeof(int32_t), cmp_i32);
        /* values: k-order, product rounded to FP32, then added */
        for (int32_t p = a_rp[r]; p < a_rp[r + 1]; p++)
        {
            int32_t k = a_ci[p];
            float a = a_v[p];
            for (int32_t q = b_rp[k]; q < b_rp[k + 1]; q++)
            {
                float prod = a * b_v[q];
                acc[b_ci[q]] = acc[b_ci[q]] + prod;
            }
        }
        for (int64_t t = start; t < pos; t++)
        {
            c_v[t] = acc[c_ci[t]];
            acc[c_ci[t]] = 0.0f;
            seen[c_ci[t]] = 0;
        }
        c_rp[r - row_begin + 1] = pos;
    }
    free(seen);
    free(acc);
    return ORACLE_OK;
}

/*
 * FP64 numeric pass over a given output pattern (rows [row_begin, row_end),
 * c_rp relative as produced above). Inputs are the FP32 values widened to
 * double; the products and sums are exact-ish double arithmetic. This is the
 * yardstick for the relative error of FP32 results.
 */
int oracle_numeric_f64(int32_t row_begin, int32_t row_end, int32_t n_cols,
                       const int32_t *a_rp, const int32_t *a_ci, const float *a_v,
                       const int32_t *b_rp, const int32_t *b_ci, const float *b_v,
                       const int64_t *c_rp, const int32_t *c_ci, double *c_v)
{
    double *acc = (double *)calloc((size_t)(n_cols > 0 ? n_cols : 1), sizeof(double));
    if (!acc)
        return ORACLE_ERR_ALLOC;
    for (int32_t r = row_begin; r < row_end; r++)
    {
        for (int32_t p = a_rp[r]; p < a_rp[r + 1]; p++)
        {
            int32_t k = a_ci[p];
            double a = (double)a_v[p];
            for (int32_t q = b_rp[k]; q < b_rp[k + 1]; q++)
                acc[b_ci[q]] += a * (double)b_v[q];
        }
        for (int64_t t = c_rp[r - row_begin]; t < c_rp[r - row_begin + 1]; t++)
        {
            c_v[t] = acc[c_ci[t]];
            acc[c_ci[t]] = 0.0;
        }
    }
    free(acc);
    return ORACLE_OK;
}

/*
 * Numeric-only FP32 pass over a given pattern, the descriptor-reuse path
 * (rv-sparse src/core/spgemm_descr.c:257-355 with filled_into == C->col_idx:
 * the structure is kept and only the values are recomputed).
 */
int oracle_numeric_f32(int32_t row_begin, int32_t row_end, int32_t n_cols,
                       const int32_t *a_rp, const int32_t *a_ci, const float *a_v,
                       const int32_t *b_rp, const int32_t *b_ci, const float *b_v,
                       const int64_t *c_rp, const int32_t *c_ci, float *c_v)
{
    float *acc = (float *)calloc((size_t)(n_cols > 0 ? n_cols : 1), sizeof(float));
    if (!acc)
        return ORACLE_ERR_ALLOC;
    for (int32_t r = row_begin; r < row_end; r++)
    {
        for (int32_t p = a_rp[r]; p < a_rp[r + 1]; p++)
        {
            int32_t k = a_ci[p];
            float a = a_v[p];
            for (int32_t q = b_rp[k]; q < b_rp[k + 1]; q++)
            {
                float prod = a * b_v[q];
                acc[b_ci[q]] = acc[b_ci[q]] + prod;
            }
        }
        for (int64_t t = c_rp[r - row_begin]; t < c_rp[r - row_begin + 1]; t++)
        {
            c_v[t] = acc[c_ci[t]];
            acc[c_ci[t]] = 0.0f;
        }
    }
    free(acc);
    return ORACLE_OK;
}

/*
 * Legacy-dtype products for rows [row_begin, row_end): distinct columns in
 * ascending order, acc[j] += a * b in A-row order starting from zero, entries
 * whose sum is zero dropped (csr_scalar_f64.c:226-245, csr_scalar_i8.c:
 * 131-175). c_rp is relative (c_rp[0] = 0); c_ci / c_v must hold the
 * symbolic total for the range (an upper bound). INT8 products and sums are
 * formed in 32-bit two's complement.
 */
#define ORACLE_LEGACY(NAME, IN_T, ACC_T, MUL, ADD)                              \
    int NAME(int32_t row_begin, int32_t row_end, int32_t n_cols,                \
             const int32_t *a_rp, const int32_t *a_ci, const IN_T *a_v,         \
             const int32_t *b_rp, const int32_t *b_ci, const IN_T *b_v,         \
             int64_t *c_rp, int32_t *c_ci, ACC_T *c_v)                          \
    {                                                                           \
        size_t n = (size_t)(n_cols > 0 ? n_cols : 1);                           \
        uint8_t *seen = (uint8_t *)calloc(n, 1);                                \
        ACC_T *acc = (ACC_T *)calloc(n, sizeof(ACC_T));                         \
        int32_t *cols = (int32_t *)malloc(n * sizeof(int32_t));                 \
        if (!seen || !acc || !cols)                                             \
        {                                                                       \
            free(seen);                                                         \
            free(acc);                                                          \
            free(cols);                                                         \
            return ORACLE_ERR_ALLOC;                                            \
        }                                                                       \
        int64_t pos = 0;                                                        \
        c_rp[0] = 0;                                                            \
        for (int32_t r = row_begin; r < row_end; r++)                           \
        {                                                                       \
            int32_t m = 0;                                                      \
            for (int32_t p = a_rp[r]; p < a_rp[r + 1]; p++)                     \
            {                                                                   \
                int32_t k = a_ci[p];                                            \
                for (int32_t q = b_rp[k]; q < b_rp[k + 1]; q++)                 \
                {                                                               \
                    int32_t j = b_ci[q];                                        \
                    if (!seen[j])                                               \
                    {                                                           \
                        seen[j] = 1;                                            \
                        acc[j] = 0;                                             \
                        cols[m++] = j;                                          \
                    }                                                           \
                    acc[j] = ADD(acc[j], MUL(a_v[p], b_v[q]));                  \
                }                                                               \
            }                                                                   \
            qsort(cols, (size_t)m, sizeof(int32_t), cmp_i32);                   \
            for (int32_t t = 0; t < m; t++)                                     \
            {                                                                   \
                int32_t j = cols[t];                                            \
                if (acc[j] != 0)                                                \
                {                                                               \
                    c_ci[pos] = j;                                              \
                    c_v[pos] = acc[j];                                          \
                    pos++;                                                      \
                }                                                               \
                seen[j] = 0;                                                    \
            }                                                                   \
            c_rp[r - row_begin + 1] = pos;                                      \
        }                                                                       \
        free(seen);                                                             \
        free(acc);                                                              \
        free(cols);                                                             \
        return ORACLE_OK;                                                       \
    }

#define MUL_F64(a, b) ((a) * (b))
#define ADD_F64(x, y) ((x) + (y))
#define MUL_I8(a, b) ((int32_t)((uint32_t)(int32_t)(a) * (uint32_t)(int32_t)(b)))
#define ADD_I32(x, y) ((int32_t)((uint32_t)(x) + (uint32_t)(y)))

ORACLE_LEGACY(oracle_spgemm_f64, double, double, MUL_F64, ADD_F64)
ORACLE_LEGACY(oracle_spgemm_i8, int8_t, int32_t, MUL_I8, ADD_I32)

/*
 * COO -> canonical CSR (mtx_to_csr_formatter.c:219-330 with canonicalise_rows
 * :74-151): with symmetric, every off-diagonal entry's mirror is appended
 * after all stored entries (:221-244); entries are ordered by (row, column)
 * keeping COO order among equal pairs (row buckets filled in COO order,
 * :286-300, then a stable sort by column); each run of equal pairs is summed
 * left to right from its first value (:120-131). coo_val may be NULL (1.0f
 * each). c_rp has rows + 1 entries; c_ci / c_v hold up to 2n entries.
 * Returns the output nnz, or a negative code.
 */
typedef struct
{
    int64_t key;
    int64_t idx;
} oracle_ki_t;

static int cmp_ki(const void *x, const void *y)
{
    const oracle_ki_t *a = (const oracle_ki_t *)x, *b = (const oracle_ki_t *)y;
    if (a->key != b->key)
        return (a->key > b->key) - (a->key < b->key);
    return (a->idx > b->idx) - (a->idx < b->idx);
}

int64_t oracle_coo_to_csr(int32_t rows, int32_t cols, int64_t n, const int32_t *coo_row,
                          const int32_t *coo_col, const float *coo_val, int symmetric,
                          int64_t *c_rp, int32_t *c_ci, float *c_v)
{
    int64_t m = n;
    if (symmetric)
        for (int64_t k = 0; k < n; k++)
            m += coo_row[k] != coo_col[k];
    oracle_ki_t *e = (oracle_ki_t *)malloc((size_t)(m > 0 ? m : 1) * sizeof(oracle_ki_t));
    float *val = (float *)malloc((size_t)(m > 0 ? m : 1) * sizeof(float));
    if (!e || !val)
    {
        free(e);
        free(val);
        return ORACLE_ERR_ALLOC;
    }
    int64_t t = 0;
    for (int64_t k = 0; k < n; k++)
    {
        if (coo_row[k] < 0 || coo_row[k] >= rows || coo_col[k] < 0 || coo_col[k] >= cols)
        {
            free(e);
            free(val);
            return ORACLE_ERR_INVALID;
        }
        e[t].key = (int64_t)coo_row[k] * cols + coo_col[k];
        e[t].idx = t;
        val[t] = coo_val ? coo_val[k] : 1.0f;
        t++;
    }
    if (symmetric)
        for (int64_t k = 0; k < n; k++)
            if (coo_row[k] != coo_col[k])
            {
                e[t].key = (int64_t)coo_col[k] * cols + coo_row[k];
                e[t].idx = t;
                val[t] = coo_val ? coo_val[k] : 1.0f;
                t++;
            }
    qsort(e, (size_t)m, sizeof(oracle_ki_t), cmp_ki);
    int64_t out = 0;
    for (int32_t r = 0; r <= rows; r++)
        c_rp[r] = 0;
    for (int64_t i = 0; i < m;)
    {
        const int64_t key = e[i].key;
        float acc = val[e[i].idx];
        int64_t j = i + 1;
        for (; j < m && e[j].key == key; j++)
            acc += val[e[j].idx];
        c_ci[out] = (int32_t)(key % cols);
        c_v[out] = acc;
        c_rp[key / cols + 1]++;
        out++;
        i = j;
    }
    for (int32_t r = 0; r < rows; r++)
        c_rp[r + 1] += c_rp[r];
    free(e);
    free(val);
    return out;
}
