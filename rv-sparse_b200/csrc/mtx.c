/*
 * Matrix Market reader for the CUDA backend: the host half of the reference's
 * loader assemble_csr_matrix (rv-sparse tools/src/mtx_to_csr_formatter.c:
 * 153-330), whose canonicalisation half runs on the device
 * (rvsp_cuda_coo_to_csr, coo.cu).
 *
 * Parsing follows the reference: the %%MatrixMarket banner on the first line
 * decides "pattern" (every value 1.0f) and "symmetric" (:36-57); further
 * comment lines are skipped (:26-33); the dimensions line is "M N L"; then up
 * to L entries "row col [value]", 1-based, read with the same scanf formats
 * (a short file ends the list early, :199-217).
 */

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "rv_sparse_types.h"
#include "rvsp_cuda.h"

int rvsp_cuda_mtx_read(const char *path, int32_t *rows, int32_t *cols, int64_t *n,
                       int32_t **coo_row, int32_t **coo_col, float **coo_val, int *symmetric)
{
    if (!path || !rows || !cols || !n || !coo_row || !coo_col || !coo_val || !symmetric)
        return RVSP_ERROR_NULL_POINTER;
    *coo_row = NULL;
    *coo_col = NULL;
    *coo_val = NULL;
    *n = 0;
    FILE *f = fopen(path, "r");
    if (!f)
        return RVSP_ERROR_INVALID_ARGUMENT;
    char buf[2048];
    int pattern = 0, sym = 0;
    if (!fgets(buf, sizeof(buf), f))
    {
        fclose(f);
        return RVSP_ERROR_INVALID_ARGUMENT;
    }
    if (strncmp(buf, "%%MatrixMarket", 14) == 0)
    {
        char object[64], format[64], field[64], symmetry[64];
        if (sscanf(buf, "%%%%MatrixMarket %63s %63s %63s %63s", object, format, field,
                   symmetry) >= 4)
        {
            pattern = strcmp(field, "pattern") == 0;
            sym = strcmp(symmetry, "symmetric") == 0;
        }
    }
    /* the dimensions line: the first line that is not a comment */
    while (buf[0] == '%')
    {
        if (!fgets(buf, sizeof(buf), f))
        {
            fclose(f);
            return RVSP_ERROR_INVALID_ARGUMENT;
        }
    }
    int M, N, L;
    if (sscanf(buf, "%d %d %d", &M, &N, &L) != 3 || M <= 0 || N <= 0 || L < 0)
    {
        fclose(f);
        return RVSP_ERROR_INVALID_ARGUMENT;
    }
    size_t cap = L > 0 ? (size_t)L : 1;
    int32_t *r = (int32_t *)malloc(cap * sizeof(int32_t));
    int32_t *c = (int32_t *)malloc(cap * sizeof(int32_t));
    float *v = (float *)malloc(cap * sizeof(float));
    if (!r || !c || !v)
    {
        free(r);
        free(c);
        free(v);
        fclose(f);
        return RVSP_ERROR_ALLOCATION_FAILED;
    }
    int64_t k = 0;
    for (int l = 0; l < L; l++)
    {
        int row, col;
        float val = 1.0f;
        if (pattern)
        {
            if (fscanf(f, "%d %d", &row, &col) != 2)
                break;
        }
        else if (fscanf(f, "%d %d %f", &row, &col, &val) != 3)
        {
            break;
        }
        r[k] = row - 1;
        c[k] = col - 1;
        v[k] = val;
        k++;
    }
    fclose(f);
    *rows = M;
    *cols = N;
    *n = k;
    *coo_row = r;
    *coo_col = c;
    *coo_val = v;
    *symmetric = sym;
    return RVSP_SUCCESS;
}

int rvsp_cuda_mtx_to_csr(const char *path, int device_out, int32_t *rows, int32_t *cols,
                         int32_t *nnz, int32_t **row_ptr, int32_t **col_idx, float **values)
{
    if (!rows || !cols || !nnz || !row_ptr || !col_idx || !values)
        return RVSP_ERROR_NULL_POINTER;
    int32_t *r, *c;
    float *v;
    int64_t n;
    int sym;
    int st = rvsp_cuda_mtx_read(path, rows, cols, &n, &r, &c, &v, &sym);
    if (st != RVSP_SUCCESS)
        return st;
    st = rvsp_cuda_coo_to_csr(*rows, *cols, n, r, c, v, sym, device_out, row_ptr, col_idx, values,
                              nnz);
    free(r);
    free(c);
    free(v);
    return st;
}
