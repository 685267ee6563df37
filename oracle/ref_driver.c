/*
 * Thin drivers around the reference's own scalar SpGEMM, linked against the
 * reference sources by oracle/Makefile into oracle/_ref/librvsp_ref.so.
 *
 * TEST AND BASELINE INFRASTRUCTURE ONLY. Used by tests/ to pin the oracle and
 * the CUDA backend to the reference's real output, and by bench.py's
 * reference arm and cpu_baseline leg to time the reference on host cores.
 *
 * Timed scope follows rv-sparse bench/bench.c:856-861: the whole raw-kernel
 * call (symbolic count, C malloc, fill + sort, numeric), inputs already in
 * memory, workspace allocated outside the timed region.
 *
 * The reference kernel is single-threaded. The *_panels drivers run it on
 * disjoint row panels of A, one POSIX thread per panel; output rows are
 * independent, so each panel's result is the reference's result for those
 * rows. Panel outputs are left in per-panel buffers (not concatenated).
 */

#define _POSIX_C_SOURCE 200809L
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "mtx_to_csr_formatter.h"
#include "rv_sparse.h"
#include "rvsp_spgemm.h"

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* One raw-kernel call; returns status and the callee-malloc'd C arrays. */
int ref_spgemm_raw(int32_t a_rows, int32_t a_cols, int32_t b_cols,
                   const int32_t *a_rp, const int32_t *a_ci, const float *a_v,
                   const int32_t *b_rp, const int32_t *b_ci, const float *b_v,
                   int32_t **c_rp, int32_t **c_ci, float **c_v, int32_t *c_nnz,
                   int64_t *ops_out)
{
    size_t ws_bytes = 0;
    if (rvsp_spgemm_buffer_size(b_cols, &ws_bytes) != RVSP_SUCCESS)
        return -2;
    void *ws = malloc(ws_bytes);
    if (!ws)
        return -6;
    int st = rvsp_spgemm_scalar_f32(a_rows, a_cols, b_cols, a_rp, a_ci, a_v,
                                    b_rp, b_ci, b_v, ws, ws_bytes,
                                    c_rp, c_ci, c_v, c_nnz, ops_out);
    free(ws);
    return st;
}

void ref_free(void *p)
{
    free(p);
}

/* The reference's Matrix Market loader (tools/src/mtx_to_csr_formatter.c:
 * 153-330); its CSR arrays copied into malloc'd ones. */
int ref_mtx_load(const char *path, int32_t *rows, int32_t *nnz, int32_t **rp, int32_t **ci,
                 float **v)
{
    struct CSR m = assemble_csr_matrix(path);
    if (!m.row_ptr || !m.col_ind || !m.val)
        return -1;
    size_t nr = vector_size(m.row_ptr), nz = vector_size(m.col_ind);
    *rows = (int32_t)nr - 1;
    *nnz = (int32_t)nz;
    *rp = (int32_t *)malloc(nr * sizeof(int32_t));
    *ci = (int32_t *)malloc((nz ? nz : 1) * sizeof(int32_t));
    *v = (float *)malloc((nz ? nz : 1) * sizeof(float));
    if (*rp && *ci && *v)
    {
        memcpy(*rp, m.row_ptr->data, nr * sizeof(int32_t));
        memcpy(*ci, m.col_ind->data, nz * sizeof(int32_t));
        memcpy(*v, m.val->data, nz * sizeof(float));
    }
    vector_free(m.row_ptr);
    vector_free(m.col_ind);
    vector_free(m.val);
    return (*rp && *ci && *v) ? 0 : -6;
}

typedef struct
{
    int32_t r0, r1, a_cols, b_cols;
    const int32_t *a_rp, *a_ci, *b_rp, *b_ci;
    const float *a_v, *b_v;
    /* numeric-only inputs */
    const int32_t *c_rp, *c_ci;
    float *c_v;
    int repeats;
    int status;
    void *ws;
    size_t ws_bytes;
} panel_t;

static void *panel_oneshot(void *arg)
{
    panel_t *p = (panel_t *)arg;
    for (int rep = 0; rep < p->repeats; rep++)
    {
        int32_t *rp = NULL, *ci = NULL, nnz = 0;
        float *v = NULL;
        /* a_rp + r0: row offsets stay absolute into the shared col_idx. */
        p->status = rvsp_spgemm_scalar_f32(p->r1 - p->r0, p->a_cols, p->b_cols,
                                           p->a_rp + p->r0, p->a_ci, p->a_v,
                                           p->b_rp, p->b_ci, p->b_v,
                                           p->ws, p->ws_bytes, &rp, &ci, &v, &nnz, NULL);
        free(rp);
        free(ci);
        free(v);
    }
    return NULL;
}

static void *panel_numeric(void *arg)
{
    panel_t *p = (panel_t *)arg;
    float *acc = (float *)p->ws;
    memset(acc, 0, (size_t)p->b_cols * sizeof(float));
    for (int rep = 0; rep < p->repeats; rep++)
        rvsp_spgemm_scalar_f32_numeric(p->r1 - p->r0, p->a_rp + p->r0, p->a_ci, p->a_v,
                                       p->b_rp, p->b_ci, p->b_v, acc,
                                       p->c_rp + p->r0, p->c_ci, p->c_v);
    p->status = 0;
    return NULL;
}

/* Split rows so each panel carries about the same number of products. */
static void split_rows(int32_t row_begin, int32_t row_end, int nthreads,
                       const int32_t *a_rp, const int32_t *a_ci, const int32_t *b_rp,
                       int32_t *bounds)
{
    double total = 0.0;
    for (int32_t r = row_begin; r < row_end; r++)
        for (int32_t p = a_rp[r]; p < a_rp[r + 1]; p++)
            total += (double)(b_rp[a_ci[p] + 1] - b_rp[a_ci[p]]) + 1.0;
    bounds[0] = row_begin;
    int t = 1;
    double acc = 0.0;
    for (int32_t r = row_begin; r < row_end && t < nthreads; r++)
    {
        for (int32_t p = a_rp[r]; p < a_rp[r + 1]; p++)
            acc += (double)(b_rp[a_ci[p] + 1] - b_rp[a_ci[p]]) + 1.0;
        if (acc >= total * (double)t / (double)nthreads)
            bounds[t++] = r + 1;
    }
    while (t <= nthreads)
        bounds[t++] = row_end;
}

/*
 * Times `repeats` one-shot raw-kernel calls over rows [row_begin, row_end)
 * on `nthreads` threads (row panels). Returns wall seconds for all repeats.
 */
double ref_time_oneshot(int nthreads, int repeats, int32_t row_begin, int32_t row_end,
                        int32_t a_cols, int32_t b_cols,
                        const int32_t *a_rp, const int32_t *a_ci, const float *a_v,
                        const int32_t *b_rp, const int32_t *b_ci, const float *b_v)
{
    if (nthreads < 1)
        nthreads = 1;
    int32_t *bounds = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nthreads + 1));
    panel_t *ps = (panel_t *)calloc((size_t)nthreads, sizeof(panel_t));
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
    split_rows(row_begin, row_end, nthreads, a_rp, a_ci, b_rp, bounds);
    size_t ws_bytes = 0;
    rvsp_spgemm_buffer_size(b_cols, &ws_bytes);
    for (int t = 0; t < nthreads; t++)
    {
        ps[t] = (panel_t){bounds[t], bounds[t + 1], a_cols, b_cols, a_rp, a_ci, b_rp, b_ci,
                          a_v, b_v, NULL, NULL, NULL, repeats, 0, malloc(ws_bytes), ws_bytes};
    }
    double t0 = now_s();
    for (int t = 0; t < nthreads; t++)
        if (ps[t].r1 > ps[t].r0)
            pthread_create(&th[t], NULL, panel_oneshot, &ps[t]);
    for (int t = 0; t < nthreads; t++)
        if (ps[t].r1 > ps[t].r0)
            pthread_join(th[t], NULL);
    double dt = now_s() - t0;
    int bad = 0;
    for (int t = 0; t < nthreads; t++)
    {
        bad |= ps[t].status != 0;
        free(ps[t].ws);
    }
    free(bounds);
    free(ps);
    free(th);
    return bad ? -1.0 : dt;
}

/*
 * Times `repeats` numeric-only passes (the descriptor-reuse path: the
 * reference's numeric function with a fixed C pattern) over rows
 * [row_begin, row_end) on `nthreads` threads. c_rp is the full absolute C
 * row pointer; c_v receives the values. Returns wall seconds.
 */
double ref_time_numeric(int nthreads, int repeats, int32_t row_begin, int32_t row_end,
                        int32_t b_cols,
                        const int32_t *a_rp, const int32_t *a_ci, const float *a_v,
                        const int32_t *b_rp, const int32_t *b_ci, const float *b_v,
                        const int32_t *c_rp, const int32_t *c_ci, float *c_v)
{
    if (nthreads < 1)
        nthreads = 1;
    int32_t *bounds = (int32_t *)malloc(sizeof(int32_t) * (size_t)(nthreads + 1));
    panel_t *ps = (panel_t *)calloc((size_t)nthreads, sizeof(panel_t));
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)nthreads);
    split_rows(row_begin, row_end, nthreads, a_rp, a_ci, b_rp, bounds);
    for (int t = 0; t < nthreads; t++)
    {
        ps[t] = (panel_t){bounds[t], bounds[t + 1], 0, b_cols, a_rp, a_ci, b_rp, b_ci,
                          a_v, b_v, c_rp, c_ci, c_v, repeats, 0,
                          malloc((size_t)b_cols * sizeof(float)), 0};
    }
    double t0 = now_s();
    for (int t = 0; t < nthreads; t++)
        if (ps[t].r1 > ps[t].r0)
            pthread_create(&th[t], NULL, panel_numeric, &ps[t]);
    for (int t = 0; t < nthreads; t++)
        if (ps[t].r1 > ps[t].r0)
            pthread_join(th[t], NULL);
    double dt = now_s() - t0;
    for (int t = 0; t < nthreads; t++)
        free(ps[t].ws);
    free(bounds);
    free(ps);
    free(th);
    return dt;
}
