// COO -> canonical CSR on the device: the canonicalisation the reference's
// Matrix Market loader does on the host (rv-sparse
// tools/src/mtx_to_csr_formatter.c:219-330 and canonicalise_rows :74-151):
// symmetric storage expanded by appending the mirror of every off-diagonal
// entry after all stored ones (:221-244); entries bucketed by row in COO
// order (:246-300); each row sorted by column and repeated (row, column)
// entries summed (:112-131).
//
// Here: one stable LSD radix sort of the packed keys (row << cb | column)
// with the COO index as payload, so entries with equal keys stay in COO
// order; then each run of equal keys is summed left to right, starting from
// its first value like the reference (acc = first; acc += next ...), and the
// row pointer is read off the sorted rows. Every pass is a device kernel;
// the only host work is the launch sequence and one read of the output size.

#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <utility>

#include "rv_sparse_types.h"
#include "rvsp_cuda.h"
#include "rvsp_internal.h"

using namespace rvsp;

namespace {

constexpr int RS_TPB = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_TPB * RS_ITEMS;  // keys per block and pass
constexpr int RS_WARPS = RS_TPB / 32;

__device__ __forceinline__ int c_lane() { return threadIdx.x & 31; }

// Keys and payloads; the mirrored entries of a symmetric matrix go after the
// stored ones, in the stored order (mpos = exclusive scan of off-diagonal
// flags). Rows or columns out of range set *bad.
__global__ void k_coo_keys(int64_t n, int32_t rows, int32_t cols, int cb,
                           const int32_t* __restrict__ r, const int32_t* __restrict__ c,
                           int symmetric, const int64_t* __restrict__ mpos,
                           uint64_t* __restrict__ keys, int64_t* __restrict__ idx,
                           int32_t* __restrict__ bad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int32_t ri = r[i], ci = c[i];
    if ((unsigned)ri >= (unsigned)rows || (unsigned)ci >= (unsigned)cols ||
        (symmetric && ((unsigned)ci >= (unsigned)rows || (unsigned)ri >= (unsigned)cols))) {
        atomicOr(bad, 1);
        keys[i] = 0;
        idx[i] = i;
        return;
    }
    keys[i] = ((uint64_t)ri << cb) | (uint64_t)ci;
    idx[i] = i;
    if (symmetric && ri != ci) {
        const int64_t j = n + mpos[i];
        keys[j] = ((uint64_t)ci << cb) | (uint64_t)ri;
        idx[j] = i;  // the mirror carries the stored entry's value
    }
}

__global__ void k_offdiag(int64_t n, const int32_t* __restrict__ r, const int32_t* __restrict__ c,
                          int32_t* __restrict__ flag) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = r[i] != c[i];
}

// Per-block histogram of one 8-bit digit, digit-major: hist[d * blocks + b].
__global__ void __launch_bounds__(RS_TPB)
    k_rs_hist(int64_t n, const uint64_t* __restrict__ keys, int shift, int32_t* __restrict__ hist) {
    __shared__ int32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * RS_TILE;
    for (int k = 0; k < RS_ITEMS; ++k) {
        const int64_t i = base + (int64_t)k * RS_TPB + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255], 1);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * gridDim.x + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one digit: the block walks its tile in order, 256 keys
// at a time; within a step ranks follow warp then lane order (match_any per
// warp, per-digit warp counts prefix-summed by one thread per digit).
__global__ void __launch_bounds__(RS_TPB)
    k_rs_scatter(int64_t n, const uint64_t* __restrict__ keys, const int64_t* __restrict__ idx,
                 int shift, const int32_t* __restrict__ off, uint64_t* __restrict__ keys_out,
                 int64_t* __restrict__ idx_out) {
    __shared__ int32_t cursor[256];
    __shared__ int32_t wcnt[RS_WARPS][256];
    const int t = threadIdx.x, warp = t >> 5, lane = c_lane();
    cursor[t] = off[(int64_t)t * gridDim.x + blockIdx.x];
    for (int w = 0; w < RS_WARPS; ++w) wcnt[w][t] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * RS_TILE;
    for (int k = 0; k < RS_ITEMS; ++k) {
        const int64_t i = base + (int64_t)k * RS_TPB + t;
        const bool ok = i < n;
        uint64_t key = 0;
        int64_t pl = 0;
        int d = 256 + lane;  // idle lanes: keys no real digit matches
        if (ok) {
            key = keys[i];
            pl = idx[i];
            d = (int)((key >> shift) & 255);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int rank = __popc(peers & ((1u << lane) - 1));
        if (ok && lane == __ffs(peers) - 1) wcnt[warp][d] = __popc(peers);
        __syncthreads();
        // thread t: digit t's base for every warp of this step, in warp order
        int run = cursor[t];
        int wbase[RS_WARPS];
#pragma unroll
        for (int w = 0; w < RS_WARPS; ++w) {
            wbase[w] = run;
            run += wcnt[w][t];
        }
        __syncthreads();
#pragma unroll
        for (int w = 0; w < RS_WARPS; ++w) wcnt[w][t] = wbase[w];
        cursor[t] = run;
        __syncthreads();
        if (ok) {
            const int pos = wcnt[warp][d] + rank;
            keys_out[pos] = key;
            idx_out[pos] = pl;
        }
        __syncthreads();
        for (int w = 0; w < RS_WARPS; ++w) wcnt[w][t] = 0;
        __syncthreads();
    }
}

__global__ void k_run_heads(int64_t n, const uint64_t* __restrict__ keys,
                            int32_t* __restrict__ head) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) head[i] = i == 0 || keys[i] != keys[i - 1];
}

// One output entry per run of equal keys: its column, and the run's values
// summed in COO order from the first value (no added zero: a lone -0.0 stays).
__global__ void k_run_sum(int64_t n, const uint64_t* __restrict__ keys,
                          const int64_t* __restrict__ idx, const int32_t* __restrict__ head,
                          const int64_t* __restrict__ pos, int cb, const float* __restrict__ v,
                          int32_t* __restrict__ out_row, int32_t* __restrict__ out_ci,
                          float* __restrict__ out_v) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !head[i]) return;
    const uint64_t key = keys[i];
    float acc = v ? v[idx[i]] : 1.0f;
    for (int64_t j = i + 1; j < n && keys[j] == key; ++j) acc += v ? v[idx[j]] : 1.0f;
    const int64_t o = pos[i];
    out_row[o] = (int32_t)(key >> cb);
    out_ci[o] = (int32_t)(key & ((1ull << cb) - 1));
    out_v[o] = acc;
}

// Row pointer of the sorted output: entry o starts every row after the
// previous entry's row up to its own.
__global__ void k_row_ptr_from_rows(int64_t m, int32_t rows, const int32_t* __restrict__ out_row,
                                    int32_t* __restrict__ rp) {
    const int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (o > m) return;
    const int32_t cur = o < m ? out_row[o] : rows;
    const int32_t prev = o > 0 ? out_row[o - 1] : -1;
    for (int32_t r = prev + 1; r <= cur; ++r) rp[r] = (int32_t)o;
}

int bits_for(int64_t x) {  // bits to hold 0 .. x - 1
    int b = 0;
    while (b < 63 && ((int64_t)1 << b) < x) ++b;
    return b;
}

struct Bufs {
    cudaStream_t st;
    void* p[24] = {};
    int n = 0;
    template <class T>
    cudaError_t get(T** out, size_t bytes) {
        void* q = nullptr;
        cudaError_t e = cudaMallocAsync(&q, bytes ? bytes : 16, st);
        if (e == cudaSuccess) p[n++] = q;
        *out = static_cast<T*>(q);
        return e;
    }
    void release() {
        for (int i = 0; i < n; ++i) cudaFreeAsync(p[i], st);
        n = 0;
    }
};

thread_local rvsp_cuda_plan_t t_cplan = nullptr;
struct CooReaper {
    ~CooReaper() {
        if (t_cplan) rvsp_cuda_plan_destroy(t_cplan);
        t_cplan = nullptr;
    }
};
thread_local CooReaper t_creaper;

}  // namespace

extern "C" int rvsp_cuda_coo_to_csr(int32_t rows, int32_t cols, int64_t n, const int32_t* coo_row,
                                    const int32_t* coo_col, const float* coo_val, int symmetric,
                                    int device_out, int32_t** row_ptr_out, int32_t** col_idx_out,
                                    float** values_out, int32_t* nnz_out) {
    if (!row_ptr_out || !col_idx_out || !values_out || !nnz_out) return RVSP_ERROR_NULL_POINTER;
    if (n > 0 && (!coo_row || !coo_col)) return RVSP_ERROR_NULL_POINTER;
    if (rows <= 0 || cols <= 0 || n < 0) return RVSP_ERROR_INVALID_ARGUMENT;
    if (symmetric && rows != cols) return RVSP_ERROR_INVALID_ARGUMENT;
    *row_ptr_out = nullptr;
    *col_idx_out = nullptr;
    *values_out = nullptr;
    *nnz_out = 0;
    if (rvsp_cuda_device_count() == 0) return RVSP_ERROR_UNSUPPORTED_BACKEND;
    const int64_t total = symmetric ? 2 * n : n;  // upper bound of the expanded count
    if (total >= INT32_MAX) return RVSP_ERROR_ALLOCATION_FAILED;
    int st;
    if (!t_cplan) {
        if ((st = rvsp_cuda_plan_create(&t_cplan, RVSP_CUDA_ALGO_EXACT))) return st;
    }
    rvsp_cuda_plan_t plan = t_cplan;
    cudaStream_t s = plan->stream;
    keep_pool_memory();
    cudaError_t e;
    if ((e = plan->misc.ensure(sizeof(Misc))) != cudaSuccess) return fail(e, "misc");
    Misc* misc = plan->misc.as<Misc>();
    cudaMemsetAsync(misc, 0, sizeof(Misc), s);
    const bool dev = n > 0 && is_dev(coo_row);
    Bufs b{s};
    auto bail = [&](int code) {
        b.release();
        cudaStreamSynchronize(s);
        return code;
    };
    const int32_t *d_r = coo_row, *d_c = coo_col;
    const float* d_v = coo_val;
    if (n > 0 && !dev) {
        int32_t *tr, *tc;
        float* tv = nullptr;
        if ((e = b.get(&tr, 4 * (size_t)n)) || (e = b.get(&tc, 4 * (size_t)n)) ||
            (coo_val && (e = b.get(&tv, 4 * (size_t)n))))
            return bail(fail(e, "COO staging"));
        cudaMemcpyAsync(tr, coo_row, 4 * (size_t)n, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(tc, coo_col, 4 * (size_t)n, cudaMemcpyHostToDevice, s);
        if (coo_val) cudaMemcpyAsync(tv, coo_val, 4 * (size_t)n, cudaMemcpyHostToDevice, s);
        d_r = tr, d_c = tc, d_v = tv;
    }
    const int cb = bits_for(cols), rb = bits_for(rows);
    const int passes = (cb + rb + 7) / 8;
    uint64_t *k0, *k1;
    int64_t *i0, *i1, *mpos, *opos;
    int32_t *flag, *hist, *hoff, *head, *out_row, *rp, *ci;
    float* v;
    const int64_t nb = (total + RS_TILE - 1) / RS_TILE;
    if ((e = b.get(&k0, 8 * (size_t)total)) || (e = b.get(&k1, 8 * (size_t)total)) ||
        (e = b.get(&i0, 8 * (size_t)total)) || (e = b.get(&i1, 8 * (size_t)total)) ||
        (e = b.get(&mpos, 8 * ((size_t)n + 1))) || (e = b.get(&flag, 4 * (size_t)n)) ||
        (e = b.get(&hist, 4 * 256 * (size_t)nb)) || (e = b.get(&hoff, 4 * (256 * (size_t)nb + 1))) ||
        (e = b.get(&head, 4 * (size_t)total)) || (e = b.get(&opos, 8 * ((size_t)total + 1))) ||
        (e = b.get(&out_row, 4 * (size_t)total)))
        return bail(fail(e, "COO scratch"));
    // expanded count
    int64_t m = n;
    if (symmetric && n > 0) {
        k_offdiag<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, d_r, d_c, flag);
        if ((st = scan_counts(plan, flag, n, mpos, nullptr, &misc->scan_total2))) return bail(st);
        if ((e = cudaMemcpyAsync(&m, &misc->scan_total2, 8, cudaMemcpyDeviceToHost, s)) ||
            (e = cudaStreamSynchronize(s)))
            return bail(fail(e, "symmetric count"));
        m += n;
    }
    if (n > 0)
        k_coo_keys<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, rows, cols, cb, d_r, d_c,
                                                               symmetric, mpos, k0, i0, &misc->err);
    const int64_t mb = (m + RS_TILE - 1) / RS_TILE;
    for (int p = 0; p < passes && m > 0; ++p) {
        k_rs_hist<<<(unsigned)mb, RS_TPB, 0, s>>>(m, k0, 8 * p, hist);
        if ((st = scan_counts(plan, hist, 256 * mb, nullptr, hoff, &misc->tile_total)))
            return bail(st);
        k_rs_scatter<<<(unsigned)mb, RS_TPB, 0, s>>>(m, k0, i0, 8 * p, hoff, k1, i1);
        std::swap(k0, k1);
        std::swap(i0, i1);
    }
    int64_t out_n = 0;
    if (m > 0) {
        k_run_heads<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(m, k0, head);
        if ((st = scan_counts(plan, head, m, opos, nullptr, &misc->scan_total))) return bail(st);
    }
    int32_t bad = 0;
    if ((e = cudaMemcpyAsync(&out_n, &misc->scan_total, 8, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(&bad, &misc->err, 4, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaStreamSynchronize(s)))
        return bail(fail(e, "COO sort"));
    if (m == 0) out_n = 0;
    if (bad) {
        g_err = "COO row or column index out of range";
        return bail(RVSP_ERROR_INVALID_ARGUMENT);
    }
    const size_t on = (size_t)(out_n > 0 ? out_n : 1);
    rp = ci = nullptr;
    v = nullptr;
    if ((e = cudaMallocAsync((void**)&rp, 4 * ((size_t)rows + 1), s)) ||
        (e = cudaMallocAsync((void**)&ci, 4 * on, s)) || (e = cudaMallocAsync((void**)&v, 4 * on, s))) {
        if (rp) cudaFreeAsync(rp, s);
        if (ci) cudaFreeAsync(ci, s);
        return bail(fail(e, "CSR alloc"));
    }
    if (m > 0)
        k_run_sum<<<(unsigned)((m + 255) / 256), 256, 0, s>>>(m, k0, i0, head, opos, cb, d_v,
                                                              out_row, ci, v);
    k_row_ptr_from_rows<<<(unsigned)((out_n + 256) / 256), 256, 0, s>>>(out_n, rows, out_row, rp);
    b.release();
    if ((e = cudaGetLastError()) != cudaSuccess) {
        cudaFreeAsync(rp, s);
        cudaFreeAsync(ci, s);
        cudaFreeAsync(v, s);
        cudaStreamSynchronize(s);
        return fail(e, "COO launch");
    }
    if (!device_out) {
        int32_t* hrp = (int32_t*)malloc(4 * ((size_t)rows + 1));
        int32_t* hci = (int32_t*)malloc(4 * on);
        float* hv = (float*)malloc(4 * on);
        if (!hrp || !hci || !hv) {
            free(hrp);
            free(hci);
            free(hv);
            cudaFreeAsync(rp, s);
            cudaFreeAsync(ci, s);
            cudaFreeAsync(v, s);
            cudaStreamSynchronize(s);
            return RVSP_ERROR_ALLOCATION_FAILED;
        }
        cudaMemcpyAsync(hrp, rp, 4 * ((size_t)rows + 1), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(hci, ci, 4 * (size_t)out_n, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(hv, v, 4 * (size_t)out_n, cudaMemcpyDeviceToHost, s);
        cudaFreeAsync(rp, s);
        cudaFreeAsync(ci, s);
        cudaFreeAsync(v, s);
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) {
            free(hrp);
            free(hci);
            free(hv);
            return fail(e, "CSR copy-out");
        }
        rp = hrp, ci = hci, v = hv;
    } else if ((e = cudaStreamSynchronize(s)) != cudaSuccess) {
        return fail(e, "COO to CSR");
    }
    *row_ptr_out = rp;
    *col_idx_out = ci;
    *values_out = v;
    *nnz_out = (int32_t)out_n;
    return RVSP_SUCCESS;
}
