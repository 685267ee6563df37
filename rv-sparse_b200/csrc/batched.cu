// Batched products: C_i = A_i * B_i for many independent, uneven products in
// one pipeline instead of one pipeline (and two host round trips) each.
//
// The operands are packed once on the device into block-stacked matrices:
//   A = [A_1; A_2; ...]  with A_i's column indices shifted by K_1 + ... + K_{i-1}
//   B = [B_1; B_2; ...]  with B_i's column indices kept as they are
// Row r of A_i then references only rows of B_i, so row r of the stacked
// product is row r of C_i with C_i's own column indices, and
// C = A * B is [C_1; C_2; ...]. The stacked product runs through the normal
// plan (exact or learned): one analysis, one stable binning of every row of
// every product by size, one launch per bin and phase, so small and large
// products share the same work queues. Per-product results are row ranges
// of the packed C.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "rv_sparse_types.h"
#include "rvsp_cuda.h"
#include "rvsp_internal.h"

using namespace rvsp;

namespace {

struct PackSrc {
    const int32_t* rp;
    const int32_t* ci;
    const float* v;
    int32_t rows;
    int32_t nnz;
    int64_t row_off;  // first packed row
    int64_t nnz_off;  // first packed entry
    int32_t col_shift;
    int32_t pad;
};

constexpr int PACK_TILE = 1024;

// One block per PACK_TILE entries (or rows) of one product; tile_start maps
// blocks to products (host-built prefix, searched per block).
__global__ void __launch_bounds__(256)
    k_pack(const PackSrc* __restrict__ src, const int64_t* __restrict__ tile_start, int32_t count,
           int32_t* __restrict__ rp, int32_t* __restrict__ ci, float* __restrict__ v) {
    const int64_t blk = blockIdx.x;
    int lo = 0, hi = count;  // product i with tile_start[i] <= blk < tile_start[i+1]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (tile_start[mid] <= blk) lo = mid; else hi = mid;
    }
    const PackSrc s = src[lo];
    const int64_t t = blk - tile_start[lo];
    const int64_t span = max((int64_t)s.nnz, (int64_t)s.rows + 1);
    for (int64_t j = t * PACK_TILE + threadIdx.x; j < min((t + 1) * PACK_TILE, span);
         j += blockDim.x) {
        if (j < s.nnz) {
            ci[s.nnz_off + j] = s.ci[j] + s.col_shift;
            v[s.nnz_off + j] = s.v[j];
        }
        if (j < s.rows) rp[s.row_off + j] = (int32_t)(s.rp[j] + s.nnz_off);
    }
    if (lo == count - 1 && t == 0 && threadIdx.x == 0)
        rp[s.row_off + s.rows] = (int32_t)(s.nnz_off + s.nnz);
}

struct Packed {
    int32_t *rp = nullptr, *ci = nullptr;
    float* v = nullptr;
};

// Packs `count` CSR operands (device arrays) into one stacked CSR.
int pack(cudaStream_t st, int32_t count, const int32_t* rows, const int32_t* nnz,
         const int32_t* const* rp, const int32_t* const* ci, const float* const* v,
         const int32_t* col_shift, Packed* out, int64_t* total_rows, int64_t* total_nnz) {
    std::vector<PackSrc> src(count);
    std::vector<int64_t> tiles(count + 1, 0);
    int64_t r = 0, z = 0;
    for (int32_t i = 0; i < count; ++i) {
        src[i] = PackSrc{rp[i], ci[i], v[i], rows[i], nnz[i], r, z, col_shift ? col_shift[i] : 0, 0};
        const int64_t span = std::max<int64_t>(nnz[i], (int64_t)rows[i] + 1);
        tiles[i + 1] = tiles[i] + (span + PACK_TILE - 1) / PACK_TILE;
        r += rows[i];
        z += nnz[i];
    }
    if (r > INT32_MAX || z > INT32_MAX) {
        g_err = "batched operands exceed int32 rows or nnz";
        return RVSP_ERROR_ALLOCATION_FAILED;
    }
    *total_rows = r;
    *total_nnz = z;
    void* dsrc = nullptr;
    void* dtiles = nullptr;
    cudaError_t e = cudaMallocAsync(&dsrc, sizeof(PackSrc) * count, st);
    if (e == cudaSuccess) e = cudaMallocAsync(&dtiles, 8 * (count + 1), st);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&out->rp, 4 * (r + 1), st);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&out->ci, 4 * std::max<int64_t>(z, 1), st);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&out->v, 4 * std::max<int64_t>(z, 1), st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dsrc, src.data(), sizeof(PackSrc) * count, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dtiles, tiles.data(), 8 * (count + 1), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        k_pack<<<(unsigned)tiles[count], 256, 0, st>>>((const PackSrc*)dsrc, (const int64_t*)dtiles,
                                                       count, out->rp, out->ci, out->v);
        note_launch(nullptr, 1);
        e = cudaGetLastError();
    }
    if (dsrc) cudaFreeAsync(dsrc, st);
    if (dtiles) cudaFreeAsync(dtiles, st);
    return e == cudaSuccess ? RVSP_SUCCESS : fail(e, "batched pack");
}

void release(cudaStream_t st, Packed& p) {
    if (p.rp) cudaFreeAsync(p.rp, st);
    if (p.ci) cudaFreeAsync(p.ci, st);
    if (p.v) cudaFreeAsync(p.v, st);
    p = Packed{};
}

thread_local rvsp_cuda_plan_t t_bplan[2] = {nullptr, nullptr};

struct BatchReaper {
    ~BatchReaper() {
        for (auto& p : t_bplan)
            if (p) {
                rvsp_cuda_plan_destroy(p);
                p = nullptr;
            }
    }
};
thread_local BatchReaper t_breaper;

}  // namespace

extern "C" int rvsp_cuda_spgemm_batched_f32(
    int algo, int32_t count, const int32_t* a_rows, const int32_t* a_cols, const int32_t* b_cols,
    const int32_t* a_nnz, const int32_t* b_nnz, const int32_t* const* a_row_ptr,
    const int32_t* const* a_col_idx,
    const float* const* a_values, const int32_t* const* b_row_ptr,
    const int32_t* const* b_col_idx, const float* const* b_values, int32_t** c_row_ptr_out,
    int32_t** c_col_idx_out, float** c_values_out, int64_t* c_nnz_out, int64_t* row_offsets_out) {
    if (!a_rows || !a_cols || !b_cols || !a_nnz || !b_nnz || !a_row_ptr || !a_col_idx || !a_values || !b_row_ptr ||
        !b_col_idx || !b_values || !c_row_ptr_out || !c_col_idx_out || !c_values_out ||
        !c_nnz_out || !row_offsets_out)
        return RVSP_ERROR_NULL_POINTER;
    if (count <= 0) return RVSP_ERROR_INVALID_ARGUMENT;
    if (algo != RVSP_CUDA_ALGO_EXACT && algo != RVSP_CUDA_ALGO_LEARNED)
        return RVSP_ERROR_UNSUPPORTED_BACKEND;
    if (algo == RVSP_CUDA_ALGO_LEARNED && !rvsp_cuda_learned_available())
        return RVSP_ERROR_UNSUPPORTED_BACKEND;
    *c_row_ptr_out = nullptr;
    *c_col_idx_out = nullptr;
    *c_values_out = nullptr;
    *c_nnz_out = 0;
    int st;
    rvsp_cuda_plan_t& plan = t_bplan[algo == RVSP_CUDA_ALGO_LEARNED ? 1 : 0];
    if (!plan) {
        if ((st = rvsp_cuda_plan_create(&plan, algo))) return st;
        plan->map_policy = 0;
    }
    plan->params = default_params();
    keep_pool_memory();
    std::vector<int32_t> a_shift(count), b_rows(count);
    int64_t kshift = 0;
    int32_t max_n = 1;
    for (int32_t i = 0; i < count; ++i) {
        if (a_rows[i] <= 0 || a_cols[i] <= 0 || b_cols[i] <= 0 || a_nnz[i] < 0 || b_nnz[i] < 0)
            return RVSP_ERROR_INVALID_ARGUMENT;
        if (!a_row_ptr[i] || !a_col_idx[i] || !a_values[i] || !b_row_ptr[i] || !b_col_idx[i] ||
            !b_values[i])
            return RVSP_ERROR_NULL_POINTER;
        if (!is_dev(a_row_ptr[i]) || !is_dev(b_row_ptr[i])) {
            g_err = "batched operands must be device-resident";
            return RVSP_ERROR_INVALID_ARGUMENT;
        }
        b_rows[i] = a_cols[i];
        a_shift[i] = (int32_t)kshift;
        kshift += a_cols[i];
        max_n = std::max(max_n, b_cols[i]);
    }
    if (kshift > INT32_MAX) return RVSP_ERROR_ALLOCATION_FAILED;
    Packed pa, pb;
    int64_t ar = 0, az = 0, br = 0, bz = 0;
    if ((st = pack(plan->stream, count, a_rows, a_nnz, a_row_ptr, a_col_idx, a_values,
                   a_shift.data(), &pa, &ar, &az)) ||
        (st = pack(plan->stream, count, b_rows.data(), b_nnz, b_row_ptr, b_col_idx, b_values,
                   nullptr, &pb, &br, &bz))) {
        release(plan->stream, pa);
        release(plan->stream, pb);
        cudaStreamSynchronize(plan->stream);
        return st;
    }
    int32_t *rp = nullptr, *ci = nullptr, nnz = 0;
    float* v = nullptr;
    if (algo == RVSP_CUDA_ALGO_LEARNED) {
        st = learned_spgemm(plan, (int32_t)ar, (int32_t)kshift, (int32_t)az, pa.rp, pa.ci, pa.v,
                            (int32_t)br, max_n, (int32_t)bz, pb.rp, pb.ci, pb.v, 1, &rp, &ci, &v,
                            &nnz);
    } else {
        int64_t n64 = 0;
        size_t ws = 0;
        st = rvsp_cuda_symbolic(plan, (int32_t)ar, (int32_t)kshift, (int32_t)az, pa.rp, pa.ci,
                                (int32_t)br, max_n, (int32_t)bz, pb.rp, pb.ci, &n64, &ws);
        if (!st) {
            const size_t alloc = n64 > 0 ? (size_t)n64 : 1;
            cudaError_t e = cudaMallocAsync((void**)&rp, (ar + 1) * 4, plan->stream);
            if (e == cudaSuccess) e = cudaMallocAsync((void**)&ci, alloc * 4, plan->stream);
            if (e == cudaSuccess) e = cudaMallocAsync((void**)&v, alloc * 4, plan->stream);
            st = e == cudaSuccess ? rvsp_cuda_numeric(plan, pa.rp, pa.ci, pa.v, pb.rp, pb.ci, pb.v,
                                                      rp, ci, v, 1, nullptr)
                                  : fail(e, "batched C");
            nnz = (int32_t)n64;
        }
    }
    release(plan->stream, pa);
    release(plan->stream, pb);
    cudaError_t e = cudaStreamSynchronize(plan->stream);
    if (st || e != cudaSuccess) {
        if (rp) cudaFree(rp);
        if (ci) cudaFree(ci);
        if (v) cudaFree(v);
        return st ? st : fail(e, "batched");
    }
    int64_t off = 0;
    for (int32_t i = 0; i < count; ++i) {
        row_offsets_out[i] = off;
        off += a_rows[i];
    }
    row_offsets_out[count] = off;
    *c_row_ptr_out = rp;
    *c_col_idx_out = ci;
    *c_values_out = v;
    *c_nnz_out = nnz;
    return RVSP_SUCCESS;
}
