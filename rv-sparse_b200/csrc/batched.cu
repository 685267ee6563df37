// Batched products: C_i = A_i * B_i for many independent, uneven products in
// one call instead of one pipeline (and its host round trips) each.
//
// The operands are packed once on the device into block-stacked matrices:
//   A = [A_1; A_2; ...]  with A_i's column indices shifted by K_1 + ... + K_{i-1}
//   B = [B_1; B_2; ...]  with B_i's column indices kept as they are
// Row r of A_i then references only rows of B_i, so row r of the stacked
// product is row r of C_i with C_i's own column indices. One kernel counts
// every product's intermediate products; consecutive products are grouped so
// each group's C fits an int32 row pointer (a group's products bound its
// nnz), and each group runs the normal plan (exact or learned) as one row
// panel of the stacked A against the whole stacked B: one analysis, one
// stable binning of every row of every product in the group by size, one
// launch per bin and phase, so small and large products share the same work
// queues. All groups are analysed first; then one C is allocated for all
// products and every group fills its part. A last kernel rewrites each
// group's row pointer as every product's own row pointer (from 0) and records
// where each product's entries start (int64), so the total nnz is not bound
// by int32.

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
// An operand whose row pointer does not start at 0 (a row panel) flags
// ERR_STRUCTURE: the batched entry point takes whole matrices only.
__global__ void __launch_bounds__(256)
    k_pack(const PackSrc* __restrict__ src, const int64_t* __restrict__ tile_start, int32_t count,
           int32_t* __restrict__ rp, int32_t* __restrict__ ci, float* __restrict__ v,
           int32_t* __restrict__ err) {
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
    if (t == 0 && threadIdx.x == 0 && s.rp[0] != 0) atomicOr(err, ERR_STRUCTURE);
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
         const int32_t* col_shift, Packed* out, int64_t* total_rows, int64_t* total_nnz,
         int32_t* err) {
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
        KTime kt(st, false, KF_PACK);
        k_pack<<<(unsigned)tiles[count], 256, 0, st>>>((const PackSrc*)dsrc, (const int64_t*)dtiles,
                                                       count, out->rp, out->ci, out->v, err);
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

// Intermediate products of each packed product: block i sums the B-row
// lengths its A entries [a_off[i], a_off[i + 1]) reference (B rows are the
// stacked B's: A's columns were shifted when packing).
__global__ void __launch_bounds__(256)
    k_product_ops(const int64_t* __restrict__ a_off, const int32_t* __restrict__ aci,
                  const int32_t* __restrict__ brp, int32_t b_rows, int64_t* __restrict__ ops,
                  int32_t* __restrict__ err) {
    __shared__ unsigned long long s_sum;
    if (threadIdx.x == 0) s_sum = 0;
    __syncthreads();
    const int i = blockIdx.x;
    unsigned long long sum = 0;
    for (int64_t j = a_off[i] + threadIdx.x; j < a_off[i + 1]; j += blockDim.x) {
        const int k = aci[j];
        if ((unsigned)k >= (unsigned)b_rows) {
            atomicOr(err, ERR_STRUCTURE);
            continue;
        }
        const int len = brp[k + 1] - brp[k];
        if (len > 0) sum += (unsigned long long)len;
    }
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(FULL, sum, o);
    if ((threadIdx.x & 31) == 0 && sum) atomicAdd(&s_sum, sum);
    __syncthreads();
    if (threadIdx.x == 0) ops[i] = (int64_t)s_sum;
}

// Every product's own row pointer from its group's: slot s of the group
// (product i, row r of rows_i + 1) gets grp_rp[first_i + r] - grp_rp[first_i]
// at out_rp[out_i + r]; the r == 0 slot records where product i's entries
// start in the common C (base + grp_rp[first_i]). prod_* are the group's
// products: their first slot in the group, first row in the group, first
// slot in out_rp.
__global__ void __launch_bounds__(256)
    k_product_rows(int32_t n_prod, const int64_t* __restrict__ slot0,
                   const int32_t* __restrict__ row0, const int64_t* __restrict__ out0,
                   const int32_t* __restrict__ grp_rp, int64_t base, int32_t* __restrict__ out_rp,
                   int64_t* __restrict__ c_off) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= slot0[n_prod]) return;
    int lo = 0, hi = n_prod;  // product i with slot0[i] <= s < slot0[i + 1]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (slot0[mid] <= s) lo = mid; else hi = mid;
    }
    const int r = (int)(s - slot0[lo]);
    const int32_t first = grp_rp[row0[lo]];
    out_rp[out0[lo] + r] = grp_rp[row0[lo] + r] - first;
    if (r == 0) c_off[lo] = base + first;
}

// Plans of the groups, kept per thread between calls (their device buffers
// are reused).
thread_local std::vector<rvsp_cuda_plan_t> t_bplans[2];

struct BatchReaper {
    ~BatchReaper() {
        for (auto& v : t_bplans)
            for (auto& p : v)
                if (p) rvsp_cuda_plan_destroy(p);
    }
};
thread_local BatchReaper t_breaper;

struct Group {
    int32_t first, last;  // products [first, last)
    int32_t row0, rows;   // rows of the stacked A
    int64_t base;         // first entry in the common C
};

}  // namespace

extern "C" int rvsp_cuda_spgemm_batched_f32(
    int algo, int32_t count, const int32_t* a_rows, const int32_t* a_cols, const int32_t* b_cols,
    const int32_t* a_nnz, const int32_t* b_nnz, const int32_t* const* a_row_ptr,
    const int32_t* const* a_col_idx, const float* const* a_values,
    const int32_t* const* b_row_ptr, const int32_t* const* b_col_idx,
    const float* const* b_values, int32_t** c_row_ptr_out, int32_t** c_col_idx_out,
    float** c_values_out, int64_t* c_nnz_out, int64_t* row_offsets_out, int64_t* c_offsets_out) {
    if (!a_rows || !a_cols || !b_cols || !a_nnz || !b_nnz || !a_row_ptr || !a_col_idx ||
        !a_values || !b_row_ptr || !b_col_idx || !b_values || !c_row_ptr_out || !c_col_idx_out ||
        !c_values_out || !c_nnz_out || !row_offsets_out || !c_offsets_out)
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
    std::vector<rvsp_cuda_plan_t>& plans = t_bplans[algo == RVSP_CUDA_ALGO_LEARNED ? 1 : 0];
    int st;
    if (plans.empty()) {
        rvsp_cuda_plan_t p = nullptr;
        if ((st = rvsp_cuda_plan_create(&p, algo))) return st;
        p->map_policy = 0;
        plans.push_back(p);
    }
    cudaStream_t s0 = plans[0]->stream;
    keep_pool_memory();
    Packed pa, pb;
    int64_t ar = 0, az = 0, br = 0, bz = 0;
    std::vector<int64_t> ops(count), a_off(count + 1, 0);
    for (int32_t i = 0; i < count; ++i) a_off[i + 1] = a_off[i] + a_nnz[i];
    int32_t *rp = nullptr, *ci = nullptr;
    float* v = nullptr;
    int64_t* c_off_dev = nullptr;
    auto cleanup = [&](int status) {
        release(s0, pa);
        release(s0, pb);
        if (status) {
            if (rp) cudaFreeAsync(rp, s0);
            if (ci) cudaFreeAsync(ci, s0);
            if (v) cudaFreeAsync(v, s0);
        }
        if (c_off_dev) cudaFreeAsync(c_off_dev, s0);
        cudaStreamSynchronize(s0);
        return status;
    };
    cudaError_t e0 = plans[0]->misc.ensure(sizeof(Misc));
    if (e0 == cudaSuccess) e0 = cudaMemsetAsync(&plans[0]->misc.as<Misc>()->err, 0, 4, s0);
    if (e0 != cudaSuccess) return cleanup(fail(e0, "batched"));
    Misc* misc = plans[0]->misc.as<Misc>();
    if ((st = pack(s0, count, a_rows, a_nnz, a_row_ptr, a_col_idx, a_values, a_shift.data(), &pa,
                   &ar, &az, &misc->err)) ||
        (st = pack(s0, count, b_rows.data(), b_nnz, b_row_ptr, b_col_idx, b_values, nullptr, &pb,
                   &br, &bz, &misc->err)))
        return cleanup(st);

    // every product's intermediate products, then the groups
    {
        int64_t* d = nullptr;
        cudaError_t e = cudaMallocAsync((void**)&d, 8 * (2 * (size_t)count + 1), s0);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d + count, a_off.data(), 8 * ((size_t)count + 1),
                                cudaMemcpyHostToDevice, s0);
        if (e == cudaSuccess) {
            k_product_ops<<<count, 256, 0, s0>>>(d + count, pa.ci, pb.rp, (int32_t)br, d,
                                                  &misc->err);
            note_launch(nullptr, 1);
            e = cudaGetLastError();
        }
        int32_t err = 0;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(ops.data(), d, 8 * (size_t)count, cudaMemcpyDeviceToHost, s0);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&err, &misc->err, 4, cudaMemcpyDeviceToHost, s0);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s0);
        if (d) cudaFreeAsync(d, s0);
        if (e != cudaSuccess) return cleanup(fail(e, "batched product counts"));
        if (err) {
            g_err = "operand structure out of range (row_ptr or col_idx)";
            return cleanup(RVSP_ERROR_INVALID_CSR);
        }
    }
    std::vector<Group> groups;
    {
        int64_t acc = 0, row = 0;
        for (int32_t i = 0; i < count; ++i) {
            if (groups.empty() || (acc + ops[i] > INT32_MAX && groups.back().last > groups.back().first)) {
                groups.push_back(Group{i, i, (int32_t)row, 0, 0});
                acc = 0;
            }
            groups.back().last = i + 1;
            groups.back().rows += a_rows[i];
            acc += ops[i];
            row += a_rows[i];
        }
    }
    while (plans.size() < groups.size()) {
        rvsp_cuda_plan_t p = nullptr;
        if ((st = rvsp_cuda_plan_create(&p, algo))) return cleanup(st);
        p->map_policy = 0;
        plans.push_back(p);
    }
    // analysis of every group (the learned path also fills its slots here):
    // group g is rows [row0, row0 + rows) of the stacked A, a row panel whose
    // row pointer indexes the stacked arrays, against the whole stacked B
    std::vector<CsrView> As(groups.size());
    CsrView Bv{pb.rp, pb.ci, pb.v, (int32_t)br, max_n, (int32_t)bz};
    int64_t total = 0;
    for (size_t g = 0; g < groups.size(); ++g) {
        Group& G = groups[g];
        rvsp_cuda_plan* plan = plans[g];
        plan->params = default_params();
        plan->analysed = false;
        plan->maps_ready = false;
        plan->filled = nullptr;
        plan->filled_host = nullptr;
        reset_graph(plan);
        plan->a_rows = G.rows;
        plan->a_cols = (int32_t)kshift;
        plan->a_nnz = (int32_t)a_off[G.last];  // panel: the end offset bounds the entries
        plan->b_rows = (int32_t)br;
        plan->b_cols = max_n;
        plan->b_nnz = (int32_t)bz;
        memset(plan->key, 0, sizeof(plan->key));
        // the plan's stream starts after the packing on the first plan's stream
        cudaEvent_t ev = nullptr;
        cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(ev, s0);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(plan->stream, ev, 0);
        if (ev) cudaEventDestroy(ev);
        if (e != cudaSuccess) return cleanup(fail(e, "batched streams"));
        As[g] = CsrView{pa.rp + G.row0, pa.ci, pa.v, G.rows, (int32_t)kshift, plan->a_nnz};
        if (algo == RVSP_CUDA_ALGO_LEARNED) {
            st = learned_symbolic(plan, As[g], Bv, true);
        } else {
            st = analyze(plan, As[g], Bv, false);
            if (!st) st = count_exact(plan, As[g], Bv);
        }
        if (st) return cleanup(st);
        plan->analysed = true;
        G.base = total;
        total += plan->c_nnz;
    }
    // one C for every product; every group fills its part
    const int64_t slots = ar + count;
    cudaError_t e = cudaMallocAsync((void**)&rp, 4 * (size_t)slots, s0);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&ci, 4 * (size_t)std::max<int64_t>(total, 1), s0);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&v, 4 * (size_t)std::max<int64_t>(total, 1), s0);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&c_off_dev, 8 * ((size_t)count + 1), s0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s0);  // C exists before other streams write it
    if (e != cudaSuccess) return cleanup(fail(e, "batched C"));
    for (size_t g = 0; g < groups.size(); ++g) {
        const Group& G = groups[g];
        rvsp_cuda_plan* plan = plans[g];
        int32_t* gci = ci + G.base;
        float* gv = v + G.base;
        if (plan->c_nnz > 0) {
            if (algo == RVSP_CUDA_ALGO_LEARNED) {
                st = learned_finish(plan, As[g], Bv, gci, gv);
            } else {
                RowOut o{nullptr, plan->c_rp.as<int32_t>(), gci, gv, &plan->misc.as<Misc>()->err,
                         false};
                run_rows(plan, FILL, As[g], Bv, o);
                st = RVSP_SUCCESS;
            }
            if (st) return cleanup(st);
        }
        // the group's products: first slot in the group, first row, first out slot
        const int32_t np = G.last - G.first;
        std::vector<int64_t> meta(3 * (size_t)np + 1);
        int64_t* slot0 = meta.data();           // [np + 1]
        int64_t* out0 = meta.data() + np + 1;   // [np]
        std::vector<int32_t> row0(np);
        int64_t sl = 0, r = 0;
        for (int32_t k = 0; k < np; ++k) {
            const int32_t i = G.first + k;
            slot0[k] = sl;
            row0[k] = (int32_t)r;
            out0[k] = (int64_t)(G.row0 + r) + i;
            sl += a_rows[i] + 1;
            r += a_rows[i];
        }
        slot0[np] = sl;
        void* dm = nullptr;
        e = cudaMallocAsync(&dm, 8 * (2 * (size_t)np + 1) + 4 * (size_t)np, plan->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dm, meta.data(), 8 * (2 * (size_t)np + 1), cudaMemcpyHostToDevice,
                                plan->stream);
        int32_t* drow0 = reinterpret_cast<int32_t*>(static_cast<int64_t*>(dm) + 2 * np + 1);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(drow0, row0.data(), 4 * (size_t)np, cudaMemcpyHostToDevice,
                                plan->stream);
        if (e == cudaSuccess) {
            const int64_t* dslot0 = static_cast<int64_t*>(dm);
            k_product_rows<<<(unsigned)((sl + 255) / 256), 256, 0, plan->stream>>>(
                np, dslot0, drow0, dslot0 + np + 1, plan->c_rp.as<int32_t>(), G.base, rp,
                c_off_dev + G.first);
            note_launch(nullptr, 1);
            e = cudaGetLastError();
        }
        // the host copies of meta / row0 must outlive the copies above
        if (e == cudaSuccess) e = cudaStreamSynchronize(plan->stream);
        if (dm) cudaFreeAsync(dm, plan->stream);
        if (e != cudaSuccess) return cleanup(fail(e, "batched row pointers"));
    }
    int32_t err = 0;
    for (size_t g = 0; g < groups.size(); ++g) {
        int32_t ge = 0;
        e = cudaMemcpyAsync(&ge, &plans[g]->misc.as<Misc>()->err, 4, cudaMemcpyDeviceToHost,
                            plans[g]->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(plans[g]->stream);
        if (e != cudaSuccess) return cleanup(fail(e, "batched"));
        err |= ge;
    }
    if (err) {
        g_err = "operand structure out of range (row_ptr or col_idx)";
        return cleanup(RVSP_ERROR_INVALID_CSR);
    }
    e = cudaMemcpyAsync(c_offsets_out, c_off_dev, 8 * (size_t)count, cudaMemcpyDeviceToHost, s0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s0);
    if (e != cudaSuccess) return cleanup(fail(e, "batched offsets"));
    c_offsets_out[count] = total;
    int64_t off = 0;
    for (int32_t i = 0; i < count; ++i) {
        row_offsets_out[i] = off;
        off += a_rows[i];
    }
    row_offsets_out[count] = off;
    *c_row_ptr_out = rp;
    *c_col_idx_out = ci;
    *c_values_out = v;
    *c_nnz_out = total;
    return cleanup(RVSP_SUCCESS);
}
