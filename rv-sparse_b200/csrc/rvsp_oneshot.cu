// One-call product: rvsp_cuda_spgemm_f32, the device counterpart of the
// reference's raw kernel rvsp_spgemm_scalar_f32
// (rv-sparse src/kernels/spgemm/gustavson_core_f32.inc:66-193):
// analysis + exact count -> allocate C -> fill + numeric.
//
// Device-resident inputs get device-resident outputs, allocated from the
// CUDA stream-ordered pool of the current device (the pool keeps released
// blocks, so repeated products reuse memory instead of calling cudaMalloc);
// host inputs get malloc'd host outputs, like the reference.

#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <mutex>

#include "rv_sparse_types.h"
#include "rvsp_cuda.h"
#include "rvsp_internal.h"

using namespace rvsp;

namespace {

// One cached plan per thread and algorithm, so back-to-back one-shot calls
// keep their device buffers and stream.
thread_local rvsp_cuda_plan_t t_plan[2] = {nullptr, nullptr};

struct PlanReaper {
    ~PlanReaper() {
        for (auto& p : t_plan)
            if (p) {
                rvsp_cuda_plan_destroy(p);
                p = nullptr;
            }
    }
};
thread_local PlanReaper t_reaper;

std::once_flag g_pool_once;

}  // namespace

namespace rvsp {
// The stream-ordered pool of the current device keeps freed blocks instead
// of returning them at every synchronisation, so repeated calls reuse memory
// instead of mapping it again.
void keep_pool_memory() {
    std::call_once(g_pool_once, [] {
        int dev = 0;
        cudaMemPool_t pool;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t thr = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
        cudaGetLastError();
    });
}
}  // namespace rvsp

namespace {

// The last entries of A's and B's row pointers (their nnz), wherever they
// live: device values come back together, one host round trip for both,
// through the plan's pinned word pair.
int read_ends(rvsp_cuda_plan* plan, const int32_t* pa, const int32_t* pb, int32_t* a,
              int32_t* b) {
    const bool da = is_dev(pa), db = is_dev(pb);
    if (!da) *a = *pa;
    if (!db) *b = *pb;
    if (!da && !db) return RVSP_SUCCESS;
    cudaError_t e = cudaSuccess;
    if (!plan->host_pin && (e = cudaMallocHost((void**)&plan->host_pin, 16)) != cudaSuccess) {
        plan->host_pin = nullptr;
        cudaGetLastError();
        if (da && (e = cudaMemcpy(a, pa, 4, cudaMemcpyDeviceToHost)) != cudaSuccess)
            return fail(e, "row_ptr read");
        if (db && (e = cudaMemcpy(b, pb, 4, cudaMemcpyDeviceToHost)) != cudaSuccess)
            return fail(e, "row_ptr read");
        return RVSP_SUCCESS;
    }
    if (da) e = cudaMemcpyAsync(plan->host_pin, pa, 4, cudaMemcpyDeviceToHost, plan->stream);
    if (e == cudaSuccess && db)
        e = cudaMemcpyAsync(plan->host_pin + 1, pb, 4, cudaMemcpyDeviceToHost, plan->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(plan->stream);
    if (e != cudaSuccess) return fail(e, "row_ptr read");
    if (da) *a = plan->host_pin[0];
    if (db) *b = plan->host_pin[1];
    return RVSP_SUCCESS;
}

}  // namespace

extern "C" int rvsp_cuda_spgemm_f32(int algo, int32_t a_rows, int32_t a_cols, int32_t b_cols,
                                    const int32_t* a_rp, const int32_t* a_ci, const float* a_v,
                                    const int32_t* b_rp, const int32_t* b_ci, const float* b_v,
                                    int32_t** c_rp_out, int32_t** c_ci_out, float** c_v_out,
                                    int32_t* c_nnz_out, int64_t* op_counts_out) {
    if (!a_rp || !a_ci || !a_v || !b_rp || !b_ci || !b_v || !c_rp_out || !c_ci_out ||
        !c_v_out || !c_nnz_out)
        return RVSP_ERROR_NULL_POINTER;
    if (a_rows <= 0 || a_cols <= 0 || b_cols <= 0) return RVSP_ERROR_INVALID_ARGUMENT;
    if (algo != RVSP_CUDA_ALGO_EXACT && algo != RVSP_CUDA_ALGO_LEARNED)
        return RVSP_ERROR_UNSUPPORTED_BACKEND;
    if (algo == RVSP_CUDA_ALGO_LEARNED && !rvsp_cuda_learned_available())
        return RVSP_ERROR_UNSUPPORTED_BACKEND;
    *c_rp_out = nullptr;
    *c_ci_out = nullptr;
    *c_v_out = nullptr;
    *c_nnz_out = 0;
    int st;
    rvsp_cuda_plan_t& plan = t_plan[algo == RVSP_CUDA_ALGO_LEARNED ? 1 : 0];
    if (!plan) {
        if ((st = rvsp_cuda_plan_create(&plan, algo))) return st;
        plan->map_policy = 0;  // a one-shot product is never reused
    }
    int32_t a_nnz = -1, b_nnz = -1;
    trace_point("one-shot: enter");
    const bool dev = is_dev(a_rp);
    // every operand array on the device: the analysis reads the operands'
    // nnz itself (returned with the bin counts), no round trip of its own
    const bool all_dev = dev && is_dev(a_ci) && is_dev(a_v) && is_dev(b_rp) && is_dev(b_ci) &&
                         is_dev(b_v);
    if (!all_dev && (st = read_ends(plan, a_rp + a_rows, b_rp + a_cols, &a_nnz, &b_nnz)))
        return st;
    trace_point("one-shot: operand nnz");
    plan->params = default_params();
    keep_pool_memory();

    if (algo == RVSP_CUDA_ALGO_EXACT && all_dev) {
        int64_t nnz = 0;
        int32_t *rp = nullptr, *ci = nullptr;
        float* v = nullptr;
        st = oneshot_exact_device(plan, a_rows, a_cols, b_cols, a_rp, a_ci, a_v, b_rp, b_ci, b_v,
                                  &rp, &ci, &v, &nnz);
        if (st) return st;
        *c_rp_out = rp;
        *c_ci_out = ci;
        *c_v_out = v;
        *c_nnz_out = (int32_t)nnz;
    } else if (algo == RVSP_CUDA_ALGO_LEARNED) {
        st = learned_spgemm(plan, a_rows, a_cols, a_nnz, a_rp, a_ci, a_v, a_cols, b_cols,
                            b_nnz, b_rp, b_ci, b_v, dev ? 1 : 0, c_rp_out, c_ci_out, c_v_out,
                            c_nnz_out);
    } else {
        int64_t nnz = 0;
        size_t ws = 0;
        st = rvsp_cuda_symbolic(plan, a_rows, a_cols, a_nnz, a_rp, a_ci, a_cols, b_cols, b_nnz,
                                b_rp, b_ci, &nnz, &ws);
        if (st) return st;
        const size_t alloc = nnz > 0 ? (size_t)nnz : 1;
        int32_t *rp = nullptr, *ci = nullptr;
        float* v = nullptr;
        if (dev) {
            cudaError_t e = cudaMallocAsync((void**)&rp, ((size_t)a_rows + 1) * 4, plan->stream);
            if (e == cudaSuccess) e = cudaMallocAsync((void**)&ci, alloc * 4, plan->stream);
            if (e == cudaSuccess) e = cudaMallocAsync((void**)&v, alloc * 4, plan->stream);
            if (e != cudaSuccess) {
                if (rp) cudaFreeAsync(rp, plan->stream);
                if (ci) cudaFreeAsync(ci, plan->stream);
                cudaStreamSynchronize(plan->stream);
                return fail(e, "C alloc");
            }
        } else {
            rp = (int32_t*)host_alloc(((size_t)a_rows + 1) * 4);
            ci = (int32_t*)host_alloc(alloc * 4);
            v = (float*)host_alloc(alloc * 4);
            if (!rp || !ci || !v) {
                host_free(rp);
                host_free(ci);
                host_free(v);
                return RVSP_ERROR_ALLOCATION_FAILED;
            }
        }
        trace_point("one-shot: C allocated");
        st = rvsp_cuda_numeric(plan, a_rp, a_ci, a_v, b_rp, b_ci, b_v, rp, ci, v, 1, nullptr);
        if (st) {
            if (dev) {
                cudaFree(rp);
                cudaFree(ci);
                cudaFree(v);
            } else {
                host_free(rp);
                host_free(ci);
                host_free(v);
            }
            return st;
        }
        *c_rp_out = rp;
        *c_ci_out = ci;
        *c_v_out = v;
        *c_nnz_out = (int32_t)nnz;
    }
    if (st) return st;
    if (op_counts_out) st = rvsp_cuda_op_counts(plan, op_counts_out, a_rows);
    return st;
}

extern "C" int rvsp_cuda_oneshot_learned_stats(int64_t* out, int32_t n) {
    if (!out) return RVSP_ERROR_NULL_POINTER;
    rvsp_cuda_plan_t plan = t_plan[1];
    if (!plan) return RVSP_ERROR_INVALID_ARGUMENT;
    return rvsp_cuda_plan_learned_stats(plan, out, n);
}
