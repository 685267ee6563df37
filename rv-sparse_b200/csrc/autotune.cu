// Autotuner of a plan's bin parameters (thread-per-row threshold, hash table
// slack, largest warp table, heavy column-chunk width).
//
// Every valid parameter setting produces the same pattern and bit-identical
// values, so the tuner only measures: each trial runs the plan's own
// symbolic + structure-filling numeric on the caller's operands into scratch
// memory and keeps the best wall time of `reps` runs (the pipeline
// synchronises with the host between its phases, so wall time is what a
// caller of the one-shot or descriptor path waits). The search is coordinate
// descent, the parameters with the largest effect first; a candidate must
// beat the incumbent by 2% to replace it, which keeps timing noise from
// moving the choice.

#include <cuda_runtime.h>

#include <chrono>
#include <cstring>

#include "rv_sparse_types.h"
#include "rvsp_cuda.h"
#include "rvsp_internal.h"

using namespace rvsp;

namespace {

struct Knob {
    int32_t BinParams::*field;
    int32_t cand[4];
    int n;
    bool heavy_only;  // matters only when the product has chunked rows
};

const Knob kKnobs[] = {
    {&BinParams::warp_cap_max, {1024, 2048, 4096, 0}, 3, false},
    {&BinParams::heavy_cw_log2, {10, 11, 12, 13}, 4, true},
    {&BinParams::slack_shift, {1, 2, 3, 0}, 3, false},
    {&BinParams::tiny_ops, {16, 32, 0, 0}, 2, false},
};

struct Scratch {
    DevBuf rp, ci, v;
    void release() {
        rp.release();
        ci.release();
        v.release();
    }
};

}  // namespace

extern "C" int rvsp_cuda_plan_autotune(
    rvsp_cuda_plan_t plan, int32_t a_rows, int32_t a_cols, int32_t a_nnz, const int32_t* a_rp,
    const int32_t* a_ci, const float* a_v, int32_t b_rows, int32_t b_cols, int32_t b_nnz,
    const int32_t* b_rp, const int32_t* b_ci, const float* b_v, int32_t reps, int32_t* params_out,
    int32_t* trial_params, float* trial_ms, int32_t max_trials, int32_t* n_trials_out,
    int64_t* c_nnz_out, size_t* ws_bytes_out) {
    if (!plan || !c_nnz_out || !ws_bytes_out || !a_v || !b_v) return RVSP_ERROR_NULL_POINTER;
    if (reps < 1) reps = 1;
    if (max_trials < 0) max_trials = 0;
    const BinParams start = plan->params;
    const int saved_policy = plan->map_policy;
    plan->map_policy = 0;  // trials time the pipeline, not the recording of reuse maps
    Scratch sc;
    int ntr = 0;
    int64_t nnz = 0;
    size_t ws = 0;

    // one run of symbolic + filling numeric under p; *items: chunked rows exist
    auto run = [&](const BinParams& p, double* ms, bool* items) -> int {
        plan->params = p;
        const auto t0 = std::chrono::steady_clock::now();
        int st = rvsp_cuda_symbolic(plan, a_rows, a_cols, a_nnz, a_rp, a_ci, b_rows, b_cols,
                                    b_nnz, b_rp, b_ci, &nnz, &ws);
        if (st) return st;
        const size_t n = nnz > 0 ? (size_t)nnz : 1;
        cudaError_t e = sc.rp.ensure(((size_t)a_rows + 1) * 4);
        if (e == cudaSuccess) e = sc.ci.ensure(n * 4);
        if (e == cudaSuccess) e = sc.v.ensure(n * 4);
        if (e != cudaSuccess) return fail(e, "autotune scratch");
        st = rvsp_cuda_numeric(plan, a_rp, a_ci, a_v, b_rp, b_ci, b_v, sc.rp.as<int32_t>(),
                               sc.ci.as<int32_t>(), sc.v.as<float>(), 1, nullptr);
        if (st) return st;
        if ((e = cudaStreamSynchronize(plan->stream)) != cudaSuccess) return fail(e, "autotune");
        *ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                  .count();
        *items = plan->n_items > 0;
        return RVSP_SUCCESS;
    };
    auto trial = [&](const BinParams& p, double* best, bool* items) -> int {
        *best = 1e300;
        for (int r = 0; r < reps; ++r) {
            double ms;
            int st = run(p, &ms, items);
            if (st) return st;
            if (ms < *best) *best = ms;
        }
        if (ntr < max_trials) {
            if (trial_params) {
                int32_t* t = trial_params + (size_t)ntr * RVSP_CUDA_BIN_PARAMS;
                t[0] = p.tiny_ops;
                t[1] = p.slack_shift;
                t[2] = p.warp_cap_max;
                t[3] = p.heavy_cw_log2;
            }
            if (trial_ms) trial_ms[ntr] = (float)*best;
        }
        ++ntr;
        return RVSP_SUCCESS;
    };

    int st;
    {
        // untimed warm-up: first-call allocations of the plan and the scratch
        double ms;
        bool items;
        st = run(start, &ms, &items);
    }
    BinParams best = start;
    double best_ms = 0.0;
    bool best_items = false;
    if (!st) st = trial(best, &best_ms, &best_items);
    for (const Knob& k : kKnobs) {
        if (st) break;
        if (k.heavy_only && !best_items) continue;
        const BinParams base = best;
        for (int i = 0; i < k.n && !st; ++i) {
            if (base.*k.field == k.cand[i]) continue;
            BinParams p = base;
            p.*k.field = k.cand[i];
            double ms;
            bool items;
            st = trial(p, &ms, &items);
            if (!st && ms < best_ms * 0.98) {
                best = p;
                best_ms = ms;
                best_items = items;
            }
        }
    }
    plan->map_policy = saved_policy;
    if (st) {
        plan->params = start;
        plan->analysed = false;
        sc.release();
        return st;
    }
    // leave the plan analysed under the choice, as rvsp_cuda_symbolic would
    plan->params = best;
    st = rvsp_cuda_symbolic(plan, a_rows, a_cols, a_nnz, a_rp, a_ci, b_rows, b_cols, b_nnz, b_rp,
                            b_ci, c_nnz_out, ws_bytes_out);
    sc.release();
    if (st) return st;
    if (params_out) {
        params_out[0] = best.tiny_ops;
        params_out[1] = best.slack_shift;
        params_out[2] = best.warp_cap_max;
        params_out[3] = best.heavy_cw_log2;
    }
    if (n_trials_out) *n_trials_out = ntr;
    return RVSP_SUCCESS;
}
