// Learned-capacity SpGEMM path (RVSP_CUDA_ALGO_LEARNED).
//
// The exact path sweeps every product twice: once to count each row's
// distinct columns into tables sized by the row's upper bound
// ub = min(products, cols(B)), once to fill. Here the row-size predictor
// (mlp.cuh) sizes each row instead, and one fused sweep fills C:
//
//   analysis       k_analyze with features; k_mlp_infer on rows whose bound
//                  exceeds the tiny bin; k_learned_bins assigns each row a
//                  capacity (tiny rows: their product count, exact; others:
//                  the prediction) and a hash-table class, stable-partitioned
//   fused fill     the FILL kernels write every row's sorted columns and
//                  values into its slot of an over-allocated buffer and record
//                  its count; a row whose table fills up or whose count passes
//                  its capacity is flagged (count -1) instead
//                  heavy rows (a warp per column chunk) are sized by the
//                  prediction too: each chunk takes its place in the row's
//                  slot with an atomic add of its count, so the sweep leaves
//                  every heavy row's exact count and every chunk's count; a
//                  row whose chunks outgrow the slot is flagged
//   exact re-run   flagged table rows are counted by the exact kernels under a
//                  row mask (flagged heavy rows need no count: the sweep
//                  counted them)
//   C              scan of all counts -> row pointer; flagged rows are filled
//                  in place by the exact FILL kernels, the rest are copied from
//                  their slots (k_compact, k_compact_rows, k_compact_items)
//
// Every row is computed by the same order-preserving kernels as the exact
// path, so the result is bit-identical to it; a misprediction costs time,
// never accuracy. The plan records how many rows were predicted, how many
// overflowed, and how full the slots were.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "mlp.cuh"
#include "rv_sparse_types.h"
#include "rvsp_cuda.h"
#include "rvsp_internal.h"
#include "spgemm_types.cuh"

namespace rvsp {

bool current_model(MlpModel* out);
void launch_mlp_infer(const MlpModel& m, const float4* feat, const int32_t* ub, const uint8_t* bin,
                      int32_t n, int32_t* cap, cudaStream_t st);

constexpr int LBIN_EXACT = BIN_HEAVY;  // predicted bin of rows left to the exact path

struct LearnedBinsOut {
    uint8_t* lbin;
    int32_t* lcap;
    uint8_t* predicted;  // 1 where the row is sized by the prediction
    uint8_t* hmask;      // heavy rows sized by the prediction (null: heavy rows stay exact)
    int32_t* tile_hist;  // [NUM_BINS][tiles]
    int32_t* hist;       // [NUM_BINS]
    int64_t* slot_total;
};

__global__ void __launch_bounds__(AN_TILE)
    k_learned_bins(int32_t rows, const uint8_t* __restrict__ bin, const int64_t* __restrict__ ops,
                   const int32_t* __restrict__ ub, const int32_t* __restrict__ cap_pred,
                   LearnedBinsOut out, BinParams P) {
    __shared__ int32_t s_hist[NUM_BINS];
    __shared__ unsigned long long s_slots;
    const int t = threadIdx.x;
    if (t < NUM_BINS) s_hist[t] = 0;
    if (t == 0) s_slots = 0;
    __syncthreads();
    const int row = blockIdx.x * AN_TILE + t;
    int lb = -1, cap = 0;
    if (row < rows) {
        const int b = bin[row];
        int predicted = 0;
        if (b == BIN_EMPTY) {
            lb = BIN_EMPTY;
        } else if (b == BIN_TINY) {
            lb = BIN_TINY;
            cap = (int)ops[row];
        } else {
            // the prediction is used only where it buys a smaller table than
            // the upper bound would; otherwise the row gets the bound's table
            // and a slot of ub entries, which cannot overflow
            // With heavy slots (out.hmask) a heavy row stays heavy: the sweep
            // counts it chunk by chunk, so it never needs the exact recount,
            // which leaves heavy rows out.
            const int c = max(cap_pred[row], 1);
            const int pb = table_bin(c, P);  // table class of the prediction
            if (pb < b && !(b == BIN_HEAVY && out.hmask)) {
                lb = pb;
                cap = c;
                predicted = 1;
            } else if (b < BIN_HEAVY) {
                lb = b;
                cap = ub[row];
            } else {
                lb = LBIN_EXACT;
                if (out.hmask) {  // a slot of the predicted size for its chunks
                    cap = c;
                    predicted = 1;
                }
            }
        }
        out.lbin[row] = (uint8_t)lb;
        out.lcap[row] = cap;
        out.predicted[row] = (uint8_t)predicted;
        if (out.hmask) out.hmask[row] = (uint8_t)(lb == LBIN_EXACT && predicted);
    }
    // warp-aggregated histogram and slot total
    unsigned left = __ballot_sync(FULL, lb >= 0);
    while (left) {
        const int k = __shfl_sync(FULL, lb, __ffs(left) - 1);
        const unsigned sel = __ballot_sync(FULL, lb == k);
        if ((t & 31) == 0) atomicAdd(&s_hist[k], __popc(sel));
        left &= ~sel;
    }
    unsigned long long sl = (unsigned long long)cap;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sl += __shfl_xor_sync(FULL, sl, o);
    if ((t & 31) == 0 && sl) atomicAdd(&s_slots, sl);
    __syncthreads();
    if (t < NUM_BINS) {
        out.tile_hist[t * gridDim.x + blockIdx.x] = s_hist[t];
        if (s_hist[t]) atomicAdd(&out.hist[t], s_hist[t]);
    }
    if (t == 0 && s_slots) atomicAdd((unsigned long long*)out.slot_total, s_slots);
}

// Rows the sweep could not finish: too large for a table, or sized by the
// prediction and outgrown it. Their counts are reset for the exact kernels.
// stats: [0] rows sized by the prediction, [1] of those, rows that outgrew
//        it, [2] rows too large for a table, [3] sum of counts, [4] sum of
//        capacities and [6] sum of upper bounds of predicted rows that fit
// Heavy rows sized by the prediction (hmask; null when there are none) were
// counted by the sweep: only those whose slot overflowed (hovf) need the
// exact fill, and their counts stand.
__global__ void k_need(int32_t rows, const uint8_t* __restrict__ lbin,
                       const uint8_t* __restrict__ predicted, const int32_t* __restrict__ lcap,
                       const int32_t* __restrict__ ub, int32_t* __restrict__ cnt,
                       uint8_t* __restrict__ need, const uint8_t* __restrict__ hmask,
                       const uint8_t* __restrict__ hovf,
                       int32_t* __restrict__ n_need, int32_t* __restrict__ n_need_heavy,
                       int64_t* __restrict__ stats) {
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    bool nd = false, ovf = false, big = false, pr = false, under = false;
    int64_t fitc = 0, fitcap = 0, fitub = 0;
    if (row < rows) {
        const int lb = lbin[row];
        const bool hslot = hmask && hmask[row];
        pr = predicted[row] != 0;
        big = lb == LBIN_EXACT;
        ovf = hslot ? hovf[row] != 0 : (lb >= BIN_WARP0 && lb < LBIN_EXACT && cnt[row] < 0);
        nd = (big && !hslot) || ovf;
        under = pr && (ovf || cnt[row] > lcap[row]);
        if (pr && !ovf) {
            fitc = cnt[row];
            fitcap = lcap[row];
            fitub = ub[row];
        }
        need[row] = nd ? 1 : 0;
        if (nd && !hslot) cnt[row] = 0;
    }
    const unsigned mn = __ballot_sync(FULL, nd), mo = __ballot_sync(FULL, ovf && pr),
                   mb = __ballot_sync(FULL, big), mp = __ballot_sync(FULL, pr),
                   mu = __ballot_sync(FULL, under), mh = __ballot_sync(FULL, nd && big);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        fitc += __shfl_xor_sync(FULL, fitc, o);
        fitcap += __shfl_xor_sync(FULL, fitcap, o);
        fitub += __shfl_xor_sync(FULL, fitub, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (mn) atomicAdd(n_need, __popc(mn));
        if (mh) atomicAdd(n_need_heavy, __popc(mh));
        if (mp) atomicAdd((unsigned long long*)&stats[0], (unsigned long long)__popc(mp));
        if (mo) atomicAdd((unsigned long long*)&stats[1], (unsigned long long)__popc(mo));
        if (mb) atomicAdd((unsigned long long*)&stats[2], (unsigned long long)__popc(mb));
        if (fitc) atomicAdd((unsigned long long*)&stats[3], (unsigned long long)fitc);
        if (fitcap) atomicAdd((unsigned long long*)&stats[4], (unsigned long long)fitcap);
        if (fitub) atomicAdd((unsigned long long*)&stats[6], (unsigned long long)fitub);
        if (mu) atomicAdd((unsigned long long*)&stats[7], (unsigned long long)__popc(mu));
    }
}

// Copy finished rows from their slots into C, one warp per row (the warp-bin
// rows: tens to thousands of entries each), 128 entries per step with each
// lane's four loads issued before its stores. Coalesced on both sides.
__global__ void __launch_bounds__(256)
    k_compact_rows(const int32_t* __restrict__ rows, int32_t n, const uint8_t* __restrict__ need,
                   const int32_t* __restrict__ cnt, const int64_t* __restrict__ slot_off,
                   const int32_t* __restrict__ c_rp, const int32_t* __restrict__ tmp_ci,
                   const float* __restrict__ tmp_v, int32_t* __restrict__ c_ci,
                   float* __restrict__ c_v) {
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= n) return;
    const int row = rows[w];
    if (need[row]) return;
    const int k = cnt[row];
    const int64_t src = slot_off[row];
    const int dst = c_rp[row];
    for (int x0 = 0; x0 < k; x0 += 128) {
        int32_t ci[4];
        float v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int x = x0 + 32 * u + lane;
            if (x < k) {
                ci[u] = tmp_ci[src + x];
                v[u] = tmp_v[src + x];
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int x = x0 + 32 * u + lane;
            if (x < k) {
                c_ci[dst + x] = ci[u];
                c_v[dst + x] = v[u];
            }
        }
    }
}

// Copy finished rows from their slots into C: one warp per 32 consecutive
// list entries; the lanes load the 32 rows' counts and offsets together, then
// copy either the 32 rows' entries as one list (up to 64 entries a row on
// average) or the rows one after the other, 128 entries per step (each lane's
// four loads issued before its stores). Coalesced on both sides.
__global__ void __launch_bounds__(256)
    k_compact(const int32_t* __restrict__ rows, int32_t n, const uint8_t* __restrict__ need,
              const int32_t* __restrict__ cnt, const int64_t* __restrict__ slot_off,
              const int32_t* __restrict__ c_rp, const int32_t* __restrict__ tmp_ci,
              const float* __restrict__ tmp_v, int32_t* __restrict__ c_ci,
              float* __restrict__ c_v) {
    const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5 << 5;
    const int lane = threadIdx.x & 31;
    if (w0 >= n) return;
    const int64_t i = w0 + lane;
    int k = 0, dst = 0;
    int64_t src = 0;
    if (i < n) {
        const int row = rows[i];
        if (!need[row]) {
            k = cnt[row];
            src = slot_off[row];
            dst = c_rp[row];
        }
    }
    int incl = k;  // inclusive scan of the counts over the warp
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += y;
    }
    const int total = __shfl_sync(FULL, incl, 31);
    if (total <= 32 * 64) {
        // short rows (tiny rows: a dozen entries): the 32 rows' entries as one
        // list, 32 per step; each lane finds its row in the counts' scan
        for (int e0 = 0; e0 < total; e0 += 32) {
            const int e = e0 + lane;
            int j = 0;
#pragma unroll
            for (int st = 16; st >= 1; st >>= 1)
                if (__shfl_sync(FULL, incl, j + st - 1) <= e) j += st;
            j = min(j, 31);
            const int first = __shfl_sync(FULL, incl, j) - __shfl_sync(FULL, k, j);
            const int64_t sj = __shfl_sync(FULL, src, j);
            const int dj = __shfl_sync(FULL, dst, j);
            if (e < total) {
                c_ci[dj + (e - first)] = tmp_ci[sj + (e - first)];
                c_v[dj + (e - first)] = tmp_v[sj + (e - first)];
            }
        }
        return;
    }
    for (int j = 0; j < 32; ++j) {
        const int kj = __shfl_sync(FULL, k, j);
        const int64_t sj = __shfl_sync(FULL, src, j);
        const int dj = __shfl_sync(FULL, dst, j);
        for (int x0 = 0; x0 < kj; x0 += 128) {
            int32_t ci[4];
            float v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int x = x0 + 32 * u + lane;
                if (x < kj) {
                    ci[u] = tmp_ci[sj + x];
                    v[u] = tmp_v[sj + x];
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int x = x0 + 32 * u + lane;
                if (x < kj) {
                    c_ci[dj + x] = ci[u];
                    c_v[dj + x] = v[u];
                }
            }
        }
    }
}

// Copy the chunks of heavy rows finished in their slots (or the overflow
// pool) into C, each chunk's entries from where the sweep put them to their
// place in C (its row's start plus the counts of the row's earlier chunks).
// One warp per 32 consecutive work items (grid-stride): lane l loads item l's
// bookkeeping (all 32 items' loads in flight together), then the warp copies
// the 32 chunks' entries as one list, 128 entries per step with each lane's
// four loads issued before its stores; each lane finds its entry's chunk in
// the scan of the chunks' counts. A chunk's source and destination offsets
// are kept less the chunk's first index in the list, so an entry's two
// addresses are one shuffle each (40 registers: 6 CTAs per SM). Items of a
// row are consecutive, so the stores run contiguously through C.
__global__ void __launch_bounds__(256)
    k_compact_items(const HeavyItem* __restrict__ items, int32_t n,
                    const uint8_t* __restrict__ hmask, const uint8_t* __restrict__ need,
                    const int32_t* __restrict__ item_cnt, const int64_t* __restrict__ item_off,
                    const int64_t* __restrict__ item_scan, const int64_t* __restrict__ slot_off,
                    const int32_t* __restrict__ c_rp, const int32_t* __restrict__ tmp_ci,
                    const float* __restrict__ tmp_v, int32_t* __restrict__ c_ci,
                    float* __restrict__ c_v) {
    const int lane = threadIdx.x & 31;
    const int64_t groups = ((int64_t)n + 31) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t g = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < groups;
         g += nwarps) {
        const int64_t w = (g << 5) + lane;
        int k = 0;
        int64_t src = 0, dst = 0;
        if (w < n) {
            const HeavyItem it = items[w];
            if (hmask[it.row] && !need[it.row]) {
                k = item_cnt[w];
                src = item_off[w];
                dst = (int64_t)c_rp[it.row] + (item_scan[w] - item_scan[it.first]);
            }
        }
        int incl = k;  // inclusive scan of the chunks' counts over the warp
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += y;
        }
        const int total = __shfl_sync(FULL, incl, 31);
        src -= incl - k;
        dst -= incl - k;
        for (int e0 = 0; e0 < total; e0 += 128) {
            int32_t ci[4];
            float v[4];
            int64_t d[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int e = e0 + 32 * u + lane;
                int j = 0;
#pragma unroll
                for (int st = 16; st >= 1; st >>= 1)
                    if (__shfl_sync(FULL, incl, j + st - 1) <= e) j += st;
                j = min(j, 31);
                const int64_t sj = __shfl_sync(FULL, src, j) + e;
                d[u] = __shfl_sync(FULL, dst, j) + e;
                if (e < total) {
                    ci[u] = tmp_ci[sj];
                    v[u] = tmp_v[sj];
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (e0 + 32 * u + lane < total) {
                    c_ci[d[u]] = ci[u];
                    c_v[d[u]] = v[u];
                }
            }
        }
    }
}

// Enqueued by analyze() before its host synchronisation: prediction and
// predicted-capacity bins, so one round trip returns both histograms.
static int learned_pre_sync(rvsp_cuda_plan* plan) {
    MlpModel model;
    if (!current_model(&model)) {
        g_err = "no row-size model loaded";
        return RVSP_ERROR_UNSUPPORTED_BACKEND;
    }
    const int64_t M = plan->a_rows;
    const int64_t tiles = (M + AN_TILE - 1) / AN_TILE;
    cudaError_t e;
#define ENS(buf, bytes) \
    if ((e = (buf).ensure(bytes)) != cudaSuccess) return fail(e, "learned alloc " #buf)
    ENS(plan->pred_cap, M * 4);
    ENS(plan->lbin, M);
    ENS(plan->lcap, M * 4);
    ENS(plan->ltile_hist, NUM_BINS * tiles * 4);
    ENS(plan->ltile_off, (NUM_BINS * tiles + 1) * 4);
    ENS(plan->lbin_rows, M * 4);
    ENS(plan->need, M);
    ENS(plan->row_flag, M);
    ENS(plan->pflag, M);
    ENS(plan->hmask, M);
    ENS(plan->hovf, M);
#undef ENS
    Misc* misc = plan->misc.as<Misc>();
    {
        KTime kt(plan->stream, plan->capturing, KF_LEARNED);
        launch_mlp_infer(model, plan->feat.as<float4>(), plan->ub.as<int32_t>(),
                         plan->bin.as<uint8_t>(), (int32_t)M, plan->pred_cap.as<int32_t>(),
                         plan->stream);
        // heavy rows take predicted slots only in the fused sweep (the
        // one-shot product); the descriptor's count keeps them exact
        LearnedBinsOut lo{plan->lbin.as<uint8_t>(), plan->lcap.as<int32_t>(),
                          plan->pflag.as<uint8_t>(),
                          plan->heavy_slots ? plan->hmask.as<uint8_t>() : nullptr,
                          plan->ltile_hist.as<int32_t>(), misc->lhist, &misc->slot_total};
        k_learned_bins<<<(unsigned)tiles, AN_TILE, 0, plan->stream>>>(
            (int32_t)M, plan->bin.as<uint8_t>(), plan->ops.as<int64_t>(), plan->ub.as<int32_t>(),
            plan->pred_cap.as<int32_t>(), lo, plan->params);
    }
    note_launch(plan, 2);
    return scan_counts(plan, plan->ltile_hist.as<int32_t>(), NUM_BINS * tiles, nullptr,
                       plan->ltile_off.as<int32_t>(), &misc->ltile_total);
}

// Learned analysis, one sweep over the predicted-capacity bins, exact counts
// of the rows that sweep could not finish. On return the plan holds the exact
// row pointer of C (plan->c_rp, plan->c_nnz) and the mask of rows finished by
// the exact path (plan->need). With fused, the sweep is the FILL kernels and
// every other row's columns and values wait in its slot (tmp_ci / tmp_v at
// slot_off) for learned_finish; without, the sweep is the COUNT kernels with
// tables sized by the prediction (the descriptor's structure analysis).
int learned_symbolic(rvsp_cuda_plan* plan, CsrView& A, CsrView& B, bool fused) {
    plan->heavy_slots = fused;
    int st = analyze(plan, A, B, true, learned_pre_sync);
    if (st) return st;
    trace_point("learned: analysis + bins");
    const int64_t M = plan->a_rows;
    Misc* misc = plan->misc.as<Misc>();
    int32_t acc = 0;
    for (int b = 0; b < NUM_BINS; ++b) {
        plan->lcount[b] = plan->host_misc.lhist[b];
        plan->loffs.off[b] = acc;
        acc += plan->lcount[b];
    }
    plan->slot_total = plan->host_misc.slot_total;
    cudaError_t e;
    // heavy rows' chunks that outgrow their predicted slot share an overflow
    // pool of a quarter of the slots, after them in the same buffers
    plan->pool_cap = fused && plan->n_items > 0 ? plan->slot_total / 4 : 0;
    const int64_t tmp_total = plan->slot_total + plan->pool_cap;
    size_t free_b = SIZE_MAX, total_b = 0;
    // slot buffers that must grow past 1 GiB must fit in half the free
    // memory (queried only then: the query waits behind any other client of
    // the driver, e.g. a clock monitor, with the GPU idle)
    if (fused && (size_t)tmp_total * 4 > plan->tmp_ci.cap &&
        (size_t)plan->slot_total * 10 > (1ull << 30) &&
        (e = cudaMemGetInfo(&free_b, &total_b)) != cudaSuccess)
        return fail(e, "mem info");
    if (fused) {
        if (free_b != SIZE_MAX && (size_t)tmp_total * 8 > free_b / 2) {
            g_err = "predicted capacity exceeds the memory budget";
            return RVSP_ERROR_ALLOCATION_FAILED;
        }
        if ((e = plan->slot_off.ensure(((size_t)M + 1) * 8)) != cudaSuccess)
            return fail(e, "slots");
        if ((e = plan->tmp_ci.ensure((size_t)tmp_total * 4)) != cudaSuccess)
            return fail(e, "slots");
        if ((e = plan->tmp_v.ensure((size_t)tmp_total * 4)) != cudaSuccess)
            return fail(e, "slots");
    }
    launch_bin_scatter(plan, plan->lbin.as<uint8_t>(), plan->ltile_off.as<int32_t>(),
                       plan->lbin_rows.as<int32_t>(), false);
    if (fused && (st = scan_counts(plan, plan->lcap.as<int32_t>(), M, plan->slot_off.as<int64_t>(),
                                   nullptr, &misc->scan_total2)))
        return st;
    if ((e = cudaMemsetAsync(plan->cnt.p, 0, M * 4, plan->stream)) != cudaSuccess)
        return fail(e, "memset");
    if (plan->n_items > 0 &&
        (e = cudaMemsetAsync(plan->item_cnt.p, 0, (size_t)plan->n_items * 4, plan->stream)) !=
            cudaSuccess)
        return fail(e, "memset");
    const bool hslots = fused && plan->n_items > 0;
    if (hslots && ((e = plan->item_off.ensure((size_t)plan->n_items * 8)) != cudaSuccess ||
                   (e = cudaMemsetAsync(plan->hovf.p, 0, M, plan->stream)) != cudaSuccess))
        return fail(e, "heavy slots");
    // one sweep over the predicted-capacity bins
    RowOut fo{plan->cnt.as<int32_t>(), nullptr, plan->tmp_ci.as<int32_t>(), plan->tmp_v.as<float>(),
              &misc->err, false};
    fo.ctl.slot_off = fused ? plan->slot_off.as<int64_t>() : nullptr;
    fo.ctl.learned = 1;
    if (hslots) {
        fo.ctl.item_off = plan->item_off.as<int64_t>();
        fo.ctl.ovf = plan->hovf.as<uint8_t>();
        fo.ctl.pool_fill = &misc->pool_fill;  // zeroed with the rest of Misc by the analysis
        fo.ctl.pool_base = plan->slot_total;
        fo.ctl.pool_cap = plan->pool_cap;
    }
    fo.learned_bins = true;
    run_rows(plan, fused ? FILL : COUNT, A, B, fo);
    {
        KTime ktn(plan->stream, plan->capturing, KF_LEARNED);
        k_need<<<(unsigned)((M + 255) / 256), 256, 0, plan->stream>>>(
            (int32_t)M, plan->lbin.as<uint8_t>(), plan->pflag.as<uint8_t>(),
            plan->lcap.as<int32_t>(), plan->ub.as<int32_t>(), plan->cnt.as<int32_t>(),
            plan->need.as<uint8_t>(), hslots ? plan->hmask.as<uint8_t>() : nullptr,
            hslots ? plan->hovf.as<uint8_t>() : nullptr, &misc->n_need, &misc->n_need_heavy,
            misc->lstats);
    }
    note_launch(plan, 1);
    // exact counts of the rows the sweep could not finish (tiny rows never overflow)
    RowOut co{plan->cnt.as<int32_t>(), nullptr, nullptr, nullptr, &misc->err, false};
    co.ctl.only = plan->need.as<uint8_t>();
    const int32_t tiny = plan->bin_count[BIN_TINY];
    const int32_t items = plan->n_items;
    plan->bin_count[BIN_TINY] = 0;
    if (hslots) plan->n_items = 0;  // the sweep counted the heavy rows
    run_rows(plan, COUNT, A, B, co);
    plan->bin_count[BIN_TINY] = tiny;
    plan->n_items = items;
    if ((st = scan_counts(plan, plan->cnt.as<int32_t>(), M, nullptr, plan->c_rp.as<int32_t>(),
                          &misc->scan_total)))
        return st;
    if (plan->n_items > 0 &&
        (st = scan_counts(plan, plan->item_cnt.as<int32_t>(), plan->n_items,
                          plan->item_scan.as<int64_t>(), nullptr, &misc->tile_total)))
        return st;
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "learned launch");
    if ((e = cudaMemcpyAsync(&plan->host_misc, misc, sizeof(Misc), cudaMemcpyDeviceToHost,
                             plan->stream)) != cudaSuccess)
        return fail(e, "learned read");
    if ((e = cudaStreamSynchronize(plan->stream)) != cudaSuccess) return fail(e, "learned sweep");
    trace_point("learned: sweep (synced)");
    if (plan->host_misc.err) {
        g_err = "operand structure out of range (row_ptr or col_idx)";
        return RVSP_ERROR_INVALID_CSR;
    }
    if (plan->host_misc.overflow || plan->host_misc.scan_total > INT32_MAX) {
        g_err = "nnz(C) exceeds INT32_MAX";
        return RVSP_ERROR_ALLOCATION_FAILED;
    }
    plan->c_nnz = plan->host_misc.scan_total;
    // heavy rows sized by the prediction were never counted by column chunk
    plan->items_counted = plan->n_items == 0 || fused;
    for (int i = 0; i < 8; ++i) plan->lstats[i] = plan->host_misc.lstats[i];
    plan->lstats[5] = plan->host_misc.n_need;
    plan->lstats[8] = (int64_t)plan->host_misc.pool_fill;
    plan->lstats[9] = plan->pool_cap;
    return RVSP_SUCCESS;
}

// C from the learned sweep: exact fill of the masked rows in place, copy of
// the rest from their slots. c_ci / c_v are device arrays of nnz entries.
int learned_finish(rvsp_cuda_plan* plan, const CsrView& A, const CsrView& B, int32_t* c_ci,
                   float* c_v) {
    Misc* misc = plan->misc.as<Misc>();
    if (plan->host_misc.n_need > 0) {
        RowOut fo{nullptr, plan->c_rp.as<int32_t>(), c_ci, c_v, &misc->err, false};
        fo.ctl.only = plan->need.as<uint8_t>();
        // tiny rows never need it; heavy rows only when one of them did (the
        // heavy kernel would otherwise pull every work item just to skip it)
        const int32_t tiny = plan->bin_count[BIN_TINY], items = plan->n_items;
        plan->bin_count[BIN_TINY] = 0;
        if (plan->host_misc.n_need_heavy == 0) plan->n_items = 0;
        run_rows(plan, FILL, A, B, fo);
        plan->bin_count[BIN_TINY] = tiny;
        plan->n_items = items;
    }
    const int32_t* lrows = plan->lbin_rows.as<int32_t>();
    const int32_t nt = plan->lcount[BIN_TINY];
    KTime kt(plan->stream, plan->capturing, KF_COMPACT);
    if (nt > 0) {
        k_compact<<<(unsigned)(((int64_t)nt + 255) / 256), 256, 0, plan->stream>>>(
            lrows + plan->loffs.off[BIN_TINY], nt, plan->need.as<uint8_t>(), plan->cnt.as<int32_t>(),
            plan->slot_off.as<int64_t>(), plan->c_rp.as<int32_t>(), plan->tmp_ci.as<int32_t>(),
            plan->tmp_v.as<float>(), c_ci, c_v);
        note_launch(plan, 1);
    }
    int32_t nw = 0;
    for (int b = BIN_WARP0; b < LBIN_EXACT; ++b) nw += plan->lcount[b];
    if (nw > 0) {
        k_compact_rows<<<(unsigned)(((int64_t)nw * 32 + 255) / 256), 256, 0, plan->stream>>>(
            lrows + plan->loffs.off[BIN_WARP0], nw, plan->need.as<uint8_t>(),
            plan->cnt.as<int32_t>(), plan->slot_off.as<int64_t>(), plan->c_rp.as<int32_t>(),
            plan->tmp_ci.as<int32_t>(), plan->tmp_v.as<float>(), c_ci, c_v);
        note_launch(plan, 1);
    }
    if (plan->heavy_slots && plan->n_items > 0) {
        const int64_t grid = std::min<int64_t>(((int64_t)plan->n_items + 255) / 256, 148 * 64);
        k_compact_items<<<(unsigned)grid, 256, 0, plan->stream>>>(
            plan->items.as<HeavyItem>(), plan->n_items, plan->hmask.as<uint8_t>(),
            plan->need.as<uint8_t>(), plan->item_cnt.as<int32_t>(), plan->item_off.as<int64_t>(),
            plan->item_scan.as<int64_t>(), plan->slot_off.as<int64_t>(), plan->c_rp.as<int32_t>(),
            plan->tmp_ci.as<int32_t>(), plan->tmp_v.as<float>(), c_ci, c_v);
        note_launch(plan, 1);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? RVSP_SUCCESS : fail(e, "learned finish");
}

// Product through the learned path; C arrays allocated like rvsp_cuda_spgemm_f32.
int learned_spgemm(rvsp_cuda_plan* plan, int32_t a_rows, int32_t a_cols, int32_t a_nnz,
                   const int32_t* a_rp, const int32_t* a_ci, const float* a_v, int32_t b_rows,
                   int32_t b_cols, int32_t b_nnz, const int32_t* b_rp, const int32_t* b_ci,
                   const float* b_v, int device_out, int32_t** c_rp_out, int32_t** c_ci_out,
                   float** c_v_out, int32_t* c_nnz_out) {
    plan->analysed = false;
    plan->maps_ready = false;
    plan->filled_host = nullptr;
    reset_graph(plan);
    plan->a_rows = a_rows;
    plan->a_cols = a_cols;
    plan->a_nnz = a_nnz;
    plan->b_rows = b_rows;
    plan->b_cols = b_cols;
    plan->b_nnz = b_nnz;
    memset(plan->key, 0, sizeof(plan->key));
    CsrView A, B;
    trace_point("learned one-shot: enter");
    int st = stage_operands(plan, a_rp, a_ci, a_v, b_rp, b_ci, b_v, false, &A, &B);
    if (st) return st;
    trace_point("learned: operands staged");
    if ((st = learned_symbolic(plan, A, B, true))) return st;
    plan->analysed = true;
    const int64_t nnz = plan->c_nnz;
    const size_t alloc = nnz > 0 ? (size_t)nnz : 1;
    int32_t *rp = nullptr, *ci = nullptr;
    float* v = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&rp, ((size_t)a_rows + 1) * 4, plan->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&ci, alloc * 4, plan->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&v, alloc * 4, plan->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(rp, plan->c_rp.p, ((size_t)a_rows + 1) * 4, cudaMemcpyDeviceToDevice,
                            plan->stream);
    if (e == cudaSuccess && nnz > 0) {
        st = learned_finish(plan, A, B, ci, v);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && st == RVSP_SUCCESS) e = cudaStreamSynchronize(plan->stream);
    trace_point("learned: finish (synced)");
    if (e != cudaSuccess || st) {
        cudaFree(rp);
        cudaFree(ci);
        cudaFree(v);
        return st ? st : fail(e, "learned product");
    }
    if (!device_out) {  // host inputs: hand back host arrays that free() releases
        int32_t* hrp = (int32_t*)host_alloc(((size_t)a_rows + 1) * 4);
        int32_t* hci = (int32_t*)host_alloc(alloc * 4);
        float* hv = (float*)host_alloc(alloc * 4);
        if (!hrp || !hci || !hv) {
            host_free(hrp);
            host_free(hci);
            host_free(hv);
            cudaFreeAsync(rp, plan->stream);
            cudaFreeAsync(ci, plan->stream);
            cudaFreeAsync(v, plan->stream);
            return RVSP_ERROR_ALLOCATION_FAILED;
        }
        trace_point("learned: host C allocated");
        e = copy_to_host(hrp, rp, ((size_t)a_rows + 1) * 4, plan->stream);
        if (e == cudaSuccess) e = copy_to_host(hci, ci, (size_t)nnz * 4, plan->stream);
        if (e == cudaSuccess) e = copy_to_host(hv, v, (size_t)nnz * 4, plan->stream);
        cudaFreeAsync(rp, plan->stream);
        cudaFreeAsync(ci, plan->stream);
        cudaFreeAsync(v, plan->stream);
        if (e != cudaSuccess) {
            host_free(hrp);
            host_free(hci);
            host_free(hv);
            return fail(e, "learned copy-out");
        }
        rp = hrp;
        ci = hci;
        v = hv;
    }
    *c_rp_out = rp;
    *c_ci_out = ci;
    *c_v_out = v;
    *c_nnz_out = (int32_t)nnz;
    return RVSP_SUCCESS;
}

}  // namespace rvsp

using namespace rvsp;

extern "C" {

int rvsp_cuda_plan_learned_stats(rvsp_cuda_plan_t plan, int64_t* out, int32_t n) {
    if (!plan || !out) return RVSP_ERROR_NULL_POINTER;
    if (n < 7) return RVSP_ERROR_INVALID_ARGUMENT;
    if (plan->algo != RVSP_CUDA_ALGO_LEARNED || !plan->analysed) return RVSP_ERROR_INVALID_ARGUMENT;
    memcpy(out, plan->lstats, sizeof(int64_t) * (n < 10 ? n : 10));
    return RVSP_SUCCESS;
}

}  // extern "C"
