// C-ABI implementation of the B200 SpGEMM backend (include/rvsp_cuda.h).
//
// A plan is the device-side half of an rv-sparse descriptor
// (rv-sparse src/core/spgemm_descr.c:19-37): it keeps the analysed structure
// of C on the device (row pointer, per-row op counts, row bins, heavy work
// items), staging copies of host-resident operands, and the CUDA graph of the
// numeric-only pass used when the descriptor is reused.
//
// Pipeline of one product (all on the plan's stream):
//   analysis   k_analyze -> (bin histogram to host) -> k_bin_scatter
//   count      k_tiny / k_warp / k_heavy in COUNT mode -> k_scan_* -> nnz
//   fill       the same kernels in FILL mode write sorted columns + values
//   reuse      REUSE mode writes values on the known pattern (graph replay)

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "rv_sparse_types.h"
#include "rvsp_cuda.h"
#include "rvsp_internal.h"
#include "spgemm_kernels.cuh"

using namespace rvsp;

namespace rvsp {

thread_local std::string g_err;
std::atomic<long long> g_launches{0};

int fail(cudaError_t e, const char* what) {
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? RVSP_ERROR_ALLOCATION_FAILED
                                          : RVSP_ERROR_DEVICE_FAILURE;
}

bool trace_on() {
    static const bool on = [] {
        const char* e = getenv("RVSP_TRACE");
        return e && e[0] == '1';
    }();
    return on;
}

bool is_dev(const void* p) {
    if (!p) return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// ---------------------------------------------------------------------------
// kernel-family timing (rvsp_cuda_kernel_timing / rvsp_cuda_kernel_times)
// ---------------------------------------------------------------------------
static std::atomic<bool> g_ktime_on{false};
static std::mutex g_ktime_mu;
struct KPending {
    int fam;
    cudaEvent_t e0, e1;
};
static std::vector<KPending> g_ktime_pending;
// events read out by a drain, reused by later scopes: creating and destroying
// events are driver calls, which wait behind any other client of the driver
// (a clock monitor, say) while the GPU runs dry inside the timed scope
static std::vector<cudaEvent_t> g_ktime_free;
static double g_ktime_ms[KF_NUM];
static int64_t g_ktime_n[KF_NUM];

bool ktime_enabled() { return g_ktime_on.load(std::memory_order_relaxed); }

// Reads every queued pair (waiting for its end event) into the totals; the
// events go back to the free list.
static void ktime_drain_locked() {
    for (const KPending& k : g_ktime_pending) {
        float ms = 0.0f;
        if (cudaEventSynchronize(k.e1) == cudaSuccess &&
            cudaEventElapsedTime(&ms, k.e0, k.e1) == cudaSuccess) {
            g_ktime_ms[k.fam] += ms;
            g_ktime_n[k.fam] += 1;
            g_ktime_free.push_back(k.e0);
            g_ktime_free.push_back(k.e1);
        } else {
            cudaEventDestroy(k.e0);
            cudaEventDestroy(k.e1);
        }
    }
    g_ktime_pending.clear();
    cudaGetLastError();
}

// An event recorded on `stream`: a reused one when the free list has one
// (a reused event that will not record, e.g. one from another device, is
// destroyed and a new one made), else a new one; null on failure.
static cudaEvent_t ktime_record(cudaStream_t stream) {
    cudaEvent_t ev = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_ktime_mu);
        if (!g_ktime_free.empty()) {
            ev = g_ktime_free.back();
            g_ktime_free.pop_back();
        }
    }
    if (ev && cudaEventRecord(ev, stream) == cudaSuccess) return ev;
    if (ev) cudaEventDestroy(ev);
    cudaGetLastError();
    ev = nullptr;
    if (cudaEventCreate(&ev) != cudaSuccess || cudaEventRecord(ev, stream) != cudaSuccess) {
        if (ev) cudaEventDestroy(ev);
        cudaGetLastError();
        return nullptr;
    }
    return ev;
}

KTime::KTime(cudaStream_t stream, bool capturing, int family) {
    if (!ktime_enabled() || capturing) return;
    e0 = ktime_record(stream);
    if (!e0) return;
    st = stream;
    fam = family;
}

KTime::~KTime() {
    if (!e0) return;
    cudaEvent_t e1 = ktime_record(st);
    if (!e1) {
        cudaEventDestroy(e0);
        return;
    }
    std::lock_guard<std::mutex> lk(g_ktime_mu);
    g_ktime_pending.push_back({fam, e0, e1});
    if (g_ktime_pending.size() >= 4096) ktime_drain_locked();
}

cudaError_t DevBuf::ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    const size_t want = bytes < 256 ? 256 : bytes;
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
}

void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}

// ---------------------------------------------------------------------------
// kernel configuration
// ---------------------------------------------------------------------------
template <int CAP, int MODE>
constexpr int warps_for() {
    constexpr int per = warp_smem_bytes<CAP, MODE>();
    constexpr int w = 65536 / per;
    return w > 8 ? 8 : (w < 1 ? 1 : w);
}


// warps per CTA of the map-replay reuse kernel (a float per slot)
template <int CAP>
constexpr int map_warps() {
    constexpr int w = 65536 / (4 * CAP);
    return w > 8 ? 8 : (w < 1 ? 1 : w);
}

constexpr int HEAVY_SMEM_MAX = 227 * 1024;  // largest dynamic shared memory of one CTA

// resident CTAs per SM of every warp-bin kernel (launches fill the GPU once
// and the warps pull rows from a counter)
static int g_warp_ctas[3][NUM_WARP_BINS];

template <int CAP, int MODE>
static void set_warp_attr() {
    constexpr int W = warps_for<CAP, MODE>();
    cudaFuncSetAttribute(k_warp<CAP, W, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         W * warp_smem_bytes<CAP, MODE>());
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_warp<CAP, W, MODE>, W * 32,
                                                      W * warp_smem_bytes<CAP, MODE>()) != cudaSuccess)
        n = 1;
    g_warp_ctas[MODE][__builtin_ctz(CAP / WARP_CAP_MIN)] = n > 0 ? n : 1;
    if (MODE == REUSE) {
        constexpr int WM = map_warps<CAP>();
        cudaFuncSetAttribute(k_warp_reuse_map<CAP, WM>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, WM * 4 * CAP);
    }
}

template <int MODE>
static void set_mode_attrs() {
    set_warp_attr<64, MODE>();
    set_warp_attr<128, MODE>();
    set_warp_attr<256, MODE>();
    set_warp_attr<512, MODE>();
    set_warp_attr<1024, MODE>();
    set_warp_attr<2048, MODE>();
    set_warp_attr<4096, MODE>();
    cudaFuncSetAttribute(k_heavy<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         HEAVY_SMEM_MAX);
}

// Heavy kernel shape for every mode and chunk width: warps per CTA chosen to
// keep the most warps resident per SM (each warp holds its own accumulator
// and bitmap in shared memory), and the resident CTAs per SM; the launches
// fill the GPU once and the CTAs pull batches of work items from a counter.
static int g_heavy_w[3][HEAVY_CW_LOG2_MAX + 1];
// dynamic shared memory of a heavy CTA of W warps: their accumulators and
// bitmaps, then the CTA's work-batch word
static size_t heavy_launch_smem(int mode, int cl, int W) {
    return (size_t)W * heavy_smem_bytes(mode, 1 << cl) + 16;
}
static int g_heavy_ctas[3][HEAVY_CW_LOG2_MAX + 1];
static int g_sms = 148;

static std::once_flag g_attr_once;
void init_kernel_attributes() {
    std::call_once(g_attr_once, [] {
        set_mode_attrs<COUNT>();
        set_mode_attrs<FILL>();
        set_mode_attrs<REUSE>();
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess)
            cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
        for (int cl = HEAVY_CW_LOG2_MIN; cl <= HEAVY_CW_LOG2_MAX; ++cl) {
            const void* fns[3] = {(const void*)k_heavy<COUNT>, (const void*)k_heavy<FILL>,
                                  (const void*)k_heavy<REUSE>};
            for (int m = 0; m < 3; ++m) {
                int best_w = 1, best_n = 1, best = 0;
                for (int W = 1; W <= HEAVY_MAX_WARPS; ++W) {
                    const size_t bytes = heavy_launch_smem(m, cl, W);
                    if (bytes > (size_t)HEAVY_SMEM_MAX) break;
                    int n = 0;
                    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fns[m], W * 32, bytes) !=
                        cudaSuccess) {
                        cudaGetLastError();
                        continue;
                    }
                    // at equal resident warps the larger CTA: its item
                    // batches (twice its warps) take fewer counter atomics
                    if (n * W >= best) {
                        best = n * W;
                        best_w = W;
                        best_n = n;
                    }
                }
                g_heavy_w[m][cl] = best_w;
                g_heavy_ctas[m][cl] = best_n;
            }
        }
        cudaGetLastError();
    });
}

static std::mutex g_params_mu;
static BinParams g_default_params = DEFAULT_BIN_PARAMS;

// RVSP_CUDA_BIN_PARAMS="tiny_ops,slack_shift,warp_cap_max,heavy_cw_log2" in
// the environment replaces the built-in default at the first use (ignored
// unless all four values parse and are in range).
static std::once_flag g_params_env_once;

BinParams default_params() {
    std::call_once(g_params_env_once, [] {
        const char* e = getenv("RVSP_CUDA_BIN_PARAMS");
        BinParams p;
        if (e && sscanf(e, "%d,%d,%d,%d", &p.tiny_ops, &p.slack_shift, &p.warp_cap_max,
                        &p.heavy_cw_log2) == 4 && bin_params_valid(p)) {
            std::lock_guard<std::mutex> lk(g_params_mu);
            g_default_params = p;
        }
    });
    std::lock_guard<std::mutex> lk(g_params_mu);
    return g_default_params;
}

void note_launch(rvsp_cuda_plan* plan, int n) {
    if (plan && plan->capturing)
        plan->graph_kernels += n;
    else
        g_launches += n;
}

template <int CAP, int MODE>
static void launch_warp(rvsp_cuda_plan* plan, const CsrView& A, const CsrView& B, int b,
                        const RowOut& o) {
    const int n = o.learned_bins ? plan->lcount[b] : plan->bin_count[b];
    const int32_t* rows = o.learned_bins ? plan->lbin_rows.as<int32_t>() + plan->loffs.off[b]
                                         : plan->bin_rows.as<int32_t>() + plan->offs.off[b];
    const int32_t* lo = plan->list_off.as<int32_t>() + plan->offs.off[b];
    uint16_t* pm = plan->pm16.as<uint16_t>() + plan->pm16_base[b];
    KTime kt(plan->stream, plan->capturing, KF_WARP_COUNT + MODE);
    if (MODE == REUSE && o.maps) {
        constexpr int WM = map_warps<CAP>();
        k_warp_reuse_map<CAP, WM><<<(n + WM - 1) / WM, WM * 32, WM * 4 * CAP, plan->stream>>>(
            A, B, rows, n, o.c_rp, o.c_v, lo, pm, o.err);
    } else {
        constexpr int W = warps_for<CAP, MODE>();
        const int fill = g_sms * g_warp_ctas[MODE][b - BIN_WARP0];
        const int grid = std::min((n + W - 1) / W, fill);
        int32_t* queue = &plan->misc.as<Misc>()->row_queue;
        cudaMemsetAsync(queue, 0, sizeof(int32_t), plan->stream);
        k_warp<CAP, W, MODE><<<grid, W * 32, W * warp_smem_bytes<CAP, MODE>(), plan->stream>>>(
            A, B, rows, n, plan->ops.as<int64_t>(), o.cnt, o.c_rp, o.c_ci, o.c_v,
            o.maps ? lo : nullptr, o.maps ? pm : nullptr, o.err, o.ctl, queue);
    }
    note_launch(plan, 1);
}

template <int MODE>
static void launch_bins(rvsp_cuda_plan* plan, const CsrView& A, const CsrView& B,
                        const RowOut& o) {
    const int32_t* rows = o.learned_bins ? plan->lbin_rows.as<int32_t>() : plan->bin_rows.as<int32_t>();
    for (int b = BIN_TINY; b < NUM_BINS; ++b) {
        const int n = o.learned_bins ? plan->lcount[b] : plan->bin_count[b];
        if (n == 0) continue;
        // heavy rows in the learned sweep: into their predicted slots when
        // the sweep fills (ctl.item_off), else left to the exact path
        if (o.learned_bins && b == BIN_HEAVY && !o.ctl.item_off) continue;
        const int32_t* r = rows + (o.learned_bins ? plan->loffs.off[b] : plan->offs.off[b]);
        if (b == BIN_TINY) {
            KTime kt(plan->stream, plan->capturing, KF_TINY_COUNT + MODE);
            const int32_t* lo = plan->list_off.as<int32_t>() + plan->offs.off[b];
            const int grid = (n + TINY_TPB - 1) / TINY_TPB;
            if (MODE == REUSE && o.maps)
                k_tiny_reuse_map<<<(n + 32 * TRM_WARPS - 1) / (32 * TRM_WARPS), 32 * TRM_WARPS, 0,
                                   plan->stream>>>(A, B, r, n, o.c_rp, o.c_v, lo,
                                                   plan->pm8.as<uint8_t>(), o.rp_out, o.err);
            else
                k_tiny<MODE><<<grid, TINY_TPB, 0, plan->stream>>>(
                    A, B, r, n, o.cnt, o.c_rp, o.c_ci, o.c_v, o.maps ? lo : nullptr,
                    o.maps ? plan->pm8.as<uint8_t>() : nullptr, o.err, o.ctl);
            note_launch(plan, 1);
        } else if (b < BIN_HEAVY) {
            switch (WARP_CAP_MIN << (b - BIN_WARP0)) {
                case 64: launch_warp<64, MODE>(plan, A, B, b, o); break;
                case 128: launch_warp<128, MODE>(plan, A, B, b, o); break;
                case 256: launch_warp<256, MODE>(plan, A, B, b, o); break;
                case 512: launch_warp<512, MODE>(plan, A, B, b, o); break;
                case 1024: launch_warp<1024, MODE>(plan, A, B, b, o); break;
                case 2048: launch_warp<2048, MODE>(plan, A, B, b, o); break;
                default: launch_warp<4096, MODE>(plan, A, B, b, o); break;
            }
        } else if (plan->n_items > 0) {
            KTime kt(plan->stream, plan->capturing, KF_HEAVY_COUNT + MODE);
            // (the learned sweep reaches here only with heavy slots, where every
            // row of the heavy items is kept heavy: no row mask to check)
            RowCtl ctl = o.ctl;
            const int cl = plan->params.heavy_cw_log2;
            const int W = g_heavy_w[MODE][cl];
            const int64_t fill = (int64_t)g_sms * g_heavy_ctas[MODE][cl];
            const int grid = (int)std::min<int64_t>((plan->n_items + W - 1) / W, fill);
            const HeavyAux aux{plan->bmeta.as<int4>(), plan->bdoff.as<int64_t>(),
                               plan->dir_ok ? plan->bdir.as<int32_t>() : nullptr,
                               plan->ameta_ok ? plan->ameta.as<int4>() : nullptr,
                               plan->ameta_ok ? plan->adoff.as<int32_t>() : nullptr,
                               plan->smask_words ? plan->bsmask.as<uint32_t>() : nullptr,
                               plan->smask_words};
            int32_t* queue = &plan->misc.as<Misc>()->heavy_queue;
            cudaMemsetAsync(queue, 0, sizeof(int32_t), plan->stream);
            k_heavy<MODE><<<grid, W * 32, heavy_launch_smem(MODE, cl, W), plan->stream>>>(
                A, B, plan->items.as<HeavyItem>(), plan->n_items, plan->item_cnt.as<int32_t>(),
                o.cnt, plan->item_scan.as<int64_t>(), o.c_rp, o.c_ci, o.c_v, o.err, ctl, cl,
                aux, queue);
            note_launch(plan, 1);
        }
    }
}

void run_rows(rvsp_cuda_plan* plan, int mode, const CsrView& A, const CsrView& B,
              const RowOut& o) {
    if (mode == COUNT) launch_bins<COUNT>(plan, A, B, o);
    else if (mode == FILL) launch_bins<FILL>(plan, A, B, o);
    else launch_bins<REUSE>(plan, A, B, o);
}

// Exclusive scan of n int32 counts. total_dev receives the sum.
// arrays of at most this many scan tiles (2048 counts each) take the
// one-CTA scan
constexpr int64_t SCAN_SINGLE_TILES = 4;

int scan_counts(rvsp_cuda_plan* plan, const int32_t* in, int64_t n, int64_t* out64,
                int32_t* out32, int64_t* total_dev) {
    const int64_t ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (ntiles == 0) return RVSP_SUCCESS;
    cudaError_t e = plan->scan_tmp.ensure((size_t)ntiles * sizeof(int64_t));
    if (e != cudaSuccess) return fail(e, "scan workspace");
    int64_t* tmp = plan->scan_tmp.as<int64_t>();
    KTime kt(plan->stream, plan->capturing, KF_SCAN);
    if (ntiles <= SCAN_SINGLE_TILES) {
        k_scan_single<<<1, SCAN_TPB, 0, plan->stream>>>(in, n, total_dev, out64, out32,
                                                        &plan->misc.as<Misc>()->overflow);
        note_launch(plan, 1);
        return RVSP_SUCCESS;
    }
    k_scan_reduce<<<(unsigned)ntiles, SCAN_TPB, 0, plan->stream>>>(in, n, tmp);
    k_scan_tiles<<<1, SCAN_TPB, 0, plan->stream>>>(tmp, ntiles, total_dev);
    k_scan_apply<<<(unsigned)ntiles, SCAN_TPB, 0, plan->stream>>>(
        in, n, tmp, total_dev, out64, out32, &plan->misc.as<Misc>()->overflow);
    note_launch(plan, 3);
    return RVSP_SUCCESS;
}

// Resolves an array to device memory, staging host memory into buf.
// Index arrays (cache_ok) are re-used when the same host pointer was staged
// before; values are always re-uploaded.
template <class T>
static int resolve(rvsp_cuda_plan* plan, DevBuf& buf, const void*& key, const T* ptr, size_t n,
                   bool cache_ok, const T** out) {
    if (n == 0) {
        cudaError_t e = buf.ensure(sizeof(T));
        if (e != cudaSuccess) return fail(e, "staging");
        *out = buf.as<T>();
        return RVSP_SUCCESS;
    }
    if (is_dev(ptr)) {
        *out = ptr;
        return RVSP_SUCCESS;
    }
    if (!(cache_ok && key == ptr && buf.p)) {
        cudaError_t e = buf.ensure(n * sizeof(T));
        if (e != cudaSuccess) return fail(e, "staging alloc");
        e = copy_to_device(buf.p, ptr, n * sizeof(T), plan->stream);
        if (e != cudaSuccess) return fail(e, "staging copy");
        key = ptr;
    }
    *out = buf.as<T>();
    return RVSP_SUCCESS;
}

int stage_operands(rvsp_cuda_plan* plan, const int32_t* a_rp, const int32_t* a_ci,
                   const float* a_v, const int32_t* b_rp, const int32_t* b_ci,
                   const float* b_v, bool cache_index, CsrView* A, CsrView* B) {
    int st;
    const int32_t *d_arp, *d_aci, *d_brp, *d_bci;
    const float *d_av = nullptr, *d_bv = nullptr;
    const size_t an = (size_t)plan->a_nnz, bn = (size_t)plan->b_nnz;
    if ((st = resolve(plan, plan->s_arp, plan->key[0], a_rp, (size_t)plan->a_rows + 1,
                      cache_index, &d_arp)))
        return st;
    if ((st = resolve(plan, plan->s_aci, plan->key[1], a_ci, an, cache_index, &d_aci))) return st;
    const void* dummy = nullptr;
    if (a_v && (st = resolve(plan, plan->s_av, dummy, a_v, an, false, &d_av))) return st;
    if (b_rp == a_rp && b_ci == a_ci && plan->b_rows == plan->a_rows && bn == an) {
        d_brp = d_arp;  // C = A * A: one staged copy serves both operands
        d_bci = d_aci;
    } else {
        if ((st = resolve(plan, plan->s_brp, plan->key[2], b_rp, (size_t)plan->b_rows + 1,
                          cache_index, &d_brp)))
            return st;
        if ((st = resolve(plan, plan->s_bci, plan->key[3], b_ci, bn, cache_index, &d_bci)))
            return st;
    }
    if (b_v) {
        if (b_v == a_v && bn == an) d_bv = d_av;
        else if ((st = resolve(plan, plan->s_bv, dummy, b_v, bn, false, &d_bv))) return st;
    }
    *A = CsrView{d_arp, d_aci, d_av, plan->a_rows, plan->a_cols, plan->a_nnz};
    *B = CsrView{d_brp, d_bci, d_bv, plan->b_rows, plan->b_cols, plan->b_nnz};
    return RVSP_SUCCESS;
}

// Analysis + binning. Leaves per-row op counts, bins and heavy items in the
// plan; one device->host read of the bin histogram.
int analyze(rvsp_cuda_plan* plan, CsrView& A, CsrView& B, bool features,
            int (*pre_sync)(rvsp_cuda_plan*)) {
    const int64_t M = plan->a_rows;
    cudaError_t e;
#define ENS(buf, bytes)                                        \
    if ((e = (buf).ensure(bytes)) != cudaSuccess) return fail(e, "plan alloc " #buf)
    ENS(plan->ops, M * 8);
    ENS(plan->ub, M * 4);
    ENS(plan->bin, M);
    ENS(plan->chunk_lo, M * 4);
    ENS(plan->nchunks, M * 4);
    ENS(plan->cnt, M * 4);
    ENS(plan->c_rp, (M + 1) * 4);
    ENS(plan->bin_rows, M * 4);
    ENS(plan->misc, sizeof(Misc));
    const int64_t tiles = (M + AN_TILE - 1) / AN_TILE;
    ENS(plan->tile_hist, NUM_BINS * tiles * 4);
    ENS(plan->tile_off, (NUM_BINS * tiles + 1) * 4);
    if (features) ENS(plan->feat, M * 16);
    Misc* misc = plan->misc.as<Misc>();
    if ((e = cudaMemsetAsync(misc, 0, sizeof(Misc), plan->stream)) != cudaSuccess)
        return fail(e, "memset");
    AnalyzeOut out{plan->ops.as<int64_t>(), plan->ub.as<int32_t>(), plan->bin.as<uint8_t>(),
                   plan->chunk_lo.as<int32_t>(), plan->nchunks.as<int32_t>(),
                   features ? plan->feat.as<float4>() : nullptr, misc->hist,
                   plan->tile_hist.as<int32_t>(), misc->totals, misc->bin_prod, &misc->err,
                   misc->nnz_ab};
    {
        KTime kt(plan->stream, plan->capturing, KF_ANALYSIS);
        k_analyze<<<(unsigned)tiles, AN_TILE, 0, plan->stream>>>(A, B, out, plan->params);
    }
    note_launch(plan, 1);
    int st = scan_counts(plan, plan->tile_hist.as<int32_t>(), NUM_BINS * tiles, nullptr,
                         plan->tile_off.as<int32_t>(), &misc->tile_total);
    if (st) return st;
    if (pre_sync && (st = pre_sync(plan))) return st;
    if ((e = cudaMemcpyAsync(&plan->host_misc, misc, sizeof(Misc), cudaMemcpyDeviceToHost,
                             plan->stream)) != cudaSuccess)
        return fail(e, "histogram read");
    if ((e = cudaStreamSynchronize(plan->stream)) != cudaSuccess) return fail(e, "analysis");
    trace_point("analysis (synced)");
    if (plan->host_misc.err) {
        g_err = "operand structure out of range (row_ptr or col_idx)";
        return RVSP_ERROR_INVALID_CSR;
    }
    // operands whose nnz the host did not know (-1): the analysis read it
    if (plan->a_nnz < 0 || plan->b_nnz < 0) {
        if (plan->host_misc.nnz_ab[0] < 0 || plan->host_misc.nnz_ab[1] < 0) {
            g_err = "operand row pointer ends below zero";
            return RVSP_ERROR_INVALID_CSR;
        }
        plan->a_nnz = A.nnz = plan->host_misc.nnz_ab[0];
        plan->b_nnz = B.nnz = plan->host_misc.nnz_ab[1];
    }
    int32_t acc = 0;
    for (int b = 0; b < NUM_BINS; ++b) {
        plan->bin_count[b] = plan->host_misc.hist[b];
        plan->offs.off[b] = acc;
        acc += plan->bin_count[b];
    }
    plan->n_items = (int32_t)plan->host_misc.totals[0];
    plan->products = plan->host_misc.totals[1];
    ENS(plan->items, (size_t)plan->n_items * sizeof(HeavyItem));
    ENS(plan->item_cnt, (size_t)plan->n_items * 4);
    ENS(plan->item_scan, ((size_t)plan->n_items + 1) * 8);
#undef ENS
    launch_bin_scatter(plan, plan->bin.as<uint8_t>(), plan->tile_off.as<int32_t>(),
                       plan->bin_rows.as<int32_t>(), true);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "analysis launch");
    if (plan->n_items > 0 && (st = build_heavy_aux(plan, A, B))) return st;
    return RVSP_SUCCESS;
}

// Per-B-row lookups of the heavy kernel (HeavyAux): metadata of every B row,
// and the chunk directory of long rows spanning several chunks, unless the
// directory would pass 2^28 entries (the kernel then binary-searches); then
// both copied beside the heavy rows' A entries when the copies fit in L2.
// One device->host read of the directory size.
int build_heavy_aux(rvsp_cuda_plan* plan, const CsrView& A, const CsrView& B) {
    const int64_t K = plan->b_rows;
    const int cl = plan->params.heavy_cw_log2;
    cudaError_t e;
    if ((e = plan->bmeta.ensure(K * 16)) != cudaSuccess ||
        (e = plan->bdcount.ensure(K * 4)) != cudaSuccess ||
        (e = plan->bdscan.ensure((K + 1) * 8)) != cudaSuccess ||
        (e = plan->bdoff.ensure(K * 8)) != cudaSuccess)
        return fail(e, "heavy lookups");
    Misc* misc = plan->misc.as<Misc>();
    {
        KTime kt(plan->stream, plan->capturing, KF_ANALYSIS);
        k_bmeta<<<(unsigned)((K + 255) / 256), 256, 0, plan->stream>>>(
            B, cl, plan->bmeta.as<int4>(), plan->bdcount.as<int32_t>(), &misc->err);
    }
    note_launch(plan, 1);
    int st = scan_counts(plan, plan->bdcount.as<int32_t>(), K, plan->bdscan.as<int64_t>(), nullptr,
                         &misc->dir_total);
    if (st) return st;
    int64_t total = 0;
    if ((e = cudaMemcpyAsync(&total, &misc->dir_total, 8, cudaMemcpyDeviceToHost,
                             plan->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(plan->stream)) != cudaSuccess)
        return fail(e, "directory size");
    plan->dir_ok = total > 0 && total <= (int64_t(1) << 28) &&
                   plan->bdir.ensure((size_t)total * 4) == cudaSuccess;
    cudaGetLastError();  // a refused directory allocation only costs the searches
    KTime kt(plan->stream, plan->capturing, KF_ANALYSIS);
    if (plan->dir_ok) {
        k_bdir<<<(unsigned)((K * 32 + 255) / 256), 256, 0, plan->stream>>>(
            B, cl, plan->bmeta.as<int4>(), plan->bdcount.as<int32_t>(),
            plan->bdscan.as<int64_t>(), plan->bdoff.as<int64_t>(), plan->bdir.as<int32_t>());
        note_launch(plan, 1);
    }
    // Chunk presence masks of the B rows left without a directory, when
    // their words stay small: a visit of such a row whose chunk bit is clear
    // skips its two binary searches (on R-MAT 2^20, 96 % of those searches
    // found no entry).
    {
        const int64_t nchunks = ((int64_t)plan->b_cols + (1 << cl) - 1) >> cl;
        const int64_t words = (nchunks + 31) / 32;
        const size_t mbytes = (size_t)(K * words * 4);
        constexpr size_t SMASK_MAX_BYTES = 128u << 20;
        plan->smask_words = 0;
        if (K > 0 && nchunks > 1 && mbytes <= SMASK_MAX_BYTES &&
            plan->bsmask.ensure(mbytes) == cudaSuccess &&
            cudaMemsetAsync(plan->bsmask.p, 0, mbytes, plan->stream) == cudaSuccess) {
            plan->smask_words = (int32_t)words;
            k_bmask<<<(unsigned)((K * 32 + 255) / 256), 256, 0, plan->stream>>>(
                B, cl, plan->bmeta.as<int4>(), plan->dir_ok ? plan->bdoff.as<int64_t>() : nullptr,
                plan->smask_words, plan->bsmask.as<uint32_t>());
            note_launch(plan, 1);
        }
        cudaGetLastError();  // without masks the searches run
    }
    // The copies are read once per (item, entry): they pay only while they
    // stay in L2 (measured: R-MAT 2^18, 84 MB of copies, 5 % faster; R-MAT
    // 2^20, 335 MB, 12 % slower than the column-index walk whose per-B-row
    // metadata stays in L2).
    // (no free-memory query: it is a driver call that waits behind any other
    // client of the driver, e.g. a clock monitor, with the GPU idle)
    const int32_t nh = plan->bin_count[BIN_HEAVY];
    const size_t abytes = 20 * (size_t)plan->a_nnz;
    constexpr size_t AMETA_MAX_BYTES = 96u << 20;
    plan->ameta_ok = nh > 0 && abytes <= AMETA_MAX_BYTES &&
                     plan->ameta.ensure(16 * (size_t)plan->a_nnz) == cudaSuccess &&
                     plan->adoff.ensure(4 * (size_t)plan->a_nnz) == cudaSuccess;
    cudaGetLastError();  // without the copies the walk looks up through A.ci
    if (plan->ameta_ok) {
        k_ameta<<<(unsigned)(((int64_t)nh * 32 + 255) / 256), 256, 0, plan->stream>>>(
            A, B, plan->bin_rows.as<int32_t>() + plan->offs.off[BIN_HEAVY], nh,
            plan->bmeta.as<int4>(), plan->dir_ok ? plan->bdoff.as<int64_t>() : nullptr,
            plan->ameta.as<int4>(), plan->adoff.as<int32_t>(), &misc->err);
        note_launch(plan, 1);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "heavy lookups launch");
    return RVSP_SUCCESS;
}

// Stable partition of the plan's rows by bin (k_bin_scatter); with
// heavy_items the heavy rows also get their column-chunk work items.
void launch_bin_scatter(rvsp_cuda_plan* plan, const uint8_t* bin, const int32_t* tile_off,
                        int32_t* bin_rows, bool heavy_items) {
    const int64_t M = plan->a_rows;
    Misc* misc = plan->misc.as<Misc>();
    KTime kt(plan->stream, plan->capturing, KF_ANALYSIS);
    k_bin_scatter<<<(unsigned)((M + AN_TILE - 1) / AN_TILE), AN_TILE, 0, plan->stream>>>(
        (int32_t)M, bin, tile_off, plan->chunk_lo.as<int32_t>(), plan->nchunks.as<int32_t>(),
        bin_rows, &misc->item_cursor, heavy_items ? plan->items.as<HeavyItem>() : nullptr);
    note_launch(plan, 1);
}

// Exact count + scan: C's row pointer in plan->c_rp, nnz in plan->c_nnz.
int count_exact(rvsp_cuda_plan* plan, const CsrView& A, const CsrView& B) {
    int st = count_launch(plan, A, B);
    return st ? st : count_read(plan);
}

// The count kernels and scans, enqueued only: C's row pointer lands in
// plan->c_rp, the heavy chunks' offsets in plan->item_scan, nnz(C) in
// Misc::scan_total.
int count_launch(rvsp_cuda_plan* plan, const CsrView& A, const CsrView& B) {
    cudaError_t e;
    const int64_t M = plan->a_rows;
    if ((e = cudaMemsetAsync(plan->cnt.p, 0, M * 4, plan->stream)) != cudaSuccess)
        return fail(e, "memset");
    Misc* misc = plan->misc.as<Misc>();
    RowOut o{plan->cnt.as<int32_t>(), nullptr, nullptr, nullptr, &misc->err, false};
    run_rows(plan, COUNT, A, B, o);
    int st = scan_counts(plan, plan->cnt.as<int32_t>(), M, nullptr, plan->c_rp.as<int32_t>(),
                         &misc->scan_total);
    if (st) return st;
    if (plan->n_items > 0) {
        st = scan_counts(plan, plan->item_cnt.as<int32_t>(), plan->n_items,
                         plan->item_scan.as<int64_t>(), nullptr, &misc->scan_total2);
        if (st) return st;
    }
    plan->items_counted = true;
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "count launch");
    return RVSP_SUCCESS;
}

// Waits for count_launch's work and takes nnz(C) into plan->c_nnz.
int count_read(rvsp_cuda_plan* plan) {
    cudaError_t e;
    Misc* misc = plan->misc.as<Misc>();
    if ((e = cudaMemcpyAsync(&plan->host_misc, misc, sizeof(Misc), cudaMemcpyDeviceToHost,
                             plan->stream)) != cudaSuccess)
        return fail(e, "count read");
    if ((e = cudaStreamSynchronize(plan->stream)) != cudaSuccess) return fail(e, "count");
    trace_point("exact count (synced)");
    if (plan->host_misc.err) {
        g_err = "operand structure out of range (row_ptr or col_idx)";
        return RVSP_ERROR_INVALID_CSR;
    }
    if (plan->host_misc.overflow || plan->host_misc.scan_total > INT32_MAX) {
        g_err = "nnz(C) exceeds INT32_MAX";
        return RVSP_ERROR_ALLOCATION_FAILED;
    }
    plan->c_nnz = plan->host_misc.scan_total;
    return RVSP_SUCCESS;
}

// Allocates the position maps and their offsets (an exclusive scan of the
// per-row product counts in bin-list order) when the plan records them and
// they fit: total products below 2^31 and map bytes within a quarter of the
// device memory currently free. Returns whether the next FILL records them.
bool prepare_maps(rvsp_cuda_plan* plan) {
    plan->maps_ready = false;
    if (!plan->map_policy || plan->products <= 0 || plan->products >= INT32_MAX) return false;
    int64_t p8 = plan->host_misc.bin_prod[BIN_TINY], p16 = 0;
    for (int b = BIN_WARP0; b < BIN_HEAVY; ++b) {
        plan->pm16_base[b] = p16;
        p16 += plan->host_misc.bin_prod[b];
    }
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const int64_t M = plan->a_rows;
    const size_t need = (size_t)p8 + 2 * (size_t)p16 + 8 * (size_t)(M + 1);
    if (need > free_b / 4) return false;
    if (plan->pm8.ensure((size_t)p8) != cudaSuccess || plan->pm16.ensure(2 * (size_t)p16) != cudaSuccess ||
        plan->list_ops.ensure(4 * (size_t)M) != cudaSuccess ||
        plan->list_off.ensure(4 * (size_t)(M + 1)) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    Misc* misc = plan->misc.as<Misc>();
    k_list_ops<<<(unsigned)((M + 255) / 256), 256, 0, plan->stream>>>(
        plan->bin_rows.as<int32_t>(), (int32_t)M, plan->ops.as<int64_t>(),
        plan->list_ops.as<int32_t>(), &misc->overflow);
    note_launch(plan, 1);
    if (scan_counts(plan, plan->list_ops.as<int32_t>(), M, nullptr, plan->list_off.as<int32_t>(),
                    &misc->list_total) != RVSP_SUCCESS)
        return false;
    return cudaGetLastError() == cudaSuccess;
}

void reset_graph(rvsp_cuda_plan* plan) {
    if (plan->gexec) cudaGraphExecDestroy(plan->gexec);
    plan->gexec = nullptr;
    plan->graph_kernels = 0;
    memset(plan->gkey, 0, sizeof(plan->gkey));
}

// Numeric-only pass on a known pattern, replayed from a CUDA graph keyed on
// the device pointers it reads and writes.
int reuse_numeric(rvsp_cuda_plan* plan, const CsrView& A, const CsrView& B, const int32_t* c_ci,
                  float* c_v, int32_t* rp_out) {
    const void* key[9] = {A.rp, A.ci, A.v, B.rp, B.ci, B.v, c_ci, c_v, rp_out};
    cudaError_t e;
    if (!(plan->gexec && memcmp(key, plan->gkey, sizeof(key)) == 0)) {
        reset_graph(plan);
        cudaGraph_t g = nullptr;
        if ((e = cudaStreamBeginCapture(plan->stream, cudaStreamCaptureModeThreadLocal)) !=
            cudaSuccess)
            return fail(e, "begin capture");
        plan->capturing = true;
        RowOut o{nullptr, plan->c_rp.as<int32_t>(), const_cast<int32_t*>(c_ci), c_v,
                 &plan->misc.as<Misc>()->err, plan->maps_ready};
        o.rp_out = rp_out;
        run_rows(plan, REUSE, A, B, o);
        plan->capturing = false;
        e = cudaStreamEndCapture(plan->stream, &g);
        if (e != cudaSuccess) return fail(e, "end capture");
        e = cudaGraphInstantiate(&plan->gexec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            plan->gexec = nullptr;
            return fail(e, "graph instantiate");
        }
        memcpy(plan->gkey, key, sizeof(key));
    }
    if ((e = cudaGraphLaunch(plan->gexec, plan->stream)) != cudaSuccess)
        return fail(e, "graph launch");
    g_launches += plan->graph_kernels;
    return RVSP_SUCCESS;
}

}  // namespace rvsp

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int rvsp_cuda_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

const char* rvsp_cuda_last_error(void) { return g_err.c_str(); }

int rvsp_cuda_is_device_pointer(const void* p) { return is_dev(p) ? 1 : 0; }

void rvsp_cuda_free(void* p) {
    if (p) cudaFree(p);
}

int64_t rvsp_cuda_launch_count(void) { return (int64_t)g_launches.load(); }

int rvsp_cuda_kernel_timing(int on) {
    std::lock_guard<std::mutex> lk(g_ktime_mu);
    ktime_drain_locked();
    for (int i = 0; i < KF_NUM; ++i) {
        g_ktime_ms[i] = 0.0;
        g_ktime_n[i] = 0;
    }
    g_ktime_on.store(on != 0);
    return RVSP_SUCCESS;
}

int rvsp_cuda_kernel_times(double* ms_out, int64_t* launches_out, int32_t n) {
    if (!ms_out) return RVSP_ERROR_NULL_POINTER;
    if (n < KF_NUM) return RVSP_ERROR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(g_ktime_mu);
    ktime_drain_locked();
    for (int i = 0; i < KF_NUM; ++i) {
        ms_out[i] = g_ktime_ms[i];
        if (launches_out) launches_out[i] = g_ktime_n[i];
    }
    return RVSP_SUCCESS;
}

const char* rvsp_cuda_kernel_family(int32_t i) {
    static const char* names[KF_NUM] = {
        "k_tiny<COUNT>", "k_tiny<FILL>", "k_tiny_reuse", "k_warp<COUNT>", "k_warp<FILL>",
        "k_warp_reuse", "k_heavy<COUNT>", "k_heavy<FILL>", "k_heavy<REUSE>", "analysis",
        "scan", "learned_sizing", "k_compact", "batched_pack"};
    return i >= 0 && i < KF_NUM ? names[i] : nullptr;
}

int rvsp_cuda_plan_create(rvsp_cuda_plan_t* out, int algo) {
    if (!out) return RVSP_ERROR_NULL_POINTER;
    *out = nullptr;
    if (algo != RVSP_CUDA_ALGO_EXACT && algo != RVSP_CUDA_ALGO_LEARNED)
        return RVSP_ERROR_UNSUPPORTED_BACKEND;
    if (rvsp_cuda_device_count() == 0) {
        g_err = "no CUDA device";
        return RVSP_ERROR_UNSUPPORTED_BACKEND;
    }
    init_kernel_attributes();
    rvsp_cuda_plan* p = new (std::nothrow) rvsp_cuda_plan();
    if (!p) return RVSP_ERROR_ALLOCATION_FAILED;
    p->algo = algo;
    p->params = default_params();
    // A blocking stream: work the caller queued on the legacy default stream
    // (e.g. filling device-resident operands) is ordered before the plan's
    // kernels, and the caller's later default-stream work after them.
    cudaError_t e = cudaStreamCreateWithFlags(&p->stream, cudaStreamDefault);
    if (e != cudaSuccess) {
        delete p;
        return fail(e, "stream create");
    }
    *out = p;
    return RVSP_SUCCESS;
}

void rvsp_cuda_plan_destroy(rvsp_cuda_plan_t p) {
    if (!p) return;
    if (p->stream) cudaStreamSynchronize(p->stream);
    reset_graph(p);
    DevBuf* bufs[] = {&p->s_arp, &p->s_aci, &p->s_av, &p->s_brp, &p->s_bci, &p->s_bv,
                      &p->ops, &p->ub, &p->bin, &p->chunk_lo, &p->nchunks, &p->feat,
                      &p->cnt, &p->c_rp, &p->bin_rows, &p->items, &p->item_cnt,
                      &p->item_scan, &p->scan_tmp, &p->misc, &p->s_cci, &p->s_cv,
                      &p->pred_cap, &p->slot_off, &p->tmp_ci, &p->tmp_v, &p->row_flag,
                      &p->tile_hist, &p->tile_off, &p->pm8, &p->pm16, &p->list_ops,
                      &p->list_off, &p->lbin, &p->lcap, &p->ltile_hist, &p->ltile_off,
                      &p->lbin_rows, &p->need, &p->pflag, &p->hmask, &p->hovf,
                      &p->item_off, &p->bmeta, &p->bdcount, &p->bdscan, &p->bdoff, &p->bdir,
                      &p->ameta, &p->adoff, &p->bsmask};
    for (DevBuf* b : bufs) b->release();
    if (p->side) {
        cudaStreamSynchronize(p->side);
        cudaStreamDestroy(p->side);
    }
    if (p->side_fork) cudaEventDestroy(p->side_fork);
    if (p->host_pin) cudaFreeHost(p->host_pin);
    if (p->stream) cudaStreamDestroy(p->stream);
    delete p;
}

int rvsp_cuda_plan_set_async(rvsp_cuda_plan_t p, int async) {
    if (!p) return RVSP_ERROR_NULL_POINTER;
    p->async = async ? 1 : 0;
    return RVSP_SUCCESS;
}

void* rvsp_cuda_plan_stream(rvsp_cuda_plan_t p) { return p ? (void*)p->stream : nullptr; }

static int params_from(const int32_t* v, int32_t n, BinParams* out) {
    if (!v) return RVSP_ERROR_NULL_POINTER;
    if (n < BIN_PARAMS_N) return RVSP_ERROR_INVALID_ARGUMENT;
    const BinParams p{v[0], v[1], v[2], v[3]};
    if (!bin_params_valid(p)) {
        g_err = "bin parameters out of range";
        return RVSP_ERROR_INVALID_ARGUMENT;
    }
    *out = p;
    return RVSP_SUCCESS;
}

static int params_to(const BinParams& p, int32_t* v, int32_t n) {
    if (!v) return RVSP_ERROR_NULL_POINTER;
    if (n < BIN_PARAMS_N) return RVSP_ERROR_INVALID_ARGUMENT;
    v[0] = p.tiny_ops;
    v[1] = p.slack_shift;
    v[2] = p.warp_cap_max;
    v[3] = p.heavy_cw_log2;
    return RVSP_SUCCESS;
}

int rvsp_cuda_plan_set_params(rvsp_cuda_plan_t p, const int32_t* params, int32_t n) {
    if (!p) return RVSP_ERROR_NULL_POINTER;
    BinParams bp;
    int st = params_from(params, n, &bp);
    if (st) return st;
    if (p->stream) cudaStreamSynchronize(p->stream);
    p->params = bp;
    // the analysed bins and heavy items belong to the old parameters
    p->analysed = false;
    p->maps_ready = false;
    p->filled = nullptr;
    p->filled_host = nullptr;
    reset_graph(p);
    return RVSP_SUCCESS;
}

int rvsp_cuda_plan_get_params(rvsp_cuda_plan_t p, int32_t* params, int32_t n) {
    if (!p) return RVSP_ERROR_NULL_POINTER;
    return params_to(p->params, params, n);
}

int rvsp_cuda_set_default_params(const int32_t* params, int32_t n) {
    (void)default_params();  // the environment's value is read first, then replaced
    BinParams bp = DEFAULT_BIN_PARAMS;
    if (params) {
        int st = params_from(params, n, &bp);
        if (st) return st;
    }
    std::lock_guard<std::mutex> lk(g_params_mu);
    g_default_params = bp;
    return RVSP_SUCCESS;
}

int rvsp_cuda_get_default_params(int32_t* params, int32_t n) {
    return params_to(default_params(), params, n);
}

int rvsp_cuda_symbolic(rvsp_cuda_plan_t plan, int32_t a_rows, int32_t a_cols, int32_t a_nnz,
                       const int32_t* a_rp, const int32_t* a_ci, int32_t b_rows, int32_t b_cols,
                       int32_t b_nnz, const int32_t* b_rp, const int32_t* b_ci,
                       int64_t* c_nnz_out, size_t* ws_bytes_out) {
    if (!plan || !a_rp || !b_rp || !c_nnz_out || !ws_bytes_out) return RVSP_ERROR_NULL_POINTER;
    if ((a_nnz > 0 && !a_ci) || (b_nnz > 0 && !b_ci)) return RVSP_ERROR_NULL_POINTER;
    if (a_rows <= 0 || a_cols <= 0 || b_rows <= 0 || b_cols <= 0 || a_nnz < 0 || b_nnz < 0)
        return RVSP_ERROR_INVALID_ARGUMENT;
    if (a_cols != b_rows) return RVSP_ERROR_INVALID_ARGUMENT;
    plan->analysed = false;
    plan->maps_ready = false;
    plan->filled = nullptr;
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
    trace_point("symbolic: enter");
    int st = stage_operands(plan, a_rp, a_ci, nullptr, b_rp, b_ci, nullptr, false, &A, &B);
    if (st) return st;
    trace_point("symbolic: operands staged");
    if (plan->algo == RVSP_CUDA_ALGO_LEARNED) {
        if ((st = learned_symbolic(plan, A, B, false))) return st;
    } else {
        if ((st = analyze(plan, A, B, plan->features))) return st;
        if ((st = count_exact(plan, A, B))) return st;
    }
    plan->analysed = true;
    *c_nnz_out = plan->c_nnz;
    *ws_bytes_out = 256;
    return RVSP_SUCCESS;
}

// Waits, when it goes out of scope, for the side stream's copy into the
// caller's host memory.
struct SideCopy {
    cudaStream_t s = nullptr;
    ~SideCopy() {
        if (s) cudaStreamSynchronize(s);
    }
};

static bool side_stream(rvsp_cuda_plan* plan) {
    if (plan->side) return true;
    cudaStream_t s = nullptr;
    cudaEvent_t ev = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
        if (s) cudaStreamDestroy(s);
        cudaGetLastError();
        return false;  // the copy stays on the plan's stream
    }
    plan->side = s;
    plan->side_fork = ev;
    return true;
}

int rvsp_cuda_numeric(rvsp_cuda_plan_t plan, const int32_t* a_rp, const int32_t* a_ci,
                      const float* a_v, const int32_t* b_rp, const int32_t* b_ci,
                      const float* b_v, int32_t* c_rp, int32_t* c_ci, float* c_v,
                      int fill_structure, void* workspace) {
    (void)workspace;
    if (!plan || !a_rp || !b_rp || !c_rp || !c_ci || !c_v) return RVSP_ERROR_NULL_POINTER;
    if (!a_ci || !a_v || !b_ci || !b_v) return RVSP_ERROR_NULL_POINTER;
    if (!plan->analysed) return RVSP_ERROR_INVALID_ARGUMENT;
    cudaError_t e;
    const int64_t M = plan->a_rows, nnz = plan->c_nnz;
    const bool dev_rp = is_dev(c_rp), dev_ci = is_dev(c_ci), dev_v = is_dev(c_v);
    // Row pointer: the analysed structure, final before this call. Into host
    // memory it is copied on the side stream, so the device->host copy runs
    // beside the operands' host->device copies (PCIe carries both directions
    // at once); every return waits for it.
    SideCopy side_rp;
    // Value-only reuse of a product whose rows are all tiny: the map-replay
    // kernel writes the row pointer beside the values, no separate copy.
    const bool rp_fused = dev_rp && !fill_structure && nnz > 0 && plan->maps_ready &&
                          plan->bin_count[BIN_TINY] == M;
    if (!rp_fused) {
        if (!dev_rp && side_stream(plan)) {
            if ((e = cudaEventRecord(plan->side_fork, plan->stream)) != cudaSuccess ||
                (e = cudaStreamWaitEvent(plan->side, plan->side_fork, 0)) != cudaSuccess ||
                (e = cudaMemcpyAsync(c_rp, plan->c_rp.p, (M + 1) * 4, cudaMemcpyDeviceToHost,
                                     plan->side)) != cudaSuccess)
                return fail(e, "row_ptr copy");
            side_rp.s = plan->side;
        } else if ((e = cudaMemcpyAsync(c_rp, plan->c_rp.p, (M + 1) * 4,
                                        dev_rp ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                        plan->stream)) != cudaSuccess) {
            return fail(e, "row_ptr copy");
        }
    }
    CsrView A, B;
    int st = stage_operands(plan, a_rp, a_ci, a_v, b_rp, b_ci, b_v, true, &A, &B);
    if (st) return st;
    int32_t* d_ci = c_ci;
    float* d_v = c_v;
    if (!dev_ci) {
        if ((e = plan->s_cci.ensure((size_t)nnz * 4)) != cudaSuccess) return fail(e, "C staging");
        d_ci = plan->s_cci.as<int32_t>();
    }
    if (!dev_v) {
        if ((e = plan->s_cv.ensure((size_t)nnz * 4)) != cudaSuccess) return fail(e, "C staging");
        d_v = plan->s_cv.as<float>();
    }
    if (nnz > 0) {
        if (fill_structure) {
            if (!plan->items_counted && plan->n_items > 0) {
                // heavy rows the learned analysis sized by prediction: count
                // their column chunks now so the chunk fills know their offsets
                k_heavy_uncounted<<<(unsigned)((M + 255) / 256), 256, 0, plan->stream>>>(
                    (int32_t)M, plan->bin.as<uint8_t>(), plan->need.as<uint8_t>(),
                    plan->row_flag.as<uint8_t>());
                RowOut ho{nullptr, nullptr, nullptr, nullptr, &plan->misc.as<Misc>()->err, false};
                ho.ctl.only = plan->row_flag.as<uint8_t>();
                const int32_t saved[NUM_BINS - 1] = {};
                int32_t keep[NUM_BINS];
                memcpy(keep, plan->bin_count, sizeof(keep));
                memcpy(plan->bin_count, saved, sizeof(saved));  // heavy bin only
                run_rows(plan, COUNT, A, B, ho);
                memcpy(plan->bin_count, keep, sizeof(keep));
                if ((st = scan_counts(plan, plan->item_cnt.as<int32_t>(), plan->n_items,
                                      plan->item_scan.as<int64_t>(), nullptr,
                                      &plan->misc.as<Misc>()->tile_total)))
                    return st;
                plan->items_counted = true;
            }
            const bool maps = prepare_maps(plan);
            RowOut o{nullptr, plan->c_rp.as<int32_t>(), d_ci, d_v, &plan->misc.as<Misc>()->err,
                     maps};
            run_rows(plan, FILL, A, B, o);
            if (maps) {
                plan->maps_ready = true;
                reset_graph(plan);
            }
            if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "fill launch");
            if (!dev_ci) {
                if ((e = copy_to_host(c_ci, d_ci, (size_t)nnz * 4, plan->stream)) != cudaSuccess)
                    return fail(e, "col_idx copy");
                plan->filled_host = c_ci;
            }
        } else {
            if (!dev_ci && plan->filled_host != c_ci) {
                if ((e = cudaMemcpyAsync(d_ci, c_ci, (size_t)nnz * 4, cudaMemcpyHostToDevice,
                                         plan->stream)) != cudaSuccess)
                    return fail(e, "col_idx upload");
                plan->filled_host = c_ci;
            }
            if ((st = reuse_numeric(plan, A, B, d_ci, d_v, rp_fused ? c_rp : nullptr))) return st;
        }
        if (!dev_v && (e = copy_to_host(c_v, d_v, (size_t)nnz * 4, plan->stream)) != cudaSuccess)
            return fail(e, "values copy");
    }
    const bool all_dev = dev_rp && dev_ci && dev_v;
    if (!(plan->async && all_dev)) {
        int32_t err = 0;
        if ((e = cudaMemcpyAsync(&plan->host_misc.err, &plan->misc.as<Misc>()->err, 4,
                                 cudaMemcpyDeviceToHost, plan->stream)) != cudaSuccess)
            return fail(e, "error word read");
        if ((e = cudaStreamSynchronize(plan->stream)) != cudaSuccess) return fail(e, "numeric");
        trace_point("numeric (synced)");
        err = plan->host_misc.err;
        if (err) {
            g_err = "operand structure out of range (row_ptr or col_idx)";
            return RVSP_ERROR_INVALID_CSR;
        }
    }
    return RVSP_SUCCESS;
}

}  // extern "C"

namespace rvsp {

// Products up to which the one-shot allocates C at the product count (an
// upper bound on nnz(C): at most 256 MB of C) and runs count, scan and fill
// back to back, reading nnz(C) back once at the end instead of between the
// count and the fill.
constexpr int64_t ONESHOT_FUSED_PRODUCTS = int64_t(1) << 25;

int oneshot_exact_device(rvsp_cuda_plan* plan, int32_t a_rows, int32_t a_cols, int32_t b_cols,
                         const int32_t* a_rp, const int32_t* a_ci, const float* a_v,
                         const int32_t* b_rp, const int32_t* b_ci, const float* b_v,
                         int32_t** c_rp_out, int32_t** c_ci_out, float** c_v_out,
                         int64_t* c_nnz_out) {
    plan->analysed = false;
    plan->maps_ready = false;
    plan->filled = nullptr;
    plan->filled_host = nullptr;
    reset_graph(plan);
    plan->a_rows = a_rows;
    plan->a_cols = a_cols;
    plan->a_nnz = -1;  // read by the analysis
    plan->b_rows = a_cols;
    plan->b_cols = b_cols;
    plan->b_nnz = -1;
    memset(plan->key, 0, sizeof(plan->key));
    CsrView A, B;
    int st = stage_operands(plan, a_rp, a_ci, a_v, b_rp, b_ci, b_v, false, &A, &B);
    if (st) return st;
    if ((st = analyze(plan, A, B, plan->features))) return st;
    const int64_t M = a_rows;
    const bool fused = plan->products <= ONESHOT_FUSED_PRODUCTS;
    int64_t cap;
    if (fused) {
        if ((st = count_launch(plan, A, B))) return st;
        cap = plan->products;
    } else {
        if ((st = count_exact(plan, A, B))) return st;
        cap = plan->c_nnz;
    }
    int32_t *rp = nullptr, *ci = nullptr;
    float* v = nullptr;
    const size_t alloc = cap > 0 ? (size_t)cap : 1;
    cudaError_t e = cudaMallocAsync((void**)&rp, ((size_t)M + 1) * 4, plan->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&ci, alloc * 4, plan->stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&v, alloc * 4, plan->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(rp, plan->c_rp.p, ((size_t)M + 1) * 4, cudaMemcpyDeviceToDevice,
                            plan->stream);
    Misc* misc = plan->misc.as<Misc>();
    if (e == cudaSuccess) {
        RowOut o{nullptr, plan->c_rp.as<int32_t>(), ci, v, &misc->err, false};
        run_rows(plan, FILL, A, B, o);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&plan->host_misc, misc, sizeof(Misc), cudaMemcpyDeviceToHost,
                            plan->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(plan->stream);
    trace_point("one-shot exact (synced)");
    const auto release = [&] {
        if (rp) cudaFreeAsync(rp, plan->stream);
        if (ci) cudaFreeAsync(ci, plan->stream);
        if (v) cudaFreeAsync(v, plan->stream);
    };
    if (e != cudaSuccess) {
        release();
        return fail(e, "one-shot product");
    }
    if (plan->host_misc.err) {
        release();
        g_err = "operand structure out of range (row_ptr or col_idx)";
        return RVSP_ERROR_INVALID_CSR;
    }
    if (fused) {
        if (plan->host_misc.overflow || plan->host_misc.scan_total > INT32_MAX) {
            release();
            g_err = "nnz(C) exceeds INT32_MAX";
            return RVSP_ERROR_ALLOCATION_FAILED;
        }
        plan->c_nnz = plan->host_misc.scan_total;
    }
    plan->analysed = true;
    *c_rp_out = rp;
    *c_ci_out = ci;
    *c_v_out = v;
    *c_nnz_out = plan->c_nnz;
    return RVSP_SUCCESS;
}

}  // namespace rvsp

extern "C" {

int rvsp_cuda_op_counts(rvsp_cuda_plan_t plan, int64_t* out, int32_t n) {
    if (!plan || !out) return RVSP_ERROR_NULL_POINTER;
    if (!plan->analysed) return RVSP_ERROR_INVALID_ARGUMENT;
    if (n < plan->a_rows) return RVSP_ERROR_INVALID_ARGUMENT;
    cudaError_t e = cudaMemcpyAsync(out, plan->ops.p, (size_t)plan->a_rows * 8,
                                    is_dev(out) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                    plan->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(plan->stream);
    return e == cudaSuccess ? RVSP_SUCCESS : fail(e, "op counts");
}

static int csr_check_impl(bool canonical, int32_t rows, int32_t cols, int32_t nnz,
                          const int32_t* rp, const int32_t* ci, int32_t* bad_row_out) {
    if (bad_row_out) *bad_row_out = -1;
    if (rows < 0 || cols < 0 || nnz < 0 || !rp) return 1;
    if (nnz > 0 && !ci) return 1;
    const bool dev = is_dev(rp);
    int32_t first = 0;
    cudaError_t e = cudaSuccess;
    if (dev) {
        if ((e = cudaMemcpy(&first, rp, 4, cudaMemcpyDeviceToHost)) != cudaSuccess)
            return fail(e, "csr check");
    } else {
        first = rp[0];
    }
    if (first != 0) return 1;
    if (rows == 0) return 0;
    const int32_t *d_rp = rp, *d_ci = ci;
    void *tmp_rp = nullptr, *tmp_ci = nullptr, *worst = nullptr;
    if (!dev) {
        if ((e = cudaMalloc(&tmp_rp, ((size_t)rows + 1) * 4)) != cudaSuccess) return fail(e, "csr check");
        cudaMemcpy(tmp_rp, rp, ((size_t)rows + 1) * 4, cudaMemcpyHostToDevice);
        d_rp = (const int32_t*)tmp_rp;
    }
    if (!is_dev(ci) && nnz > 0) {
        if ((e = cudaMalloc(&tmp_ci, (size_t)nnz * 4)) != cudaSuccess) {
            cudaFree(tmp_rp);
            return fail(e, "csr check");
        }
        cudaMemcpy(tmp_ci, ci, (size_t)nnz * 4, cudaMemcpyHostToDevice);
        d_ci = (const int32_t*)tmp_ci;
    }
    unsigned long long init = ~0ull, res = ~0ull;
    e = cudaMalloc(&worst, 8);
    if (e == cudaSuccess) e = cudaMemcpy(worst, &init, 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        if (canonical)
            k_csr_check<true><<<(rows + 255) / 256, 256>>>(rows, cols, nnz, d_rp, d_ci,
                                                           (unsigned long long*)worst);
        else
            k_csr_check<false><<<(rows + 255) / 256, 256>>>(rows, cols, nnz, d_rp, d_ci,
                                                            (unsigned long long*)worst);
        note_launch(nullptr, 1);
        e = cudaMemcpy(&res, worst, 8, cudaMemcpyDeviceToHost);
    }
    cudaFree(worst);
    cudaFree(tmp_rp);
    cudaFree(tmp_ci);
    if (e != cudaSuccess) return fail(e, "csr check");
    if (res == ~0ull) return 0;
    if (bad_row_out) *bad_row_out = (int32_t)(res >> 8);
    return (int)(res & 0xff);
}

int rvsp_cuda_csr_check(int32_t rows, int32_t cols, int32_t nnz, const int32_t* rp,
                        const int32_t* ci, int32_t* bad_row_out) {
    return csr_check_impl(true, rows, cols, nnz, rp, ci, bad_row_out);
}

int rvsp_cuda_csr_validate(int32_t rows, int32_t cols, int32_t nnz, const int32_t* rp,
                           const int32_t* ci) {
    if (!rp || (nnz > 0 && !ci)) return RVSP_ERROR_NULL_POINTER;
    if (rows <= 0 || cols <= 0 || nnz < 0) return RVSP_ERROR_INVALID_ARGUMENT;
    int32_t last = 0;
    cudaError_t e = is_dev(rp) ? cudaMemcpy(&last, rp + rows, 4, cudaMemcpyDeviceToHost)
                               : (last = rp[rows], cudaSuccess);
    if (e != cudaSuccess) return fail(e, "csr validate");
    if (last != nnz) return RVSP_ERROR_INVALID_CSR;
    const int st = csr_check_impl(false, rows, cols, nnz, rp, ci, nullptr);
    if (st < 0) return st;
    return st == 0 ? RVSP_SUCCESS : RVSP_ERROR_INVALID_CSR;
}

int rvsp_cuda_plan_collect_features(rvsp_cuda_plan_t plan, int on) {
    if (!plan) return RVSP_ERROR_NULL_POINTER;
    plan->features = on != 0;
    return RVSP_SUCCESS;
}

int rvsp_cuda_plan_row_stats(rvsp_cuda_plan_t plan, float* feat_out, int32_t* cnt_out,
                             int32_t* ub_out, int32_t n) {
    if (!plan) return RVSP_ERROR_NULL_POINTER;
    if (!plan->analysed || n < plan->a_rows) return RVSP_ERROR_INVALID_ARGUMENT;
    const bool have_feat = plan->features || plan->algo == RVSP_CUDA_ALGO_LEARNED;
    if (feat_out && !have_feat) return RVSP_ERROR_INVALID_ARGUMENT;
    const size_t M = (size_t)plan->a_rows;
    cudaError_t e = cudaSuccess;
    auto kind = [](const void* p) {
        return is_dev(p) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    };
    if (feat_out) e = cudaMemcpyAsync(feat_out, plan->feat.p, M * 16, kind(feat_out), plan->stream);
    // exact counts: C's row pointer differences are exact on every path
    if (e == cudaSuccess && cnt_out) {
        std::vector<int32_t> rp(M + 1);
        e = cudaMemcpyAsync(rp.data(), plan->c_rp.p, (M + 1) * 4, cudaMemcpyDeviceToHost,
                            plan->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(plan->stream);
        if (e == cudaSuccess) {
            std::vector<int32_t> c(M);
            for (size_t i = 0; i < M; ++i) c[i] = rp[i + 1] - rp[i];
            e = cudaMemcpyAsync(cnt_out, c.data(), M * 4,
                                is_dev(cnt_out) ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost,
                                plan->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(plan->stream);
        }
    }
    if (e == cudaSuccess && ub_out)
        e = cudaMemcpyAsync(ub_out, plan->ub.p, M * 4, kind(ub_out), plan->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(plan->stream);
    return e == cudaSuccess ? RVSP_SUCCESS : fail(e, "row stats");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free row pointer from per-row counts.
//
// For callers that cannot allocate device memory at the point they need C's
// row pointer: code recording a CUDA graph under stream capture (cudaMalloc
// there is illegal or stays out of the graph), latency-critical or real-time
// loops that cannot afford the device-wide synchronisation cudaFree implies,
// and hosts where another allocator already owns the device memory budget.
// The scan's scratch (one int64 partial sum per 2048-row tile, the total and
// an overflow flag) lives in the file-scope array below instead of a plan.
//
// The array is a single static allocation of about 32 KiB that every GPU
// holding this library keeps until the process exits, so the row count is
// capped at NOALLOC_MAX_ROWS. All calls on a device share it and it keeps the
// last call's contents: the overflow flag is cleared at the start of every
// call (the partial sums and total are fully rewritten), and calls whose work
// overlaps on the GPU (different streams, no ordering between them) race on
// it and must be serialised by the caller.
// ---------------------------------------------------------------------------
namespace {

constexpr int64_t NOALLOC_MAX_TILES = 4096;
constexpr int64_t NOALLOC_MAX_ROWS = NOALLOC_MAX_TILES * SCAN_TILE;  // 8,388,608 rows

struct NoAllocScratch {
    int64_t tile_sums[NOALLOC_MAX_TILES];
    int64_t total;
    int32_t overflow;
    int32_t pad;
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
// the scratch array's device address per device, and the context it was
// resolved in (a cudaDeviceReset makes a new context, in which the module,
// and with it the array, may load at another address)
struct NoAllocAddr {
    unsigned long long ctx_id;
    NoAllocScratch* addr;
};
NoAllocAddr g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};

}  // namespace

namespace rvsp {

// Unique id of the calling thread's current CUDA context (cuCtxGetId: never
// reused within the process), or 0 when the driver cannot tell, in which case
// the caller resolves the address again.
unsigned long long current_context_id() {
    using GetCurrent = int (*)(void**);
    using GetId = int (*)(void*, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
        cudaGetLastError();
    });
    if (!get_current || !get_id) return 0;
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

}  // namespace rvsp

extern "C" {

int rvsp_cuda_row_ptr_noalloc(const int32_t* counts, int32_t n, int32_t* row_ptr,
                              int64_t* total_out, void* stream) {
    if (!counts || !row_ptr) return RVSP_ERROR_NULL_POINTER;
    if (n <= 0 || (int64_t)n > NOALLOC_MAX_ROWS) {
        g_err = "rvsp_cuda_row_ptr_noalloc: n must be in [1, 8388608] (static scratch of 4096 "
                "tiles x 2048 rows)";
        return RVSP_ERROR_INVALID_ARGUMENT;
    }
    if (!is_dev(counts) || !is_dev(row_ptr)) {
        g_err = "rvsp_cuda_row_ptr_noalloc: counts and row_ptr must be device memory";
        return RVSP_ERROR_INVALID_ARGUMENT;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(e, "rvsp_cuda_row_ptr_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
        g_err = "rvsp_cuda_row_ptr_noalloc: device index too large";
        return RVSP_ERROR_INVALID_ARGUMENT;
    }
    NoAllocScratch* scratch = nullptr;
    {
        // once per device (and context), with that device current: the
        // host-side name of a __device__ array is not a device address, so
        // resolve it here
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        NoAllocAddr& slot = g_noalloc_addr[dev];
        const unsigned long long ctx = current_context_id();
        if (!slot.addr || ctx == 0 || slot.ctx_id != ctx) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) {
                slot.addr = nullptr;
                return fail(e, "rvsp_cuda_row_ptr_noalloc: cudaGetSymbolAddress");
            }
            slot.addr = static_cast<NoAllocScratch*>(p);
            slot.ctx_id = current_context_id();
        }
        scratch = slot.addr;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t ntiles = ((int64_t)n + SCAN_TILE - 1) / SCAN_TILE;
    e = cudaMemsetAsync(&scratch->overflow, 0, sizeof(int32_t), st);
    if (e != cudaSuccess) return fail(e, "rvsp_cuda_row_ptr_noalloc: clear");
    k_scan_reduce<<<(unsigned)ntiles, SCAN_TPB, 0, st>>>(counts, n, scratch->tile_sums);
    k_scan_tiles<<<1, SCAN_TPB, 0, st>>>(scratch->tile_sums, ntiles, &scratch->total);
    k_scan_apply<<<(unsigned)ntiles, SCAN_TPB, 0, st>>>(counts, n, scratch->tile_sums,
                                                        &scratch->total, nullptr, row_ptr,
                                                        &scratch->overflow);
    note_launch(nullptr, 3);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e, "rvsp_cuda_row_ptr_noalloc");
    if (total_out) {
        int64_t host[2] = {0, 0};  // total, then the overflow flag in the low word
        e = cudaMemcpyAsync(host, &scratch->total, sizeof(host), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail(e, "rvsp_cuda_row_ptr_noalloc: read total");
        *total_out = host[0];
        if ((int32_t)(host[1] & 0xffffffff) != 0 || host[0] > INT32_MAX) {
            g_err = "rvsp_cuda_row_ptr_noalloc: total exceeds INT32_MAX";
            return RVSP_ERROR_ALLOCATION_FAILED;
        }
    }
    return RVSP_SUCCESS;
}

}  // extern "C"
