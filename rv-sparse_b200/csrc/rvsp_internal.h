// Internal state shared by the C-ABI translation units of the B200 backend.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <string>

#include "spgemm_types.cuh"

namespace rvsp {

// Grow-only device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes);
    void release();
    template <class T>
    T* as() const {
        return reinterpret_cast<T*>(p);
    }
};

// Small device-side block of counters and flags of one plan.
struct Misc {
    int32_t hist[NUM_BINS];    // rows per bin
    int32_t cursor[NUM_BINS];  // bin scatter cursors
    int64_t totals[2];         // heavy items, products
    int32_t item_cursor;
    int32_t overflow;          // a 32-bit row pointer would overflow
    int64_t scan_total;        // nnz(C)
    int64_t scan_total2;       // heavy item total / learned capacity total
    int32_t n_overflow_rows;   // learned path: rows that outgrew their capacity
    int32_t pad;
    int64_t overflow_ub;       // learned path: sum of upper bounds of those rows
    int32_t err;               // ERR_* bits raised by kernels
    int32_t pad2;
    int64_t bin_prod[NUM_BINS];  // products per bin
    int64_t tile_total;        // scratch total of the tile-histogram scan
    int64_t list_total;        // scratch total of the product-offset scan
    int32_t lhist[NUM_BINS];   // learned path: rows per predicted-capacity bin
    int32_t n_need;            // learned path: rows sent to the exact path
    int32_t n_need_heavy;      //   of which heavy rows
    int64_t slot_total;        // learned path: sum of predicted capacities
    int64_t lstats[8];         // learned path statistics (see rvsp_cuda_plan_learned_stats)
    int64_t ltile_total;
    int64_t dir_total;         // heavy-row B directory entries
    int32_t heavy_queue;       // next heavy work item of the running launch
    int32_t row_queue;         // next row of the running warp-bin launch
    unsigned long long pool_fill;  // learned path: entries placed in the overflow pool
    int32_t nnz_ab[2];         // nnz of A and B as the analysis read them (operands
                               // whose nnz the host did not know)
};

// Output pointers of a row-kernel launch.
struct RowOut {
    int32_t* cnt;
    const int32_t* c_rp;
    int32_t* c_ci;
    float* c_v;
    int32_t* err;
    bool maps;           // FILL: record position maps; REUSE: replay them
    RowCtl ctl = {nullptr, nullptr, 0, nullptr, nullptr, nullptr, 0, 0};
    bool learned_bins = false;  // iterate the predicted-capacity bins instead
    // REUSE, every row a tiny row: the map-replay kernel also writes the
    // caller's row pointer (the copy of the analysed one is skipped)
    int32_t* rp_out = nullptr;
};

extern thread_local std::string g_err;
extern std::atomic<long long> g_launches;

int fail(cudaError_t e, const char* what);

// Host-side phase tracer: with RVSP_TRACE=1 in the environment, every trace
// point prints the host time since the previous one (per thread) to stderr.
bool trace_on();
inline void trace_point(const char* what) {
    if (!trace_on()) return;
    static thread_local std::chrono::steady_clock::time_point last;
    const auto now = std::chrono::steady_clock::now();
    fprintf(stderr, "[rvsp] %-28s %9.1f us\n", what,
            std::chrono::duration<double, std::micro>(now - last).count());
    last = now;
}
bool is_dev(const void* p);
// Unique id of the calling thread's current CUDA context, 0 when unknown.
unsigned long long current_context_id();
// Host arrays for results: free()-compatible; large ones 2 MiB aligned with
// transparent huge pages advised, or a released one taken from the cache.
void* host_alloc(size_t bytes);
// Release a host array (any free()-compatible block): large ones go to the
// cache that host_alloc draws from, the rest to free().
void host_free(void* p);
// Device->host copy of bytes into dst, finished on return (enqueued only on a
// stream that is recording a graph); large copies into pageable memory are
// staged through pinned pieces and host threads.
cudaError_t copy_to_host(void* dst, const void* src, size_t bytes, cudaStream_t stream);
// Host->device copy of bytes from src, enqueued on stream; large copies from
// pageable memory are staged through the pinned pieces (those return once
// the upload has completed), the rest are plain cudaMemcpyAsync calls.
cudaError_t copy_to_device(void* dst, const void* src, size_t bytes, cudaStream_t stream);

// Opt-in device timing of the kernels by family (rvsp_cuda_kernel_timing):
// a KTime scope records a CUDA event pair around the launches it covers on
// the plan's stream (none while the plan records a graph); the pairs are
// read when the totals are queried.
enum KernelFamily : int {
    KF_TINY_COUNT = 0, KF_TINY_FILL, KF_TINY_REUSE,
    KF_WARP_COUNT, KF_WARP_FILL, KF_WARP_REUSE,
    KF_HEAVY_COUNT, KF_HEAVY_FILL, KF_HEAVY_REUSE,
    KF_ANALYSIS,  // row analysis, binning, heavy-row lookups
    KF_SCAN,      // prefix sums
    KF_LEARNED,   // inference, predicted bins, re-run masks
    KF_COMPACT,   // slot -> C copies of the learned path
    KF_PACK,      // batched products: operands stacked into one product
    KF_NUM
};
bool ktime_enabled();
struct KTime {
    cudaEvent_t e0 = nullptr;
    cudaStream_t st = nullptr;
    int fam = 0;
    KTime(cudaStream_t stream, bool capturing, int family);
    ~KTime();
};

void init_kernel_attributes();
BinParams default_params();  // the process-wide default of new and internal plans
void keep_pool_memory();     // the device pool keeps freed blocks (one-shot entry points)

}  // namespace rvsp

struct rvsp_cuda_plan {
    int algo = 4;
    int async = 0;
    cudaStream_t stream = nullptr;
    // side stream for a host-resident C row pointer's copy, which overlaps
    // the operands' host->device copies (created on first use)
    cudaStream_t side = nullptr;
    cudaEvent_t side_fork = nullptr;
    int32_t* host_pin = nullptr;  // pinned words for small device->host reads
    bool analysed = false;
    bool capturing = false;
    int32_t a_rows = 0, a_cols = 0, a_nnz = 0, b_rows = 0, b_cols = 0, b_nnz = 0;
    // bin parameters of the next analysis (the plan's own once set, else the
    // process default at plan creation)
    rvsp::BinParams params = rvsp::DEFAULT_BIN_PARAMS;

    // staging copies of host-resident operands; key[] holds the host
    // pointers of the staged index arrays (a_rp, a_ci, b_rp, b_ci)
    rvsp::DevBuf s_arp, s_aci, s_av, s_brp, s_bci, s_bv;
    const void* key[4] = {nullptr, nullptr, nullptr, nullptr};

    // analysed structure
    rvsp::DevBuf ops, ub, bin, chunk_lo, nchunks, feat, cnt, c_rp, bin_rows, tile_hist, tile_off;
    rvsp::DevBuf items, item_cnt, item_scan, scan_tmp, misc;
    // per-B-row lookups of the heavy kernel (HeavyAux), built by the analysis
    // when the product has chunked rows; dir_ok when the directory exists
    rvsp::DevBuf bmeta, bdcount, bdscan, bdoff, bdir;
    rvsp::DevBuf ameta, adoff;  // per A entry of heavy rows (HeavyAux)
    rvsp::DevBuf bsmask;        // chunk presence of B rows without a directory
    bool ameta_ok = false;
    bool dir_ok = false;
    int32_t smask_words = 0;    // words per B row of bsmask, 0: no masks
    int32_t bin_count[rvsp::NUM_BINS] = {};
    rvsp::BinOffsets offs = {};
    int32_t n_items = 0;
    int64_t c_nnz = 0;
    int64_t products = 0;
    rvsp::Misc host_misc = {};

    // device staging of a host-resident C; filled_host is the host col_idx
    // whose structure the staging currently holds
    rvsp::DevBuf s_cci, s_cv;
    const int32_t* filled = nullptr;
    const int32_t* filled_host = nullptr;

    // per-product output positions, recorded by the first fill and replayed by
    // numeric-only reuse (uint8 for tiny rows, uint16 for warp-bin rows);
    // list_off is the product offset of every entry of bin_rows
    int map_policy = 1;   // 0: never record (one-shot plans)
    bool features = false;  // analysis also writes the per-row model features
    bool items_counted = true;  // every heavy work item's count (item_scan) is valid
    bool maps_ready = false;
    rvsp::DevBuf pm8, pm16, list_ops, list_off;
    int64_t pm16_base[rvsp::NUM_BINS] = {};

    // learned path: predicted capacities, their bins (stable partition like
    // the exact bins), slot offsets of the over-allocated output, the mask of
    // rows sent back to the exact path
    rvsp::DevBuf lbin, lcap, ltile_hist, ltile_off, lbin_rows, need, pflag;
    int32_t lcount[rvsp::NUM_BINS] = {};
    rvsp::BinOffsets loffs = {};
    int64_t slot_total = 0;
    int64_t lstats[10] = {};  // see rvsp_cuda_plan_learned_stats
    rvsp::DevBuf pred_cap, slot_off, tmp_ci, tmp_v, row_flag;
    // heavy rows of the learned sweep: rows kept heavy (hmask), rows whose
    // chunks found no room (hovf), where each chunk went in the slot buffer
    // (item_off), the size of the shared overflow pool after the slots
    rvsp::DevBuf hmask, hovf, item_off;
    int64_t pool_cap = 0;

    bool heavy_slots = false;  // the last learned analysis sized heavy rows by prediction

    // numeric-only CUDA graph
    cudaGraphExec_t gexec = nullptr;
    const void* gkey[9] = {};
    int graph_kernels = 0;
};

namespace rvsp {
int stage_operands(rvsp_cuda_plan* plan, const int32_t* a_rp, const int32_t* a_ci,
                   const float* a_v, const int32_t* b_rp, const int32_t* b_ci, const float* b_v,
                   bool cache_index, CsrView* A, CsrView* B);
int analyze(rvsp_cuda_plan* plan, CsrView& A, CsrView& B, bool features,
            int (*pre_sync)(rvsp_cuda_plan*) = nullptr);
int count_exact(rvsp_cuda_plan* plan, const CsrView& A, const CsrView& B);
int count_launch(rvsp_cuda_plan* plan, const CsrView& A, const CsrView& B);
int count_read(rvsp_cuda_plan* plan);
// One-shot exact product of device-resident operands into new device arrays
// (rvsp_cuda_spgemm_f32's exact path when every operand array is on the
// device; the operands' nnz are read by the analysis).
int oneshot_exact_device(rvsp_cuda_plan* plan, int32_t a_rows, int32_t a_cols, int32_t b_cols,
                         const int32_t* a_rp, const int32_t* a_ci, const float* a_v,
                         const int32_t* b_rp, const int32_t* b_ci, const float* b_v,
                         int32_t** c_rp_out, int32_t** c_ci_out, float** c_v_out,
                         int64_t* c_nnz_out);
void run_rows(rvsp_cuda_plan* plan, int mode, const CsrView& A, const CsrView& B,
              const RowOut& o);
int scan_counts(rvsp_cuda_plan* plan, const int32_t* in, int64_t n, int64_t* out64,
                int32_t* out32, int64_t* total_dev);
void note_launch(rvsp_cuda_plan* plan, int n);
void reset_graph(rvsp_cuda_plan* plan);
int build_heavy_aux(rvsp_cuda_plan* plan, const CsrView& A, const CsrView& B);
void launch_bin_scatter(rvsp_cuda_plan* plan, const uint8_t* bin, const int32_t* tile_off,
                        int32_t* bin_rows, bool heavy_items);
int learned_symbolic(rvsp_cuda_plan* plan, CsrView& A, CsrView& B, bool fused);
int learned_finish(rvsp_cuda_plan* plan, const CsrView& A, const CsrView& B, int32_t* c_ci,
                   float* c_v);
int learned_spgemm(rvsp_cuda_plan* plan, int32_t a_rows, int32_t a_cols, int32_t a_nnz,
                   const int32_t* a_rp, const int32_t* a_ci, const float* a_v, int32_t b_rows,
                   int32_t b_cols, int32_t b_nnz, const int32_t* b_rp, const int32_t* b_ci,
                   const float* b_v, int device_out, int32_t** c_rp_out, int32_t** c_ci_out,
                   float** c_v_out, int32_t* c_nnz_out);
}  // namespace rvsp
