// Types and constants shared by the B200 SpGEMM kernels and their host-side
// launchers: operand views, row bins, heavy work items.

#pragma once

#include <cstdint>
#include <climits>
#include <cuda_runtime.h>

namespace rvsp {


constexpr unsigned FULL = 0xffffffffu;

enum Mode : int { COUNT = 0, FILL = 1, REUSE = 2 };

struct CsrView {
    const int32_t* __restrict__ rp;
    const int32_t* __restrict__ ci;
    const float* __restrict__ v;
    int32_t rows;
    int32_t cols;
    int32_t nnz;
};

// Bits of the per-plan device error word.
constexpr int ERR_STRUCTURE = 1;  // an operand's row pointer or column index is out of range

// ---------------------------------------------------------------------------
// Bins. A row's upper bound ub = min(ops, b_cols) bounds its distinct columns.
// Which rows go to which bin, how many threads a row gets and how large its
// table is are runtime parameters of a plan (BinParams, chosen by the
// autotuner or left at their defaults); the constants below are the
// compiled limits those parameters range over.
// ---------------------------------------------------------------------------
constexpr int TINY_CAP = 32;      // thread-per-row rows hold at most 32 products
constexpr int WARP_CAP_MIN = 64;  // warp-per-row hash tables: 64 .. 4096 slots
constexpr int NUM_WARP_BINS = 7;
constexpr int WARP_CAP_MAX = WARP_CAP_MIN << (NUM_WARP_BINS - 1);
constexpr int BIN_EMPTY = 0;
constexpr int BIN_TINY = 1;
constexpr int BIN_WARP0 = 2;
constexpr int BIN_HEAVY = BIN_WARP0 + NUM_WARP_BINS;
constexpr int NUM_BINS = BIN_HEAVY + 1;
constexpr int HEAVY_CW_LOG2_MIN = 9;    // heavy column chunks: 512 ..
constexpr int HEAVY_CW_LOG2_MAX = 13;   // .. 8192 columns per work item
constexpr int AN_TILE = 256;    // rows per analysis / binning tile

// Runtime bin parameters of a plan.
//   tiny_ops       rows with at most tiny_ops products run one thread per row
//                  (0 .. TINY_CAP); the others get a warp
//   slack_shift    a warp row's hash table holds at least ub + (ub >> slack_shift)
//                  slots (1 .. 4: load factor at most 2/3, 4/5, 8/9, 16/17)
//   warp_cap_max   largest warp table (64 .. 4096, a power of two); rows that
//                  need more are heavy: a warp per column chunk
//   heavy_cw_log2  log2 of the columns per heavy work item (9 .. 13)
struct BinParams {
    int32_t tiny_ops;
    int32_t slack_shift;
    int32_t warp_cap_max;
    int32_t heavy_cw_log2;
};
constexpr int BIN_PARAMS_N = 4;
constexpr BinParams DEFAULT_BIN_PARAMS = {TINY_CAP, 2, 2048, 11};

__host__ __device__ inline bool bin_params_valid(const BinParams& p) {
    const bool pow2 = p.warp_cap_max > 0 && (p.warp_cap_max & (p.warp_cap_max - 1)) == 0;
    return p.tiny_ops >= 0 && p.tiny_ops <= TINY_CAP && p.slack_shift >= 1 && p.slack_shift <= 4 &&
           pow2 && p.warp_cap_max >= WARP_CAP_MIN && p.warp_cap_max <= WARP_CAP_MAX &&
           p.heavy_cw_log2 >= HEAVY_CW_LOG2_MIN && p.heavy_cw_log2 <= HEAVY_CW_LOG2_MAX;
}

// Work item of the heavy kernel: a column chunk of a heavy row.
struct HeavyItem {
    int32_t row;
    int32_t chunk;
    int32_t first;  // index of the row's first item
    int32_t pad;
};

// Per-B-row lookups for the heavy kernel, built by the analysis when the
// product has chunked rows: meta[k] = {row start, row end, first column, last
// column}; for rows of at least DIR_MIN_LEN entries that span several column
// chunks, doff[k] >= 0 and dir[doff[k] + i] is the first position of the
// row whose column is >= (first chunk + i) * chunk width, for i = 0 .. (last
// chunk - first chunk + 1); doff[k] = -1 otherwise (dir may be null).
struct HeavyAux {
    const int4* meta;
    const int64_t* doff;
    const int32_t* dir;
    // the same per A entry of the heavy rows (ameta[j] = meta[A.ci[j]];
    // adoff[j] = the directory offset of B row k = A.ci[j], or -(k + 2) when
    // it has none), or null: looked up through A.ci
    const int4* ameta;
    const int32_t* adoff;
    // chunk presence of the B rows that span several chunks without a
    // directory: bit c of row k's smask_words words is set when the row has
    // an entry in column chunk c (a clear bit spares the row's two binary
    // searches), or null
    const uint32_t* smask;
    int32_t smask_words;
};
constexpr int DIR_MIN_LEN = 32;

struct BinOffsets {
    int32_t off[NUM_BINS];
};

// Extra controls of a row-kernel launch, used by the learned path.
//   slot_off  FILL writes row r at slot_off[r] instead of c_rp[r]; the slot
//             holds slot_off[r+1] - slot_off[r] entries; the row's count goes
//             to cnt[r]
//   only      when set, row r is processed only if only[r] != 0
//   learned   tables are sized by a prediction: a row whose table fills up
//             (or, with slot_off, whose count passes its slot) gets cnt[r] = -1
//             and is left for the exact path instead of raising an error
//   item_off  heavy FILL into slots: every chunk takes its place in the row's
//             slot with an atomic add of its count to cnt[r] (so cnt[r] ends
//             as the row's exact count and item_cnt holds every chunk's); a
//             chunk past the slot's end takes a place in the shared overflow
//             pool [pool_base, pool_base + pool_cap) of the same buffer
//             (*pool_fill counts its use); item_off[w] is where the chunk
//             went, or -1 when the pool was full too, in which case ovf[r] is
//             set and the row is left for the exact fill
struct RowCtl {
    const int64_t* slot_off;
    const uint8_t* only;
    int learned;
    int64_t* item_off;
    uint8_t* ovf;
    unsigned long long* pool_fill;
    int64_t pool_base;
    int64_t pool_cap;
};

// Table bin of a warp row holding up to ub distinct columns: the smallest
// warp table with ub + (ub >> slack_shift) slots, BIN_HEAVY past warp_cap_max.
__host__ __device__ inline int table_bin(int32_t ub, const BinParams& p) {
    const int64_t need = (int64_t)ub + (ub >> p.slack_shift);
    int cap = WARP_CAP_MIN, b = BIN_WARP0;
    while (cap < need && cap < p.warp_cap_max) {
        cap <<= 1;
        ++b;
    }
    return cap < need ? BIN_HEAVY : b;
}

__host__ __device__ inline int bin_of(int64_t ops, int32_t ub, const BinParams& p) {
    if (ub <= 0) return BIN_EMPTY;
    if (ops <= p.tiny_ops) return BIN_TINY;
    return table_bin(ub, p);
}

}  // namespace rvsp
