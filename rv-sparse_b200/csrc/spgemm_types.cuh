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
// ---------------------------------------------------------------------------
constexpr int TINY_CAP = 32;      // thread-per-row: rows with ops <= 32
constexpr int WARP_CAP_MIN = 64;  // warp-per-row hash tables: 64 .. 4096 slots
constexpr int NUM_WARP_BINS = 7;
constexpr int WARP_CAP_MAX = WARP_CAP_MIN << (NUM_WARP_BINS - 1);
constexpr int BIN_EMPTY = 0;
constexpr int BIN_TINY = 1;
constexpr int BIN_WARP0 = 2;
constexpr int BIN_HEAVY = BIN_WARP0 + NUM_WARP_BINS;
constexpr int NUM_BINS = BIN_HEAVY + 1;
constexpr int HEAVY_CW = 8192;  // columns per heavy work item
constexpr int AN_TILE = 256;    // rows per analysis / binning tile

struct HeavyItem {
    int32_t row;
    int32_t chunk;
    int32_t first;  // index of the row's first item
    int32_t pad;
};

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
struct RowCtl {
    const int64_t* slot_off;
    const uint8_t* only;
    int learned;
};

__host__ __device__ inline int bin_of(int64_t ops, int32_t ub) {
    if (ub <= 0) return BIN_EMPTY;
    if (ops <= TINY_CAP) return BIN_TINY;
    int64_t need = (int64_t)ub + (ub >> 2);  // load factor <= 0.8
    int cap = WARP_CAP_MIN, b = BIN_WARP0;
    while (cap < need && b < BIN_HEAVY) {
        cap <<= 1;
        ++b;
    }
    return b;  // BIN_HEAVY when need > WARP_CAP_MAX
}

}  // namespace rvsp
