// Device kernels of the B200 CSR SpGEMM backend (C = A * B, FP32).
//
// Gustavson row-wise product, as in rv-sparse
// src/kernels/spgemm/gustavson_core_f32.inc:18-64 (numeric) and
// src/kernels/spgemm/rvsp_symbolic.c:13-137 (symbolic count and fill),
// restructured for the GPU:
//
//   k_analyze      per-row op count (rvsp_symbolic.c:41), upper bound on the
//                  row's distinct columns, learned-model features, bin id
//   k_bin_scatter  rows grouped by bin; heavy rows expanded into
//                  (row, column-chunk) work items
//   k_tiny<MODE>   thread per row, rows with <= 32 products
//   k_warp<CAP,..> warp per row, shared-memory hash table of CAP slots
//   k_heavy<..>    warp per (row, column chunk), dense shared-memory
//                  accumulator + occupancy bitmap over CW columns
//   k_scan_*       exclusive scan of row counts into C's row pointer
//
// Each row kernel runs in one of three modes:
//   COUNT  distinct output columns per row (rvsp_symbolic_count)
//   FILL   sorted column indices and values (rvsp_symbolic_fill + numeric)
//   REUSE  values only, on a known sorted pattern (descriptor reuse)
//
// Order of operations. The reference adds, per output column, the FP32
// products a*b in A-row order starting from +0.0f, with no FMA contraction
// (accum_scalar_f32.c:69 under -std=c11). Every kernel here reproduces that
// order exactly: products are formed with __fmul_rn and added with
// __fadd_rn; a thread or warp owns a whole row (or a whole column chunk of a
// row); when one warp step holds several products of the same column, they
// are combined in lane order, which is A-row order (ordered_add below).
// Values are therefore bit-identical to the reference scalar kernel.

#pragma once

#include "spgemm_types.cuh"

namespace rvsp {

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// Row range [*s, *e) of row r of M. Rows outside the matrix or offsets outside
// [0, nnz] flag ERR_STRUCTURE and read as empty, so a malformed operand can
// never send a kernel outside its arrays.
__device__ __forceinline__ void row_range(const CsrView& M, int r, int* s, int* e,
                                          int32_t* err) {
    if ((unsigned)r >= (unsigned)M.rows) {
        *s = *e = 0;
        atomicOr(err, ERR_STRUCTURE);
        return;
    }
    const int a = M.rp[r], b = M.rp[r + 1];
    if (a < 0 || b < a || b > M.nnz) {
        *s = *e = 0;
        atomicOr(err, ERR_STRUCTURE);
        return;
    }
    *s = a;
    *e = b;
}

__device__ __forceinline__ int warp_incl_scan(int x) {
    const int lane = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

__device__ __forceinline__ uint32_t hash_slot(int32_t col, int log2cap) {
    return ((uint32_t)col * 0x9E3779B1u) >> (32 - log2cap);
}

// First index in [lo, hi) with a[idx] >= target (hi if none); a sorted
// ascending. Warp-cooperative 32-ary search; all lanes get the result.
__device__ __forceinline__ int warp_lower_bound(const int32_t* __restrict__ a, int lo, int hi,
                                                int target) {
    const int lane = lane_id();
    while (hi - lo > 32) {
        const int n = hi - lo;
        const int stride = (n + 31) >> 5;
        const int idx = lo + lane * stride;
        const bool pred = idx < hi && a[idx] < target;
        const int c = __popc(__ballot_sync(FULL, pred));
        if (c == 0) return lo;
        const int nlo = lo + (c - 1) * stride + 1;
        const int nhi = min(lo + c * stride, hi);
        lo = nlo;
        hi = nhi;
    }
    const int idx = lo + lane;
    const bool pred = idx < hi && a[idx] < target;
    return lo + __popc(__ballot_sync(FULL, pred));
}

// Position of col in the sorted smem array keys[0, n) (col must be present).
__device__ __forceinline__ int smem_lower_bound(const int32_t* keys, int n, int32_t col) {
    int pos = 0;
    int step = 1;
    while ((step << 1) <= n) step <<= 1;
    for (; step > 0; step >>= 1)
        if (pos + step <= n && keys[pos + step - 1] < col) pos += step;
    return pos;
}

// vals[slot] += prod for every active lane, in lane order when several lanes
// share a slot. Lanes hold consecutive products of the row's flattened
// (A entry, B entry) sequence, so lane order is the reference's order.
__device__ __forceinline__ void ordered_add(float* vals, int slot, bool active, float prod) {
    const int lane = lane_id();
    const int key = active ? slot : (0x40000000 | lane);
    const unsigned peers = __match_any_sync(FULL, key);
    const int n = __popc(peers);
    const int maxn = __reduce_max_sync(FULL, (unsigned)n);
    if (maxn == 1) {
        if (active) vals[slot] = __fadd_rn(vals[slot], prod);
        return;
    }
    const int leader = __ffs(peers) - 1;
    const bool lead = active && lane == leader;
    float acc = lead ? vals[slot] : 0.0f;
    unsigned m = peers;
    for (int r = 0; r < maxn; ++r) {
        const int src = m ? (__ffs(m) - 1) : lane;
        const float v = __shfl_sync(FULL, prod, src);
        if (lead && m) acc = __fadd_rn(acc, v);
        m &= m - 1;
    }
    if (lead) vals[slot] = acc;
}
// ---------------------------------------------------------------------------
// Analysis: one CTA per tile of AN_TILE rows; threads stride over the tile's
// A entries (a contiguous range of col_idx) so long rows are shared.
// ---------------------------------------------------------------------------

struct AnalyzeOut {
    int64_t* ops;        // [rows] intermediate products per row
    int32_t* ub;         // [rows] min(ops, b_cols)
    uint8_t* bin;        // [rows]
    int32_t* chunk_lo;   // [rows] first heavy column chunk
    int32_t* nchunks;    // [rows] heavy column chunks (0 for other bins)
    float4* feat;        // [rows] learned-model features (optional)
    int32_t* hist;       // [NUM_BINS] rows per bin
    int32_t* tile_hist;  // [NUM_BINS][tiles] rows per bin per tile (stable binning)
    int64_t* totals;     // [0] heavy items, [1] products
    int64_t* bin_prod;   // [NUM_BINS] products per bin
    int32_t* err;        // ERR_* bits
    int32_t* nnz_ab;     // [2] nnz of A and B as the kernel used them (read back with the bins)
};

// Sum of a 64-bit value over the whole warp (result on every lane).
__device__ __forceinline__ unsigned long long warp_sum64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// Per-key counts and 64-bit sums of a warp into shared counters, one atomic
// per distinct key present in the warp (keys < nkeys; others are skipped).
__device__ __forceinline__ void warp_bin_add(int key, int nkeys, unsigned long long val,
                                             int32_t* cnt, unsigned long long* sum) {
    const int lane = lane_id();
    unsigned left = __ballot_sync(FULL, key >= 0 && key < nkeys);
    while (left) {
        const int k = __shfl_sync(FULL, key, __ffs(left) - 1);
        const unsigned sel = __ballot_sync(FULL, key == k);
        const unsigned long long tot = warp_sum64(key == k ? val : 0ull);
        if (lane == 0) {
            atomicAdd(&cnt[k], __popc(sel));
            if (sum && tot) atomicAdd(&sum[k], tot);
        }
        left &= ~sel;
    }
}

// Rows of at most AN_SHORT entries are summarised by their own thread;
// longer rows by the whole CTA striding over their entries.
constexpr int AN_SHORT = 32;

__global__ void __launch_bounds__(AN_TILE)
    k_analyze(CsrView A, CsrView B, AnalyzeOut out, BinParams P) {
    __shared__ int32_t s_rp[AN_TILE + 1];
    __shared__ unsigned long long s_ops[AN_TILE];
    __shared__ int32_t s_maxlen[AN_TILE];
    __shared__ int32_t s_minc[AN_TILE];
    __shared__ int32_t s_maxc[AN_TILE];
    __shared__ int32_t s_hist[NUM_BINS];
    __shared__ unsigned long long s_bprod[NUM_BINS];
    __shared__ unsigned long long s_items, s_prod;
    __shared__ int s_long;

    // An operand's nnz passed as -1 is not known on the host (a device-
    // resident one-shot operand): it is the last entry of its row pointer,
    // read here instead of in a host round trip of its own, and returned
    // with the bin counts.
    if (A.nnz < 0) A.nnz = A.rp[A.rows];
    if (B.nnz < 0) B.nnz = B.rp[B.rows];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        out.nnz_ab[0] = A.nnz;
        out.nnz_ab[1] = B.nnz;
    }
    const int r0 = blockIdx.x * AN_TILE;
    const int nr = min(AN_TILE, A.rows - r0);
    const int t = threadIdx.x;
    for (int i = t; i <= nr; i += blockDim.x) s_rp[i] = A.rp[r0 + i];
    if (t < NUM_BINS) {
        s_hist[t] = 0;
        s_bprod[t] = 0;
    }
    if (t == 0) {
        s_items = 0;
        s_prod = 0;
        s_long = 0;
    }
    __syncthreads();
    // short rows: one thread each, no atomics
    if (t < nr) {
        const int s0 = s_rp[t], s1 = s_rp[t + 1];
        unsigned long long ops = 0;
        int maxlen = 0, minc = INT_MAX, maxc = -1;
        if (s0 < 0 || s1 < s0 || s1 > A.nnz) {
            atomicOr(out.err, ERR_STRUCTURE);
        } else if (s1 - s0 <= AN_SHORT) {
            // four entries at a time, phase by phase (their B rows, the rows'
            // bounds, the rows' first and last columns), so each phase's
            // loads are in flight together instead of one chain per entry
            for (int p0 = s0; p0 < s1; p0 += 4) {
                int k[4], bs[4], be[4], first[4], last[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) k[u] = p0 + u < s1 ? A.ci[p0 + u] : 0;
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    bs[u] = be[u] = 0;
                    if (p0 + u < s1) row_range(B, k[u], &bs[u], &be[u], out.err);
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    first[u] = 0;
                    last[u] = -1;
                    if (be[u] > bs[u]) {
                        first[u] = B.ci[bs[u]];
                        last[u] = B.ci[be[u] - 1];
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int len = be[u] - bs[u];
                    if (len <= 0) continue;
                    if (first[u] < 0 || last[u] >= B.cols || last[u] < first[u]) {
                        atomicOr(out.err, ERR_STRUCTURE);
                        continue;
                    }
                    ops += (unsigned long long)len;
                    maxlen = max(maxlen, len);
                    minc = min(minc, first[u]);
                    maxc = max(maxc, last[u]);
                }
            }
        } else {
            s_long = 1;
        }
        s_ops[t] = ops;
        s_maxlen[t] = maxlen;
        s_minc[t] = minc;
        s_maxc[t] = maxc;
    }
    __syncthreads();
    if (s_long) {
        // long rows: the CTA strides over the tile's entries, skipping short
        // rows; a warp whose entries all fall in one row (a long row's
        // stretch) combines them in registers and updates the row once,
        // instead of 32 lanes contending for the same shared counters
        const int p0 = max(s_rp[0], 0), p1 = min(s_rp[nr], A.nnz);
        const int lane = t & 31;
        for (int base = p0 + (t & ~31); base < p1; base += blockDim.x) {
            const int p = base + lane;
            int lo = -1, len = 0, first = INT_MAX, last = -1;
            if (p < p1) {
                int l = 0, h = nr;  // largest i with s_rp[i] <= p
                while (h - l > 1) {
                    const int mid = (l + h) >> 1;
                    if (s_rp[mid] <= p) l = mid; else h = mid;
                }
                if (s_rp[l + 1] - s_rp[l] > AN_SHORT) {
                    int bs, be;
                    row_range(B, A.ci[p], &bs, &be, out.err);
                    if (be > bs) {
                        const int f = B.ci[bs], g = B.ci[be - 1];
                        if (f < 0 || g >= B.cols || g < f) {
                            atomicOr(out.err, ERR_STRUCTURE);
                        } else {
                            lo = l;
                            len = be - bs;
                            first = f;
                            last = g;
                        }
                    }
                }
            }
            const unsigned has = __ballot_sync(FULL, lo >= 0);
            if (!has) continue;
            const int lead = __ffs(has) - 1;
            const int lrow = __shfl_sync(FULL, lo, lead);
            if (__all_sync(FULL, lo < 0 || lo == lrow)) {
                unsigned long long sum = (unsigned long long)len;
                int mxl = len, mnc = first, mxc = last;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    sum += __shfl_xor_sync(FULL, sum, o);
                    mxl = max(mxl, __shfl_xor_sync(FULL, mxl, o));
                    mnc = min(mnc, __shfl_xor_sync(FULL, mnc, o));
                    mxc = max(mxc, __shfl_xor_sync(FULL, mxc, o));
                }
                if (lane == lead) {
                    atomicAdd(&s_ops[lrow], sum);
                    atomicMax(&s_maxlen[lrow], mxl);
                    atomicMin(&s_minc[lrow], mnc);
                    atomicMax(&s_maxc[lrow], mxc);
                }
            } else if (lo >= 0) {
                atomicAdd(&s_ops[lo], (unsigned long long)len);
                atomicMax(&s_maxlen[lo], len);
                atomicMin(&s_minc[lo], first);
                atomicMax(&s_maxc[lo], last);
            }
        }
        __syncthreads();
    }
    // per row: bound, bin, heavy chunks, features; warp-aggregated counters
    const bool live = t < nr;
    const int row = r0 + t;
    const int64_t ops = live ? (int64_t)s_ops[t] : 0;
    const int32_t ub = (int32_t)min(ops, (int64_t)B.cols);
    const int b = live ? bin_of(ops, ub, P) : -1;
    int nch = 0;
    if (live) {
        out.ops[row] = ops;
        out.ub[row] = ub;
        out.bin[row] = (uint8_t)b;
        int clo = 0;
        if (b == BIN_HEAVY) {
            clo = s_minc[t] >> P.heavy_cw_log2;
            nch = (s_maxc[t] >> P.heavy_cw_log2) - clo + 1;
        }
        out.chunk_lo[row] = clo;
        out.nchunks[row] = nch;
        if (out.feat) {
            const int anz = s_rp[t + 1] - s_rp[t];
            const int span = ops > 0 ? s_maxc[t] - s_minc[t] + 1 : 0;
            out.feat[row] = make_float4((float)anz, (float)ops, (float)s_maxlen[t], (float)span);
        }
    }
    warp_bin_add(b, NUM_BINS, (unsigned long long)ops, s_hist, s_bprod);
    const unsigned long long wprod = warp_sum64((unsigned long long)ops);
    const unsigned long long witems = warp_sum64((unsigned long long)nch);
    if (lane_id() == 0) {
        if (wprod) atomicAdd(&s_prod, wprod);
        if (witems) atomicAdd(&s_items, witems);
    }
    __syncthreads();
    if (t < NUM_BINS) {
        out.tile_hist[t * gridDim.x + blockIdx.x] = s_hist[t];
        if (s_hist[t]) atomicAdd(&out.hist[t], s_hist[t]);
        if (s_bprod[t]) atomicAdd((unsigned long long*)&out.bin_prod[t], s_bprod[t]);
    }
    if (t == 0) {
        if (s_items) atomicAdd((unsigned long long*)&out.totals[0], s_items);
        atomicAdd((unsigned long long*)&out.totals[1], s_prod);
    }
}

// Stable partition of rows by bin: tile_off[b * tiles + tile] is where the
// tile's rows of bin b start in bin_rows (an exclusive scan of tile_hist), so
// every bin lists its rows in ascending order. Heavy rows reserve a block of
// consecutive work items.
__global__ void __launch_bounds__(AN_TILE)
    k_bin_scatter(int32_t rows, const uint8_t* __restrict__ bin,
                  const int32_t* __restrict__ tile_off, const int32_t* __restrict__ chunk_lo,
                  const int32_t* __restrict__ nchunks, int32_t* __restrict__ bin_rows,
                  int32_t* __restrict__ item_cursor, HeavyItem* __restrict__ items) {
    __shared__ int32_t s_wc[AN_TILE / 32][NUM_BINS];
    const int t = threadIdx.x, lane = lane_id(), warp = t >> 5;
    const int row = blockIdx.x * AN_TILE + t;
    const int b = row < rows ? (int)bin[row] : NUM_BINS;
    for (int i = t; i < (AN_TILE / 32) * NUM_BINS; i += blockDim.x) (&s_wc[0][0])[i] = 0;
    __syncthreads();
    const unsigned peers = __match_any_sync(FULL, b);
    if (b < NUM_BINS && lane == __ffs(peers) - 1) s_wc[warp][b] = __popc(peers);
    __syncthreads();
    if (b >= NUM_BINS) return;
    int before = 0;
    for (int w = 0; w < warp; ++w) before += s_wc[w][b];
    const int pos = tile_off[b * gridDim.x + blockIdx.x] + before +
                    __popc(peers & ((1u << lane) - 1));
    bin_rows[pos] = row;
    if (b == BIN_HEAVY && items) {
        const int n = nchunks[row];
        const int first = atomicAdd(item_cursor, n);
        const int lo = chunk_lo[row];
        for (int c = 0; c < n; ++c) items[first + c] = HeavyItem{row, lo + c, first, 0};
    }
}

// Per-row product counts in bin-list order (int32; rows beyond INT32_MAX
// products flag *overflow), the input of the position-map offsets.
__global__ void k_list_ops(const int32_t* __restrict__ bin_rows, int32_t n,
                           const int64_t* __restrict__ ops, int32_t* __restrict__ out,
                           int32_t* __restrict__ overflow) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t v = ops[bin_rows[i]];
    if (v > INT32_MAX) atomicExch(overflow, 1);
    out[i] = (int32_t)min(v, (int64_t)INT32_MAX);
}

// ---------------------------------------------------------------------------
// Tiny rows (ops <= 32): one thread per row, the reference loop verbatim.
// Per-thread scratch is interleaved with a padded stride (element x of thread
// t at x*TINY_LD + t): threads touching the same element never share a bank,
// and neither do lanes reading one thread's elements during the coalesced
// write-out, where each warp stores its 32 rows one row at a time.
//
// FILL mode can also record, for every product in reference order, the
// position of its column within the output row (pm, one byte per product;
// rows start at list_off[i] - list_off[0]), which the reuse kernel replays.
// ---------------------------------------------------------------------------
constexpr int TINY_TPB = 128;
constexpr int TINY_LD = TINY_TPB + 1;
constexpr int TINY_AB = 8;    // A entries whose B-row ranges are loaded together
constexpr int TINY_VALS = 5;  // B entries loaded together

// One tiny row's products in the reference order, with many loads in flight:
// A's entries TINY_AB at a time (column indices and values, then the B-row
// ranges, as two batches), each B row TINY_VALS entries at a time.
// f(col, product value) runs once per product, in A-row order then B-row
// order; VALUES loads A's and B's values too.
template <bool VALUES, class F>
__device__ __forceinline__ void tiny_walk(const CsrView& A, const CsrView& B, int a0, int a1,
                                          int32_t* err, F&& f) {
    for (int p0 = a0; p0 < a1; p0 += TINY_AB) {
        int k[TINY_AB];
        float a[TINY_AB];
#pragma unroll
        for (int u = 0; u < TINY_AB; ++u) {
            k[u] = p0 + u < a1 ? A.ci[p0 + u] : -1;
            a[u] = VALUES && p0 + u < a1 ? A.v[p0 + u] : 0.0f;
        }
        int q0[TINY_AB], q1[TINY_AB];
#pragma unroll
        for (int u = 0; u < TINY_AB; ++u) {
            q0[u] = q1[u] = 0;
            if (p0 + u < a1) {
                if ((unsigned)k[u] < (unsigned)B.rows) {
                    q0[u] = B.rp[k[u]];
                    q1[u] = B.rp[k[u] + 1];
                } else {
                    atomicOr(err, ERR_STRUCTURE);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < TINY_AB; ++u) {
            if (q0[u] < 0 || q1[u] < q0[u] || q1[u] > B.nnz) {
                atomicOr(err, ERR_STRUCTURE);
                q1[u] = q0[u] = 0;
            }
            for (int m0 = q0[u]; m0 < q1[u]; m0 += TINY_VALS) {
                int c[TINY_VALS];
                float v[TINY_VALS];
#pragma unroll
                for (int t = 0; t < TINY_VALS; ++t) {
                    const bool in = m0 + t < q1[u];
                    c[t] = in ? __ldg(B.ci + m0 + t) : -1;
                    v[t] = VALUES && in ? __ldg(B.v + m0 + t) : 0.0f;
                }
#pragma unroll
                for (int t = 0; t < TINY_VALS; ++t)
                    if (m0 + t < q1[u]) f(c[t], __fmul_rn(a[u], v[t]));
            }
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(TINY_TPB)
    k_tiny(CsrView A, CsrView B, const int32_t* __restrict__ rows, int nrows,
           int32_t* __restrict__ cnt, const int32_t* __restrict__ c_rp,
           int32_t* __restrict__ c_ci, float* __restrict__ c_v,
           const int32_t* __restrict__ list_off, uint8_t* __restrict__ pm,
           int32_t* __restrict__ err, RowCtl ctl) {
    __shared__ int32_t s_col[TINY_CAP * TINY_LD];
    __shared__ float s_val[(MODE == COUNT ? 1 : TINY_CAP) * TINY_LD];
    const int t = threadIdx.x, lane = lane_id(), wbase = t & ~31;
    const int i = blockIdx.x * TINY_TPB + t;
    int row = i < nrows ? rows[i] : 0;
    const bool live = i < nrows && !(ctl.only && !ctl.only[row]);
#define COL(x) s_col[(x) * TINY_LD + t]
#define VAL(x) s_val[(x) * TINY_LD + t]
    int n = 0;
    int64_t c0 = 0;
    if (live) {
        int a0, a1;
        row_range(A, row, &a0, &a1, err);
        if (MODE == REUSE) {
            c0 = c_rp[row];
            n = min((int)(c_rp[row + 1] - c0), TINY_CAP);
            for (int x = 0; x < n; ++x) COL(x) = c_ci[c0 + x];
        } else if (MODE == FILL && !pm) {
            // one walk: (column, product) pairs in A-row order, a stable
            // insertion sort by column, then each run of equal columns summed
            // left to right from +0.0f -- the reference's order per column
            tiny_walk<true>(A, B, a0, a1, err, [&](int col, float pv) {
                if (n < TINY_CAP) {
                    COL(n) = col;
                    VAL(n) = pv;
                    ++n;
                }
            });
            for (int x = 1; x < n; ++x) {
                const int key = COL(x);
                const float v = VAL(x);
                int y = x - 1;
                while (y >= 0 && COL(y) > key) {
                    COL(y + 1) = COL(y);
                    VAL(y + 1) = VAL(y);
                    --y;
                }
                COL(y + 1) = key;
                VAL(y + 1) = v;
            }
            int m = 0;
            for (int x = 0; x < n;) {
                const int c = COL(x);
                float acc = 0.0f;
                for (; x < n && COL(x) == c; ++x) acc = __fadd_rn(acc, VAL(x));
                COL(m) = c;
                VAL(m) = acc;
                ++m;
            }
            n = m;
            if (ctl.slot_off) {
                c0 = ctl.slot_off[row];
                cnt[row] = n;
            } else {
                c0 = c_rp[row];
            }
        } else {
            tiny_walk<false>(A, B, a0, a1, err, [&](int col, float) {
                if (n < TINY_CAP) COL(n++) = col;
            });
            for (int x = 1; x < n; ++x) {  // insertion sort
                const int key = COL(x);
                int y = x - 1;
                while (y >= 0 && COL(y) > key) {
                    COL(y + 1) = COL(y);
                    --y;
                }
                COL(y + 1) = key;
            }
            int m = 0;  // unique
            for (int x = 0; x < n; ++x) {
                const int c = COL(x);
                if (m == 0 || COL(m - 1) != c) COL(m++) = c;
            }
            n = m;
            if (MODE == COUNT) {
                cnt[row] = n;
            } else if (ctl.slot_off) {
                c0 = ctl.slot_off[row];
                cnt[row] = n;
            } else {
                c0 = c_rp[row];
            }
        }
        if (MODE == REUSE || (MODE == FILL && pm)) {
            uint8_t* pp = pm ? pm + (list_off[i] - list_off[0]) : nullptr;
            for (int x = 0; x < n; ++x) VAL(x) = 0.0f;
            tiny_walk<true>(A, B, a0, a1, err, [&](int col, float pv) {
                int pos = 0, step = 16;
                for (; step > 0; step >>= 1)
                    if (pos + step <= n && COL(pos + step - 1) < col) pos += step;
                if (pp) *pp++ = (uint8_t)pos;
                if (pos < n) VAL(pos) = __fadd_rn(VAL(pos), pv);
            });
        }
    }
    if (MODE == COUNT) return;
    __syncwarp();
    for (int j = 0; j < 32; ++j) {  // coalesced write-out, one row per step
        const int64_t cj = __shfl_sync(FULL, (long long)c0, j);
        const int nj = __shfl_sync(FULL, n, j);
        if (lane < nj) {
            if (MODE == FILL) c_ci[cj + lane] = s_col[lane * TINY_LD + wbase + j];
            c_v[cj + lane] = s_val[lane * TINY_LD + wbase + j];
        }
    }
#undef COL
#undef VAL
}

// Reuse with a position map: the numeric loop of the reference with the
// output position of every product read from pm instead of searched for.
// Neither B's nor C's column indices are read.
//
// One thread per row, as in the reference loop, organised so each thread
// keeps many independent loads in flight: A entries are taken 8 at a time
// (their column indices, values and B-row ranges loaded as two batches), and
// each B row's values and positions are loaded TRM_VALS at a time before
// they are accumulated. Values accumulate in a per-warp buffer laid out in C
// order, so a warp whose 32 rows are consecutive writes C back as one
// contiguous range.
// (Staging the warp's map bytes and A entries in shared memory first halves
// the L1 sectors but costs more in instructions and occupancy than it saves.)
constexpr int TRM_WARPS = 4;
constexpr int TRM_VALS = 5;  // B values per step of the inner loop
constexpr int TRM_CCAP = 32 * TINY_CAP;  // C entries of one warp's rows

__global__ void __launch_bounds__(TRM_WARPS * 32)
    k_tiny_reuse_map(CsrView A, CsrView B, const int32_t* __restrict__ rows, int nrows,
                     const int32_t* __restrict__ c_rp, float* __restrict__ c_v,
                     const int32_t* __restrict__ list_off, const uint8_t* __restrict__ pm,
                     int32_t* __restrict__ rp_out, int32_t* __restrict__ err) {
    __shared__ float s_acc[TRM_WARPS][TRM_CCAP];
    const int w = threadIdx.x >> 5, lane = lane_id();
    const int i = (blockIdx.x * TRM_WARPS + w) * 32 + lane;
    if ((blockIdx.x * TRM_WARPS + w) * 32 >= nrows) return;  // whole warp idle
    const bool live = i < nrows;
    int row = -1, c0 = 0, c1 = 0, a0 = 0, a1 = 0, pb = 0;
    if (live) {
        row = rows[i];
        c0 = c_rp[row];
        c1 = c_rp[row + 1];
        row_range(A, row, &a0, &a1, err);
        pb = list_off[i] - list_off[0];
        if (rp_out) {  // every row of C is a tiny row: this launch writes the row pointer
            rp_out[row] = c0;
            if (row == A.rows - 1) rp_out[A.rows] = c1;
        }
    }
    const int n = min(c1 - c0, TINY_CAP);
    const int last = __popc(__ballot_sync(FULL, live)) - 1;  // live lanes are a prefix
    const int row_first = __shfl_sync(FULL, row, 0), row_last = __shfl_sync(FULL, row, last);
    const int cbase = __shfl_sync(FULL, c0, 0), cend = __shfl_sync(FULL, c1, last);
    const bool contig = row_last - row_first == last && cend - cbase <= TRM_CCAP;
    int coff, ctotal;
    if (contig) {
        coff = c0 - cbase;
        ctotal = cend - cbase;
    } else {
        const int incl = warp_incl_scan(n);
        coff = incl - n;
        ctotal = __shfl_sync(FULL, incl, 31);
    }
    float* acc = s_acc[w];
    for (int e = lane; e < ctotal; e += 32) acc[e] = 0.0f;
    __syncwarp();
    if (live) {
        const uint8_t* sp = pm + pb;
        float* mine = acc + coff;
        for (int p0 = a0; p0 < a1; p0 += 8) {
            int k[8];
            float a[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                k[u] = p0 + u < a1 ? A.ci[p0 + u] : -1;
                a[u] = p0 + u < a1 ? A.v[p0 + u] : 0.0f;
            }
            int q0[8], q1[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                q0[u] = q1[u] = 0;
                if (p0 + u < a1) {
                    if ((unsigned)k[u] < (unsigned)B.rows) {
                        q0[u] = B.rp[k[u]];
                        q1[u] = B.rp[k[u] + 1];
                    } else {
                        atomicOr(err, ERR_STRUCTURE);
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                if (q0[u] < 0 || q1[u] < q0[u] || q1[u] > B.nnz) {
                    atomicOr(err, ERR_STRUCTURE);
                    q1[u] = q0[u] = 0;
                }
                const float* src = B.v + q0[u];
                const int len = q1[u] - q0[u];
                // B rows of tiny rows are short: 5 values in flight per step
                // wastes fewer issue slots than 8 on rows of up to 5 entries
                // (the 5-point stencil, low-degree graphs) and loses little on
                // longer ones (measured: 70 us against 74 us per pass on the
                // 1024^2 Poisson product)
                for (int m0 = 0; m0 < len; m0 += TRM_VALS) {
                    float v[TRM_VALS];
                    int x[TRM_VALS];
#pragma unroll
                    for (int t = 0; t < TRM_VALS; ++t) {
                        const bool in = m0 + t < len;
                        v[t] = in ? __ldg(src + m0 + t) : 0.0f;
                        x[t] = in ? (int)__ldg(sp + m0 + t) : TINY_CAP;
                    }
#pragma unroll
                    for (int t = 0; t < TRM_VALS; ++t)
                        if (x[t] < n) mine[x[t]] = __fadd_rn(mine[x[t]], __fmul_rn(a[u], v[t]));
                }
                sp += len;
            }
        }
    }
    __syncwarp();
    if (contig) {
        for (int e = lane; e < ctotal; e += 32) c_v[cbase + e] = acc[e];
    } else {
        for (int j = 0; j <= last; ++j) {
            const int cj = __shfl_sync(FULL, c0, j);
            const int nj = __shfl_sync(FULL, n, j);
            const int oj = __shfl_sync(FULL, coff, j);
            if (lane < nj) c_v[cj + lane] = acc[oj + lane];
        }
    }
}

// ---------------------------------------------------------------------------
// Medium rows: one warp per row, CAP-slot shared-memory table per warp.
// The row's products are processed 32 at a time in flattened
// (A entry, B entry) order; each lane locates its A entry with a 5-step
// search over the warp's inclusive scan of B-row lengths.
// FILL mode can record each product's output position (pm, uint16, rows
// starting at list_off[w] - list_off[0]) for the reuse kernel.
// ---------------------------------------------------------------------------
template <int CAP, int MODE>
__host__ __device__ constexpr int warp_smem_bytes() {
    // COUNT: keys; REUSE: keys + values; FILL: keys + values + radix
    // histogram (9-bit digits from 1024 slots up, where the extra 1 KB does
    // not cost a CTA per SM) + the radix sort's ping-pong buffer
    return (MODE == COUNT ? 4 : MODE == REUSE ? 8 : 12) * CAP +
           (MODE == FILL ? 4 * (CAP >= 1024 ? 512 : 256) : 0);
}

// Lane's product p of the current 32-entry A chunk: its B position and the
// A value. incl is the warp's inclusive scan of the chunk's B-row lengths.
struct ProductRef {
    int q;
    float a;
};

__device__ __forceinline__ ProductRef locate_product(int p, int incl, int bl, int bs, float av) {
    int e = 0;
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        const int cand = __shfl_sync(FULL, incl, e + s - 1);
        if (cand <= p) e += s;
    }
    e = min(e, 31);
    const int e_incl = __shfl_sync(FULL, incl, e);
    const int e_bl = __shfl_sync(FULL, bl, e);
    const int e_bs = __shfl_sync(FULL, bs, e);
    const float e_av = __shfl_sync(FULL, av, e);
    return ProductRef{e_bs + (p - (e_incl - e_bl)), e_av};
}

// Walks row [a0, a1) of A times B in the reference's product order:
// f(k, pv, col, bv, av, distinct) runs on every lane for the product with
// row-local index k (pv false on idle lanes) and returns a warp-uniform
// "stop". A's entries are taken 32 at a time; runs of short B rows are walked
// flattened, 32 products per step spread over their entries (distinct false:
// two lanes may hold the same column), and a B row of WALK_SEG or more
// entries is walked on its own, 32 of its entries per step (distinct true:
// the lanes' columns differ). VALUES loads B's and A's values too.
constexpr int WALK_SEG = 12;

template <bool VALUES, class F>
__device__ __forceinline__ void walk_products(const CsrView& A, const CsrView& B, int a0, int a1,
                                              int32_t* err, F&& f) {
    const int lane = lane_id();
    int before = 0;
    for (int base = a0; base < a1; base += 32) {
        const int j = base + lane;
        int bs = 0, bl = 0;
        float av = 0.0f;
        if (j < a1) {
            int be;
            row_range(B, A.ci[j], &bs, &be, err);
            bl = be - bs;
            if (VALUES) av = A.v[j];
        }
        const int incl = warp_incl_scan(bl);
        const unsigned longm = __ballot_sync(FULL, bl >= WALK_SEG);
        int e = 0;
        while (e < 32) {
            const unsigned rest = (longm >> e) << e;
            const int nl = rest ? __ffs(rest) - 1 : 32;
            if (nl > e) {
                const int pstart = e > 0 ? __shfl_sync(FULL, incl, (e - 1) & 31) : 0;
                const int pend = __shfl_sync(FULL, incl, nl - 1);
                for (int f0 = pstart; f0 < pend; f0 += 32) {
                    const int p = f0 + lane;
                    const bool pv = p < pend;
                    const ProductRef pr = locate_product(p, incl, bl, bs, av);
                    int col = -1;
                    float bv = 0.0f;
                    if (pv) {
                        col = B.ci[pr.q];
                        if (VALUES) bv = B.v[pr.q];
                    }
                    const bool stop = f(before + p, pv, col, bv, pr.a, false);
                    __syncwarp();
                    if (stop) return;
                }
                e = nl;
            }
            if (e < 32) {
                const int se = __shfl_sync(FULL, bs, e);
                const int le = __shfl_sync(FULL, bl, e);
                const float ae = __shfl_sync(FULL, av, e);
                const int kb = before + __shfl_sync(FULL, incl, e) - le;
                for (int q0 = 0; q0 < le; q0 += 32) {
                    const int q = q0 + lane;
                    const bool pv = q < le;
                    int col = -1;
                    float bv = 0.0f;
                    if (pv) {
                        col = B.ci[se + q];
                        if (VALUES) bv = B.v[se + q];
                    }
                    const bool stop = f(kb + q, pv, col, bv, ae, true);
                    __syncwarp();
                    if (stop) return;
                }
                ++e;
            }
        }
        before += __shfl_sync(FULL, incl, 31);
    }
}

// One warp's stable LSD radix sort of the 32-bit words keys[0, n) by the
// DB-bit digits of (word - sub) >> base_shift, `passes` of them, with tmp[0, n)
// as the ping-pong buffer and hist 2^DB ints. Ranks within a digit follow lane
// order chunk by chunk, so each pass is stable. Result in keys.
template <int DB>
__device__ void warp_radix_sort_core(int32_t* keys, int32_t* tmp, int n, uint32_t sub,
                                     int base_shift, int passes, int32_t* hist) {
    constexpr int NB = 1 << DB, PER = NB / 32;
    const int lane = lane_id();
    int32_t* src = keys;
    int32_t* dst = tmp;
    for (int pass = 0; pass < passes; ++pass) {
        const int shift = base_shift + DB * pass;
        for (int i = lane; i < NB; i += 32) hist[i] = 0;
        __syncwarp();
        for (int i = lane; i < n; i += 32)
            atomicAdd(&hist[(((uint32_t)src[i] - sub) >> shift) & (NB - 1)], 1);
        __syncwarp();
        int v[PER], s = 0;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            v[j] = hist[lane * PER + j];
            s += v[j];
        }
        int run = warp_incl_scan(s) - s;
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            hist[lane * PER + j] = run;
            run += v[j];
        }
        __syncwarp();
        for (int base = 0; base < n; base += 32) {
            const int i = base + lane;
            const bool ok = i < n;
            const int32_t k = ok ? src[i] : 0;
            const int d = ok ? (int)((((uint32_t)k - sub) >> shift) & (NB - 1)) : NB + lane;
            const unsigned peers = __match_any_sync(FULL, d);
            const int leader = __ffs(peers) - 1;
            int start = 0;
            if (ok && lane == leader) {
                start = hist[d];
                hist[d] = start + __popc(peers);
            }
            start = __shfl_sync(FULL, start, leader);
            if (ok) dst[start + __popc(peers & ((1u << lane) - 1))] = k;
            __syncwarp();
        }
        int32_t* t = src;
        src = dst;
        dst = t;
    }
    if (src != keys) {
        for (int i = lane; i < n; i += 32) keys[i] = src[i];
        __syncwarp();
    }
}

// Packed (column - min) << 12 | index words of one row, columns spanning
// range < 2^20: 8-bit digits, except that with a 512-entry histogram (H9) a
// span of 2^16..2^18 takes two 9-bit passes instead of three 8-bit ones
// (and no copy back from the ping-pong buffer).
template <bool H9>
__device__ __forceinline__ void sort_packed_columns(int32_t* keys, int32_t* tmp, int n,
                                                    uint32_t range, int32_t* hist) {
    if (n <= 1) return;
    if (H9 && range >= (1u << 16) && range < (1u << 18))
        warp_radix_sort_core<9>(keys, tmp, n, 0u, 12, 2, hist);
    else
        warp_radix_sort_core<8>(keys, tmp, n, 0u, 12, range < (1u << 8) ? 1 : range < (1u << 16) ? 2 : 3,
                                hist);
}

// Keys[0, n) ascending: digits of key - min, as many passes as the key range
// needs.
__device__ void warp_radix_sort(int32_t* keys, int32_t* tmp, int n, int32_t* hist) {
    const int lane = lane_id();
    if (n <= 1) return;
    int mn = INT_MAX, mx = INT_MIN;
    for (int i = lane; i < n; i += 32) {
        mn = min(mn, keys[i]);
        mx = max(mx, keys[i]);
    }
    mn = __reduce_min_sync(FULL, mn);
    mx = __reduce_max_sync(FULL, mx);
    const uint32_t range = (uint32_t)mx - (uint32_t)mn;
    const int passes = range < (1u << 8) ? 1 : range < (1u << 16) ? 2 : range < (1u << 24) ? 3 : 4;
    warp_radix_sort_core<8>(keys, tmp, n, (uint32_t)mn, 0, passes, hist);
}

// Work from a launch's counter in CTA batches. The CTA's warps draw
// indices one at a time from a (batch base, next index) word in shared
// memory; the warp that draws index `batch` fetches the next batch from the
// counter. Warps that arrive while that fetch is in flight (index > batch)
// take a single index straight from the counter instead of waiting, so no
// warp ever waits on another, and every index is handed out exactly once.
// The batches keep the order of the list (each CTA works on neighbouring
// entries, the grid sweeps the list front to back) while the counter takes
// one atomic per batch instead of one per entry: hundreds of millions of
// atomics on one address otherwise (R-MAT 2^20 heavy items). The word
// starts at `batch` (set before a __syncthreads), so the first draw
// fetches. Called by lane 0; returns the index drawn.
__device__ __forceinline__ long long draw_batched(unsigned long long* s_q, int32_t* queue,
                                                  long long batch) {
    const unsigned long long o = atomicAdd(s_q, 1ull);
    const long long b = (long long)(o >> 32);
    const long long c = (long long)(o & 0xffffffffull);
    if (c < batch) return b + c;
    if (c == batch) {
        const int nb = atomicAdd(queue, (int)batch);
        atomicExch(s_q, ((unsigned long long)(unsigned)nb << 32) | 1ull);
        return nb;
    }
    return atomicAdd(queue, 1);
}

// Medium rows: one warp per row, a CAP-slot shared-memory table per warp.
//   COUNT  hash-insert the row's columns, count the new ones
//   FILL   COUNT's insert, compaction, radix sort -> sorted columns written;
//          then the values: every product finds its column's position by
//          binary search and is added in order (ordered_add); the positions
//          are recorded in pm when requested (uint16, rows starting at
//          list_off[w] - list_off[0])
//   REUSE  the value pass alone, on the stored sorted columns
template <int CAP, int WARPS, int MODE>
__global__ void __launch_bounds__(WARPS * 32)
    k_warp(CsrView A, CsrView B, const int32_t* __restrict__ rows, int nrows,
           const int64_t* __restrict__ ops, int32_t* __restrict__ cnt,
           const int32_t* __restrict__ c_rp,
           int32_t* __restrict__ c_ci, float* __restrict__ c_v,
           const int32_t* __restrict__ list_off, uint16_t* __restrict__ pm,
           int32_t* __restrict__ err, RowCtl ctl, int32_t* __restrict__ queue) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int LOG2CAP = __builtin_ctz(CAP);
    const int warp = threadIdx.x >> 5, lane = lane_id();
    unsigned char* mine = smem + warp * warp_smem_bytes<CAP, MODE>();
    int32_t* keys = reinterpret_cast<int32_t*>(mine);
    float* vals = reinterpret_cast<float*>(keys + CAP);
    int32_t* hist = reinterpret_cast<int32_t*>(mine + 8 * CAP);
    constexpr bool HIST9 = CAP >= 1024;  // histogram of 512 entries: 9-bit digits
    int32_t* sorttmp = reinterpret_cast<int32_t*>(mine + 8 * CAP + 4 * (HIST9 ? 512 : 256));  // FILL only
    volatile int32_t* vkeys = keys;
    // learned: a table that fills up means the row outgrew its predicted
    // capacity; the row is flagged for the exact path instead of an error
    const bool learned = MODE != REUSE && ctl.learned;

    for (;;) {
        // rows are pulled one at a time from the launch's counter (a CTA
        // batch word like k_heavy's would cost the 512- and 1024-slot FILL
        // tables a resident CTA per SM; one in global memory measured slower)
        int w = 0;
        if (lane == 0) w = atomicAdd(queue, 1);
        w = __shfl_sync(FULL, w, 0);
        if (w >= nrows) break;
        const int row = rows[w];
        if (ctl.only && !ctl.only[row]) continue;
        int a0, a1;
        row_range(A, row, &a0, &a1, err);
        int n = 0;          // distinct columns (COUNT/FILL) or stored row length (REUSE)
        int64_t o = 0;      // where the row's C entries go
        if (MODE == REUSE) {
            o = c_rp[row];
            n = min(c_rp[row + 1] - (int)o, CAP);
            for (int x = lane; x < n; x += 32) keys[x] = c_ci[o + x];
        } else {
            bool wide = false;  // columns span 2^20 or more: the two-walk path
            // the row's length: counted (exact) or its predicted slots (learned)
            const int64_t room = MODE != FILL ? 0
                                 : learned   ? ctl.slot_off[row + 1] - ctl.slot_off[row]
                                             : (int64_t)(c_rp[row + 1] - c_rp[row]);
            if (MODE == FILL && !pm && ops[row] <= CAP && 2 * room >= ops[row]) {
                // Every product fits the table and at most every other one
                // repeats a column: expand, sort, compress. Each product's
                // column and value go to its row-local index; a stable sort
                // of packed (column - min) << 12 | index words brings equal
                // columns together in A-row order, and each run is summed
                // left to right from +0.0f, the reference's order. No
                // hashing, no ordered combine, no compaction; the sort holds
                // the products instead of the distinct columns, which costs
                // more than the hashing saves once most products repeat.
                const int P = (int)ops[row];
                int mn = INT_MAX, mx = INT_MIN;
                walk_products<true>(A, B, a0, a1, err, [&](int k, bool pv, int col, float bv,
                                                           float av, bool) {
                    if (pv && k < P) {
                        keys[k] = col;
                        vals[k] = __fmul_rn(av, bv);
                        mn = min(mn, col);
                        mx = max(mx, col);
                    } else if (pv) {
                        atomicOr(err, ERR_STRUCTURE);  // more products than analysed
                    }
                    return false;
                });
                __syncwarp();
                mn = __reduce_min_sync(FULL, mn);
                mx = __reduce_max_sync(FULL, mx);
                const uint32_t range = (uint32_t)mx - (uint32_t)mn;
                if (mn <= mx && range < (1u << 20)) {
                    for (int x = lane; x < P; x += 32)
                        keys[x] = (int32_t)((((uint32_t)keys[x] - (uint32_t)mn) << 12) | (uint32_t)x);
                    __syncwarp();
                    sort_packed_columns<HIST9>(keys, sorttmp, P, range, hist);
                    int nexp = (int)room;
                    if (learned) {
                        // the distinct columns must fit the predicted slots
                        int heads = 0;
                        for (int x = lane; x < P; x += 32)
                            heads += x == 0 || ((uint32_t)keys[x - 1] >> 12) != ((uint32_t)keys[x] >> 12);
                        heads = __reduce_add_sync(FULL, heads);
                        if (heads > room) {
                            if (lane == 0) cnt[row] = -1;
                            __syncwarp();
                            continue;
                        }
                        nexp = heads;
                        if (lane == 0) cnt[row] = heads;
                    }
                    o = learned ? ctl.slot_off[row] : (int64_t)c_rp[row];
                    int out = 0;
                    for (int b0 = 0; b0 < P; b0 += 32) {
                        const int x = b0 + lane;
                        const uint32_t w = x < P ? (uint32_t)keys[x] : 0u;
                        const bool head = x < P && (x == 0 || ((uint32_t)keys[x - 1] >> 12) != (w >> 12));
                        const unsigned hm = __ballot_sync(FULL, head);
                        if (head) {
                            float sum = __fadd_rn(0.0f, vals[w & 4095u]);
                            for (int y = x + 1; y < P; ++y) {
                                const uint32_t wy = (uint32_t)keys[y];
                                if ((wy >> 12) != (w >> 12)) break;
                                sum = __fadd_rn(sum, vals[wy & 4095u]);
                            }
                            const int d = out + __popc(hm & ((1u << lane) - 1));
                            if (d < nexp) {
                                c_ci[o + d] = (int32_t)((w >> 12) + (uint32_t)mn);
                                c_v[o + d] = sum;
                            }
                        }
                        out += __popc(hm);
                    }
                    if (out != nexp && lane == 0) atomicOr(err, ERR_STRUCTURE);
                    __syncwarp();
                    continue;
                }
                wide = mn <= mx;
            }
            if (MODE == FILL && !pm && !wide) {
                // One walk: each product finds or inserts its column's slot
                // and is added to the slot's accumulator in A-row order; then
                // the occupied slots are compacted and sorted by column as
                // packed words (column - min) << 12 | compacted index, and the
                // values are gathered through the index at write-out. Rows
                // whose columns span 2^20 or more take the two-walk path below.
                for (int x = lane; x < CAP; x += 32) {
                    keys[x] = -1;
                    vals[x] = 0.0f;
                }
                __syncwarp();
                bool ovf = false;
                walk_products<true>(A, B, a0, a1, err, [&](int, bool pv, int col, float bv, float av,
                                                           bool distinct) {
                    int slot = -1;
                    bool inserted = false, ok = true;
                    if (pv) {
                        uint32_t h = hash_slot(col, LOG2CAP);
                        ok = false;
                        for (int probe = 0; probe < CAP; ++probe) {
                            const int cur = vkeys[h];
                            if (cur == col) {
                                ok = true;
                                break;
                            }
                            if (cur == -1) {
                                const int old = atomicCAS(&keys[h], -1, col);
                                if (old == -1 || old == col) {
                                    inserted = old == -1;
                                    ok = true;
                                    break;
                                }
                            }
                            h = (h + 1) & (CAP - 1);
                        }
                        if (ok) slot = (int)h;
                        else if (!learned) atomicOr(err, ERR_STRUCTURE);
                    }
                    n += __popc(__ballot_sync(FULL, inserted));
                    if (distinct) {
                        if (slot >= 0) vals[slot] = __fadd_rn(vals[slot], __fmul_rn(av, bv));
                    } else {
                        ordered_add(vals, slot, slot >= 0, __fmul_rn(av, bv));
                    }
                    if (learned) ovf = __any_sync(FULL, !ok);
                    return ovf;
                });
                __syncwarp();
                if (learned && (ovf || n > ctl.slot_off[row + 1] - ctl.slot_off[row])) {
                    if (lane == 0) cnt[row] = -1;
                    continue;
                }
                int out = 0;
                int mn = INT_MAX, mx = INT_MIN;
                for (int b0 = 0; b0 < CAP; b0 += 32) {
                    const int key = keys[b0 + lane];
                    const float v = vals[b0 + lane];
                    const bool occ = key != -1;
                    const unsigned m = __ballot_sync(FULL, occ);
                    __syncwarp();
                    if (occ) {
                        const int d = out + __popc(m & ((1u << lane) - 1));
                        keys[d] = key;
                        vals[d] = v;
                        mn = min(mn, key);
                        mx = max(mx, key);
                    }
                    out += __popc(m);
                    __syncwarp();
                }
                mn = __reduce_min_sync(FULL, mn);
                mx = __reduce_max_sync(FULL, mx);
                const uint32_t range = n > 0 ? (uint32_t)mx - (uint32_t)mn : 0u;
                if (range < (1u << 20) && n < 4096) {
                    for (int x = lane; x < n; x += 32)
                        keys[x] = (int32_t)((((uint32_t)keys[x] - (uint32_t)mn) << 12) | (uint32_t)x);
                    __syncwarp();
                    sort_packed_columns<HIST9>(keys, sorttmp, n, range, hist);
                    o = learned ? ctl.slot_off[row] : (int64_t)c_rp[row];
                    for (int x = lane; x < n; x += 32) {
                        const uint32_t w = (uint32_t)keys[x];
                        c_ci[o + x] = (int32_t)((w >> 12) + (uint32_t)mn);
                        c_v[o + x] = vals[w & 4095u];
                    }
                    if (learned && lane == 0) cnt[row] = n;
                    __syncwarp();
                    continue;
                }
                n = 0;  // wide row: start over on the two-walk path
            }
            for (int x = lane; x < CAP; x += 32) keys[x] = -1;
            __syncwarp();
            bool ovf = false;
            walk_products<false>(A, B, a0, a1, err, [&](int, bool pv, int col, float, float, bool) {
                bool inserted = false, ok = true;
                if (pv) {
                    // at most CAP probes: a table can only fill up when an
                    // operand breaks the column-range contract (or, learned,
                    // when the prediction was too small)
                    uint32_t h = hash_slot(col, LOG2CAP);
                    ok = false;
                    for (int probe = 0; probe < CAP; ++probe) {
                        const int cur = vkeys[h];
                        if (cur == col) {
                            ok = true;
                            break;
                        }
                        if (cur == -1) {
                            const int old = atomicCAS(&keys[h], -1, col);
                            if (old == -1 || old == col) {
                                inserted = old == -1;
                                ok = true;
                                break;
                            }
                        }
                        h = (h + 1) & (CAP - 1);
                    }
                    if (!ok && !learned) atomicOr(err, ERR_STRUCTURE);
                }
                n += __popc(__ballot_sync(FULL, inserted));
                if (learned) ovf = __any_sync(FULL, !ok);
                return ovf;
            });
            __syncwarp();
            if (learned && (ovf || (MODE == FILL && n > ctl.slot_off[row + 1] - ctl.slot_off[row]))) {
                if (lane == 0) cnt[row] = -1;
                continue;
            }
            if (MODE == COUNT) {
                if (lane == 0) cnt[row] = n;
                continue;
            }
            // FILL: compact occupied slots to the front (left moves only)
            int out = 0;
            for (int b0 = 0; b0 < CAP; b0 += 32) {
                const int key = keys[b0 + lane];
                const bool occ = key != -1;
                const unsigned m = __ballot_sync(FULL, occ);
                __syncwarp();
                if (occ) keys[out + __popc(m & ((1u << lane) - 1))] = key;
                out += __popc(m);
                __syncwarp();
            }
            warp_radix_sort(keys, reinterpret_cast<int32_t*>(vals), n, hist);
            o = learned ? ctl.slot_off[row] : (int64_t)c_rp[row];
            for (int x = lane; x < n; x += 32) c_ci[o + x] = keys[x];
            if (learned && lane == 0) cnt[row] = n;
        }
        // values: every product to its column's position, in order
        for (int x = lane; x < n; x += 32) vals[x] = 0.0f;
        __syncwarp();
        uint16_t* pp = (MODE == FILL && pm) ? pm + (list_off[w] - list_off[0]) : nullptr;
        walk_products<true>(A, B, a0, a1, err, [&](int k, bool pv, int col, float bv, float av,
                                                   bool distinct) {
            int pos = -1;
            if (pv) {
                pos = smem_lower_bound(keys, n, col);
                if (pp) pp[k] = (uint16_t)pos;
            }
            if (distinct) {
                if (pv && pos < n) vals[pos] = __fadd_rn(vals[pos], __fmul_rn(av, bv));
            } else {
                ordered_add(vals, pos, pv && pos < n, __fmul_rn(av, bv));
            }
            return false;
        });
        __syncwarp();
        for (int x = lane; x < n; x += 32) c_v[o + x] = vals[x];
        __syncwarp();
    }
}

// Reuse with a position map: like REUSE, but every product's slot comes
// from pm, so B's and C's column indices are not read and no search runs.
template <int CAP, int WARPS>
__global__ void __launch_bounds__(WARPS * 32)
    k_warp_reuse_map(CsrView A, CsrView B, const int32_t* __restrict__ rows, int nrows,
                     const int32_t* __restrict__ c_rp, float* __restrict__ c_v,
                     const int32_t* __restrict__ list_off, const uint16_t* __restrict__ pm,
                     int32_t* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = lane_id();
    float* vals = reinterpret_cast<float*>(smem) + warp * CAP;
    for (int w = blockIdx.x * WARPS + warp; w < nrows; w += gridDim.x * WARPS) {
        const int row = rows[w];
        const int c0 = c_rp[row];
        const int L = min(c_rp[row + 1] - c0, CAP);
        for (int x = lane; x < L; x += 32) vals[x] = 0.0f;
        __syncwarp();
        const uint16_t* pp = pm + (list_off[w] - list_off[0]);
        int a0, a1;
        row_range(A, row, &a0, &a1, err);
        for (int base = a0; base < a1; base += 32) {
            const int j = base + lane;
            int bs = 0, bl = 0;
            float av = 0.0f;
            if (j < a1) {
                int be;
                row_range(B, A.ci[j], &bs, &be, err);
                bl = be - bs;
                av = A.v[j];
            }
            const int incl = warp_incl_scan(bl);
            const int total = __shfl_sync(FULL, incl, 31);
            for (int f = 0; f < total; f += 32) {
                const int p = f + lane;
                const bool pv = p < total;
                const ProductRef pr = locate_product(p, incl, bl, bs, av);
                int slot = -1;
                float bv = 0.0f;
                if (pv) {
                    slot = pp[p];
                    bv = B.v[pr.q];
                }
                const bool ok = pv && slot < L;
                ordered_add(vals, slot, ok, __fmul_rn(pr.a, bv));
                __syncwarp();
            }
            pp += total;
        }
        __syncwarp();
        for (int x = lane; x < L; x += 32) c_v[c0 + x] = vals[x];
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Heavy rows: one warp per (row, chunk of cw = 2^cw_log2 columns). The warp
// walks the row's A entries 32 at a time; each lane finds the part of its B
// row that falls in the chunk (a binary search only when the B row straddles
// a chunk edge). In A-row order, a run of short in-chunk segments is walked
// flattened (products spread over the lanes, two steps of 32 in flight,
// same-column products of a step combined in lane order by ordered_add),
// and a segment of HEAVY_SEG or more products is walked with the lanes over
// its own columns, which are distinct, so it needs neither the product
// search nor the ordered combine. COUNT and FILL set bits of a presence
// bitmap; FILL and REUSE add into a dense accumulator of cw floats started
// at +0.0f, the reference's start. FILL writes the chunk's entries in column
// order straight from the bitmap. The A row is re-read once per chunk; the
// products once in all.
// ---------------------------------------------------------------------------
constexpr int HEAVY_SEG = 12;  // in-chunk B segments this long are walked on their own

// COUNT walks up to HEAVY_COUNT_SPAN neighbouring chunks of a row at once
// (k_heavy): a bitmap of HEAVY_COUNT_SPAN cw bits.
constexpr int HEAVY_COUNT_SPAN = 8;
__host__ __device__ constexpr int heavy_smem_bytes(int mode, int cw) {
    return mode == COUNT ? HEAVY_COUNT_SPAN * cw / 8 : 4 * cw + (mode == REUSE ? 0 : cw / 8);
}

// First index in [lo, hi) with a[idx] >= target (hi if none); one thread.
__device__ __forceinline__ int seq_lower_bound(const int32_t* __restrict__ a, int lo, int hi,
                                               int target) {
    while (lo < hi) {
        const int mid = lo + ((hi - lo) >> 1);
        if (__ldg(a + mid) < target) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Per-B-row metadata and directory sizes (HeavyAux). Rows whose structure is
// out of range flag ERR_STRUCTURE and read as empty.
__global__ void k_bmeta(CsrView B, int cw_log2, int4* __restrict__ meta,
                        int32_t* __restrict__ dcount, int32_t* __restrict__ err) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= B.rows) return;
    int bs, be;
    row_range(B, k, &bs, &be, err);
    int first = 0, last = -1, dc = 0;
    if (be > bs) {
        first = B.ci[bs];
        last = B.ci[be - 1];
        if (first < 0 || last >= B.cols || last < first) {
            atomicOr(err, ERR_STRUCTURE);
            be = bs;
            first = 0;
            last = -1;
        } else {
            const int fc = first >> cw_log2, lc = last >> cw_log2;
            if (be - bs >= DIR_MIN_LEN && lc > fc) dc = lc - fc + 2;
        }
    }
    meta[k] = make_int4(bs, be, first, last);
    dcount[k] = dc;
}

// Directory fill: one warp per B row with a directory; the entry at q writes
// itself as the start of every chunk from just after its predecessor's chunk
// up to its own; the row end closes the list. doff[k] = -1 for the others.
__global__ void k_bdir(CsrView B, int cw_log2, const int4* __restrict__ meta,
                       const int32_t* __restrict__ dcount, const int64_t* __restrict__ dscan,
                       int64_t* __restrict__ doff, int32_t* __restrict__ dir) {
    const int k = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = lane_id();
    if (k >= B.rows) return;
    const int dc = dcount[k];
    if (dc == 0) {
        if (lane == 0) doff[k] = -1;
        return;
    }
    const int64_t off = dscan[k];
    const int4 m = meta[k];
    const int fc = m.z >> cw_log2, lc = m.w >> cw_log2;
    if (lane == 0) {
        doff[k] = off;
        dir[off + (lc - fc + 1)] = m.y;
    }
    for (int q = m.x + lane; q < m.y; q += 32) {
        const int c = B.ci[q] >> cw_log2;
        const int prev = q > m.x ? (B.ci[q - 1] >> cw_log2) : fc - 1;
        // clamped to [fc, lc]: an unsorted row (a broken operand) cannot
        // write outside its directory
        for (int x = max(prev + 1, fc); x <= min(c, lc); ++x) dir[off + (x - fc)] = q;
    }
}

// Chunk presence masks (HeavyAux::smask, zeroed before): one warp per B row
// that spans several column chunks and has no directory; each entry sets its
// chunk's bit. Rows with a directory or within one chunk keep zero words
// (the heavy walk never reads them).
__global__ void k_bmask(CsrView B, int cw_log2, const int4* __restrict__ meta,
                        const int64_t* __restrict__ doff, int words, uint32_t* __restrict__ smask) {
    const int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = lane_id();
    if (k >= B.rows) return;
    const int4 m = meta[k];
    if (m.y <= m.x || (m.z >> cw_log2) == (m.w >> cw_log2)) return;
    if (doff && doff[k] >= 0) return;
    uint32_t* row = smask + k * words;
    for (int q = m.x + lane; q < m.y; q += 32) {
        const int c = B.ci[q] >> cw_log2;
        // an unsorted row (a broken operand) cannot write outside its words
        if (c >= 0 && (c >> 5) < words) atomicOr(row + (c >> 5), 1u << (c & 31));
    }
}

// Heavy rows' A entries with their B row's metadata and directory offset
// copied beside them (HeavyAux::ameta / adoff; -(k + 2) for a B row k
// without a directory): the heavy walk then reads one coalesced word pair
// per entry instead of a column index followed by two gathers. One warp per
// heavy row; a column out of range flags ERR_STRUCTURE and records an empty
// row.
__global__ void k_ameta(CsrView A, CsrView B, const int32_t* __restrict__ rows, int nrows,
                        const int4* __restrict__ meta, const int64_t* __restrict__ doff,
                        int4* __restrict__ ameta, int32_t* __restrict__ adoff,
                        int32_t* __restrict__ err) {
    const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = lane_id();
    if (w >= nrows) return;
    int a0, a1;
    row_range(A, rows[w], &a0, &a1, err);
    for (int j = a0 + lane; j < a1; j += 32) {
        const int k = A.ci[j];
        int4 m = make_int4(0, 0, 0, -1);
        int d = -1;
        if ((unsigned)k < (unsigned)B.rows) {
            m = meta[k];
            d = doff ? (int)doff[k] : -1;
            if (d < 0) d = -(k + 2);
        } else {
            atomicOr(err, ERR_STRUCTURE);
        }
        ameta[j] = m;
        adoff[j] = d;
    }
}

// Accumulates, for the calling warp, the in-chunk B segments of 32 A entries
// (lane l: positions [s, s + len) of its entry's B row, A value av) into the
// chunk [lo, lo + cw) in A-row order. A run of short segments is walked
// flattened (products spread over the lanes, two steps of 32 in flight,
// same-column products of a step combined in lane order by ordered_add); a
// segment of HEAVY_SEG or more products is walked with the lanes over its own
// columns, which are distinct, so it needs neither the product search nor
// the ordered combine. COUNT and FILL set bits of the presence bitmap; FILL
// and REUSE add into the accumulator.
template <int MODE>
__device__ __forceinline__ void heavy_segments(const CsrView& B, int s, int len, float av, int lo,
                                               int cw, float* acc, unsigned* bits,
                                               int32_t* err) {
    const int lane = lane_id();
    const int incl = warp_incl_scan(len);
    const unsigned longm = __ballot_sync(FULL, len >= HEAVY_SEG);
    int e = 0;
    while (e < 32) {
        const unsigned rest = (longm >> e) << e;
        const int nl = rest ? __ffs(rest) - 1 : 32;
        if (nl > e) {
            const int pstart = e > 0 ? __shfl_sync(FULL, incl, (e - 1) & 31) : 0;
            const int pend = __shfl_sync(FULL, incl, nl - 1);
            for (int f0 = pstart; f0 < pend; f0 += 64) {
                // two steps located and loaded before either is accumulated
                const int p0 = f0 + lane, p1 = f0 + 32 + lane;
                const ProductRef r0 = locate_product(p0, incl, len, s, av);
                const ProductRef r1 = locate_product(p1, incl, len, s, av);
                int c0 = 0, c1 = 0;
                float b0 = 0.0f, b1 = 0.0f;
                if (p0 < pend) {
                    c0 = __ldg(B.ci + r0.q) - lo;
                    if (MODE != COUNT) b0 = __ldg(B.v + r0.q);
                }
                if (p1 < pend) {
                    c1 = __ldg(B.ci + r1.q) - lo;
                    if (MODE != COUNT) b1 = __ldg(B.v + r1.q);
                }
                const bool ok0 = p0 < pend && (unsigned)c0 < (unsigned)cw;
                const bool ok1 = p1 < pend && (unsigned)c1 < (unsigned)cw;
                if ((p0 < pend && !ok0) || (p1 < pend && !ok1))
                    atomicOr(err, ERR_STRUCTURE);  // B row not sorted
                if (MODE != REUSE) {
                    if (ok0) atomicOr(&bits[c0 >> 5], 1u << (c0 & 31));
                    if (ok1) atomicOr(&bits[c1 >> 5], 1u << (c1 & 31));
                }
                if (MODE != COUNT) {
                    ordered_add(acc, ok0 ? c0 : 0, ok0, __fmul_rn(r0.a, b0));
                    __syncwarp();
                    if (f0 + 32 < pend) ordered_add(acc, ok1 ? c1 : 0, ok1, __fmul_rn(r1.a, b1));
                }
                __syncwarp();
            }
            e = nl;
        }
        if (e < 32) {
            const int se = __shfl_sync(FULL, s, e);
            const int qe = se + __shfl_sync(FULL, len, e);
            const float ae = __shfl_sync(FULL, av, e);
            for (int q0 = se; q0 < qe; q0 += 64) {
                const int qa = q0 + lane, qb = q0 + 32 + lane;
                const bool two = q0 + 32 < qe;  // warp-uniform
                int ca = 0, cb = 0;
                float va = 0.0f, vb = 0.0f;
                if (qa < qe) {
                    ca = __ldg(B.ci + qa) - lo;
                    if (MODE != COUNT) va = __ldg(B.v + qa);
                }
                if (two && qb < qe) {
                    cb = __ldg(B.ci + qb) - lo;
                    if (MODE != COUNT) vb = __ldg(B.v + qb);
                }
                const bool oka = qa < qe && (unsigned)ca < (unsigned)cw;
                const bool okb = two && qb < qe && (unsigned)cb < (unsigned)cw;
                if ((qa < qe && !oka) || (two && qb < qe && !okb)) atomicOr(err, ERR_STRUCTURE);
                if (MODE != REUSE) {
                    if (oka) atomicOr(&bits[ca >> 5], 1u << (ca & 31));
                    if (okb) atomicOr(&bits[cb >> 5], 1u << (cb & 31));
                }
                if (MODE != COUNT) {
                    if (oka) acc[ca] = __fadd_rn(acc[ca], __fmul_rn(ae, va));
                    if (okb) acc[cb] = __fadd_rn(acc[cb], __fmul_rn(ae, vb));
                }
            }
            __syncwarp();
            ++e;
        }
    }
}

// End of a heavy work item w (row `row`, chunk starting at column lo) for
// the calling warp, whose accumulator and bitmap hold the chunk: COUNT
// records the chunk's count (and adds it to the row's); FILL writes the
// chunk's columns in order with their values at the chunk's place in C (or,
// in the learned sweep, in the row's slot or the overflow pool, RowCtl);
// REUSE writes the values at the chunk's known positions in C. The bitmap
// and accumulator are left zeroed for the warp's next item (REUSE zeroes its
// accumulator when it starts an item).
template <int MODE>
__device__ __forceinline__ void heavy_finish(
    const CsrView& B, int w, const HeavyItem& it, int row, int lo, int cw, float* acc,
    unsigned* bits, int32_t* __restrict__ item_cnt, int32_t* __restrict__ row_cnt,
    const int64_t* __restrict__ item_scan, const int32_t* __restrict__ c_rp,
    int32_t* __restrict__ c_ci, float* __restrict__ c_v, int32_t* __restrict__ err,
    const RowCtl& ctl) {
    const int lane = lane_id();
    const int nw = cw >> 5;
    __syncwarp();
    if (MODE == COUNT) {
        int c = 0;
        for (int x = lane; x < nw; x += 32) {
            c += __popc(bits[x]);
            bits[x] = 0u;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(FULL, c, o);
        if (lane == 0) {
            item_cnt[w] = c;
            if (c && row_cnt) atomicAdd(&row_cnt[row], c);
        }
    } else if (MODE == FILL) {
        // lane l writes the present columns of bitmap word x0 + l; the
        // words' popcounts give each lane its first output position
        int64_t out;
        bool keep = true;
        if (ctl.item_off) {
            // learned sweep: the chunk takes the next place in its row's
            // slot (c_ci / c_v are the slot buffers), else in the shared
            // overflow pool; a chunk that finds no room only clears its
            // bitmap and accumulator
            int c = 0;
            for (int x = lane; x < nw; x += 32) c += __popc(bits[x]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(FULL, c, o);
            long long dst = -1;
            if (lane == 0) {
                item_cnt[w] = c;
                const int off = atomicAdd(&row_cnt[row], c);
                const int64_t s0 = ctl.slot_off[row], cap = ctl.slot_off[row + 1] - s0;
                if ((int64_t)off + c <= cap) {
                    dst = s0 + off;
                } else if (c > 0) {
                    const unsigned long long p =
                        atomicAdd(ctl.pool_fill, (unsigned long long)c);
                    if ((int64_t)p + c <= ctl.pool_cap) dst = ctl.pool_base + (int64_t)p;
                } else {
                    dst = s0;  // an empty chunk needs no room
                }
                ctl.item_off[w] = dst;
                if (dst < 0) ctl.ovf[row] = 1;
            }
            dst = __shfl_sync(FULL, dst, 0);
            keep = dst >= 0;
            out = dst;
        } else {
            out = (int64_t)c_rp[row] + (item_scan[w] - item_scan[it.first]);
        }
        // writes into C stay inside the row (counts that disagree with
        // this fill would only come from an operand changed in between)
        const int64_t lim = ctl.item_off ? INT64_MAX : (int64_t)c_rp[row + 1];
        for (int x0 = 0; x0 < nw; x0 += 32) {
            unsigned word = 0u;
            if (x0 + lane < nw) {
                word = bits[x0 + lane];
                bits[x0 + lane] = 0u;
            }
            const int pc = __popc(word);
            const int incl = warp_incl_scan(pc);
            int64_t pos = out + (incl - pc);
            while (word) {
                const int b = __ffs(word) - 1;
                word &= word - 1;
                const int col = (x0 + lane) * 32 + b;
                if (keep && pos < lim) {
                    c_ci[pos] = lo + col;
                    c_v[pos] = acc[col];
                } else if (keep) {
                    atomicOr(err, ERR_STRUCTURE);
                }
                acc[col] = 0.0f;
                ++pos;
            }
            out += __shfl_sync(FULL, incl, 31);
        }
    } else {
        const int hi = (int)min((int64_t)lo + cw, (int64_t)B.cols);
        const int r0 = c_rp[row], r1 = c_rp[row + 1];
        const int s = warp_lower_bound(c_ci, r0, r1, lo);
        const int t2 = warp_lower_bound(c_ci, s, r1, hi);
        for (int q = s + lane; q < t2; q += 32) {
            const int col = c_ci[q] - lo;
            c_v[q] = (unsigned)col < (unsigned)cw ? acc[col] : 0.0f;
        }
    }
    __syncwarp();
}

// Whether B row k (a row without a directory) has an entry in chunks
// [c, c + span) by its presence mask (span <= 32: at most two words).
__device__ __forceinline__ bool heavy_mask_any(const HeavyAux& aux, int k, int c, int span) {
    const uint32_t* m = aux.smask + (int64_t)k * aux.smask_words;
    const int w0 = c >> 5, b0 = c & 31;
    uint64_t bits = m[w0] >> b0;
    if (b0 + span > 32) bits |= (uint64_t)m[w0 + 1] << (32 - b0);
    const uint64_t want = span >= 64 ? ~0ull : ((1ull << span) - 1);
    return (bits & want) != 0;
}

// Heavy rows: one warp per work item (row, chunk of cw = 2^cw_log2
// columns), items pulled from a counter (in CTA batches, below) by a grid
// that fills the GPU once (a warp that drew a light item takes the next one
// instead of idling beside a heavy one). The warp walks the row's A entries 32 at a
// time; each lane finds the part of its B row that falls in the chunk from
// the B row's metadata and, for long rows, its column-chunk directory (for
// the others the chunk's presence bit, then a binary search only when the
// bit is set), and heavy_segments accumulates the segments in A-row order. The A row is re-read once per chunk; the products once in
// all.
constexpr int HEAVY_MAX_WARPS = 32;

template <int MODE>
__global__ void __launch_bounds__(HEAVY_MAX_WARPS * 32)
    k_heavy(CsrView A, CsrView B, const HeavyItem* __restrict__ items, int nitems,
            int32_t* __restrict__ item_cnt, int32_t* __restrict__ row_cnt,
            const int64_t* __restrict__ item_scan, const int32_t* __restrict__ c_rp,
            int32_t* __restrict__ c_ci, float* __restrict__ c_v, int32_t* __restrict__ err,
            RowCtl ctl, int cw_log2, HeavyAux aux, int32_t* __restrict__ queue) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int cw = 1 << cw_log2;
    const int nw = cw >> 5;  // bitmap words
    const int warp = threadIdx.x >> 5, lane = lane_id();
    unsigned char* mine = smem + warp * heavy_smem_bytes(MODE, cw);
    float* acc = reinterpret_cast<float*>(mine);
    unsigned* bits = reinterpret_cast<unsigned*>(mine + (MODE == COUNT ? 0 : 4 * cw));

    // The accumulator and the bitmap start at zero once; every item clears
    // what it set (COUNT and FILL while reading the bitmap out, REUSE by
    // zeroing its chunk), so no item pays for zeroing a whole chunk.
    if (MODE != COUNT) {
        float4* a4 = reinterpret_cast<float4*>(acc);
        for (int x = lane; x < (cw >> 2); x += 32) a4[x] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (MODE != REUSE)
        for (int x = lane; x < (MODE == COUNT ? HEAVY_COUNT_SPAN * nw : nw); x += 32) bits[x] = 0u;
    __syncwarp();
    // work items in CTA batches of twice the CTA's warps (draw_batched); the
    // batch word follows the warps' accumulators and bitmaps
    const long long batch = 2 * (long long)(blockDim.x >> 5);
    unsigned long long* s_q = reinterpret_cast<unsigned long long*>(
        smem + (blockDim.x >> 5) * heavy_smem_bytes(MODE, cw));
    if (threadIdx.x == 0) *s_q = (unsigned long long)batch;
    __syncthreads();
    for (;;) {
        long long wq = 0;
        if (lane == 0) wq = draw_batched(s_q, queue, batch);
        wq = __shfl_sync(FULL, wq, 0);
        if (wq >= nitems) break;
        const int w = (int)wq;
        const HeavyItem it = items[w];
        const int row = it.row;
        if (ctl.only && !ctl.only[row]) continue;
        // COUNT takes a row's chunks HEAVY_COUNT_SPAN at a time (its items
        // k .. k + span - 1 for k a multiple of the span, one walk over their
        // columns): fewer walks of the A row, fewer lookups; the other items
        // of a group are skipped here
        int span = 1;
        if constexpr (MODE == COUNT) {
            const int k = w - it.first;
            if (k % HEAVY_COUNT_SPAN) continue;
            // the group's items that belong to this row (a row's items are
            // consecutive)
            const bool same = lane > 0 && lane < HEAVY_COUNT_SPAN && w + lane < nitems &&
                              items[w + lane].first == it.first;
            const unsigned m = __ballot_sync(FULL, same) | 1u;
            span = __ffs(~m) - 1;
        }
        const int wcw = span << cw_log2;  // columns walked
        const int lo = it.chunk << cw_log2;
        const int hi = (int)min((int64_t)lo + wcw, (int64_t)B.cols);
        if (MODE == REUSE) {
            float4* a4 = reinterpret_cast<float4*>(acc);
            for (int x = lane; x < (cw >> 2); x += 32) a4[x] = make_float4(0.f, 0.f, 0.f, 0.f);
            __syncwarp();
        }
        int a0, a1;
        row_range(A, row, &a0, &a1, err);
        for (int base = a0; base < a1; base += 32) {
            const int j = base + lane;
            int s = 0, len = 0;
            float av = 0.0f;
            if (j < a1) {
                // {start, end, first column, last column} of B row k =
                // A.ci[j], and its directory offset (or k when it has none)
                int4 m = make_int4(0, 0, 0, -1);
                int64_t d = -1;
                int k = -1;
                if (aux.ameta) {
                    m = aux.ameta[j];
                    const int x = aux.adoff[j];
                    if (x >= 0) d = x; else k = -(x + 2);
                } else {
                    k = A.ci[j];
                    if ((unsigned)k >= (unsigned)B.rows) {
                        atomicOr(err, ERR_STRUCTURE);
                    } else {
                        m = aux.meta[k];
                        if (aux.dir) d = aux.doff[k];
                    }
                }
                if (m.y > m.x && m.w >= lo && m.z < hi) {
                    int t;
                    if (d >= 0 && aux.dir) {
                        const int c = it.chunk - (m.z >> cw_log2);
                        s = m.z >= lo ? m.x : aux.dir[d + c];
                        t = m.w < hi ? m.y : aux.dir[d + c + span];
                        // only an unsorted row (a broken operand) leaves a
                        // directory entry unwritten: stay inside the row
                        s = min(max(s, m.x), m.y);
                        t = min(max(t, s), m.y);
                    } else if (m.z >= lo && m.w < hi) {
                        s = m.x;  // the whole row lies in the chunk
                        t = m.y;
                    } else if (aux.smask && k >= 0 &&
                               !heavy_mask_any(aux, k, it.chunk, span)) {
                        t = s;  // no entry of the row in these chunks
                    } else {
                        s = m.z >= lo ? m.x : seq_lower_bound(B.ci, m.x, m.y, lo);
                        t = m.w < hi ? m.y : seq_lower_bound(B.ci, s, m.y, hi);
                    }
                    len = t - s;
                    if (MODE != COUNT && len > 0) av = A.v[j];
                }
            }
            if (__any_sync(FULL, len > 0))
                heavy_segments<MODE>(B, s, len, av, lo, wcw, acc, bits, err);
        }
        if constexpr (MODE == COUNT) {
            // each chunk of the walk: its count from its half of the bitmap
            __syncwarp();
            for (int h = 0; h < span; ++h) {
                int c = 0;
                for (int x = lane; x < nw; x += 32) {
                    c += __popc(bits[h * nw + x]);
                    bits[h * nw + x] = 0u;
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(FULL, c, o);
                if (lane == 0) {
                    item_cnt[w + h] = c;
                    if (c && row_cnt) atomicAdd(&row_cnt[row], c);
                }
            }
            __syncwarp();
        } else {
            heavy_finish<MODE>(B, w, it, row, lo, cw, acc, bits, item_cnt, row_cnt, item_scan,
                               c_rp, c_ci, c_v, err, ctl);
        }
    }
}

// Heavy rows whose column-chunk counts are still missing (rows the learned
// structure analysis sized by prediction rather than counting by chunk).
__global__ void k_heavy_uncounted(int32_t rows, const uint8_t* __restrict__ bin,
                                  const uint8_t* __restrict__ need, uint8_t* __restrict__ mask) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < rows) mask[r] = bin[r] == BIN_HEAVY && !need[r];
}

// ---------------------------------------------------------------------------
// Exclusive scan of int32 counts (reduce -> scan tile sums -> apply).
// ---------------------------------------------------------------------------
constexpr int SCAN_TPB = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_TPB * SCAN_ITEMS;

__device__ __forceinline__ int64_t block_excl_scan64(int64_t x, int64_t* total) {
    __shared__ int64_t s_warp[SCAN_TPB / 32];
    const int lane = lane_id(), warp = threadIdx.x >> 5;
    int64_t incl = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(FULL, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const int64_t v = lane < SCAN_TPB / 32 ? s_warp[lane] : 0;
        int64_t vi = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(FULL, vi, o);
            if (lane >= o) vi += y;
        }
        if (lane < SCAN_TPB / 32) s_warp[lane] = vi - v;
        if (lane == SCAN_TPB / 32 - 1) *total = vi;
    }
    __syncthreads();
    const int64_t r = s_warp[warp] + incl - x;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(SCAN_TPB)
    k_scan_reduce(const int32_t* __restrict__ in, int64_t n, int64_t* __restrict__ tile_sums) {
    __shared__ int64_t s_total;
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    int64_t s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i)
        if (base + i < n) s += in[base + i];
    block_excl_scan64(s, &s_total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = s_total;
}

// One CTA: exclusive scan of the tile sums in place; total to *total.
__global__ void __launch_bounds__(SCAN_TPB)
    k_scan_tiles(int64_t* __restrict__ tile_sums, int64_t ntiles, int64_t* __restrict__ total) {
    __shared__ int64_t s_total;
    int64_t carry = 0;
    for (int64_t b0 = 0; b0 < ntiles; b0 += SCAN_TPB) {
        const int64_t i = b0 + threadIdx.x;
        const int64_t v = i < ntiles ? tile_sums[i] : 0;
        const int64_t ex = block_excl_scan64(v, &s_total);
        if (i < ntiles) tile_sums[i] = carry + ex;
        carry += s_total;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

// out64[i] / out32[i] = exclusive prefix; out[n] = total. Sets *overflow
// when a 32-bit output would exceed INT32_MAX.
__global__ void __launch_bounds__(SCAN_TPB)
    k_scan_apply(const int32_t* __restrict__ in, int64_t n, const int64_t* __restrict__ tile_sums,
                 const int64_t* __restrict__ total, int64_t* __restrict__ out64,
                 int32_t* __restrict__ out32, int32_t* __restrict__ overflow) {
    __shared__ int64_t s_total;
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    int32_t v[SCAN_ITEMS];
    int64_t s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        v[i] = base + i < n ? in[base + i] : 0;
        s += v[i];
    }
    int64_t run = tile_sums[blockIdx.x] + block_excl_scan64(s, &s_total);
    bool ovf = false;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        if (base + i < n) {
            if (out64) out64[base + i] = run;
            if (out32) {
                out32[base + i] = (int32_t)run;
                ovf |= run > INT32_MAX;
            }
        }
        run += v[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const int64_t tot = *total;
        if (out64) out64[n] = tot;
        if (out32) {
            out32[n] = (int32_t)tot;
            ovf |= tot > INT32_MAX;
        }
    }
    if (ovf) atomicExch(overflow, 1);
}

// Short arrays: the whole exclusive scan in one CTA, tile after tile with a
// running carry (one launch instead of three); outputs as k_scan_apply's.
__global__ void __launch_bounds__(SCAN_TPB)
    k_scan_single(const int32_t* __restrict__ in, int64_t n, int64_t* __restrict__ total,
                  int64_t* __restrict__ out64, int32_t* __restrict__ out32,
                  int32_t* __restrict__ overflow) {
    __shared__ int64_t s_total;
    int64_t carry = 0;
    bool ovf = false;
    for (int64_t t0 = 0; t0 < n; t0 += SCAN_TILE) {
        const int64_t base = t0 + (int64_t)threadIdx.x * SCAN_ITEMS;
        int32_t v[SCAN_ITEMS];
        int64_t s = 0;
#pragma unroll
        for (int i = 0; i < SCAN_ITEMS; ++i) {
            v[i] = base + i < n ? in[base + i] : 0;
            s += v[i];
        }
        int64_t run = carry + block_excl_scan64(s, &s_total);
#pragma unroll
        for (int i = 0; i < SCAN_ITEMS; ++i) {
            if (base + i < n) {
                if (out64) out64[base + i] = run;
                if (out32) {
                    out32[base + i] = (int32_t)run;
                    ovf |= run > INT32_MAX;
                }
            }
            run += v[i];
        }
        carry += s_total;
        __syncthreads();  // every thread has read s_total before the next tile's scan
    }
    if (threadIdx.x == 0) {
        *total = carry;
        if (out64) out64[n] = carry;
        if (out32) {
            out32[n] = (int32_t)carry;
            ovf |= carry > INT32_MAX;
        }
    }
    if (ovf) atomicExch(overflow, 1);
}

// ---------------------------------------------------------------------------
// Canonical CSR check (rv-sparse src/kernels/spgemm/rvsp_support.c:37-127):
// thread per row; the lowest failing row wins. Row offsets outside [0, nnz]
// are reported as a bad row pointer before any column is read.
// ---------------------------------------------------------------------------
// With CANONICAL == false only the row pointer and the column range are
// checked (rv-sparse src/core/matrix.c:51-90, rvsp_csr_validate).
template <bool CANONICAL>
__global__ void k_csr_check(int32_t rows, int32_t cols, int32_t nnz,
                            const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                            unsigned long long* __restrict__ worst) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const int s = rp[r], e = rp[r + 1];
    int code = 0;
    if (e < s || s < 0 || e > nnz) {
        code = 1;
    } else {
        int last = -1;
        for (int p = s; p < e && !code; ++p) {
            const int c = ci[p];
            if (c < 0 || c >= cols) code = 2;
            else if (CANONICAL && c == last) code = 4;
            else if (CANONICAL && c < last) code = 3;
            last = c;
        }
    }
    if (code) atomicMin(worst, ((unsigned long long)(uint32_t)r << 8) | (unsigned)code);
}

}  // namespace rvsp
