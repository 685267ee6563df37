// The reference's two other dtypes on the CUDA backend: FP64 x FP64 -> FP64
// and INT8 x INT8 -> INT32, one call each (rvsp_cuda_spgemm_f64 / _i8), the
// device counterparts of the reference's legacy raw kernels
// rvsp_spgemm_csr_scalar_f64_raw and rvsp_spgemm_csr_scalar_i8_raw
// (rv-sparse src/kernels/spgemm/legacy/csr_scalar_f64.c:49-272,
// csr_scalar_i8.c:24-196).
//
// Semantics kept from those kernels: per output column acc += a * b in A-row
// order starting from zero (FP64 products and sums rounded to nearest, no
// FMA; INT32 products and sums in two's complement), columns ascending, and
// entries whose sum is exactly zero are not stored (the FP32 path keeps
// them, as the reference's FP32 path does).
//
// Pipeline: the structure comes from the FP32 machinery (exact analysis,
// count, fill with zero-valued operands, which only the column indices of
// are used); a warp per output row then recomputes the values in the typed
// arithmetic, positions found by binary search in the row's sorted columns
// (staged in shared memory for rows of up to TYPED_STAGE entries, read in
// place otherwise); last, the rows are compacted without their zero sums.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "rv_sparse_types.h"
#include "rvsp_cuda.h"
#include "rvsp_internal.h"

using namespace rvsp;

namespace {

__device__ __forceinline__ int t_lane() { return threadIdx.x & 31; }

__device__ __forceinline__ int t_incl_scan(int x) {
    const int lane = t_lane();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// Row range of row r of M; out-of-range rows or offsets flag ERR_STRUCTURE
// and read as empty.
__device__ __forceinline__ void t_row_range(const CsrView& M, int r, int* s, int* e,
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

struct F64Ops {
    using In = double;
    using Out = double;
    static __device__ __forceinline__ Out mul(In a, In b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ Out add(Out x, Out y) { return __dadd_rn(x, y); }
};

struct I8Ops {
    using In = int8_t;
    using Out = int32_t;
    static __device__ __forceinline__ Out mul(In a, In b) {
        return (int32_t)((uint32_t)(int32_t)a * (uint32_t)(int32_t)b);
    }
    static __device__ __forceinline__ Out add(Out x, Out y) {
        return (int32_t)((uint32_t)x + (uint32_t)y);
    }
};

constexpr int TYPED_WARPS = 4;
constexpr int TYPED_STAGE = 1024;  // row entries staged in shared memory

// vals[slot] = add(vals[slot], prod) for every active lane, lanes sharing a
// slot combined in lane order (= A-row order).
template <class Ops>
__device__ __forceinline__ void typed_ordered_add(typename Ops::Out* vals, int slot, bool active,
                                                  typename Ops::Out prod) {
    using T = typename Ops::Out;
    const int lane = t_lane();
    const int key = active ? slot : (0x40000000 | lane);
    const unsigned peers = __match_any_sync(FULL, key);
    const int maxn = __reduce_max_sync(FULL, (unsigned)__popc(peers));
    if (maxn == 1) {
        if (active) vals[slot] = Ops::add(vals[slot], prod);
        return;
    }
    const bool lead = active && lane == __ffs(peers) - 1;
    T acc = lead ? vals[slot] : T(0);
    unsigned m = peers;
    for (int r = 0; r < maxn; ++r) {
        const int src = m ? (__ffs(m) - 1) : lane;
        const T v = __shfl_sync(FULL, prod, src);
        if (lead && m) acc = Ops::add(acc, v);
        m &= m - 1;
    }
    if (lead) vals[slot] = acc;
}

// First index in [0, n) of cols with cols[idx] >= col (n if none).
__device__ __forceinline__ int typed_lower_bound(const int32_t* cols, int n, int32_t col) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (cols[mid] < col) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Values of every output row on its known sorted structure, one warp per row.
template <class Ops>
__global__ void __launch_bounds__(TYPED_WARPS * 32)
    k_typed_numeric(CsrView A, CsrView B, const typename Ops::In* __restrict__ av,
                    const typename Ops::In* __restrict__ bv, const int32_t* __restrict__ c_rp,
                    const int32_t* __restrict__ c_ci, typename Ops::Out* __restrict__ c_v,
                    int32_t* __restrict__ err) {
    using T = typename Ops::Out;
    __shared__ int32_t s_cols[TYPED_WARPS][TYPED_STAGE];
    __shared__ T s_acc[TYPED_WARPS][TYPED_STAGE];
    const int warp = threadIdx.x >> 5, lane = t_lane();
    for (int row = blockIdx.x * TYPED_WARPS + warp; row < A.rows; row += gridDim.x * TYPED_WARPS) {
        const int c0 = c_rp[row], n = c_rp[row + 1] - c0;
        const bool staged = n <= TYPED_STAGE;
        const int32_t* cols = staged ? s_cols[warp] : c_ci + c0;
        T* acc = staged ? s_acc[warp] : c_v + c0;
        for (int x = lane; x < n; x += 32) {
            if (staged) s_cols[warp][x] = c_ci[c0 + x];
            acc[x] = T(0);
        }
        __syncwarp();
        int a0, a1;
        t_row_range(A, row, &a0, &a1, err);
        for (int base = a0; base < a1; base += 32) {
            const int j = base + lane;
            int bs = 0, bl = 0;
            T a = T(0);
            if (j < a1) {
                int be;
                t_row_range(B, A.ci[j], &bs, &be, err);
                bl = be - bs;
                a = (T)av[j];
            }
            const int incl = t_incl_scan(bl);
            const int total = __shfl_sync(FULL, incl, 31);
            for (int f0 = 0; f0 < total; f0 += 32) {
                const int p = f0 + lane;
                // entry of product p: the number of entries whose products end at or before p
                int e = 0;
#pragma unroll
                for (int st = 16; st >= 1; st >>= 1) {
                    const int cand = __shfl_sync(FULL, incl, e + st - 1);
                    if (cand <= p) e += st;
                }
                e = min(e, 31);
                const int e_incl = __shfl_sync(FULL, incl, e);
                const int e_bl = __shfl_sync(FULL, bl, e);
                const int e_bs = __shfl_sync(FULL, bs, e);
                const T ea = __shfl_sync(FULL, a, e);
                int pos = -1;
                T prod = T(0);
                if (p < total) {
                    const int q = e_bs + (p - (e_incl - e_bl));
                    pos = typed_lower_bound(cols, n, B.ci[q]);
                    if (pos >= n || cols[pos] != B.ci[q]) {
                        atomicOr(err, ERR_STRUCTURE);  // the structure does not hold the column
                        pos = -1;
                    } else {
                        prod = Ops::mul((typename Ops::In)ea, bv[q]);
                    }
                }
                typed_ordered_add<Ops>(acc, pos < 0 ? 0 : pos, pos >= 0, prod);
                __syncwarp();
            }
        }
        __syncwarp();
        if (staged)
            for (int x = lane; x < n; x += 32) c_v[c0 + x] = acc[x];
        __syncwarp();
    }
}

// Per-row count of the entries whose value is not zero.
template <class T>
__global__ void k_nonzero_count(int32_t rows, const int32_t* __restrict__ c_rp,
                                const T* __restrict__ c_v, int32_t* __restrict__ cnt) {
    const int row = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = t_lane();
    if (row >= rows) return;
    int c = 0;
    for (int x = c_rp[row] + lane; x < c_rp[row + 1]; x += 32) c += c_v[x] != T(0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(FULL, c, o);
    if (lane == 0) cnt[row] = c;
}

// Rows copied without their zero entries, order kept.
template <class T>
__global__ void k_nonzero_compact(int32_t rows, const int32_t* __restrict__ c_rp,
                                  const int32_t* __restrict__ c_ci, const T* __restrict__ c_v,
                                  const int32_t* __restrict__ out_rp, int32_t* __restrict__ out_ci,
                                  T* __restrict__ out_v) {
    const int row = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = t_lane();
    if (row >= rows) return;
    int o = out_rp[row];
    for (int x0 = c_rp[row]; x0 < c_rp[row + 1]; x0 += 32) {
        const int x = x0 + lane;
        const bool keep = x < c_rp[row + 1] && c_v[x] != T(0);
        const unsigned m = __ballot_sync(FULL, keep);
        if (keep) {
            const int d = o + __popc(m & ((1u << lane) - 1));
            out_ci[d] = c_ci[x];
            out_v[d] = c_v[x];
        }
        o += __popc(m);
    }
}

thread_local rvsp_cuda_plan_t t_tplan = nullptr;

struct TypedReaper {
    ~TypedReaper() {
        if (t_tplan) {
            rvsp_cuda_plan_destroy(t_tplan);
            t_tplan = nullptr;
        }
    }
};
thread_local TypedReaper t_treaper;

// Stream-ordered device allocations of one call, released together.
struct Scratch {
    cudaStream_t st;
    void* p[16] = {};
    int n = 0;
    explicit Scratch(cudaStream_t s) : st(s) {}
    template <class T>
    cudaError_t get(T** out, size_t bytes) {
        void* q = nullptr;
        cudaError_t e = cudaMallocAsync(&q, bytes ? bytes : 16, st);
        if (e == cudaSuccess) p[n++] = q;
        *out = static_cast<T*>(q);
        return e;
    }
    void release() {
        for (int i = 0; i < n; ++i) cudaFreeAsync(p[i], st);
        n = 0;
    }
};

template <class Ops>
int typed_spgemm(int32_t a_rows, int32_t a_cols, int32_t b_cols, const int32_t* a_rp,
                 const int32_t* a_ci, const typename Ops::In* a_v, const int32_t* b_rp,
                 const int32_t* b_ci, const typename Ops::In* b_v, int32_t** c_rp_out,
                 int32_t** c_ci_out, typename Ops::Out** c_v_out, int32_t* c_nnz_out) {
    using In = typename Ops::In;
    using Out = typename Ops::Out;
    if (!a_rp || !a_ci || !a_v || !b_rp || !b_ci || !b_v || !c_rp_out || !c_ci_out ||
        !c_v_out || !c_nnz_out)
        return RVSP_ERROR_NULL_POINTER;
    if (a_rows <= 0 || a_cols <= 0 || b_cols <= 0) return RVSP_ERROR_INVALID_ARGUMENT;
    *c_rp_out = nullptr;
    *c_ci_out = nullptr;
    *c_v_out = nullptr;
    *c_nnz_out = 0;
    if (rvsp_cuda_device_count() == 0) return RVSP_ERROR_UNSUPPORTED_BACKEND;
    int st;
    if (!t_tplan) {
        if ((st = rvsp_cuda_plan_create(&t_tplan, RVSP_CUDA_ALGO_EXACT))) return st;
        t_tplan->map_policy = 0;
    }
    rvsp_cuda_plan_t plan = t_tplan;
    plan->params = default_params();
    keep_pool_memory();
    cudaStream_t s = plan->stream;
    const bool dev = is_dev(a_rp);
    cudaError_t e;
    int32_t a_nnz = 0, b_nnz = 0;
    if (dev) {
        if ((e = cudaMemcpy(&a_nnz, a_rp + a_rows, 4, cudaMemcpyDeviceToHost)) != cudaSuccess ||
            (e = cudaMemcpy(&b_nnz, b_rp + a_cols, 4, cudaMemcpyDeviceToHost)) != cudaSuccess)
            return fail(e, "row_ptr read");
    } else {
        a_nnz = a_rp[a_rows];
        b_nnz = b_rp[a_cols];
    }
    if (a_nnz < 0 || b_nnz < 0) return RVSP_ERROR_INVALID_CSR;
    Scratch sc(s);
    auto bail = [&](int code) {
        sc.release();
        cudaStreamSynchronize(s);
        return code;
    };
    // operands on the device (index arrays and typed values)
    const int32_t *d_arp = a_rp, *d_aci = a_ci, *d_brp = b_rp, *d_bci = b_ci;
    const In *d_av = a_v, *d_bv = b_v;
    if (!dev) {
        int32_t *t0, *t1, *t2, *t3;
        In *t4, *t5;
        if ((e = sc.get(&t0, 4 * ((size_t)a_rows + 1))) || (e = sc.get(&t1, 4 * (size_t)a_nnz)) ||
            (e = sc.get(&t2, 4 * ((size_t)a_cols + 1))) || (e = sc.get(&t3, 4 * (size_t)b_nnz)) ||
            (e = sc.get(&t4, sizeof(In) * (size_t)a_nnz)) ||
            (e = sc.get(&t5, sizeof(In) * (size_t)b_nnz)))
            return bail(fail(e, "staging"));
        cudaMemcpyAsync(t0, a_rp, 4 * ((size_t)a_rows + 1), cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(t1, a_ci, 4 * (size_t)a_nnz, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(t2, b_rp, 4 * ((size_t)a_cols + 1), cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(t3, b_ci, 4 * (size_t)b_nnz, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(t4, a_v, sizeof(In) * (size_t)a_nnz, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(t5, b_v, sizeof(In) * (size_t)b_nnz, cudaMemcpyHostToDevice, s);
        d_arp = t0, d_aci = t1, d_brp = t2, d_bci = t3, d_av = t4, d_bv = t5;
    }
    // structure: exact analysis and count, then a fill on zero-valued operands
    int64_t nnz = 0;
    size_t ws = 0;
    if ((st = rvsp_cuda_symbolic(plan, a_rows, a_cols, a_nnz, d_arp, d_aci, a_cols, b_cols, b_nnz,
                                 d_brp, d_bci, &nnz, &ws)))
        return bail(st);
    float* zeros;
    int32_t *s_rp, *s_ci, *cnt, *o_rp;
    float* s_fv;
    Out* s_v;
    const size_t zn = (size_t)std::max(a_nnz, b_nnz) + 1, cn = (size_t)(nnz > 0 ? nnz : 1);
    if ((e = sc.get(&zeros, 4 * zn)) || (e = sc.get(&s_rp, 4 * ((size_t)a_rows + 1))) ||
        (e = sc.get(&s_ci, 4 * cn)) || (e = sc.get(&s_fv, 4 * cn)) ||
        (e = sc.get(&s_v, sizeof(Out) * cn)) || (e = sc.get(&cnt, 4 * (size_t)a_rows)) ||
        (e = sc.get(&o_rp, 4 * ((size_t)a_rows + 1))))
        return bail(fail(e, "typed scratch"));
    cudaMemsetAsync(zeros, 0, 4 * zn, s);
    if ((st = rvsp_cuda_numeric(plan, d_arp, d_aci, zeros, d_brp, d_bci, zeros, s_rp, s_ci, s_fv, 1,
                                nullptr)))
        return bail(st);
    // typed values on that structure
    Misc* misc = plan->misc.as<Misc>();
    const CsrView A{d_arp, d_aci, nullptr, a_rows, a_cols, a_nnz};
    const CsrView B{d_brp, d_bci, nullptr, a_cols, b_cols, b_nnz};
    const int grid = (int)std::min<int64_t>(((int64_t)a_rows + TYPED_WARPS - 1) / TYPED_WARPS,
                                            148 * 16);
    k_typed_numeric<Ops><<<grid, TYPED_WARPS * 32, 0, s>>>(A, B, d_av, d_bv, s_rp, s_ci, s_v,
                                                          &misc->err);
    const unsigned wgrid = (unsigned)(((int64_t)a_rows * 32 + 255) / 256);
    k_nonzero_count<Out><<<wgrid, 256, 0, s>>>(a_rows, s_rp, s_v, cnt);
    note_launch(plan, 2);
    if ((st = scan_counts(plan, cnt, a_rows, nullptr, o_rp, &misc->scan_total))) return bail(st);
    int64_t total = 0;
    int32_t err = 0;
    if ((e = cudaMemcpyAsync(&total, &misc->scan_total, 8, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(&err, &misc->err, 4, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaStreamSynchronize(s)))
        return bail(fail(e, "typed numeric"));
    if (err) {
        g_err = "operand structure out of range (row_ptr or col_idx)";
        return bail(RVSP_ERROR_INVALID_CSR);
    }
    // outputs where the inputs live
    int32_t *rp = nullptr, *ci = nullptr;
    Out* v = nullptr;
    const size_t on = (size_t)(total > 0 ? total : 1);
    if ((e = cudaMallocAsync((void**)&rp, 4 * ((size_t)a_rows + 1), s)) ||
        (e = cudaMallocAsync((void**)&ci, 4 * on, s)) ||
        (e = cudaMallocAsync((void**)&v, sizeof(Out) * on, s))) {
        if (rp) cudaFreeAsync(rp, s);
        if (ci) cudaFreeAsync(ci, s);
        return bail(fail(e, "C alloc"));
    }
    cudaMemcpyAsync(rp, o_rp, 4 * ((size_t)a_rows + 1), cudaMemcpyDeviceToDevice, s);
    k_nonzero_compact<Out><<<wgrid, 256, 0, s>>>(a_rows, s_rp, s_ci, s_v, o_rp, ci, v);
    note_launch(plan, 1);
    sc.release();
    if ((e = cudaGetLastError()) != cudaSuccess) {
        cudaFreeAsync(rp, s);
        cudaFreeAsync(ci, s);
        cudaFreeAsync(v, s);
        cudaStreamSynchronize(s);
        return fail(e, "typed launch");
    }
    if (!dev) {
        int32_t* hrp = (int32_t*)malloc(4 * ((size_t)a_rows + 1));
        int32_t* hci = (int32_t*)malloc(4 * on);
        Out* hv = (Out*)malloc(sizeof(Out) * on);
        if (!hrp || !hci || !hv) {
            free(hrp);
            free(hci);
            free(hv);
            cudaFreeAsync(rp, s);
            cudaFreeAsync(ci, s);
            cudaFreeAsync(v, s);
            cudaStreamSynchronize(s);
            return RVSP_ERROR_ALLOCATION_FAILED;
        }
        cudaMemcpyAsync(hrp, rp, 4 * ((size_t)a_rows + 1), cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(hci, ci, 4 * (size_t)total, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(hv, v, sizeof(Out) * (size_t)total, cudaMemcpyDeviceToHost, s);
        cudaFreeAsync(rp, s);
        cudaFreeAsync(ci, s);
        cudaFreeAsync(v, s);
        if ((e = cudaStreamSynchronize(s)) != cudaSuccess) {
            free(hrp);
            free(hci);
            free(hv);
            return fail(e, "C copy-out");
        }
        rp = hrp, ci = hci, v = hv;
    } else if ((e = cudaStreamSynchronize(s)) != cudaSuccess) {
        return fail(e, "typed compact");
    }
    *c_rp_out = rp;
    *c_ci_out = ci;
    *c_v_out = v;
    *c_nnz_out = (int32_t)total;
    return RVSP_SUCCESS;
}

}  // namespace

extern "C" int rvsp_cuda_spgemm_f64(int32_t a_rows, int32_t a_cols, int32_t b_cols,
                                    const int32_t* a_rp, const int32_t* a_ci, const double* a_v,
                                    const int32_t* b_rp, const int32_t* b_ci, const double* b_v,
                                    int32_t** c_rp_out, int32_t** c_ci_out, double** c_v_out,
                                    int32_t* c_nnz_out) {
    return typed_spgemm<F64Ops>(a_rows, a_cols, b_cols, a_rp, a_ci, a_v, b_rp, b_ci, b_v,
                                c_rp_out, c_ci_out, c_v_out, c_nnz_out);
}

extern "C" int rvsp_cuda_spgemm_i8(int32_t a_rows, int32_t a_cols, int32_t b_cols,
                                   const int32_t* a_rp, const int32_t* a_ci, const int8_t* a_v,
                                   const int32_t* b_rp, const int32_t* b_ci, const int8_t* b_v,
                                   int32_t** c_rp_out, int32_t** c_ci_out, int32_t** c_v_out,
                                   int32_t* c_nnz_out) {
    return typed_spgemm<I8Ops>(a_rows, a_cols, b_cols, a_rp, a_ci, a_v, b_rp, b_ci, b_v,
                               c_rp_out, c_ci_out, c_v_out, c_nnz_out);
}
