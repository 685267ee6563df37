"""ctypes binding of librvsp_b200.so (the rv-sparse C API on the B200 backend).

The library is the product; this module only loads it and mirrors its C
declarations (include/rv_sparse.h, include/rv_sparse_types.h,
include/rvsp_cuda.h) so tests and benchmarks can drive it from Python. It
never computes a product itself: when the shared library is missing every
entry point raises instead of falling back to anything.

Array arguments accept numpy arrays (host memory) or objects exposing a
device pointer via ``data_ptr()`` (e.g. CUDA tensors), matching the library's
per-pointer residency rule.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "lib", "librvsp_b200.so")

# rv_sparse_types.h
RVSP_SUCCESS = 0
RVSP_ERROR_NULL_POINTER = -1
RVSP_ERROR_INVALID_ARGUMENT = -2
RVSP_ERROR_INVALID_CSR = -3
RVSP_ERROR_UNSUPPORTED_DTYPE = -4
RVSP_ERROR_UNSUPPORTED_BACKEND = -5
RVSP_ERROR_ALLOCATION_FAILED = -6
RVSP_ERROR_DEVICE_FAILURE = -7

RVSP_DTYPE_INT8, RVSP_DTYPE_INT32, RVSP_DTYPE_BF16, RVSP_DTYPE_FP32, RVSP_DTYPE_FP64 = range(5)
RVSP_FORMAT_CSR = 0
(RVSP_BACKEND_SCALAR, RVSP_BACKEND_SCALAR_UNROLL4, RVSP_BACKEND_RVV_INTRINSICS,
 RVSP_BACKEND_CUDA, RVSP_BACKEND_CUDA_LEARNED) = range(5)
(RVSP_SPGEMM_ALGO_DEFAULT, RVSP_SPGEMM_ALGO_RVV, RVSP_SPGEMM_ALGO_CONTIG,
 RVSP_SPGEMM_ALGO_ADAPTIVE, RVSP_SPGEMM_ALGO_CUDA, RVSP_SPGEMM_ALGO_CUDA_LEARNED) = range(6)
RVSP_OWNS_HOST = 1
RVSP_OWNS_DEVICE = 2
RVSP_CUDA_ALGO_EXACT = 4
RVSP_CUDA_ALGO_LEARNED = 5


class CsrMatrix(C.Structure):
    """rvsp_csr_matrix_t"""
    _fields_ = [("rows", C.c_int32), ("cols", C.c_int32), ("nnz", C.c_int32),
                ("row_ptr", C.c_void_p), ("col_idx", C.c_void_p), ("values", C.c_void_p),
                ("dtype", C.c_int), ("format", C.c_int), ("owns_data", C.c_int)]


class SpgemmOptions(C.Structure):
    """rvsp_spgemm_options_t"""
    _fields_ = [("backend", C.c_int), ("input_dtype", C.c_int), ("output_dtype", C.c_int)]


class RvspError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        super().__init__(f"{what}: status {status} ({status_string(status)}) {last_error()}")


_lib = None

_VP = C.c_void_p
_I32 = C.c_int32
_I64 = C.c_int64

_PROTOS = {
    # rv_sparse.h
    "rvsp_get_version": (C.c_char_p, []),
    "rvsp_status_to_string": (C.c_char_p, [C.c_int]),
    "rvsp_csr_create": (C.c_int, [C.POINTER(CsrMatrix), _I32, _I32, _I32, _VP, _VP, _VP, C.c_int]),
    "rvsp_csr_validate": (C.c_int, [C.POINTER(CsrMatrix)]),
    "rvsp_csr_destroy": (None, [C.POINTER(CsrMatrix)]),
    "rvsp_spgemm_csr": (C.c_int, [C.POINTER(CsrMatrix), C.POINTER(CsrMatrix), C.POINTER(CsrMatrix),
                                  C.POINTER(SpgemmOptions)]),
    "rvsp_spgemm_descr_create": (C.c_int, [C.POINTER(_VP)]),
    "rvsp_spgemm_descr_destroy": (None, [_VP]),
    "rvsp_spgemm_set_algo": (C.c_int, [_VP, C.c_int]),
    "rvsp_spgemm_work_estimation": (C.c_int, [_VP, C.POINTER(CsrMatrix), C.POINTER(CsrMatrix),
                                              C.POINTER(C.c_size_t), C.POINTER(_I32)]),
    "rvsp_spgemm_compute": (C.c_int, [_VP, C.POINTER(CsrMatrix), C.POINTER(CsrMatrix),
                                      C.POINTER(CsrMatrix), _VP]),
    "rvsp_spgemm_get_op_counts": (C.c_int, [_VP, _VP, _I32]),
    "rvsp_spgemm_invalidate_structure": (None, [_VP]),
    # rvsp_cuda.h
    "rvsp_cuda_device_count": (C.c_int, []),
    "rvsp_cuda_last_error": (C.c_char_p, []),
    "rvsp_cuda_is_device_pointer": (C.c_int, [_VP]),
    "rvsp_cuda_free": (None, [_VP]),
    "rvsp_cuda_host_free": (None, [_VP]),
    "rvsp_cuda_plan_create": (C.c_int, [C.POINTER(_VP), C.c_int]),
    "rvsp_cuda_plan_destroy": (None, [_VP]),
    "rvsp_cuda_plan_set_async": (C.c_int, [_VP, C.c_int]),
    "rvsp_cuda_plan_stream": (_VP, [_VP]),
    "rvsp_cuda_symbolic": (C.c_int, [_VP, _I32, _I32, _I32, _VP, _VP, _I32, _I32, _I32, _VP, _VP,
                                     C.POINTER(_I64), C.POINTER(C.c_size_t)]),
    "rvsp_cuda_numeric": (C.c_int, [_VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, C.c_int, _VP]),
    "rvsp_cuda_op_counts": (C.c_int, [_VP, _VP, _I32]),
    "rvsp_cuda_spgemm_f32": (C.c_int, [C.c_int, _I32, _I32, _I32, _VP, _VP, _VP, _VP, _VP, _VP,
                                       C.POINTER(_VP), C.POINTER(_VP), C.POINTER(_VP),
                                       C.POINTER(_I32), _VP]),
    "rvsp_cuda_spgemm_f64": (C.c_int, [_I32, _I32, _I32, _VP, _VP, _VP, _VP, _VP, _VP,
                                       C.POINTER(_VP), C.POINTER(_VP), C.POINTER(_VP),
                                       C.POINTER(_I32)]),
    "rvsp_cuda_spgemm_i8": (C.c_int, [_I32, _I32, _I32, _VP, _VP, _VP, _VP, _VP, _VP,
                                      C.POINTER(_VP), C.POINTER(_VP), C.POINTER(_VP),
                                      C.POINTER(_I32)]),
    "rvsp_cuda_coo_to_csr": (C.c_int, [_I32, _I32, _I64, _VP, _VP, _VP, C.c_int, C.c_int,
                                       C.POINTER(_VP), C.POINTER(_VP), C.POINTER(_VP),
                                       C.POINTER(_I32)]),
    "rvsp_cuda_mtx_read": (C.c_int, [C.c_char_p, C.POINTER(_I32), C.POINTER(_I32),
                                     C.POINTER(_I64), C.POINTER(_VP), C.POINTER(_VP),
                                     C.POINTER(_VP), C.POINTER(C.c_int)]),
    "rvsp_cuda_mtx_to_csr": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(_I32), C.POINTER(_I32),
                                       C.POINTER(_I32), C.POINTER(_VP), C.POINTER(_VP),
                                       C.POINTER(_VP)]),
    "rvsp_cuda_csr_check": (C.c_int, [_I32, _I32, _I32, _VP, _VP, C.POINTER(_I32)]),
    "rvsp_cuda_csr_validate": (C.c_int, [_I32, _I32, _I32, _VP, _VP]),
    "rvsp_cuda_launch_count": (_I64, []),
    "rvsp_cuda_kernel_timing": (C.c_int, [C.c_int]),
    "rvsp_cuda_kernel_times": (C.c_int, [_VP, _VP, _I32]),
    "rvsp_cuda_kernel_family": (C.c_char_p, [_I32]),
    "rvsp_cuda_learned_available": (C.c_int, []),
    "rvsp_cuda_mlp_load": (C.c_int, [C.c_char_p]),
    "rvsp_cuda_mlp_set": (C.c_int, [_VP, _I32]),
    "rvsp_cuda_mlp_get": (C.c_int, [_VP, _I32]),
    "rvsp_cuda_mlp_save": (C.c_int, [C.c_char_p, _VP, _I32]),
    "rvsp_cuda_mlp_grad": (C.c_int, [_VP, _VP, _VP, _VP, _I32, _VP, _VP]),
    "rvsp_cuda_mlp_train": (C.c_int, [_VP, _VP, _VP, _VP, _I32, _I32, _I32, C.c_float,
                                      C.c_uint64, _VP]),
    "rvsp_cuda_mlp_infer": (C.c_int, [_VP, _I32, _VP, _VP, _I32, _VP, _VP, _VP]),
    "rvsp_cuda_plan_collect_features": (C.c_int, [_VP, C.c_int]),
    "rvsp_cuda_plan_row_stats": (C.c_int, [_VP, _VP, _VP, _VP, _I32]),
    "rvsp_cuda_plan_learned_stats": (C.c_int, [_VP, _VP, _I32]),
    "rvsp_cuda_oneshot_learned_stats": (C.c_int, [_VP, _I32]),
    "rvsp_cuda_row_ptr_noalloc": (C.c_int, [_VP, _I32, _VP, C.POINTER(_I64), _VP]),
    "rvsp_cuda_plan_set_params": (C.c_int, [_VP, _VP, _I32]),
    "rvsp_cuda_plan_get_params": (C.c_int, [_VP, _VP, _I32]),
    "rvsp_cuda_set_default_params": (C.c_int, [_VP, _I32]),
    "rvsp_cuda_get_default_params": (C.c_int, [_VP, _I32]),
    "rvsp_cuda_plan_autotune": (C.c_int, [_VP, _I32, _I32, _I32, _VP, _VP, _VP, _I32, _I32, _I32,
                                          _VP, _VP, _VP, _I32, _VP, _VP, _VP, _I32,
                                          C.POINTER(_I32), C.POINTER(_I64),
                                          C.POINTER(C.c_size_t)]),
    "rvsp_cuda_spgemm_batched_f32": (C.c_int, [C.c_int, _I32, _VP, _VP, _VP, _VP, _VP,
                                               _VP, _VP, _VP, _VP, _VP, _VP,
                                               C.POINTER(_VP), C.POINTER(_VP), C.POINTER(_VP),
                                               C.POINTER(_I64), _VP, _VP]),
}

BIN_PARAMS = 4  # tiny_ops, slack_shift, warp_cap_max, heavy_cw_log2
BIN_PARAM_NAMES = ("tiny_ops", "slack_shift", "warp_cap_max", "heavy_cw_log2")
DEFAULT_BIN_PARAMS = (32, 2, 2048, 11)
MLP_PARAMS = 1282
MLP_FLOATS = 1291  # [mean(4), inv_std(4), z, params(1282)]


def build() -> None:
    """Compile the library in-tree for sm_100a (make -C rv-sparse_b200)."""
    subprocess.run(["make", "-s", "-j8", "-C", PKG_DIR], check=True)


def lib():
    """The loaded librvsp_b200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: run `make -C {PKG_DIR}`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def status_string(st: int) -> str:
    return lib().rvsp_status_to_string(st).decode()


def last_error() -> str:
    return lib().rvsp_cuda_last_error().decode()


def device_count() -> int:
    return lib().rvsp_cuda_device_count()


def launch_count() -> int:
    return lib().rvsp_cuda_launch_count()


KERNEL_FAMILIES = 14


def kernel_timing(on: bool) -> None:
    """Start (resetting the totals) or stop per-family device timing."""
    check(lib().rvsp_cuda_kernel_timing(1 if on else 0), "kernel_timing")


def kernel_times() -> dict:
    """{family: (total ms, launches)} of the timed launches so far."""
    L = lib()
    ms = np.zeros(KERNEL_FAMILIES, np.float64)
    n = np.zeros(KERNEL_FAMILIES, np.int64)
    check(L.rvsp_cuda_kernel_times(ms.ctypes.data, n.ctypes.data, KERNEL_FAMILIES), "kernel_times")
    return {L.rvsp_cuda_kernel_family(i).decode(): (float(ms[i]), int(n[i]))
            for i in range(KERNEL_FAMILIES)}


def ptr(a) -> int | None:
    """Address of a numpy array or of a device tensor (data_ptr())."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data if a.size else _EMPTY.ctypes.data
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return int(a)


_EMPTY = np.zeros(4, np.int32)


def check(st: int, what: str = "") -> None:
    if st != RVSP_SUCCESS:
        raise RvspError(st, what)


def csr_struct(rows, cols, nnz, row_ptr, col_idx, values, dtype=RVSP_DTYPE_FP32) -> CsrMatrix:
    M = CsrMatrix()
    M.rows, M.cols, M.nnz = rows, cols, nnz
    M.row_ptr, M.col_idx, M.values = ptr(row_ptr), ptr(col_idx), ptr(values)
    M.dtype, M.format, M.owns_data = dtype, RVSP_FORMAT_CSR, 0
    return M


def from_csr(M) -> CsrMatrix:
    """rvsp_csr_matrix_t view of an object with rows, cols, row_ptr, col_idx, values."""
    return csr_struct(M.rows, M.cols, int(M.row_ptr[-1]) if isinstance(M.row_ptr, np.ndarray)
                      else int(M.nnz), M.row_ptr, M.col_idx, M.values)


def spgemm(A, B, backend=RVSP_BACKEND_CUDA):
    """One-shot C = A * B on host numpy CSR through rvsp_spgemm_csr.

    Returns (row_ptr, col_idx, values) as numpy arrays (copies); C is
    released with rvsp_csr_destroy.
    """
    L = lib()
    a, b = from_csr(A), from_csr(B)
    c = CsrMatrix()
    opts = SpgemmOptions(backend, RVSP_DTYPE_FP32, RVSP_DTYPE_FP32)
    check(L.rvsp_spgemm_csr(C.byref(a), C.byref(b), C.byref(c), C.byref(opts)), "rvsp_spgemm_csr")
    try:
        n = c.nnz
        rp = np.ctypeslib.as_array(C.cast(c.row_ptr, C.POINTER(C.c_int32)), (A.rows + 1,)).copy()
        ci = (np.ctypeslib.as_array(C.cast(c.col_idx, C.POINTER(C.c_int32)), (n,)).copy()
              if n else np.zeros(0, np.int32))
        v = (np.ctypeslib.as_array(C.cast(c.values, C.POINTER(C.c_float)), (n,)).copy()
             if n else np.zeros(0, np.float32))
    finally:
        L.rvsp_csr_destroy(C.byref(c))
    return rp, ci, v


class Descriptor:
    """rvsp_spgemm_descr_t with its create / set_algo / estimate / compute cycle."""

    def __init__(self, algo=RVSP_SPGEMM_ALGO_CUDA):
        self.L = lib()
        self.h = C.c_void_p()
        check(self.L.rvsp_spgemm_descr_create(C.byref(self.h)), "descr_create")
        if algo is not None:
            check(self.L.rvsp_spgemm_set_algo(self.h, algo), "set_algo")

    def close(self):
        if self.h:
            self.L.rvsp_spgemm_descr_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def work_estimation(self, a: CsrMatrix, b: CsrMatrix):
        ws = C.c_size_t(0)
        nnz = C.c_int32(0)
        st = self.L.rvsp_spgemm_work_estimation(self.h, C.byref(a), C.byref(b), C.byref(ws),
                                                C.byref(nnz))
        return st, ws.value, nnz.value

    def compute(self, a: CsrMatrix, b: CsrMatrix, c: CsrMatrix, ws) -> int:
        return self.L.rvsp_spgemm_compute(self.h, C.byref(a), C.byref(b), C.byref(c), ptr(ws))

    def op_counts(self, n):
        out = np.zeros(max(n, 1), np.int64)
        st = self.L.rvsp_spgemm_get_op_counts(self.h, out.ctypes.data, n)
        return st, out[:n]

    def invalidate(self):
        self.L.rvsp_spgemm_invalidate_structure(self.h)


class Plan:
    """rvsp_cuda_plan_t: the device-side half of a descriptor, driven directly."""

    def __init__(self, algo=RVSP_CUDA_ALGO_EXACT, features=False):
        self.L = lib()
        self.h = C.c_void_p()
        check(self.L.rvsp_cuda_plan_create(C.byref(self.h), algo), "plan_create")
        if features:
            check(self.L.rvsp_cuda_plan_collect_features(self.h, 1))
        self.rows = 0

    def close(self):
        if self.h:
            self.L.rvsp_cuda_plan_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def symbolic(self, A, B, a_nnz=None, b_nnz=None):
        """A, B: objects with rows, cols, row_ptr, col_idx (numpy or device tensors)."""
        nnz = C.c_int64()
        ws = C.c_size_t()
        a_nnz = int(A.row_ptr[-1]) if a_nnz is None else a_nnz
        b_nnz = int(B.row_ptr[-1]) if b_nnz is None else b_nnz
        st = self.L.rvsp_cuda_symbolic(self.h, A.rows, A.cols, a_nnz, ptr(A.row_ptr),
                                       ptr(A.col_idx), B.rows, B.cols, b_nnz, ptr(B.row_ptr),
                                       ptr(B.col_idx), C.byref(nnz), C.byref(ws))
        self.rows = A.rows
        return st, nnz.value

    def numeric(self, A, B, c_rp, c_ci, c_v, fill=True):
        return self.L.rvsp_cuda_numeric(self.h, ptr(A.row_ptr), ptr(A.col_idx), ptr(A.values),
                                        ptr(B.row_ptr), ptr(B.col_idx), ptr(B.values), ptr(c_rp),
                                        ptr(c_ci), ptr(c_v), 1 if fill else 0, None)

    def set_params(self, params):
        """Bin parameters (BIN_PARAM_NAMES order) for the next symbolic call."""
        v = np.asarray(params, np.int32)
        return self.L.rvsp_cuda_plan_set_params(self.h, v.ctypes.data, v.size)

    def get_params(self):
        v = np.zeros(BIN_PARAMS, np.int32)
        check(self.L.rvsp_cuda_plan_get_params(self.h, v.ctypes.data, BIN_PARAMS), "get_params")
        return tuple(int(x) for x in v)

    def autotune(self, A, B, reps=2, max_trials=16):
        """Symbolic analysis after choosing the bin parameters for A * B.

        Returns (status, nnz(C), chosen parameters, [(parameters, ms), ...])."""
        best = np.zeros(BIN_PARAMS, np.int32)
        tp = np.zeros((max_trials, BIN_PARAMS), np.int32)
        tms = np.zeros(max_trials, np.float32)
        ntr = C.c_int32()
        nnz = C.c_int64()
        ws = C.c_size_t()
        st = self.L.rvsp_cuda_plan_autotune(
            self.h, A.rows, A.cols, int(A.row_ptr[-1]), ptr(A.row_ptr), ptr(A.col_idx),
            ptr(A.values), B.rows, B.cols, int(B.row_ptr[-1]), ptr(B.row_ptr), ptr(B.col_idx),
            ptr(B.values), reps, best.ctypes.data, tp.ctypes.data, tms.ctypes.data, max_trials,
            C.byref(ntr), C.byref(nnz), C.byref(ws))
        self.rows = A.rows
        n = min(ntr.value, max_trials)
        trials = [(tuple(int(x) for x in tp[i]), float(tms[i])) for i in range(n)]
        return st, nnz.value, tuple(int(x) for x in best), trials

    def row_stats(self):
        n = self.rows
        feat = np.zeros((max(n, 1), 4), np.float32)
        cnt = np.zeros(max(n, 1), np.int32)
        ub = np.zeros(max(n, 1), np.int32)
        check(self.L.rvsp_cuda_plan_row_stats(self.h, feat.ctypes.data, cnt.ctypes.data,
                                              ub.ctypes.data, n), "row_stats")
        return feat[:n], cnt[:n], ub[:n]

    def learned_stats(self):
        out = np.zeros(len(LEARNED_STATS), np.int64)
        check(self.L.rvsp_cuda_plan_learned_stats(self.h, out.ctypes.data, out.size),
              "learned_stats")
        return dict(zip(LEARNED_STATS, out.tolist()))


LEARNED_STATS = ("predicted_rows", "overflowed_rows", "exact_by_size_rows", "fit_nnz",
                 "fit_capacity", "exact_rows", "fit_upper_bound", "underpredicted_rows",
                 "pool_entries", "pool_capacity")


def oneshot_learned_stats():
    """Learned-path statistics of this thread's last learned one-shot product."""
    out = np.zeros(len(LEARNED_STATS), np.int64)
    check(lib().rvsp_cuda_oneshot_learned_stats(out.ctypes.data, out.size), "oneshot stats")
    return dict(zip(LEARNED_STATS, out.tolist()))


def set_default_params(params=None):
    """Process-wide bin parameters of new plans and of the one-shot and batched
    entry points; None restores the built-in default."""
    if params is None:
        return lib().rvsp_cuda_set_default_params(None, 0)
    v = np.asarray(params, np.int32)
    return lib().rvsp_cuda_set_default_params(v.ctypes.data, v.size)


def get_default_params():
    v = np.zeros(BIN_PARAMS, np.int32)
    check(lib().rvsp_cuda_get_default_params(v.ctypes.data, BIN_PARAMS), "get_default_params")
    return tuple(int(x) for x in v)


def model_to_vector(mean, inv_std, z, params):
    v = np.zeros(MLP_FLOATS, np.float32)
    v[0:4] = mean
    v[4:8] = inv_std
    v[8] = z
    v[9:] = params
    return v


def model_from_vector(v):
    v = np.asarray(v, np.float32)
    return v[0:4].copy(), v[4:8].copy(), float(v[8]), v[9:].copy()


def unpack_params(p):
    """Flat parameter vector -> dict of W1 (32,4) b1 W2 (32,32) b2 W3 (2,32) b3."""
    p = np.asarray(p)
    o = 0
    out = {}
    for name, shape in (("W1", (32, 4)), ("b1", (32,)), ("W2", (32, 32)), ("b2", (32,)),
                        ("W3", (2, 32)), ("b3", (2,))):
        size = int(np.prod(shape))
        out[name] = p[o:o + size].reshape(shape)
        o += size
    return out


def pack_params(d):
    return np.concatenate([np.asarray(d[k], np.float32).ravel()
                           for k in ("W1", "b1", "W2", "b2", "W3", "b3")])


def spgemm_batched(pairs_dev, algo=RVSP_CUDA_ALGO_EXACT):
    """Batched product of device operand pairs (objects with rows, cols, nnz,
    row_ptr, col_idx, values as device tensors). Returns the library-owned C
    device pointers (rp, ci, v), the total nnz, the row offsets and the entry
    offsets: product i's row pointer (from 0) starts at rp + row_offs[i] + i,
    its entries at ci / v + c_offs[i]. Release the pointers with
    free_device()."""
    L = lib()
    n = len(pairs_dev)
    i32 = lambda xs: np.ascontiguousarray(xs, np.int32)  # noqa: E731
    vp = lambda xs: (C.c_void_p * n)(*[ptr(x) for x in xs])  # noqa: E731
    a_rows = i32([a.rows for a, b in pairs_dev])
    a_cols = i32([a.cols for a, b in pairs_dev])
    b_cols = i32([b.cols for a, b in pairs_dev])
    a_nnz = i32([a.nnz for a, b in pairs_dev])
    b_nnz = i32([b.nnz for a, b in pairs_dev])
    arrs = [vp([a.row_ptr for a, b in pairs_dev]), vp([a.col_idx for a, b in pairs_dev]),
            vp([a.values for a, b in pairs_dev]), vp([b.row_ptr for a, b in pairs_dev]),
            vp([b.col_idx for a, b in pairs_dev]), vp([b.values for a, b in pairs_dev])]
    prp, pci, pv = C.c_void_p(), C.c_void_p(), C.c_void_p()
    nnz = C.c_int64()
    offs = np.zeros(n + 1, np.int64)
    c_offs = np.zeros(n + 1, np.int64)
    st = L.rvsp_cuda_spgemm_batched_f32(algo, n, a_rows.ctypes.data, a_cols.ctypes.data,
                                        b_cols.ctypes.data, a_nnz.ctypes.data, b_nnz.ctypes.data,
                                        *[C.cast(x, C.c_void_p) for x in arrs], C.byref(prp),
                                        C.byref(pci), C.byref(pv), C.byref(nnz), offs.ctypes.data,
                                        c_offs.ctypes.data)
    check(st, "rvsp_cuda_spgemm_batched_f32")
    return (prp.value, pci.value, pv.value), nnz.value, offs, c_offs


_libc = None


def _host_array(p, n, ctype, np_dtype):
    """Copy n elements of a library-malloc'd host array and free it."""
    global _libc
    if _libc is None:
        _libc = C.CDLL(None)
        _libc.free.argtypes = [C.c_void_p]
    out = (np.ctypeslib.as_array(C.cast(p, C.POINTER(ctype)), (n,)).copy()
           if n else np.zeros(0, np_dtype))
    _libc.free(p)
    return out


def mtx_read(path):
    """Matrix Market file -> (rows, cols, coo_row, coo_col, coo_val, symmetric),
    0-based COO, parsed by the library's C reader."""
    rows, cols, n, sym = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int()
    pr, pc, pv = C.c_void_p(), C.c_void_p(), C.c_void_p()
    check(lib().rvsp_cuda_mtx_read(str(path).encode(), C.byref(rows), C.byref(cols), C.byref(n),
                                   C.byref(pr), C.byref(pc), C.byref(pv), C.byref(sym)), "mtx_read")
    k = n.value
    return (rows.value, cols.value, _host_array(pr, k, C.c_int32, np.int32),
            _host_array(pc, k, C.c_int32, np.int32), _host_array(pv, k, C.c_float, np.float32),
            bool(sym.value))


def free_device(*ptrs):
    for p in ptrs:
        if p:
            lib().rvsp_cuda_free(p)
