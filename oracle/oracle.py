"""CPU oracle for FP32 CSR SpGEMM -- test and baseline infrastructure only.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's cpu_baseline /
reference legs may import this module, and only as the checker or the timed
CPU baseline. The CUDA library never links or calls anything here.

Two checkers are exposed:

* ``liboracle`` -- this repository's C restatement of the reference's scalar
  Gustavson path (``oracle/rvsp_oracle.c``; each function cites the reference
  file:line it follows), built by ``oracle/Makefile``.
* ``libref`` -- the reference's own scalar FP32 path compiled from its
  sources (rv-sparse ``src/kernels/spgemm/accum_scalar_f32.c``,
  ``rvsp_symbolic.c``, ``rvsp_support.c``, ``src/core/spgemm_descr.c``) plus
  ``oracle/ref_driver.c``; present when the build ran next to a reference
  checkout, and shipped prebuilt otherwise.

The restatement is pinned against the reference's golden fixtures
(rv-sparse ``tests/csr_fixtures.h:42-153``, committed as
``tests/golden/csr_fixtures.json``) and against ``libref`` outputs on seeded
inputs (``tests/golden/ref_outputs.json``).

The reference's legacy FP64 and INT8 -> INT32 one-shot kernels are restated
too (``spgemm_typed``) and, in ``libref``, compiled from their sources
(rv-sparse ``src/kernels/spgemm/legacy/csr_scalar_f64.c``, ``csr_scalar_i8.c``;
``ref_spgemm_typed``).

An FP64 MLP forward/backward (``mlp_forward_backward_f64``) is the gradient
oracle for the learned row-size predictor; it has no reference counterpart.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "librvsp_ref.so")

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")

_lib = None
_ref = None


def build(ref_dir: str | None = None) -> None:
    """Compile the restatement; with a reference checkout (ref_dir, or
    $RVSP_REFERENCE_DIR) also the reference library and the reference's own
    C tests and examples (against both libraries)."""
    targets = ["oracle"]
    ref_dir = ref_dir or os.environ.get("RVSP_REFERENCE_DIR", "")
    if ref_dir and os.path.isdir(os.path.join(ref_dir, "src", "kernels", "spgemm")):
        targets += ["ref", "reftests"]
    subprocess.run(["make", "-s", "-C", HERE, f"REF={ref_dir}"] + targets, check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.oracle_csr_check.restype = C.c_int
        L.oracle_csr_check.argtypes = [C.c_int32, C.c_int32, _i32p, _i32p, C.POINTER(C.c_int32)]
        L.oracle_symbolic.restype = C.c_int64
        L.oracle_symbolic.argtypes = [C.c_int32, C.c_int32, C.c_int32, _i32p, _i32p, _i32p, _i32p,
                                      _i64p, _i64p]
        L.oracle_spgemm_f32.restype = C.c_int
        L.oracle_spgemm_f32.argtypes = [C.c_int32, C.c_int32, C.c_int32,
                                        _i32p, _i32p, _f32p, _i32p, _i32p, _f32p,
                                        _i64p, _i32p, _f32p]
        L.oracle_numeric_f64.restype = C.c_int
        L.oracle_numeric_f64.argtypes = [C.c_int32, C.c_int32, C.c_int32,
                                         _i32p, _i32p, _f32p, _i32p, _i32p, _f32p,
                                         _i64p, _i32p, _f64p]
        _i8p = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")
        L.oracle_spgemm_f64.restype = C.c_int
        L.oracle_spgemm_f64.argtypes = [C.c_int32, C.c_int32, C.c_int32,
                                        _i32p, _i32p, _f64p, _i32p, _i32p, _f64p,
                                        _i64p, _i32p, _f64p]
        L.oracle_spgemm_i8.restype = C.c_int
        L.oracle_spgemm_i8.argtypes = [C.c_int32, C.c_int32, C.c_int32,
                                       _i32p, _i32p, _i8p, _i32p, _i32p, _i8p,
                                       _i64p, _i32p, _i32p]
        L.oracle_coo_to_csr.restype = C.c_int64
        L.oracle_coo_to_csr.argtypes = [C.c_int32, C.c_int32, C.c_int64, _i32p, _i32p, C.c_void_p,
                                        C.c_int, _i64p, _i32p, _f32p]
        L.oracle_numeric_f32.restype = C.c_int
        L.oracle_numeric_f32.argtypes = [C.c_int32, C.c_int32, C.c_int32,
                                         _i32p, _i32p, _f32p, _i32p, _i32p, _f32p,
                                         _i64p, _i32p, _f32p]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(f"{REF_SO} missing: build it next to a reference checkout")
        L = C.CDLL(REF_SO)
        L.ref_spgemm_raw.restype = C.c_int
        L.ref_spgemm_raw.argtypes = [C.c_int32, C.c_int32, C.c_int32,
                                     _i32p, _i32p, _f32p, _i32p, _i32p, _f32p,
                                     C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                     C.POINTER(C.c_void_p), C.POINTER(C.c_int32), _i64p]
        L.ref_free.argtypes = [C.c_void_p]
        L.ref_time_oneshot.restype = C.c_double
        L.ref_time_oneshot.argtypes = [C.c_int, C.c_int, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                       _i32p, _i32p, _f32p, _i32p, _i32p, _f32p]
        L.ref_time_numeric.restype = C.c_double
        L.ref_time_numeric.argtypes = [C.c_int, C.c_int, C.c_int32, C.c_int32, C.c_int32,
                                       _i32p, _i32p, _f32p, _i32p, _i32p, _f32p,
                                       _i32p, _i32p, _f32p]
        for nm in ("rvsp_spgemm_csr_scalar_f64_raw", "rvsp_spgemm_csr_scalar_i8_raw"):
            fn = getattr(L, nm)
            fn.restype = C.c_int
            fn.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                           C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p),
                           C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_int32)]
        L.ref_mtx_load.restype = C.c_int
        L.ref_mtx_load.argtypes = [C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                   C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                   C.POINTER(C.c_void_p)]
        L.rvsp_csr_check.restype = C.c_int
        L.rvsp_csr_check.argtypes = [C.c_int32, C.c_int32, _i32p, _i32p, C.POINTER(C.c_int32)]
        _ref = L
    return _ref


def _arrs(M):
    return (np.ascontiguousarray(M.row_ptr, np.int32), np.ascontiguousarray(M.col_idx, np.int32),
            np.ascontiguousarray(M.values, np.float32))


def csr_check(rows, cols, row_ptr, col_idx):
    """Canonical-CSR status (0 ok, 1 bad row_ptr, 2 range, 3 unsorted, 4 dup), bad row."""
    bad = C.c_int32(-1)
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col_idx, np.int32)
    if ci.size == 0:
        ci = np.zeros(1, np.int32)
    st = lib().oracle_csr_check(rows, cols, rp, ci, C.byref(bad))
    return st, bad.value


def symbolic(A, B, row_begin=0, row_end=None):
    """(ops per row int64, distinct output columns per row int64) for rows [row_begin, row_end)."""
    row_end = A.rows if row_end is None else row_end
    a_rp, a_ci, _ = _arrs(A)
    b_rp, b_ci, _ = _arrs(B)
    n = row_end - row_begin
    ops = np.zeros(max(n, 1), np.int64)
    cnt = np.zeros(max(n, 1), np.int64)
    lib().oracle_symbolic(row_begin, row_end, B.cols, a_rp, _nz(a_ci), b_rp, _nz(b_ci), ops, cnt)
    return ops[:n], cnt[:n]


def _nz(a):
    return a if a.size else np.zeros(1, a.dtype)


def spgemm_f32(A, B, row_begin=0, row_end=None):
    """Reference-order FP32 product of rows [row_begin, row_end).

    Returns (row_ptr int64 relative to row_begin, col_idx int32, values float32).
    """
    row_end = A.rows if row_end is None else row_end
    a_rp, a_ci, a_v = _arrs(A)
    b_rp, b_ci, b_v = _arrs(B)
    _, cnt = symbolic(A, B, row_begin, row_end)
    total = int(cnt.sum())
    rp = np.zeros(row_end - row_begin + 1, np.int64)
    ci = np.zeros(max(total, 1), np.int32)
    v = np.zeros(max(total, 1), np.float32)
    st = lib().oracle_spgemm_f32(row_begin, row_end, B.cols, a_rp, _nz(a_ci), _nz(a_v),
                                 b_rp, _nz(b_ci), _nz(b_v), rp, ci, v)
    if st != 0:
        raise MemoryError("oracle_spgemm_f32 failed")
    return rp, ci[:total], v[:total]


def numeric_f64(A, B, c_rp, c_ci, row_begin=0, row_end=None):
    """FP64 values over a given pattern (c_rp relative to row_begin)."""
    row_end = A.rows if row_end is None else row_end
    a_rp, a_ci, a_v = _arrs(A)
    b_rp, b_ci, b_v = _arrs(B)
    c_rp = np.ascontiguousarray(c_rp, np.int64)
    c_ci = np.ascontiguousarray(c_ci, np.int32)
    out = np.zeros(max(int(c_rp[-1] - c_rp[0]) if c_rp.size else 0, 1), np.float64)
    lib().oracle_numeric_f64(row_begin, row_end, B.cols, a_rp, _nz(a_ci), _nz(a_v),
                             b_rp, _nz(b_ci), _nz(b_v), c_rp, _nz(c_ci), out)
    return out[: int(c_rp[-1])]


def numeric_f32(A, B, c_rp, c_ci, row_begin=0, row_end=None):
    """Reference-order FP32 values over a given pattern (descriptor reuse)."""
    row_end = A.rows if row_end is None else row_end
    a_rp, a_ci, a_v = _arrs(A)
    b_rp, b_ci, b_v = _arrs(B)
    c_rp = np.ascontiguousarray(c_rp, np.int64)
    c_ci = np.ascontiguousarray(c_ci, np.int32)
    out = np.zeros(max(int(c_rp[-1]), 1), np.float32)
    lib().oracle_numeric_f32(row_begin, row_end, B.cols, a_rp, _nz(a_ci), _nz(a_v),
                             b_rp, _nz(b_ci), _nz(b_v), c_rp, _nz(c_ci), out)
    return out[: int(c_rp[-1])]


def ref_spgemm(A, B):
    """Run the reference's raw scalar kernel; returns (row_ptr, col_idx, values, ops, status)."""
    L = ref()
    a_rp, a_ci, a_v = _arrs(A)
    b_rp, b_ci, b_v = _arrs(B)
    p_rp, p_ci, p_v = C.c_void_p(), C.c_void_p(), C.c_void_p()
    nnz = C.c_int32(0)
    ops = np.zeros(max(A.rows, 1), np.int64)
    st = L.ref_spgemm_raw(A.rows, A.cols, B.cols, a_rp, _nz(a_ci), _nz(a_v), b_rp, _nz(b_ci),
                          _nz(b_v), C.byref(p_rp), C.byref(p_ci), C.byref(p_v), C.byref(nnz), ops)
    if st != 0:
        return None, None, None, ops[: A.rows], st
    n = nnz.value
    rp = np.ctypeslib.as_array(C.cast(p_rp, C.POINTER(C.c_int32)), (A.rows + 1,)).copy()
    ci = (np.ctypeslib.as_array(C.cast(p_ci, C.POINTER(C.c_int32)), (n,)).copy()
          if n else np.zeros(0, np.int32))
    v = (np.ctypeslib.as_array(C.cast(p_v, C.POINTER(C.c_float)), (n,)).copy()
         if n else np.zeros(0, np.float32))
    for p in (p_rp, p_ci, p_v):
        L.ref_free(p)
    return rp, ci, v, ops[: A.rows], 0


def ref_time_oneshot(A, B, nthreads=1, repeats=1, row_begin=0, row_end=None):
    row_end = A.rows if row_end is None else row_end
    a_rp, a_ci, a_v = _arrs(A)
    b_rp, b_ci, b_v = _arrs(B)
    return ref().ref_time_oneshot(nthreads, repeats, row_begin, row_end, A.cols, B.cols,
                                  a_rp, _nz(a_ci), _nz(a_v), b_rp, _nz(b_ci), _nz(b_v))


def ref_time_numeric(A, B, c_rp, c_ci, c_v, nthreads=1, repeats=1, row_begin=0, row_end=None):
    row_end = A.rows if row_end is None else row_end
    a_rp, a_ci, a_v = _arrs(A)
    b_rp, b_ci, b_v = _arrs(B)
    return ref().ref_time_numeric(nthreads, repeats, row_begin, row_end, B.cols,
                                  a_rp, _nz(a_ci), _nz(a_v), b_rp, _nz(b_ci), _nz(b_v),
                                  np.ascontiguousarray(c_rp, np.int32), _nz(c_ci), c_v)


# ---------------------------------------------------------------------------
# FP64 MLP oracle for the learned row-size predictor (no reference counterpart)
# ---------------------------------------------------------------------------

def mlp_forward_backward_f64(params, X, y, w_loss):
    """Forward + backward of the 4-32-32-2 ReLU MLP in float64.

    params: dict W1 (32,4) b1 (32) W2 (32,32) b2 (32) W3 (2,32) b3 (2).
    Output o = [mu, s]; loss per row = w * (0.5 * ((y - mu) / sigma)^2 + log sigma),
    sigma = softplus(s) + 1e-3 (a Gaussian negative log-likelihood on log2(nnz+1)).
    Returns (mean loss, grads dict).
    """
    P = {k: np.asarray(v, np.float64) for k, v in params.items()}
    X = np.asarray(X, np.float64)
    y = np.asarray(y, np.float64)
    w = np.asarray(w_loss, np.float64)
    n = X.shape[0]
    z1 = X @ P["W1"].T + P["b1"]
    h1 = np.maximum(z1, 0)
    z2 = h1 @ P["W2"].T + P["b2"]
    h2 = np.maximum(z2, 0)
    o = h2 @ P["W3"].T + P["b3"]
    mu, s = o[:, 0], o[:, 1]
    sp = np.logaddexp(0, s)
    sig = sp + 1e-3
    r = (y - mu) / sig
    loss = w * (0.5 * r * r + np.log(sig))
    L = loss.sum() / n
    dmu = w * (-r / sig) / n
    dsig = w * (-r * r / sig + 1.0 / sig) / n
    ds = dsig * (1.0 / (1.0 + np.exp(-s)))
    do = np.stack([dmu, ds], 1)
    g = {}
    g["W3"] = do.T @ h2
    g["b3"] = do.sum(0)
    dh2 = do @ P["W3"]
    dz2 = dh2 * (z2 > 0)
    g["W2"] = dz2.T @ h1
    g["b2"] = dz2.sum(0)
    dh1 = dz2 @ P["W2"]
    dz1 = dh1 * (z1 > 0)
    g["W1"] = dz1.T @ X
    g["b1"] = dz1.sum(0)
    return L, g


_TYPED = {"f64": (np.float64, np.float64), "i8": (np.int8, np.int32)}


def spgemm_typed(A, B, dtype, row_begin=0, row_end=None):
    """Legacy-dtype product (dtype "f64": FP64 -> FP64, "i8": INT8 -> INT32) of rows
    [row_begin, row_end): (row_ptr int64 relative, col_idx, values), zero sums dropped."""
    in_t, out_t = _TYPED[dtype]
    row_end = A.rows if row_end is None else row_end
    a_rp = np.ascontiguousarray(A.row_ptr, np.int32)
    a_ci = np.ascontiguousarray(A.col_idx, np.int32)
    b_rp = np.ascontiguousarray(B.row_ptr, np.int32)
    b_ci = np.ascontiguousarray(B.col_idx, np.int32)
    a_v = np.ascontiguousarray(A.values, in_t)
    b_v = np.ascontiguousarray(B.values, in_t)
    _, cnt = symbolic(A, B, row_begin, row_end)
    total = int(cnt.sum())
    rp = np.zeros(row_end - row_begin + 1, np.int64)
    ci = np.zeros(max(total, 1), np.int32)
    v = np.zeros(max(total, 1), out_t)
    fn = lib().oracle_spgemm_f64 if dtype == "f64" else lib().oracle_spgemm_i8
    if fn(row_begin, row_end, B.cols, a_rp, _nz(a_ci), _nz(a_v), b_rp, _nz(b_ci), _nz(b_v),
          rp, ci, v) != 0:
        raise MemoryError("oracle legacy-dtype product failed")
    n = int(rp[-1])
    return rp, ci[:n], v[:n]


def ref_spgemm_typed(A, B, dtype):
    """The reference's own legacy raw kernel (csr_scalar_f64.c / csr_scalar_i8.c);
    returns (row_ptr, col_idx, values, status)."""
    in_t, out_t = _TYPED[dtype]
    L = ref()
    fn = L.rvsp_spgemm_csr_scalar_f64_raw if dtype == "f64" else L.rvsp_spgemm_csr_scalar_i8_raw
    arrs = [np.ascontiguousarray(A.row_ptr, np.int32), _nz(np.ascontiguousarray(A.col_idx, np.int32)),
            _nz(np.ascontiguousarray(A.values, in_t)), np.ascontiguousarray(B.row_ptr, np.int32),
            _nz(np.ascontiguousarray(B.col_idx, np.int32)), _nz(np.ascontiguousarray(B.values, in_t))]
    p_rp, p_ci, p_v = C.c_void_p(), C.c_void_p(), C.c_void_p()
    nnz = C.c_int32(0)
    st = fn(A.rows, A.cols, B.cols, *[a.ctypes.data for a in arrs], C.byref(p_rp), C.byref(p_ci),
            C.byref(p_v), C.byref(nnz))
    if st != 0:
        return None, None, None, st
    n = nnz.value
    ctype = C.c_double if dtype == "f64" else C.c_int32
    rp = np.ctypeslib.as_array(C.cast(p_rp, C.POINTER(C.c_int32)), (A.rows + 1,)).copy()
    ci = (np.ctypeslib.as_array(C.cast(p_ci, C.POINTER(C.c_int32)), (n,)).copy()
          if n else np.zeros(0, np.int32))
    v = (np.ctypeslib.as_array(C.cast(p_v, C.POINTER(ctype)), (n,)).copy()
         if n else np.zeros(0, out_t))
    for p in (p_rp, p_ci, p_v):
        L.ref_free(p)
    return rp, ci, v, 0


def coo_to_csr(rows, cols, coo_row, coo_col, coo_val=None, symmetric=False):
    """Canonical CSR of a COO list the way the reference's Matrix Market loader
    builds it (mirrors appended, stable (row, col) order, runs summed from their
    first value); returns (row_ptr int64, col_idx, values)."""
    r = np.ascontiguousarray(coo_row, np.int32)
    c = np.ascontiguousarray(coo_col, np.int32)
    n = r.size
    cap = max(2 * n, 1)
    rp = np.zeros(rows + 1, np.int64)
    ci = np.zeros(cap, np.int32)
    v = np.zeros(cap, np.float32)
    vv = None if coo_val is None else np.ascontiguousarray(coo_val, np.float32)
    m = lib().oracle_coo_to_csr(rows, cols, n, _nz(r), _nz(c),
                                None if vv is None else _nz(vv).ctypes.data, 1 if symmetric else 0,
                                rp, ci, v)
    if m < 0:
        raise ValueError(f"oracle_coo_to_csr failed: {m}")
    return rp, ci[:m], v[:m]


def ref_mtx_load(path):
    """The reference's own loader (assemble_csr_matrix) on a file: (row_ptr, col_idx, values)."""
    L = ref()
    rows, nnz = C.c_int32(), C.c_int32()
    prp, pci, pv = C.c_void_p(), C.c_void_p(), C.c_void_p()
    if L.ref_mtx_load(path.encode(), C.byref(rows), C.byref(nnz), C.byref(prp), C.byref(pci),
                      C.byref(pv)) != 0:
        raise RuntimeError("reference loader failed")
    n = nnz.value
    rp = np.ctypeslib.as_array(C.cast(prp, C.POINTER(C.c_int32)), (rows.value + 1,)).copy()
    ci = (np.ctypeslib.as_array(C.cast(pci, C.POINTER(C.c_int32)), (n,)).copy()
          if n else np.zeros(0, np.int32))
    v = (np.ctypeslib.as_array(C.cast(pv, C.POINTER(C.c_float)), (n,)).copy()
         if n else np.zeros(0, np.float32))
    for p in (prp, pci, pv):
        L.ref_free(p)
    return rp, ci, v
