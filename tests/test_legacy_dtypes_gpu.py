"""FP64 -> FP64 and INT8 -> INT32 products on the CUDA backend against the
oracle's restatement of the reference's legacy kernels (itself checked
against the compiled reference in test_oracle.py): same structure after the
zero sums are dropped, values bit for bit (FP64 in the reference's order,
INT32 exact)."""

import ctypes as C

import numpy as np
import pytest

import oracle
import rvsp_b200 as rv
from conftest import TypedMat, typed_pair
from gpu_util import d2h, dev
from rvsp_b200 import gen
from test_parity_gpu import _bin_sweep_matrix

pytestmark = pytest.mark.gpu

OUT = {"f64": (np.float64, C.c_double), "i8": (np.int32, C.c_int32)}


def cuda_typed(A, B, dtype, device=True):
    L = rv.lib()
    fn = L.rvsp_cuda_spgemm_f64 if dtype == "f64" else L.rvsp_cuda_spgemm_i8
    arrs = [A.row_ptr, A.col_idx, A.values, B.row_ptr, B.col_idx, B.values]
    if device:
        keep = [dev(a) for a in arrs]
        ptrs = [t.data_ptr() for t in keep]
    else:
        keep = [np.ascontiguousarray(a if a.size else np.zeros(1, a.dtype)) for a in arrs]
        ptrs = [a.ctypes.data for a in keep]
    prp, pci, pv = C.c_void_p(), C.c_void_p(), C.c_void_p()
    nnz = C.c_int32()
    st = fn(A.rows, A.cols, B.cols, *ptrs, C.byref(prp), C.byref(pci), C.byref(pv), C.byref(nnz))
    rv.check(st, f"rvsp_cuda_spgemm_{dtype}")
    n = nnz.value
    np_t, c_t = OUT[dtype]
    if device:
        rp = d2h(prp.value, A.rows + 1, np.int32)
        ci = d2h(pci.value, n, np.int32)
        v = d2h(pv.value, n, np_t)
        rv.free_device(prp.value, pci.value, pv.value)
    else:
        libc = C.CDLL(None)
        rp = np.ctypeslib.as_array(C.cast(prp, C.POINTER(C.c_int32)), (A.rows + 1,)).copy()
        ci = (np.ctypeslib.as_array(C.cast(pci, C.POINTER(C.c_int32)), (n,)).copy()
              if n else np.zeros(0, np.int32))
        v = (np.ctypeslib.as_array(C.cast(pv, C.POINTER(c_t)), (n,)).copy()
             if n else np.zeros(0, np_t))
        for p in (prp, pci, pv):
            libc.free(p)
    return rp, ci, v


def assert_typed_same(got, want, dtype, name):
    rp, ci, v = got
    wrp, wci, wv = want
    assert np.array_equal(np.asarray(rp, np.int64), np.asarray(wrp, np.int64)), f"{name}: row_ptr"
    assert np.array_equal(ci, wci), f"{name}: col_idx"
    if dtype == "f64":
        assert np.array_equal(v.view(np.uint64), np.asarray(wv, np.float64).view(np.uint64)), name
    else:
        assert np.array_equal(v, wv), name


def _cases():
    S, T = _bin_sweep_matrix(11)  # tiny, every warp table and chunked rows
    return [("rmat_s11", *(gen.rmat(scale=11, edge_factor=8, seed=3),) * 2),
            ("uniform", *(gen.uniform_fixed(700, 700, 11, seed=5),) * 2),
            ("bin_sweep", S, T)]


@pytest.mark.parametrize("dtype", ["f64", "i8"])
@pytest.mark.parametrize("device", [True, False])
def test_legacy_dtype_products(gpu_lib, dtype, device):
    for name, M1, M2 in _cases():
        A, B = typed_pair(M1, M2, dtype, seed=9)
        want = oracle.spgemm_typed(A, B, dtype)
        got = cuda_typed(A, B, dtype, device)
        _, cnt = oracle.symbolic(A, B)
        assert int(want[0][-1]) < int(cnt.sum()), name  # the case has cancelled entries
        assert_typed_same(got, want, dtype, f"{name}/{dtype}/{'dev' if device else 'host'}")


@pytest.mark.parametrize("dtype", ["f64", "i8"])
def test_legacy_dtype_public_api(gpu_lib, dtype):
    M = gen.rmat(scale=9, edge_factor=8, seed=1)
    A, B = typed_pair(M, M, dtype, seed=4)
    want = oracle.spgemm_typed(A, B, dtype)
    dt_in = rv.RVSP_DTYPE_FP64 if dtype == "f64" else rv.RVSP_DTYPE_INT8
    dt_out = rv.RVSP_DTYPE_FP64 if dtype == "f64" else rv.RVSP_DTYPE_INT32
    a = rv.csr_struct(A.rows, A.cols, A.nnz, A.row_ptr, A.col_idx, A.values, dtype=dt_in)
    b = rv.csr_struct(B.rows, B.cols, B.nnz, B.row_ptr, B.col_idx, B.values, dtype=dt_in)
    c = rv.CsrMatrix()
    L = rv.lib()
    opts = rv.SpgemmOptions(rv.RVSP_BACKEND_CUDA, dt_in, dt_out)
    rv.check(L.rvsp_spgemm_csr(C.byref(a), C.byref(b), C.byref(c), C.byref(opts)), "spgemm_csr")
    assert c.dtype == dt_out and c.nnz == want[1].size
    np_t, c_t = OUT[dtype]
    rp = np.ctypeslib.as_array(C.cast(c.row_ptr, C.POINTER(C.c_int32)), (A.rows + 1,)).copy()
    ci = np.ctypeslib.as_array(C.cast(c.col_idx, C.POINTER(C.c_int32)), (c.nnz,)).copy()
    v = np.ctypeslib.as_array(C.cast(c.values, C.POINTER(c_t)), (c.nnz,)).copy()
    L.rvsp_csr_destroy(C.byref(c))
    assert_typed_same((rp, ci, v), want, dtype, f"public/{dtype}")
    # the legacy wrappers' codes for a dtype mismatch
    fa = rv.csr_struct(A.rows, A.cols, A.nnz, A.row_ptr, A.col_idx,
                       A.values.astype(np.float32), dtype=rv.RVSP_DTYPE_FP32)
    c2 = rv.CsrMatrix()
    st = L.rvsp_spgemm_csr(C.byref(fa), C.byref(b), C.byref(c2), C.byref(opts))
    assert st == (rv.RVSP_ERROR_INVALID_ARGUMENT if dtype == "f64"
                  else rv.RVSP_ERROR_UNSUPPORTED_DTYPE)


def test_legacy_dtype_empty_and_all_cancelling(gpu_lib):
    # an all-empty A; and a product whose every sum cancels (a row [1, -1] times
    # two identical B rows)
    A = TypedMat(2, 3, [0, 0, 0], [], np.zeros(0, np.float64))
    B = TypedMat(3, 4, [0, 1, 1, 2], [0, 3], np.array([1.0, 2.0]))
    assert_typed_same(cuda_typed(A, B, "f64"), oracle.spgemm_typed(A, B, "f64"), "f64", "empty")
    A = TypedMat(1, 2, [0, 2], [0, 1], np.array([1, -1], np.int8))
    B = TypedMat(2, 3, [0, 2, 4], [0, 2, 0, 2], np.array([5, 7, 5, 7], np.int8))
    rp, ci, v = cuda_typed(A, B, "i8")
    assert list(rp) == [0, 0] and ci.size == 0 and v.size == 0
