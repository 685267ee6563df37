"""COO -> canonical CSR on the device (the reference Matrix Market loader's
canonicalisation) against the oracle, which test_oracle.py pins to the
reference's own loader: structure and values bit for bit."""

import ctypes as C

import numpy as np
import pytest

import oracle
import rvsp_b200 as rv
from conftest import mtx_cases
from gpu_util import d2h, dev
from rvsp_b200 import gen

pytestmark = pytest.mark.gpu


def _take(rows, prp, pci, pv, n, device_out):
    if device_out:
        rp = d2h(prp.value, rows + 1, np.int32)
        ci = d2h(pci.value, n, np.int32)
        v = d2h(pv.value, n, np.float32)
        rv.free_device(prp.value, pci.value, pv.value)
        return rp, ci, v
    return (rv._host_array(prp, rows + 1, C.c_int32, np.int32),
            rv._host_array(pci, n, C.c_int32, np.int32),
            rv._host_array(pv, n, C.c_float, np.float32))


def coo_to_csr(rows, cols, r, c, v, symmetric, device_in, device_out):
    arrs = [np.ascontiguousarray(r, np.int32), np.ascontiguousarray(c, np.int32),
            None if v is None else np.ascontiguousarray(v, np.float32)]
    keep = [None if a is None else (dev(a) if device_in else a) for a in arrs]
    ptrs = [None if a is None else rv.ptr(a) for a in keep]
    prp, pci, pv = C.c_void_p(), C.c_void_p(), C.c_void_p()
    nnz = C.c_int32()
    st = rv.lib().rvsp_cuda_coo_to_csr(rows, cols, len(arrs[0]), ptrs[0], ptrs[1], ptrs[2],
                                       1 if symmetric else 0, 1 if device_out else 0,
                                       C.byref(prp), C.byref(pci), C.byref(pv), C.byref(nnz))
    if st:
        return st, None
    return 0, _take(rows, prp, pci, pv, nnz.value, device_out)


def same(got, want, name):
    rp, ci, v = got
    wrp, wci, wv = want
    assert np.array_equal(np.asarray(rp, np.int64), np.asarray(wrp, np.int64)), name
    assert np.array_equal(ci, wci), name
    assert np.array_equal(v.view(np.uint32), np.asarray(wv, np.float32).view(np.uint32)), name


@pytest.mark.parametrize("device_out", [False, True])
def test_mtx_files(gpu_lib, tmp_path, device_out):
    for name, path in mtx_cases(str(tmp_path), seed=3):
        rows, cols, r, c, v, sym = rv.mtx_read(path)
        want = oracle.coo_to_csr(rows, cols, r, c, v, sym)
        R, Cc, N = C.c_int32(), C.c_int32(), C.c_int32()
        prp, pci, pv = C.c_void_p(), C.c_void_p(), C.c_void_p()
        rv.check(rv.lib().rvsp_cuda_mtx_to_csr(path.encode(), 1 if device_out else 0, C.byref(R),
                                               C.byref(Cc), C.byref(N), C.byref(prp), C.byref(pci),
                                               C.byref(pv)), name)
        assert (R.value, Cc.value) == (rows, cols)
        same(_take(rows, prp, pci, pv, N.value, device_out), want, name)


@pytest.mark.parametrize("device_in", [False, True])
def test_large_shuffled_coo(gpu_lib, device_in):
    """1.5 M entries over 300k x 2^21: several radix passes and many tiles;
    a third of the entries repeated, pattern and valued, plain and symmetric."""
    rng = np.random.default_rng(5)
    rows, cols, n = 300_000, 1 << 21, 1_000_000
    r = rng.integers(0, rows, n).astype(np.int32)
    c = rng.integers(0, cols, n).astype(np.int32)
    rep = rng.integers(0, n, n // 2)
    r = np.concatenate([r, r[rep]])
    c = np.concatenate([c, c[rep]])
    v = rng.uniform(-1, 1, r.size).astype(np.float32)
    for vals in (v, None):
        st, got = coo_to_csr(rows, cols, r, c, vals, False, device_in, True)
        assert st == 0
        same(got, oracle.coo_to_csr(rows, cols, r, c, vals, False), "large")
    m = 200_000
    rs, cs = rng.integers(0, m, 400_000).astype(np.int32), rng.integers(0, m, 400_000).astype(np.int32)
    vs = rng.uniform(-1, 1, rs.size).astype(np.float32)
    st, got = coo_to_csr(m, m, rs, cs, vs, True, device_in, False)
    assert st == 0
    same(got, oracle.coo_to_csr(m, m, rs, cs, vs, True), "large symmetric")


def test_csr_round_trip_and_errors(gpu_lib):
    M = gen.rmat(scale=12, edge_factor=8, seed=2)
    r = np.repeat(np.arange(M.rows, dtype=np.int32), np.diff(M.row_ptr))
    perm = np.random.default_rng(1).permutation(M.nnz)
    st, got = coo_to_csr(M.rows, M.cols, r[perm], M.col_idx[perm], M.values[perm], False, True, True)
    assert st == 0
    same(got, (M.row_ptr, M.col_idx, M.values), "round trip")
    # empty list, and indices out of range
    st, got = coo_to_csr(5, 7, np.zeros(0, np.int32), np.zeros(0, np.int32), None, False, False, False)
    assert st == 0 and list(got[0]) == [0] * 6 and got[1].size == 0
    st, _ = coo_to_csr(5, 7, np.array([1, 5], np.int32), np.array([0, 0], np.int32), None, False,
                       False, False)
    assert st == rv.RVSP_ERROR_INVALID_ARGUMENT
    st, _ = coo_to_csr(5, 7, np.array([1, 2], np.int32), np.array([0, -1], np.int32), None, False,
                       True, True)
    assert st == rv.RVSP_ERROR_INVALID_ARGUMENT
