"""The C library without a GPU: it loads, exports every declared symbol, and
its host-side argument checks follow the reference's contract
(rv-sparse tests/test_spgemm_descr_f32.c, src/core/matrix.c)."""

import ctypes as C
import os
import re

import numpy as np
import pytest

import rvsp_b200 as rv
from conftest import ROOT, have_gpu


def declared_functions():
    names = set()
    for h in ("rv_sparse.h", "rvsp_cuda.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:RVSP_CUDA_API\s+)?[A-Za-z_][\w\s\*]*?\b(rvsp_\w+)\s*\(", text,
                             flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = rv.lib()
    names = declared_functions()
    assert len(names) >= 25, names
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    assert set(declared_functions()) <= set(rv._PROTOS), set(declared_functions()) - set(rv._PROTOS)


def test_status_strings_and_version():
    assert rv.status_string(0) == "success"
    assert rv.status_string(rv.RVSP_ERROR_INVALID_CSR) == "invalid CSR matrix"
    assert rv.status_string(rv.RVSP_ERROR_DEVICE_FAILURE) == "device failure"
    assert rv.status_string(-99) == "unknown error"
    assert rv.lib().rvsp_get_version() == b"0.1.0"


def _host_matrix(rp, ci, rows, cols):
    rp = np.array(rp, np.int32)
    ci = np.array(ci, np.int32)
    v = np.ones(max(len(ci), 1), np.float32)
    return rp, ci, v, rv.csr_struct(rows, cols, int(rp[-1]), rp, ci, v)


def test_csr_create_and_validate_host():
    L = rv.lib()
    rp, ci, v, M = _host_matrix([0, 2, 3], [0, 1, 1], 2, 2)
    out = rv.CsrMatrix()
    assert L.rvsp_csr_create(C.byref(out), 2, 2, 3, rv.ptr(rp), rv.ptr(ci), rv.ptr(v),
                             rv.RVSP_DTYPE_FP32) == 0
    assert out.owns_data == 0 and out.nnz == 3
    assert L.rvsp_csr_create(None, 2, 2, 3, rv.ptr(rp), rv.ptr(ci), rv.ptr(v), 3) == -1
    assert L.rvsp_csr_create(C.byref(out), 0, 2, 3, rv.ptr(rp), rv.ptr(ci), rv.ptr(v), 3) == -2
    bad = np.array([1, 2, 3], np.int32)
    assert L.rvsp_csr_create(C.byref(out), 2, 2, 3, rv.ptr(bad), rv.ptr(ci), rv.ptr(v), 3) == -3
    rng = np.array([0, 2, 3], np.int32)
    oob = np.array([0, 2, 1], np.int32)
    assert L.rvsp_csr_create(C.byref(out), 2, 2, 3, rv.ptr(rng), rv.ptr(oob), rv.ptr(v), 3) == -3
    # validate does not check sortedness (rv-sparse docs/api_design.md:88-94)
    uns = np.array([1, 0, 1], np.int32)
    assert L.rvsp_csr_create(C.byref(out), 2, 2, 3, rv.ptr(rng), rv.ptr(uns), rv.ptr(v), 3) == 0
    wrong_nnz = np.array([0, 2, 2], np.int32)
    assert L.rvsp_csr_create(C.byref(out), 2, 2, 3, rv.ptr(wrong_nnz), rv.ptr(ci), rv.ptr(v), 3) == -3
    L.rvsp_csr_destroy(C.byref(out))
    assert out.rows == 0 and out.row_ptr is None
    L.rvsp_csr_destroy(None)


def test_descriptor_contract_host_side():
    """Ordering and NULL rules that never reach the device."""
    L = rv.lib()
    assert L.rvsp_spgemm_descr_create(None) == rv.RVSP_ERROR_NULL_POINTER
    h = C.c_void_p()
    assert L.rvsp_spgemm_descr_create(C.byref(h)) == 0 and h
    assert L.rvsp_spgemm_set_algo(None, rv.RVSP_SPGEMM_ALGO_CUDA) == rv.RVSP_ERROR_NULL_POINTER
    # vector strategies are not provided by this build, as the reference
    # refuses them on a build without the vector extension
    for algo in (rv.RVSP_SPGEMM_ALGO_RVV, rv.RVSP_SPGEMM_ALGO_CONTIG,
                 rv.RVSP_SPGEMM_ALGO_ADAPTIVE, 99):
        assert L.rvsp_spgemm_set_algo(h, algo) == rv.RVSP_ERROR_UNSUPPORTED_BACKEND
    # the default strategy (the reference's scalar kernel) is the CUDA exact path
    expect = 0 if have_gpu() else rv.RVSP_ERROR_UNSUPPORTED_BACKEND
    assert L.rvsp_spgemm_set_algo(h, rv.RVSP_SPGEMM_ALGO_DEFAULT) == expect
    assert L.rvsp_spgemm_set_algo(h, rv.RVSP_SPGEMM_ALGO_CUDA) == expect
    rp, ci, v, A = _host_matrix([0, 2, 3], [0, 1, 1], 2, 2)
    crp, cci, cv, Cm = _host_matrix([0, 0, 0], [], 2, 2)
    ws = np.zeros(64, np.uint8)
    assert L.rvsp_spgemm_compute(h, C.byref(A), C.byref(A), C.byref(Cm), rv.ptr(ws)) == -2
    ops = np.zeros(2, np.int64)
    assert L.rvsp_spgemm_get_op_counts(h, rv.ptr(ops), 2) == -2
    assert L.rvsp_spgemm_get_op_counts(h, None, 2) == -1
    size = C.c_size_t()
    nnz = C.c_int32()
    assert L.rvsp_spgemm_work_estimation(h, None, C.byref(A), C.byref(size), C.byref(nnz)) == -1
    assert L.rvsp_spgemm_work_estimation(None, C.byref(A), C.byref(A), C.byref(size),
                                         C.byref(nnz)) == -1
    fp64 = rv.csr_struct(2, 2, 3, rp, ci, v, rv.RVSP_DTYPE_FP64)
    assert L.rvsp_spgemm_work_estimation(h, C.byref(fp64), C.byref(A), C.byref(size),
                                         C.byref(nnz)) == rv.RVSP_ERROR_UNSUPPORTED_DTYPE
    mism = rv.csr_struct(2, 3, 3, rp, ci, v)
    assert L.rvsp_spgemm_work_estimation(h, C.byref(mism), C.byref(A), C.byref(size),
                                         C.byref(nnz)) == rv.RVSP_ERROR_INVALID_ARGUMENT
    L.rvsp_spgemm_invalidate_structure(None)
    L.rvsp_spgemm_descr_destroy(None)
    L.rvsp_spgemm_descr_destroy(h)


def test_oneshot_backend_selection_host_side():
    L = rv.lib()
    rp, ci, v, A = _host_matrix([0, 2, 3], [0, 1, 1], 2, 2)
    out = rv.CsrMatrix()
    opts = rv.SpgemmOptions(rv.RVSP_BACKEND_RVV_INTRINSICS, rv.RVSP_DTYPE_FP32, rv.RVSP_DTYPE_FP32)
    assert L.rvsp_spgemm_csr(C.byref(A), C.byref(A), C.byref(out), C.byref(opts)) == -5
    # the unrolled scalar alias has no legacy dtypes in the reference either
    opts = rv.SpgemmOptions(rv.RVSP_BACKEND_SCALAR_UNROLL4, rv.RVSP_DTYPE_FP64, rv.RVSP_DTYPE_FP64)
    assert L.rvsp_spgemm_csr(C.byref(A), C.byref(A), C.byref(out), C.byref(opts)) == -5
    if not have_gpu():
        # the scalar backends run on the GPU, so without one they are refused
        for be in (rv.RVSP_BACKEND_SCALAR, rv.RVSP_BACKEND_SCALAR_UNROLL4):
            opts = rv.SpgemmOptions(be, rv.RVSP_DTYPE_FP32, rv.RVSP_DTYPE_FP32)
            assert L.rvsp_spgemm_csr(C.byref(A), C.byref(A), C.byref(out), C.byref(opts)) == -5
    assert L.rvsp_spgemm_csr(None, C.byref(A), C.byref(out), None) == -1
    if not have_gpu():
        assert L.rvsp_spgemm_csr(C.byref(A), C.byref(A), C.byref(out), None) == -5
        assert rv.device_count() == 0


def test_plan_requires_device_or_valid_algo():
    L = rv.lib()
    p = C.c_void_p()
    assert L.rvsp_cuda_plan_create(None, rv.RVSP_CUDA_ALGO_EXACT) == -1
    assert L.rvsp_cuda_plan_create(C.byref(p), 7) == rv.RVSP_ERROR_UNSUPPORTED_BACKEND
    if not have_gpu():
        assert L.rvsp_cuda_plan_create(C.byref(p), rv.RVSP_CUDA_ALGO_EXACT) == -5
    L.rvsp_cuda_plan_destroy(None)
    assert L.rvsp_cuda_is_device_pointer(rv.ptr(np.zeros(4, np.int32))) == 0


def test_host_free_takes_any_malloc_block():
    """rvsp_cuda_host_free releases host result arrays: any block malloc (or
    the library) returned, NULL included. Blocks of 64 MiB and more are kept
    for reuse, at most four at a time (the oldest are freed): a run of large
    releases passes through the keeping and the eviction."""
    L = rv.lib()
    libc = C.CDLL(None)
    libc.malloc.restype = C.c_void_p
    libc.malloc.argtypes = [C.c_size_t]
    L.rvsp_cuda_host_free(None)
    for mib in (1, 80, 80, 100, 70, 90, 200, 65, 2):
        p = libc.malloc(mib << 20)
        assert p
        C.memset(p, 0xA5, mib << 20)
        L.rvsp_cuda_host_free(p)
