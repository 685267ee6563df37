"""CUDA backend parity: bit-exact structure and values against the oracle and
the reference scalar kernel's golden outputs.

Values are compared bit for bit: the kernels add the FP32 products in the
reference's order (rv-sparse accum_scalar_f32.c:69, k-order from +0.0f, no
FMA), so there is no tolerance to state for the exact path.
"""

import ctypes as C
import hashlib

import numpy as np
import pytest

import oracle
import rvsp_b200 as rv
from conftest import Mat, ref_digests
from gpu_util import DevCSR, bits, d2h, dev, oneshot
from rvsp_b200 import gen

pytestmark = pytest.mark.gpu


def assert_same(got, want, name=""):
    rp, ci, v = got
    wrp, wci, wv = want
    assert np.array_equal(np.asarray(rp, np.int64), np.asarray(wrp, np.int64)), f"{name}: row_ptr"
    assert np.array_equal(ci, wci), f"{name}: col_idx"
    assert np.array_equal(bits(v), bits(wv)), f"{name}: values"


def oracle_full(A, B):
    rp, ci, v = oracle.spgemm_f32(A, B)
    return rp, ci, v


def test_fixtures_oneshot_device_and_host(gpu_lib, fixtures):
    for name, A, B, Cx in fixtures:
        want = (Cx.row_ptr, Cx.col_idx, Cx.values)
        assert_same(oneshot(A, B, device=True), want, name + "/device")
        assert_same(oneshot(A, B, device=False), want, name + "/host")


def test_fixtures_public_api_oneshot(gpu_lib, fixtures):
    for name, A, B, Cx in fixtures:
        assert_same(rv.spgemm(A, B), (Cx.row_ptr, Cx.col_idx, Cx.values), name)


def _descr_run(A, B, algo, device):
    d = rv.Descriptor(algo)
    if device:
        dA, dB = DevCSR(A), DevCSR(B)
        a, b = dA.struct(), dB.struct()
    else:
        a, b = rv.from_csr(A), rv.from_csr(B)
    st, ws, nnz = d.work_estimation(a, b)
    rv.check(st, "work_estimation")
    if device:
        crp, cci, cv = dev(np.zeros(A.rows + 1, np.int32)), dev(np.zeros(max(nnz, 1), np.int32)), \
            dev(np.zeros(max(nnz, 1), np.float32))
        wsb = dev(np.zeros(max(ws, 4), np.uint8))
    else:
        crp, cci, cv = np.zeros(A.rows + 1, np.int32), np.zeros(max(nnz, 1), np.int32), \
            np.zeros(max(nnz, 1), np.float32)
        wsb = np.zeros(max(ws, 4), np.uint8)
    c = rv.csr_struct(A.rows, B.cols, nnz, crp, cci, cv)
    rv.check(d.compute(a, b, c, wsb), "compute")
    if device:
        out = (crp.cpu().numpy(), cci.cpu().numpy()[:nnz], cv.cpu().numpy()[:nnz])
    else:
        out = (crp.copy(), cci[:nnz].copy(), cv[:nnz].copy())
    d.close()
    return nnz, out


@pytest.mark.parametrize("device", [True, False])
def test_fixtures_descriptor(gpu_lib, fixtures, device):
    """rv-sparse tests/test_spgemm_reference_f32.c:66-158 with the CUDA strategy."""
    for name, A, B, Cx in fixtures:
        nnz, out = _descr_run(A, B, rv.RVSP_SPGEMM_ALGO_CUDA, device)
        assert nnz == Cx.nnz, name
        assert_same(out, (Cx.row_ptr, Cx.col_idx, Cx.values), name)


def test_reference_golden_cases(gpu_lib, ref_cases):
    for name, A, B, want, ops in ref_cases:
        rp, ci, v, gops = oneshot(A, B, want_ops=True)
        assert_same((rp, ci, v), want, name)
        assert np.array_equal(gops, ops), name


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", ["uniform_4096x4096_16_seed0", "poisson2d_1024"])
def test_full_size_digests(gpu_lib, name):
    """Full 4096^2 plain product and the 1024^2 Poisson product against the
    SHA-256 of the reference kernel's output arrays."""
    d = ref_digests()[name]
    A = gen.uniform_fixed() if name.startswith("uniform") else gen.poisson2d(1024)
    rp, ci, v, ops = oneshot(A, A, want_ops=True)
    assert rp[-1] == d["c_nnz"]
    assert _sha(rp) == d["row_ptr_sha256"]
    assert _sha(ci) == d["col_idx_sha256"]
    assert _sha(v) == d["values_sha256"]
    assert _sha(ops) == d["ops_sha256"]


def test_descriptor_contract(gpu_lib, fixtures):
    """rv-sparse tests/test_spgemm_descr_f32.c with the CUDA strategy."""
    L = rv.lib()
    name, A0, B0, Cx = fixtures[0]
    a_vals = A0.values.copy()
    A = Mat(A0.rows, A0.cols, A0.row_ptr, A0.col_idx, a_vals)
    a, b = rv.from_csr(A), rv.from_csr(B0)
    h = C.c_void_p()
    assert L.rvsp_spgemm_descr_create(C.byref(h)) == 0
    assert L.rvsp_spgemm_set_algo(h, rv.RVSP_SPGEMM_ALGO_CUDA) == 0
    rp3, ci3, v3 = np.zeros(3, np.int32), np.zeros(3, np.int32), np.zeros(3, np.float32)
    tmp = rv.csr_struct(2, 2, 3, rp3, ci3, v3)
    ws0 = np.zeros(4096, np.uint8)
    assert L.rvsp_spgemm_compute(h, C.byref(a), C.byref(b), C.byref(tmp), rv.ptr(ws0)) == -2
    ops = np.zeros(2, np.int64)
    assert L.rvsp_spgemm_get_op_counts(h, rv.ptr(ops), 2) == -2
    size, nnz = C.c_size_t(), C.c_int32()
    assert L.rvsp_spgemm_work_estimation(h, C.byref(a), C.byref(b), C.byref(size), C.byref(nnz)) == 0
    assert nnz.value == Cx.nnz and size.value > 0
    assert L.rvsp_spgemm_work_estimation(h, None, C.byref(b), C.byref(size), C.byref(nnz)) == -1
    assert L.rvsp_spgemm_set_algo(h, rv.RVSP_SPGEMM_ALGO_CUDA) == -2
    assert L.rvsp_spgemm_get_op_counts(h, rv.ptr(ops), 2) == 0
    assert list(ops) == [2, 1]
    assert L.rvsp_spgemm_get_op_counts(h, rv.ptr(ops), 1) == -2
    n = nnz.value
    crp, cci, cv = np.zeros(A.rows + 1, np.int32), np.zeros(n, np.int32), np.zeros(n, np.float32)
    ws = np.zeros(size.value, np.uint8)
    c = rv.csr_struct(A.rows, B0.cols, n, crp, cci, cv)
    assert L.rvsp_spgemm_compute(h, C.byref(a), C.byref(b), C.byref(c), None) == -1
    assert L.rvsp_spgemm_compute(h, C.byref(a), C.byref(b), None, rv.ptr(ws)) == -1
    small = rv.csr_struct(A.rows, B0.cols, n - 1, crp, cci, cv)
    assert L.rvsp_spgemm_compute(h, C.byref(a), C.byref(b), C.byref(small), rv.ptr(ws)) == -2
    wrong = rv.csr_struct(A.rows + 1, B0.cols, n, crp, cci, cv)
    assert L.rvsp_spgemm_compute(h, C.byref(a), C.byref(b), C.byref(wrong), rv.ptr(ws)) == -2
    bad_a = rv.csr_struct(A.rows, A.cols, A.nnz - 1, A.row_ptr, A.col_idx, a_vals)
    assert L.rvsp_spgemm_compute(h, C.byref(bad_a), C.byref(b), C.byref(c), rv.ptr(ws)) == -2
    assert L.rvsp_spgemm_compute(h, C.byref(a), C.byref(b), C.byref(c), rv.ptr(ws)) == 0
    assert c.nnz == Cx.nnz
    assert np.array_equal(cci, Cx.col_idx) and np.array_equal(cv, Cx.values)
    a_vals *= 2.0  # reuse: same pattern, new values, no re-analysis
    assert L.rvsp_spgemm_compute(h, C.byref(a), C.byref(b), C.byref(c), rv.ptr(ws)) == 0
    assert np.array_equal(cv, 2.0 * Cx.values)
    assert np.array_equal(cci, Cx.col_idx)
    L.rvsp_spgemm_invalidate_structure(h)
    cci[:] = -7
    assert L.rvsp_spgemm_compute(h, C.byref(a), C.byref(b), C.byref(c), rv.ptr(ws)) == 0
    assert np.array_equal(cci, Cx.col_idx)
    L.rvsp_spgemm_invalidate_structure(None)
    L.rvsp_spgemm_descr_destroy(None)
    L.rvsp_spgemm_descr_destroy(h)


@pytest.mark.parametrize("device", [True, False])
def test_descriptor_reuse_rescaled_values(gpu_lib, device):
    """Poisson product reused with rescaled values (the numeric-only graph path)."""
    A = gen.poisson2d(96)
    rng = np.random.default_rng(3)
    d = rv.Descriptor(rv.RVSP_SPGEMM_ALGO_CUDA)
    vals = A.values.copy()
    if device:
        drp, dci, dv = dev(A.row_ptr), dev(A.col_idx), dev(vals)
        a = rv.csr_struct(A.rows, A.cols, A.nnz, drp, dci, dv)
    else:
        a = rv.csr_struct(A.rows, A.cols, A.nnz, A.row_ptr, A.col_idx, vals)
    st, ws, nnz = d.work_estimation(a, a)
    rv.check(st)
    wrp, wci, _ = oracle.spgemm_f32(A, A)
    if device:
        crp, cci, cv = dev(np.zeros(A.rows + 1, np.int32)), dev(np.zeros(nnz, np.int32)), \
            dev(np.zeros(nnz, np.float32))
    else:
        crp, cci, cv = np.zeros(A.rows + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz, np.float32)
    c = rv.csr_struct(A.rows, A.cols, nnz, crp, cci, cv)
    wsb = np.zeros(max(ws, 4), np.uint8)
    for rep in range(4):
        scaled = (A.values * rng.uniform(0.5, 1.5, A.nnz).astype(np.float32)).astype(np.float32)
        if device:
            dv.copy_(dev(scaled))
            crp.fill_(-1)  # every compute writes C's row pointer
        else:
            vals[:] = scaled
            crp[:] = -1
        rv.check(d.compute(a, a, c, wsb), f"compute {rep}")
        M = Mat(A.rows, A.cols, A.row_ptr, A.col_idx, scaled)
        want = oracle.numeric_f32(M, M, wrp, wci)
        got_v = cv.cpu().numpy() if device else cv
        got_ci = cci.cpu().numpy() if device else cci
        got_rp = crp.cpu().numpy() if device else crp
        assert np.array_equal(got_rp.astype(np.int64), np.asarray(wrp, np.int64)), rep
        assert np.array_equal(got_ci, wci)
        assert np.array_equal(bits(got_v), bits(want)), rep
    d.close()


def _bin_sweep_matrix(seed=0):
    """Rows whose products span every bin: tiny, warp tables 64..4096, heavy."""
    rng = np.random.default_rng(seed)
    K, N = 3000, 40000
    b_counts = np.concatenate([rng.integers(0, 6, K - 40), rng.integers(200, 3000, 40)])
    rng.shuffle(b_counts)
    B = gen.from_keys(K, N, gen._distinct_rows(b_counts, N, rng), None, rng)
    a_counts = np.concatenate([np.zeros(50, np.int64), rng.integers(1, 4, 400),
                               rng.integers(4, 40, 300), rng.integers(40, 200, 100),
                               rng.integers(200, 900, 30)])
    rng.shuffle(a_counts)
    A = gen.from_keys(a_counts.size, K, gen._distinct_rows(a_counts, K, rng), None, rng)
    return A, B


def test_every_bin_matches_oracle(gpu_lib):
    A, B = _bin_sweep_matrix()
    ops = gen.row_products(A, B)
    ub = np.minimum(ops, B.cols)
    assert (ops == 0).any() and (ops <= 32).any() and (ub > 4096).any()
    assert_same(oneshot(A, B), oracle_full(A, B), "bin sweep")
    nnz, out = _descr_run(A, B, rv.RVSP_SPGEMM_ALGO_CUDA, True)
    assert_same(out, oracle_full(A, B), "bin sweep descriptor")


def _rows_of(rows, cols, per_row, col_pool, rng, vals=True):
    """CSR with per_row distinct columns a row, drawn from col_pool."""
    ci = np.concatenate([np.sort(rng.choice(col_pool, per_row, replace=False)) for _ in range(rows)])
    rp = np.arange(rows + 1) * per_row
    return Mat(rows, cols, rp, ci, rng.uniform(-1, 1, rows * per_row))


def test_warp_rows_fill_paths(gpu_lib):
    """Warp-table rows take one of three fill paths by what the analysis
    knows of them: few repeated columns (expand, sort, compress), mostly
    repeated columns (hash table), columns spanning 2^20 or more (two walks).
    Each is built here from rows of 20 A entries times 10-entry B rows
    (200 products, a 256-slot table) and compared with the oracle."""
    rng = np.random.default_rng(11)
    A = _rows_of(96, 256, 20, np.arange(256), rng)
    cases = {
        "distinct": _rows_of(256, 1 << 16, 10, np.arange(1 << 16), rng),
        "repeats": _rows_of(256, 4096, 10, np.arange(40) * 97, rng),
        "wide": _rows_of(256, 1 << 22, 10, np.arange(1 << 22), rng),
    }
    for name, B in cases.items():
        ops = gen.row_products(A, B)
        assert (ops == 200).all() and B.cols > 200, name
        want = oracle_full(A, B)
        nnz = np.diff(np.asarray(want[0], np.int64))
        if name == "repeats":
            assert (2 * nnz < ops).all()
        else:
            assert (2 * nnz >= ops).all()
        assert_same(oneshot(A, B), want, name)
        assert_same(oneshot(A, B, device=False), want, name + " host")


def test_rmat_matches_oracle(gpu_lib):
    R = gen.rmat(scale=13, edge_factor=8, seed=5)
    assert_same(oneshot(R, R), oracle_full(R, R), "rmat s13")


def test_rmat16_heavy_rows_sampled(gpu_lib):
    """R-MAT 2^16: chunked heavy rows over B rows long enough to get a column
    directory, several scan tiles; the hub rows and a band of middle rows are
    compared with the oracle bit for bit."""
    R = gen.rmat(scale=16, edge_factor=16, seed=0)
    rp, ci, v = oneshot(R, R)
    for r0, r1 in ((0, 1500), (30000, 30400)):
        wrp, wci, wv = oracle.spgemm_f32(R, R, r0, r1)
        lo, hi = int(rp[r0]), int(rp[r1])
        assert np.array_equal(np.asarray(rp[r0:r1 + 1], np.int64) - lo, wrp), (r0, r1)
        assert np.array_equal(ci[lo:hi], wci), (r0, r1)
        assert np.array_equal(bits(v[lo:hi]), bits(wv)), (r0, r1)


def test_tall_skinny_heavy_rows(gpu_lib):
    A, B = gen.tall_skinny(a_rows=20000, k=20000, n=20000, b_max=6000, seed=3)
    assert_same(oneshot(A, B), oracle_full(A, B), "tall skinny")


def test_edge_shapes(gpu_lib):
    cases = []
    # all-empty A
    cases.append((Mat(3, 4, [0, 0, 0, 0], [], []), Mat(4, 5, [0, 1, 1, 2, 2], [0, 4], [1.0, 2.0])))
    # empty B rows only
    cases.append((Mat(2, 3, [0, 2, 3], [0, 2, 1], [1.0, 2.0, 3.0]), Mat(3, 3, [0, 0, 0, 0], [], [])))
    # 1x1
    cases.append((Mat(1, 1, [0, 1], [0], [3.0]), Mat(1, 1, [0, 1], [0], [-2.0])))
    # single output column, many products per row (ops > 32 with ub == 1)
    rng = np.random.default_rng(0)
    K = 100
    cases.append((Mat(4, K, [0, K, 2 * K, 3 * K, 4 * K], np.tile(np.arange(K), 4), rng.uniform(-1, 1, 4 * K)),
                  Mat(K, 1, np.arange(K + 1), np.zeros(K), rng.uniform(-1, 1, K))))
    # negative zero products must sum to +0.0 like the reference
    cases.append((Mat(1, 2, [0, 2], [0, 1], [-0.0, 1.0]), Mat(2, 1, [0, 1, 2], [0, 0], [1.0, -0.0])))
    for i, (A, B) in enumerate(cases):
        want = oracle_full(A, B)
        assert_same(oneshot(A, B), want, f"edge {i}")
        assert_same(oneshot(A, B, device=False), want, f"edge {i} host")


def test_invalid_csr_rejected_on_device(gpu_lib):
    """One-shot rejects non-canonical device inputs (rv-sparse src/core/spgemm.c:45-51)."""
    L = rv.lib()
    A = gen.uniform_fixed(64, 64, 8, seed=2)
    rng = np.random.default_rng(1)
    for kind in ("dup", "unsorted", "range", "rowptr"):
        ci = A.col_idx.copy()
        rp = A.row_ptr.copy()
        r = int(rng.integers(1, 60))
        s = rp[r]
        if kind == "dup":
            ci[s + 1] = ci[s]
        elif kind == "unsorted":
            ci[s], ci[s + 1] = ci[s + 1], ci[s]
        elif kind == "range":
            ci[s] = 64
        else:
            rp[r] = rp[r + 1] + 1
        code, bad = oracle.csr_check(A.rows, A.cols, rp, ci)
        drp, dci = dev(rp), dev(ci)
        badrow = C.c_int32()
        got = L.rvsp_cuda_csr_check(A.rows, A.cols, A.nnz, rv.ptr(drp), rv.ptr(dci), C.byref(badrow))
        assert (got, badrow.value) == (code, bad), kind
        dv = dev(A.values)
        M = rv.csr_struct(A.rows, A.cols, A.nnz, drp, dci, dv)
        out = rv.CsrMatrix()
        assert L.rvsp_spgemm_csr(C.byref(M), C.byref(M), C.byref(out), None) == rv.RVSP_ERROR_INVALID_CSR


def test_nnz_overflow_reports_allocation_failed(gpu_lib):
    """nnz(C) > INT32_MAX fails like rv-sparse rvsp_symbolic.c:69, before any C allocation."""
    n = 50000
    A = Mat(n, 1, np.arange(n + 1), np.zeros(n), np.ones(n))
    B = Mat(1, n, [0, n], np.arange(n), np.ones(n))
    d = rv.Descriptor(rv.RVSP_SPGEMM_ALGO_CUDA)
    dA, dB = DevCSR(A), DevCSR(B)
    st, ws, nnz = d.work_estimation(dA.struct(), dB.struct())
    assert st == rv.RVSP_ERROR_ALLOCATION_FAILED
    d.close()


def test_op_counts_match_oracle(gpu_lib):
    A, B = _bin_sweep_matrix(3)
    d = rv.Descriptor(rv.RVSP_SPGEMM_ALGO_CUDA)
    dA, dB = DevCSR(A), DevCSR(B)
    st, ws, nnz = d.work_estimation(dA.struct(), dB.struct())
    rv.check(st)
    st, ops = d.op_counts(A.rows)
    rv.check(st)
    wops, wcnt = oracle.symbolic(A, B)
    assert np.array_equal(ops, wops)
    assert nnz == wcnt.sum()
    d.close()


def test_launch_counter_advances(gpu_lib):
    before = rv.launch_count()
    A = gen.uniform_fixed(128, 128, 8, seed=9)
    oneshot(A, A)
    assert rv.launch_count() > before


@pytest.mark.parametrize("device", [True, False])
def test_descriptor_reuse_all_bins(gpu_lib, device):
    """Reuse across tiny, warp-table and heavy rows: the position maps recorded
    by the first fill replay bit-exactly with new values in A and B."""
    A, B = _bin_sweep_matrix(7)
    rng = np.random.default_rng(11)
    d = rv.Descriptor(rv.RVSP_SPGEMM_ALGO_CUDA)
    av, bvals = A.values.copy(), B.values.copy()
    if device:
        dA, dB = DevCSR(A), DevCSR(B)
        a, b = dA.struct(), dB.struct()
    else:
        a = rv.csr_struct(A.rows, A.cols, A.nnz, A.row_ptr, A.col_idx, av)
        b = rv.csr_struct(B.rows, B.cols, B.nnz, B.row_ptr, B.col_idx, bvals)
    st, ws, nnz = d.work_estimation(a, b)
    rv.check(st)
    wrp, wci, _ = oracle.spgemm_f32(A, B)
    if device:
        crp, cci, cv = dev(np.zeros(A.rows + 1, np.int32)), dev(np.zeros(nnz, np.int32)), \
            dev(np.zeros(nnz, np.float32))
    else:
        crp, cci, cv = np.zeros(A.rows + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz, np.float32)
    c = rv.csr_struct(A.rows, B.cols, nnz, crp, cci, cv)
    wsb = np.zeros(max(ws, 4), np.uint8)
    for rep in range(3):
        na = (A.values * rng.uniform(0.5, 1.5, A.nnz)).astype(np.float32)
        nb = (B.values * rng.uniform(0.5, 1.5, B.nnz)).astype(np.float32)
        if device:
            dA.values.copy_(dev(na))
            dB.values.copy_(dev(nb))
        else:
            av[:] = na
            bvals[:] = nb
        rv.check(d.compute(a, b, c, wsb), f"compute {rep}")
        want = oracle.numeric_f32(Mat(A.rows, A.cols, A.row_ptr, A.col_idx, na),
                                  Mat(B.rows, B.cols, B.row_ptr, B.col_idx, nb), wrp, wci)
        got_v = cv.cpu().numpy() if device else cv
        got_ci = cci.cpu().numpy() if device else cci
        assert np.array_equal(got_ci, wci)
        assert np.array_equal(bits(got_v), bits(want)), rep
    d.close()


@pytest.mark.parametrize("algo", [rv.RVSP_CUDA_ALGO_EXACT, rv.RVSP_CUDA_ALGO_LEARNED])
def test_batched_products_match_oracle(gpu_lib, algo):
    """Uneven products in one batched call: each row range of the packed C is
    that product's C, bit for bit, with its own column indices."""
    if algo == rv.RVSP_CUDA_ALGO_LEARNED and not rv.lib().rvsp_cuda_learned_available():
        pytest.skip("no row-size model")
    pairs = gen.batched_uneven(count=24, lo=8, hi=4000, seed=13)
    pairs.append((gen.uniform_fixed(50, 3, 2, seed=1), gen.uniform_fixed(3, 9000, 3, seed=2)))
    dev_pairs = [(DevCSR(A), DevCSR(B)) for A, B in pairs]
    (prp, pci, pv), nnz, offs, coffs = rv.spgemm_batched(dev_pairs, algo)
    try:
        crp = d2h(prp, int(offs[-1]) + len(pairs), np.int32)
        cci = d2h(pci, nnz, np.int32)
        cv = d2h(pv, nnz, np.float32)
    finally:
        rv.free_device(prp, pci, pv)
    assert offs[-1] == sum(A.rows for A, _ in pairs) and coffs[-1] == nnz
    for i, (A, B) in enumerate(pairs):
        r0 = int(offs[i]) + i
        lrp = crp[r0:r0 + A.rows + 1]
        e0, e1 = int(coffs[i]), int(coffs[i + 1])
        wrp, wci, wv = oracle.spgemm_f32(A, B)
        assert np.array_equal(lrp, wrp), i
        assert e1 - e0 == lrp[-1], i
        assert np.array_equal(cci[e0:e1], wci), i
        assert np.array_equal(bits(cv[e0:e1]), bits(wv)), i


def test_batched_rejects_a_row_panel(gpu_lib):
    """Batched operands are whole matrices: an A whose row pointer does not
    start at 0 is refused instead of being packed with wrong offsets."""
    A = gen.uniform_fixed(40, 40, 4, seed=2)
    dA = DevCSR(A)
    panel = DevCSR(A)
    panel.rows = 20
    panel.row_ptr = dA.row_ptr[10:31]
    panel.nnz = int(A.row_ptr[30] - A.row_ptr[10])
    with pytest.raises(rv.RvspError) as e:
        rv.spgemm_batched([(dA, dA), (panel, dA)], rv.RVSP_CUDA_ALGO_EXACT)
    assert e.value.status == rv.RVSP_ERROR_INVALID_CSR
