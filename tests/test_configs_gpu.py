"""Parity of the benchmark configurations' own paths, bit for bit against the
oracle (the scalar Gustavson restatement, pinned to the reference kernel):

* the device row-panel path that runs the power-law product: A's row pointer
  offset into the full arrays (include/rvsp_cuda.h), R-MAT 2^16 split into
  panels like the 2^20 product, three panels including the heaviest, exact and
  learned;
* the full-size tall-skinny product (2,000,000 x 100,000 times 100,000^2):
  every row of the heaviest 1 % by products plus 2,000 seeded rows;
* a host C of several hundred MB (the staged device->host copy) against the
  device-resident C of the same product;
* batched uneven products: 64 seeded products of the 512-product
  configuration, including its largest, in one batched call, exact and
  learned; and all 512 in one call (their C passes 2^31 entries).

Values are compared bit for bit: every path adds the FP32 products in the
reference's order (rv-sparse accum_scalar_f32.c:69).
"""

import ctypes as C
import functools

import numpy as np
import pytest

import oracle
import rvsp_b200 as rv
from gpu_util import DevCSR, bits, d2h
from rvsp_b200 import gen, ranks

pytestmark = pytest.mark.gpu

ALGOS = (("exact", rv.RVSP_CUDA_ALGO_EXACT), ("learned", rv.RVSP_CUDA_ALGO_LEARNED))


def _panel_product(dA, dB, r0, r1, algo):
    """rvsp_cuda_spgemm_f32 on rows [r0, r1) of device A: the row pointer
    passed is a view starting at row r0, its offsets index A's full arrays."""
    L = rv.lib()
    rp_view = dA.row_ptr[r0:r1 + 1]
    prp, pci, pv = C.c_void_p(), C.c_void_p(), C.c_void_p()
    nnz = C.c_int32()
    rv.check(L.rvsp_cuda_spgemm_f32(algo, r1 - r0, dA.cols, dB.cols, rv.ptr(rp_view),
                                    rv.ptr(dA.col_idx), rv.ptr(dA.values), rv.ptr(dB.row_ptr),
                                    rv.ptr(dB.col_idx), rv.ptr(dB.values), C.byref(prp),
                                    C.byref(pci), C.byref(pv), C.byref(nnz), None), "panel")
    n = nnz.value
    out = (d2h(prp.value, r1 - r0 + 1, np.int32), d2h(pci.value, n, np.int32),
           d2h(pv.value, n, np.float32))
    for p in (prp, pci, pv):
        L.rvsp_cuda_free(p)
    return out


def _same(got, want, what):
    rp, ci, v = got
    wrp, wci, wv = want
    assert np.array_equal(np.asarray(rp, np.int64), np.asarray(wrp, np.int64)), f"{what}: row_ptr"
    assert np.array_equal(ci, wci), f"{what}: col_idx"
    assert np.array_equal(bits(v), bits(wv)), f"{what}: values"


def test_rmat_row_panels_match_oracle(gpu_lib):
    R = gen.rmat(scale=16, edge_factor=16, seed=5)
    ops = gen.row_products(R, R)
    panels = ranks.row_panels(ops, int(ops.sum()) // 4 + 1)
    assert len(panels) >= 4
    heavy = int(np.argmax([ops[a:b].sum() for a, b in panels]))
    dR = DevCSR(R)
    for pi in sorted({0, heavy, len(panels) - 2}):
        r0, r1 = panels[pi]
        want = oracle.spgemm_f32(R, R, r0, r1)
        for name, algo in ALGOS:
            _same(_panel_product(dR, dR, r0, r1, algo), want, f"panel {pi} [{r0},{r1}) {name}")


def test_host_output_of_a_large_product_matches_the_device_output(gpu_lib):
    """Host operands and a host C of several hundred MB: the one-shot copies C
    out through the pinned staging ring and its host threads (copies of 64 MiB
    and more), exact and learned; bit-identical to the device-resident C."""
    from gpu_util import oneshot
    R = gen.rmat(scale=16, edge_factor=16, seed=9)
    for name, algo in ALGOS:
        want = oneshot(R, R, algo=algo, device=True)
        assert want[1].nbytes >= 64 << 20, "C too small to take the staged copy"
        _same(oneshot(R, R, algo=algo, device=False), want, f"host C {name}")


def test_large_host_operands_are_uploaded_staged(gpu_lib):
    """Host operands of 64 MiB and more per array go up through the pinned
    pieces and host threads (B: 1,000,000 rows of 20 entries, 80 MB per
    array): C bit-identical to the product of the same operands on the
    device, exact and learned, and to the oracle."""
    from gpu_util import oneshot
    B = gen.uniform_fixed(rows=1_000_000, cols=1_000_000, per_row=20, seed=3)
    A = gen.uniform_fixed(rows=2000, cols=1_000_000, per_row=4, seed=4)
    assert B.col_idx.nbytes >= 64 << 20
    want = oracle.spgemm_f32(A, B)
    for name, algo in ALGOS:
        _same(oneshot(A, B, algo=algo, device=False), want, f"host operands {name}")
        _same(oneshot(A, B, algo=algo, device=True), want, f"device operands {name}")


def test_host_results_through_the_public_api_reuse_released_arrays(gpu_lib):
    """rvsp_spgemm_csr with host operands, twice per backend, the first C
    released by rvsp_csr_destroy before the second product (large released
    arrays are kept and handed out again): every host C bit-identical to the
    device-resident C of the same product."""
    from gpu_util import oneshot
    L = rv.lib()
    R = gen.rmat(scale=16, edge_factor=16, seed=9)
    S = gen.rmat(scale=16, edge_factor=14, seed=10)
    for backend, algo in ((rv.RVSP_BACKEND_CUDA, rv.RVSP_CUDA_ALGO_EXACT),
                          (rv.RVSP_BACKEND_CUDA_LEARNED, rv.RVSP_CUDA_ALGO_LEARNED)):
        opts = rv.SpgemmOptions(backend, rv.RVSP_DTYPE_FP32, rv.RVSP_DTYPE_FP32)
        for M in (R, S, R):
            want = oneshot(M, M, algo=algo, device=True)
            hm = rv.csr_struct(M.rows, M.cols, M.nnz, M.row_ptr, M.col_idx, M.values)
            c = rv.CsrMatrix()
            rv.check(L.rvsp_spgemm_csr(C.byref(hm), C.byref(hm), C.byref(c), C.byref(opts)),
                     "rvsp_spgemm_csr")
            assert c.owns_data == 1 and c.nnz == want[1].size
            got = (np.ctypeslib.as_array((C.c_int32 * (M.rows + 1)).from_address(c.row_ptr)).copy(),
                   np.ctypeslib.as_array((C.c_int32 * c.nnz).from_address(c.col_idx)).copy(),
                   np.ctypeslib.as_array((C.c_float * c.nnz).from_address(c.values)).copy())
            L.rvsp_csr_destroy(C.byref(c))
            _same(got, want, f"public API host C, backend {backend}")


def _row_subset(A, rows):
    """CSR of the given rows of A (in order)."""
    lens = np.diff(A.row_ptr.astype(np.int64))[rows]
    rp = np.zeros(rows.size + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    idx = np.repeat(A.row_ptr[rows].astype(np.int64) - rp[:-1], lens) + np.arange(rp[-1])
    return gen.CSR(rows.size, A.cols, rp.astype(np.int32), A.col_idx[idx], A.values[idx])


def test_tall_skinny_full_size_heaviest_and_sampled_rows(gpu_lib):
    A, B = gen.tall_skinny(a_rows=2_000_000)
    ops = gen.row_products(A, B)
    top = np.argsort(ops, kind="stable")[::-1][: A.rows // 100]
    rows = np.union1d(top, np.random.default_rng(0).choice(A.rows, 2000, replace=False))
    S = _row_subset(A, rows)
    wrp, wci, wv = oracle.spgemm_f32(S, B)
    wrp = np.asarray(wrp, np.int64)
    dA, dB = DevCSR(A), DevCSR(B)
    for name, algo in ALGOS:
        rp, ci, v = _panel_product(dA, dB, 0, A.rows, algo)
        rp = rp.astype(np.int64)
        lo, hi = rp[rows], rp[rows + 1]
        assert np.array_equal(hi - lo, np.diff(wrp)), f"{name}: row lengths"
        idx = np.repeat(lo - wrp[:-1], hi - lo) + np.arange(wrp[-1])
        assert np.array_equal(ci[idx], wci), f"{name}: col_idx"
        assert np.array_equal(bits(v[idx]), bits(wv)), f"{name}: values"


@functools.lru_cache(maxsize=1)
def _batched_pairs():
    return gen.batched_uneven(count=512)


def test_batched_uneven_products_match_oracle(gpu_lib):
    pairs = _batched_pairs()
    prods = np.array([gen.products(A, B) for A, B in pairs], np.int64)
    rng = np.random.default_rng(3)
    pick = {int(np.argmax(prods))}
    for i in rng.permutation(len(pairs)):
        if len(pick) == 64:
            break
        pick.add(int(i))
    pick = sorted(pick)
    chosen = [pairs[i] for i in pick]
    dev_pairs = [(DevCSR(A), DevCSR(B)) for A, B in chosen]
    wants = [oracle.spgemm_f32(A, B) for A, B in chosen]
    for name, algo in ALGOS:
        ptrs, n, offs, coffs = rv.spgemm_batched(dev_pairs, algo)
        crp = d2h(ptrs[0], int(offs[-1]) + len(chosen), np.int32)
        cci = d2h(ptrs[1], n, np.int32)
        cv = d2h(ptrs[2], n, np.float32)
        rv.free_device(*ptrs)
        for k, (want, i) in enumerate(zip(wants, pick)):
            r0 = int(offs[k]) + k
            e0, e1 = int(coffs[k]), int(coffs[k + 1])
            got = (crp[r0:r0 + chosen[k][0].rows + 1], cci[e0:e1], cv[e0:e1])
            _same(got, want, f"{name} product {i}")


def test_batched_all_512_products_in_one_call(gpu_lib):
    """The whole 512-product configuration (its C passes 2^31 entries) in one
    batched call: every product's row pointer and entry range are consistent,
    and eight seeded products, the largest among them, match the oracle."""
    pairs = _batched_pairs()
    prods = np.array([gen.products(A, B) for A, B in pairs], np.int64)
    dev_pairs = [(DevCSR(A), DevCSR(B)) for A, B in pairs]
    ptrs, n, offs, coffs = rv.spgemm_batched(dev_pairs, rv.RVSP_CUDA_ALGO_EXACT)
    try:
        assert coffs[-1] == n and np.all(np.diff(coffs) >= 0)
        crp = d2h(ptrs[0], int(offs[-1]) + len(pairs), np.int32)
        pick = sorted({int(np.argmax(prods))} |
                      set(np.random.default_rng(9).choice(len(pairs), 7, replace=False).tolist()))
        for i in pick:
            A, B = pairs[i]
            r0 = int(offs[i]) + i
            lrp = crp[r0:r0 + A.rows + 1]
            e0, e1 = int(coffs[i]), int(coffs[i + 1])
            assert lrp[0] == 0 and lrp[-1] == e1 - e0
            got = (lrp, d2h(ptrs[1] + 4 * e0, e1 - e0, np.int32),
                   d2h(ptrs[2] + 4 * e0, e1 - e0, np.float32))
            _same(got, oracle.spgemm_f32(A, B), f"product {i}")
    finally:
        rv.free_device(*ptrs)
