"""The CPU oracle pinned against the reference's golden vectors (CPU only)."""

import hashlib

import numpy as np
import pytest

import oracle
from conftest import ref_digests
from rvsp_b200 import gen


def test_oracle_fixtures(fixtures):
    """rv-sparse tests/csr_fixtures.h: structure exact, values exact."""
    for name, A, B, Cx in fixtures:
        rp, ci, v = oracle.spgemm_f32(A, B)
        assert np.array_equal(rp, Cx.row_ptr), name
        assert np.array_equal(ci, Cx.col_idx), name
        assert np.array_equal(v, Cx.values), name


def test_oracle_cancellation_keeps_structural_zero(fixtures):
    name, A, B, Cx = [f for f in fixtures if f[0] == "cancel"][0]
    rp, ci, v = oracle.spgemm_f32(A, B)
    assert rp[-1] == 1 and ci[0] == 0 and v[0] == 0.0 and not np.signbit(v[0])


def test_oracle_matches_reference_outputs(ref_cases):
    """Bit-exact against the reference scalar kernel's stored outputs."""
    for name, A, B, (rp, ci, v), ops in ref_cases:
        orp, oci, ov = oracle.spgemm_f32(A, B)
        assert np.array_equal(orp, rp.astype(np.int64)), name
        assert np.array_equal(oci, ci), name
        assert np.array_equal(ov.view(np.uint32), v.view(np.uint32)), name
        oops, ocnt = oracle.symbolic(A, B)
        assert np.array_equal(oops, ops), name
        assert ocnt.sum() == rp[-1]


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", ["uniform_4096x4096_16_seed0", "poisson2d_1024"])
def test_oracle_matches_reference_digests(name):
    d = ref_digests()[name]
    A = gen.uniform_fixed() if name.startswith("uniform") else gen.poisson2d(1024)
    rp, ci, v = oracle.spgemm_f32(A, A)
    assert rp[-1] == d["c_nnz"]
    assert _sha(rp.astype(np.int32)) == d["row_ptr_sha256"]
    assert _sha(ci) == d["col_idx_sha256"]
    assert _sha(v) == d["values_sha256"]
    ops, _ = oracle.symbolic(A, A)
    assert _sha(ops) == d["ops_sha256"]
    assert gen.products(A, A) == d["products"]


def test_oracle_row_ranges_compose(ref_cases):
    """A row-range call gives the same rows as the full call (sampling checks rely on it)."""
    name, A, B, (rp, ci, v), _ = ref_cases[2]
    r0, r1 = 37, 211
    srp, sci, sv = oracle.spgemm_f32(A, B, r0, r1)
    assert np.array_equal(srp + rp[r0], rp[r0:r1 + 1])
    assert np.array_equal(sci, ci[rp[r0]:rp[r1]])
    assert np.array_equal(sv.view(np.uint32), v[rp[r0]:rp[r1]].view(np.uint32))


def test_oracle_numeric_f32_and_f64(ref_cases):
    for name, A, B, (rp, ci, v), _ in ref_cases:
        nv = oracle.numeric_f32(A, B, rp.astype(np.int64), ci)
        assert np.array_equal(nv.view(np.uint32), v.view(np.uint32)), name
        dv = oracle.numeric_f64(A, B, rp.astype(np.int64), ci)
        err = np.abs(dv - v.astype(np.float64))
        assert (err <= 1e-5 + 1e-4 * np.abs(dv)).all(), name


def test_oracle_csr_check_codes():
    rp = np.array([0, 2, 4], np.int32)
    assert oracle.csr_check(2, 4, rp, np.array([0, 1, 2, 3], np.int32)) == (0, -1)
    assert oracle.csr_check(2, 4, rp, np.array([0, 1, 3, 3], np.int32)) == (4, 1)
    assert oracle.csr_check(2, 4, rp, np.array([0, 1, 3, 2], np.int32)) == (3, 1)
    assert oracle.csr_check(2, 4, rp, np.array([0, 5, 1, 2], np.int32)) == (2, 0)
    assert oracle.csr_check(2, 4, np.array([1, 2, 4], np.int32), np.zeros(4, np.int32))[0] == 1
    assert oracle.csr_check(2, 4, np.array([0, 3, 2], np.int32), np.arange(4, dtype=np.int32)) == (1, 1)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
def test_oracle_vs_live_reference_rmat():
    """Live cross-check against the compiled reference on a fresh seeded R-MAT."""
    R = gen.rmat(scale=11, edge_factor=8, seed=11)
    rrp, rci, rv, rops, st = oracle.ref_spgemm(R, R)
    assert st == 0
    orp, oci, ov = oracle.spgemm_f32(R, R)
    assert np.array_equal(orp, rrp.astype(np.int64))
    assert np.array_equal(oci, rci)
    assert np.array_equal(ov.view(np.uint32), rv.view(np.uint32))


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("dtype", ["f64", "i8"])
def test_legacy_dtypes_match_reference(dtype):
    """FP64 and INT8 -> INT32 restatements against the reference's own legacy
    kernels: same structure after zero-sum entries are dropped, values bit for bit."""
    from conftest import typed_pair
    cases = [gen.rmat(scale=10, edge_factor=8, seed=2), gen.uniform_fixed(600, 500, 9, seed=4)]
    for M in cases:
        A, B = typed_pair(M, M, dtype, seed=7)
        rrp, rci, rv, st = oracle.ref_spgemm_typed(A, B, dtype)
        assert st == 0
        orp, oci, ov = oracle.spgemm_typed(A, B, dtype)
        assert np.array_equal(orp, rrp.astype(np.int64))
        assert np.array_equal(oci, rci)
        if dtype == "f64":
            assert np.array_equal(ov.view(np.uint64), rv.view(np.uint64))
        else:
            assert np.array_equal(ov, rv)
        _, cnt = oracle.symbolic(A, B)
        assert int(orp[-1]) < int(cnt.sum())  # some sums cancelled and were dropped


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
def test_coo_canonicalisation_matches_reference_loader(tmp_path):
    """The oracle's COO -> CSR restatement against the reference's own Matrix
    Market loader on seeded files (repeated entries up to three times,
    symmetric expansion, pattern values, a short file); the files are parsed by
    the library's C reader (host code only)."""
    import rvsp_b200 as rv
    from conftest import mtx_cases
    for name, path in mtx_cases(str(tmp_path)):
        rows, cols, r, c, v, sym = rv.mtx_read(path)
        wrp, wci, wv = oracle.ref_mtx_load(path)
        orp, oci, ov = oracle.coo_to_csr(rows, cols, r, c, v, sym)
        assert np.array_equal(orp, wrp.astype(np.int64)), name
        assert np.array_equal(oci, wci), name
        assert np.array_equal(ov.view(np.uint32), wv.view(np.uint32)), name
