"""Runtime bin parameters and the autotuner.

The parameters only move rows between kernels (thread, warp hash table,
chunked dense accumulator) and resize tables, so every valid setting must give
the reference's pattern and bit-identical values; the tuner must leave its
plan analysed under the choice it reports.
"""

import numpy as np
import pytest

import oracle
import rvsp_b200 as rv
from conftest import Mat
from gpu_util import DevCSR, bits, dev, oneshot
from rvsp_b200 import gen
from test_parity_gpu import _bin_sweep_matrix, assert_same

pytestmark = pytest.mark.gpu

# extremes of every parameter: everything on warps, tiny tables, narrow chunks;
# the opposite corner; and mixed settings
PARAM_SETS = [
    (0, 1, 64, 9),
    (16, 3, 1024, 11),
    (32, 4, 4096, 13),
    (32, 2, 256, 10),
    (8, 1, 2048, 12),
]


def plan_run(A, B, params=None, algo=rv.RVSP_CUDA_ALGO_EXACT):
    """symbolic + filling numeric through a plan on device operands."""
    dA, dB = DevCSR(A), DevCSR(B)
    p = rv.Plan(algo)
    if params is not None:
        rv.check(p.set_params(params), "set_params")
        assert p.get_params() == tuple(params)
    st, nnz = p.symbolic(dA, dB)
    rv.check(st, "symbolic")
    crp = dev(np.zeros(A.rows + 1, np.int32))
    cci = dev(np.zeros(max(nnz, 1), np.int32))
    cv = dev(np.zeros(max(nnz, 1), np.float32))
    rv.check(p.numeric(dA, dB, crp, cci, cv), "numeric")
    out = (crp.cpu().numpy(), cci.cpu().numpy()[:nnz], cv.cpu().numpy()[:nnz])
    p.close()
    return out


def _cases():
    A, B = _bin_sweep_matrix(3)
    R = gen.rmat(scale=12, edge_factor=8, seed=9)
    T, S = gen.tall_skinny(a_rows=6000, k=6000, n=30000, b_max=4000, seed=4)
    return [("bin_sweep", A, B), ("rmat_s12", R, R), ("tall_skinny", T, S)]


@pytest.mark.parametrize("params", PARAM_SETS)
def test_every_param_set_is_bit_exact(gpu_lib, params):
    for name, A, B in _cases():
        want = oracle.spgemm_f32(A, B)
        assert_same(plan_run(A, B, params), want, f"{name} {params}")


def test_learned_plan_under_params(gpu_lib):
    if not rv.lib().rvsp_cuda_learned_available():
        pytest.skip("no row-size model")
    for name, A, B in _cases():
        want = oracle.spgemm_f32(A, B)
        for params in ((16, 1, 512, 10), (32, 3, 4096, 12)):
            assert_same(plan_run(A, B, params, rv.RVSP_CUDA_ALGO_LEARNED), want,
                        f"learned {name} {params}")


def test_param_validation(gpu_lib):
    p = rv.Plan()
    bad = [(33, 2, 4096, 13), (-1, 2, 4096, 13), (32, 0, 4096, 13), (32, 5, 4096, 13),
           (32, 2, 3000, 13), (32, 2, 32, 13), (32, 2, 8192, 13), (32, 2, 4096, 8),
           (32, 2, 4096, 14)]
    for b in bad:
        assert p.set_params(b) == rv.RVSP_ERROR_INVALID_ARGUMENT, b
        assert p.get_params() == rv.DEFAULT_BIN_PARAMS
    assert p.set_params((32, 2, 4096)) == rv.RVSP_ERROR_INVALID_ARGUMENT  # too few values
    p.close()


def test_set_params_discards_analysis(gpu_lib, fixtures):
    name, A, B, Cx = fixtures[0]
    dA, dB = DevCSR(A), DevCSR(B)
    p = rv.Plan()
    st, nnz = p.symbolic(dA, dB)
    rv.check(st)
    crp = dev(np.zeros(A.rows + 1, np.int32))
    cci, cv = dev(np.zeros(max(nnz, 1), np.int32)), dev(np.zeros(max(nnz, 1), np.float32))
    rv.check(p.set_params((16, 3, 1024, 11)))
    assert p.numeric(dA, dB, crp, cci, cv) == rv.RVSP_ERROR_INVALID_ARGUMENT
    st, nnz2 = p.symbolic(dA, dB)
    rv.check(st)
    assert nnz2 == nnz
    rv.check(p.numeric(dA, dB, crp, cci, cv))
    assert_same((crp.cpu().numpy(), cci.cpu().numpy()[:nnz], cv.cpu().numpy()[:nnz]),
                (Cx.row_ptr, Cx.col_idx, Cx.values), name)
    p.close()


def test_default_params_reach_oneshot_and_descriptor_reuse(gpu_lib):
    A, B = _bin_sweep_matrix(5)
    want = oracle.spgemm_f32(A, B)
    try:
        rv.check(rv.set_default_params((16, 3, 256, 10)))
        assert rv.get_default_params() == (16, 3, 256, 10)
        assert rv.Plan().get_params() == (16, 3, 256, 10)
        assert_same(oneshot(A, B), want, "one-shot under default params")
        # descriptor reuse replays its maps and the chunked rows under these bins
        d = rv.Descriptor(rv.RVSP_SPGEMM_ALGO_CUDA)
        dA, dB = DevCSR(A), DevCSR(B)
        a, b = dA.struct(), dB.struct()
        st, ws, nnz = d.work_estimation(a, b)
        rv.check(st)
        crp, cci, cv = dev(np.zeros(A.rows + 1, np.int32)), dev(np.zeros(nnz, np.int32)), \
            dev(np.zeros(nnz, np.float32))
        c = rv.csr_struct(A.rows, B.cols, nnz, crp, cci, cv)
        wsb = np.zeros(max(ws, 4), np.uint8)
        rng = np.random.default_rng(2)
        for rep in range(3):
            na = (A.values * rng.uniform(0.5, 1.5, A.nnz)).astype(np.float32)
            dA.values.copy_(dev(na))
            rv.check(d.compute(a, b, c, wsb), f"compute {rep}")
            wv = oracle.numeric_f32(Mat(A.rows, A.cols, A.row_ptr, A.col_idx, na), B,
                                    want[0], want[1])
            assert np.array_equal(cci.cpu().numpy(), want[1])
            assert np.array_equal(bits(cv.cpu().numpy()), bits(wv)), rep
        d.close()
    finally:
        rv.check(rv.set_default_params(None))
    assert rv.get_default_params() == rv.DEFAULT_BIN_PARAMS


def test_autotune_leaves_plan_analysed_under_choice(gpu_lib):
    R = gen.rmat(scale=13, edge_factor=8, seed=21)
    want = oracle.spgemm_f32(R, R)
    dR = DevCSR(R)
    p = rv.Plan()
    st, nnz, best, trials = p.autotune(dR, dR, reps=1)
    rv.check(st, "autotune")
    assert nnz == want[1].size
    assert p.get_params() == best
    assert 1 <= len(trials) <= 16
    assert trials[0][0] == rv.DEFAULT_BIN_PARAMS  # the search starts at the plan's params
    assert all(ms > 0 for _, ms in trials)
    # the choice is the fastest trial or within the 2% switching margin of it
    t_best = min(ms for prm, ms in trials if prm == best)
    assert t_best <= min(ms for _, ms in trials) / 0.98 + 1e-6
    crp = dev(np.zeros(R.rows + 1, np.int32))
    cci, cv = dev(np.zeros(nnz, np.int32)), dev(np.zeros(nnz, np.float32))
    rv.check(p.numeric(dR, dR, crp, cci, cv), "numeric after autotune")
    assert_same((crp.cpu().numpy(), cci.cpu().numpy(), cv.cpu().numpy()), want, "autotuned")
    p.close()


def test_descriptor_autotune_env(gpu_lib, fixtures, monkeypatch):
    monkeypatch.setenv("RVSP_AUTOTUNE", "1")
    for name, A, B, Cx in fixtures:
        d = rv.Descriptor(rv.RVSP_SPGEMM_ALGO_CUDA)
        a, b = rv.from_csr(A), rv.from_csr(B)
        st, ws, nnz = d.work_estimation(a, b)
        rv.check(st, name)
        crp, cci, cv = np.zeros(A.rows + 1, np.int32), np.zeros(max(nnz, 1), np.int32), \
            np.zeros(max(nnz, 1), np.float32)
        c = rv.csr_struct(A.rows, B.cols, nnz, crp, cci, cv)
        rv.check(d.compute(a, b, c, np.zeros(max(ws, 4), np.uint8)), name)
        assert_same((crp, cci[:nnz], cv[:nnz]), (Cx.row_ptr, Cx.col_idx, Cx.values), name)
        d.close()
