"""Learned row-size predictor on the GPU: training kernels against the FP64
oracle, inference against a float64 forward pass, and the learned SpGEMM path
bit-identical to the exact path (including forced mispredictions)."""

import os

import numpy as np
import pytest

import oracle
import rvsp_b200 as rv
from conftest import Mat
from gpu_util import DevCSR, bits, oneshot
from rvsp_b200 import gen

pytestmark = pytest.mark.gpu

SHIPPED = os.path.join(rv.PKG_DIR, "weights", "row_mlp_v1.bin")


def _rand_params(rng, scale=0.3):
    return {"W1": rng.normal(0, scale, (32, 4)), "b1": rng.normal(0, 0.1, 32),
            "W2": rng.normal(0, scale, (32, 32)), "b2": rng.normal(0, 0.1, 32),
            "W3": rng.normal(0, scale, (2, 32)), "b3": rng.normal(0, 0.1, 2)}


def test_gradient_kernel_matches_fp64_oracle(gpu_lib):
    """Gradient tolerance: |g_gpu - g_oracle| <= 1e-5 + 2e-3 * max|g_oracle| per tensor
    (FP32 products summed in a different order over 1000 samples)."""
    rng = np.random.default_rng(5)
    P = _rand_params(rng)
    n = 1000
    X = rng.normal(0, 1, (n, 4)).astype(np.float32)
    y = rng.uniform(0, 10, n).astype(np.float32)
    w = rng.uniform(0.5, 2.0, n).astype(np.float32)
    flat = rv.pack_params(P)
    loss = np.zeros(1, np.float32)
    grad = np.zeros(rv.MLP_PARAMS, np.float32)
    rv.check(rv.lib().rvsp_cuda_mlp_grad(flat.ctypes.data, X.ctypes.data, y.ctypes.data,
                                         w.ctypes.data, n, loss.ctypes.data, grad.ctypes.data))
    Pf = rv.unpack_params(flat.astype(np.float64))
    L, g = oracle.mlp_forward_backward_f64(Pf, X, y, w)
    assert abs(loss[0] - L) <= 1e-4 * abs(L) + 1e-5
    G = rv.unpack_params(grad)
    for k in g:
        scale = np.abs(g[k]).max()
        assert np.abs(G[k] - g[k]).max() <= 1e-5 + 2e-3 * scale, k


def test_training_kernel_reduces_loss(gpu_lib):
    rng = np.random.default_rng(7)
    n = 20000
    X = rng.normal(0, 1, (n, 4)).astype(np.float32)
    y = (3 + 1.5 * X[:, 0] - 0.7 * X[:, 1] * X[:, 2] + 0.2 * rng.normal(size=n)).astype(np.float32)
    p = rv.pack_params(_rand_params(rng, 0.2))
    losses = np.zeros(15, np.float32)
    rv.check(rv.lib().rvsp_cuda_mlp_train(p.ctypes.data, X.ctypes.data, y.ctypes.data, None, n, 15,
                                          1024, 3e-3, 11, losses.ctypes.data))
    assert losses[-1] < losses[0] - 1.0
    L, _ = oracle.mlp_forward_backward_f64(rv.unpack_params(p.astype(np.float64)), X, y,
                                           np.ones(n))
    assert abs(L - losses[-1]) < 0.5


def test_inference_kernel_matches_fp64_forward(gpu_lib):
    rng = np.random.default_rng(9)
    P = _rand_params(rng)
    mean, inv_std, z = rng.normal(0, 1, 4), rng.uniform(0.3, 1.0, 4), 1.5
    model = rv.model_to_vector(mean, inv_std, z, rv.pack_params(P))
    n = 3000
    feat = np.exp2(rng.uniform(0, 14, (n, 4))).astype(np.float32) - 1
    ub = rng.integers(0, 20000, n).astype(np.int32)
    mu = np.zeros(n, np.float32)
    sig = np.zeros(n, np.float32)
    cap = np.zeros(n, np.int32)
    rv.check(rv.lib().rvsp_cuda_mlp_infer(model.ctypes.data, rv.MLP_FLOATS, feat.ctypes.data,
                                          ub.ctypes.data, n, mu.ctypes.data, sig.ctypes.data,
                                          cap.ctypes.data))
    m = rv.model_from_vector(model)
    x = (np.log2(1.0 + feat.astype(np.float64)) - m[0]) * m[1]
    Pd = rv.unpack_params(m[3].astype(np.float64))
    h1 = np.maximum(x @ Pd["W1"].T + Pd["b1"], 0)
    h2 = np.maximum(h1 @ Pd["W2"].T + Pd["b2"], 0)
    o = h2 @ Pd["W3"].T + Pd["b3"]
    s = np.logaddexp(0, o[:, 1]) + 1e-3
    assert np.allclose(mu, o[:, 0], rtol=1e-4, atol=1e-4)
    assert np.allclose(sig, s, rtol=1e-4, atol=1e-5)
    e = np.minimum(mu.astype(np.float64) + m[2] * sig, 30.0)
    want = np.where(ub <= 0, 0, np.clip(np.ceil(np.exp2(e) - 1), 1, np.maximum(ub, 1)))
    # capacities agree except where exp2 rounding lands on an integer boundary
    assert (np.abs(cap - want) <= 1).all() and (cap == want).mean() > 0.99


def _constant_model(log2cap, sigma_raw=-20.0):
    """A model predicting the same capacity 2^log2cap - 1 for every row."""
    P = {k: np.zeros(v) for k, v in (("W1", (32, 4)), ("b1", 32), ("W2", (32, 32)), ("b2", 32),
                                     ("W3", (2, 32)), ("b3", 2))}
    P["b3"] = np.array([log2cap, sigma_raw])
    return rv.model_to_vector(np.zeros(4), np.ones(4), 0.0, rv.pack_params(P))


def _products():
    out = []
    R = gen.rmat(scale=12, edge_factor=12, seed=21)
    out.append(("rmat", R, R))
    rng = np.random.default_rng(4)
    A = gen.poisson_rows(3000, 3000, 20.0, rng)
    B = gen.poisson_rows(3000, 3000, 20.0, rng)
    out.append(("poisson20", A, B))
    A, B = gen.tall_skinny(a_rows=6000, k=5000, n=5000, b_max=3000, seed=8)
    out.append(("tall", A, B))
    out.append(("uniform", gen.uniform_fixed(1024, 1024, 16, seed=3), gen.uniform_fixed(1024, 1024, 16, seed=4)))
    return out


@pytest.mark.parametrize("log2cap", [1.0, 6.0, 30.0])
def test_learned_path_bit_exact_under_any_prediction(gpu_lib, log2cap):
    """Whatever the model predicts -- far too small (every predicted row
    overflows and is re-run exactly), mid-size, or far too large -- the
    learned path returns exactly the exact path's C."""
    L = rv.lib()
    saved = np.zeros(rv.MLP_FLOATS, np.float32)
    had = L.rvsp_cuda_mlp_get(saved.ctypes.data, rv.MLP_FLOATS) == 0
    try:
        m = _constant_model(log2cap)
        rv.check(L.rvsp_cuda_mlp_set(m.ctypes.data, rv.MLP_FLOATS))
        for name, A, B in _products():
            want = oneshot(A, B, algo=rv.RVSP_CUDA_ALGO_EXACT)
            got = oneshot(A, B, algo=rv.RVSP_CUDA_ALGO_LEARNED)
            assert np.array_equal(got[0], want[0]), name
            assert np.array_equal(got[1], want[1]), name
            assert np.array_equal(bits(got[2]), bits(want[2])), name
            host = oneshot(A, B, algo=rv.RVSP_CUDA_ALGO_LEARNED, device=False)
            assert np.array_equal(bits(host[2]), bits(want[2])), name
    finally:
        if had:
            L.rvsp_cuda_mlp_set(saved.ctypes.data, rv.MLP_FLOATS)


def test_learned_descriptor_matches_exact(gpu_lib):
    L = rv.lib()
    saved = np.zeros(rv.MLP_FLOATS, np.float32)
    had = L.rvsp_cuda_mlp_get(saved.ctypes.data, rv.MLP_FLOATS) == 0
    try:
        rv.check(L.rvsp_cuda_mlp_set(_constant_model(7.0).ctypes.data, rv.MLP_FLOATS))
        for name, A, B in _products():
            dA, dB = DevCSR(A), DevCSR(B)
            pe = rv.Plan(rv.RVSP_CUDA_ALGO_EXACT)
            pl = rv.Plan(rv.RVSP_CUDA_ALGO_LEARNED)
            st, n_e = pe.symbolic(dA, dB, A.nnz, B.nnz)
            rv.check(st)
            st, n_l = pl.symbolic(dA, dB, A.nnz, B.nnz)
            rv.check(st)
            assert n_e == n_l, name
            stats = pl.learned_stats()
            assert stats["exact_rows"] <= A.rows, name
            d = rv.Descriptor(rv.RVSP_SPGEMM_ALGO_CUDA_LEARNED)
            st, ws, nnz = d.work_estimation(dA.struct(), dB.struct())
            rv.check(st)
            assert nnz == n_e
            import torch
            crp = torch.zeros(A.rows + 1, dtype=torch.int32, device="cuda")
            cci = torch.zeros(max(nnz, 1), dtype=torch.int32, device="cuda")
            cv = torch.zeros(max(nnz, 1), dtype=torch.float32, device="cuda")
            c = rv.csr_struct(A.rows, B.cols, nnz, crp, cci, cv)
            rv.check(d.compute(dA.struct(), dB.struct(), c, np.zeros(16, np.uint8)))
            wrp, wci, wv = oracle.spgemm_f32(A, B)
            assert np.array_equal(crp.cpu().numpy(), wrp), name
            assert np.array_equal(cci.cpu().numpy()[:nnz], wci), name
            assert np.array_equal(bits(cv.cpu().numpy()[:nnz]), bits(wv)), name
            d.close()
            pe.close()
            pl.close()
    finally:
        if had:
            L.rvsp_cuda_mlp_set(saved.ctypes.data, rv.MLP_FLOATS)


@pytest.mark.skipif(not os.path.exists(SHIPPED), reason="no trained checkpoint shipped yet")
def test_trained_model_gains_over_upper_bound(gpu_lib):
    """What the trained network buys over sizing by the upper bound
    min(products, cols) alone: on products where that bound is loose (a banded
    product, where many products land on the same columns, and an R-MAT graph)
    the rows it sizes get tables and slots far below their bound, few of them
    outgrow the prediction, and C is unchanged."""
    L = rv.lib()
    assert L.rvsp_cuda_mlp_load(SHIPPED.encode()) == 0
    rng = np.random.default_rng(8)
    n = 40000
    rows = np.repeat(np.arange(n), 24)
    cols = np.clip(rows + rng.integers(-16, 17, rows.size), 0, n - 1)
    band = gen.from_keys(n, n, np.unique(rows.astype(np.int64) * n + cols), None, rng)
    R = gen.rmat(scale=14, edge_factor=16, seed=99)
    # band: many products share columns (bound >> nnz); R-MAT: moderate
    for name, M, ratio in (("band16", band, 0.8), ("rmat14", R, 0.95)):
        dM = DevCSR(M)
        p = rv.Plan(rv.RVSP_CUDA_ALGO_LEARNED)
        st, nnz = p.symbolic(dM, dM, M.nnz, M.nnz)
        rv.check(st)
        s = p.learned_stats()
        p.close()
        pred = s["predicted_rows"]
        assert pred > 0, (name, s)
        assert s["overflowed_rows"] / pred < 0.10, (name, s)
        assert s["fit_capacity"] < ratio * s["fit_upper_bound"], (name, s)
        want = oneshot(M, M, algo=rv.RVSP_CUDA_ALGO_EXACT)
        got = oneshot(M, M, algo=rv.RVSP_CUDA_ALGO_LEARNED)
        assert np.array_equal(got[1], want[1]) and np.array_equal(bits(got[2]), bits(want[2]))


@pytest.mark.skipif(not os.path.exists(SHIPPED), reason="no trained checkpoint shipped yet")
def test_trained_model_saves_time_on_a_power_law_product(gpu_lib):
    """What the trained network gains in time: on a power-law product (a row
    panel of R-MAT 2^18, heavy rows holding almost every product) the learned
    path fills C in one sweep into slots the network sizes, so it skips the
    count pass the exact path makes, and must finish faster (median of 5 one-
    shot products each) with C bit-identical. Without the network the only
    safe slot of a row is its upper bound min(products, cols): the predicted
    slots must take less (fit_capacity below fit_upper_bound)."""
    import time

    import torch

    from rvsp_b200 import ranks
    L = rv.lib()
    assert L.rvsp_cuda_mlp_load(SHIPPED.encode()) == 0
    R = gen.rmat(scale=18, edge_factor=16, seed=0)
    ops = gen.row_products(R, R)
    r0, r1 = ranks.row_panels(ops)[0]
    dR = DevCSR(R)

    def run(algo):
        import ctypes as C
        prp, pci, pv = C.c_void_p(), C.c_void_p(), C.c_void_p()
        nnz = C.c_int32()
        rv.check(L.rvsp_cuda_spgemm_f32(algo, r1 - r0, R.cols, R.cols,
                                        rv.ptr(dR.row_ptr[r0:r1 + 1]), rv.ptr(dR.col_idx),
                                        rv.ptr(dR.values), rv.ptr(dR.row_ptr), rv.ptr(dR.col_idx),
                                        rv.ptr(dR.values), C.byref(prp), C.byref(pci),
                                        C.byref(pv), C.byref(nnz), None))
        return (prp.value, pci.value, pv.value), nnz.value

    from gpu_util import d2h
    times, outs = {}, {}
    for algo in (rv.RVSP_CUDA_ALGO_EXACT, rv.RVSP_CUDA_ALGO_LEARNED):
        rv.free_device(*run(algo)[0])  # warm-up
        ts = []
        for _ in range(5):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ptrs, n = run(algo)
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
            outs[algo] = (d2h(ptrs[1], n, np.int32), d2h(ptrs[2], n, np.float32))
            rv.free_device(*ptrs)
        times[algo] = float(np.median(ts))
    assert np.array_equal(outs[rv.RVSP_CUDA_ALGO_EXACT][0], outs[rv.RVSP_CUDA_ALGO_LEARNED][0])
    assert np.array_equal(bits(outs[rv.RVSP_CUDA_ALGO_EXACT][1]),
                          bits(outs[rv.RVSP_CUDA_ALGO_LEARNED][1]))
    s = rv.oneshot_learned_stats()
    print(f"exact {times[rv.RVSP_CUDA_ALGO_EXACT] * 1e3:.2f} ms, learned "
          f"{times[rv.RVSP_CUDA_ALGO_LEARNED] * 1e3:.2f} ms, stats {s}")
    assert times[rv.RVSP_CUDA_ALGO_LEARNED] < times[rv.RVSP_CUDA_ALGO_EXACT]
    assert s["predicted_rows"] > 0 and s["fit_capacity"] < s["fit_upper_bound"]
