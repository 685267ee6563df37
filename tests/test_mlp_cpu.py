"""The FP64 MLP oracle (gradient reference for the training kernels) pinned by
finite differences, and the checkpoint format round trip (CPU only)."""

import os

import numpy as np

import oracle
import rvsp_b200 as rv


def _rand_params(rng, scale=0.3):
    return {"W1": rng.normal(0, scale, (32, 4)), "b1": rng.normal(0, 0.1, 32),
            "W2": rng.normal(0, scale, (32, 32)), "b2": rng.normal(0, 0.1, 32),
            "W3": rng.normal(0, scale, (2, 32)), "b3": rng.normal(0, 0.1, 2)}


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    P = _rand_params(rng)
    X = rng.normal(0, 1, (40, 4))
    y = rng.uniform(0, 8, 40)
    w = rng.uniform(0.5, 1.5, 40)
    L0, g = oracle.mlp_forward_backward_f64(P, X, y, w)
    eps = 1e-6
    for name in ("W1", "b1", "W2", "b2", "W3", "b3"):
        flat = P[name].ravel()
        for idx in rng.choice(flat.size, min(6, flat.size), replace=False):
            Q = {k: v.copy() for k, v in P.items()}
            Q[name].ravel()[idx] += eps
            Lp, _ = oracle.mlp_forward_backward_f64(Q, X, y, w)
            Q[name].ravel()[idx] -= 2 * eps
            Lm, _ = oracle.mlp_forward_backward_f64(Q, X, y, w)
            fd = (Lp - Lm) / (2 * eps)
            assert abs(fd - g[name].ravel()[idx]) <= 1e-6 + 1e-4 * abs(fd), (name, idx)


def test_checkpoint_round_trip(tmp_path):
    L = rv.lib()
    rng = np.random.default_rng(1)
    params = rv.pack_params(_rand_params(rng))
    model = rv.model_to_vector(rng.normal(size=4), rng.uniform(0.5, 2, 4), 1.7, params)
    path = str(tmp_path / "m.bin")
    assert L.rvsp_cuda_mlp_save(path.encode(), model.ctypes.data, rv.MLP_FLOATS) == 0
    assert L.rvsp_cuda_mlp_save(path.encode(), model.ctypes.data, 7) == rv.RVSP_ERROR_INVALID_ARGUMENT
    assert L.rvsp_cuda_mlp_load(path.encode()) == 0
    got = np.zeros(rv.MLP_FLOATS, np.float32)
    assert L.rvsp_cuda_mlp_get(got.ctypes.data, rv.MLP_FLOATS) == 0
    assert np.array_equal(got, model)
    # a corrupted file is rejected and leaves the loaded model in place
    raw = bytearray(open(path, "rb").read())
    raw[100] ^= 0xFF
    bad = str(tmp_path / "bad.bin")
    open(bad, "wb").write(bytes(raw))
    assert L.rvsp_cuda_mlp_load(bad.encode()) == rv.RVSP_ERROR_INVALID_ARGUMENT
    assert L.rvsp_cuda_mlp_load(str(tmp_path / "missing.bin").encode()) == rv.RVSP_ERROR_INVALID_ARGUMENT
    assert L.rvsp_cuda_mlp_get(got.ctypes.data, rv.MLP_FLOATS) == 0 and np.array_equal(got, model)
    # restore the shipped checkpoint if there is one
    shipped = os.path.join(rv.PKG_DIR, "weights", "row_mlp_v1.bin")
    if os.path.exists(shipped):
        assert L.rvsp_cuda_mlp_load(shipped.encode()) == 0


def test_shipped_checkpoint_is_valid():
    shipped = os.path.join(rv.PKG_DIR, "weights", "row_mlp_v1.bin")
    if not os.path.exists(shipped):
        import pytest
        pytest.skip("no trained checkpoint shipped yet")
    L = rv.lib()
    assert L.rvsp_cuda_mlp_load(shipped.encode()) == 0
    assert L.rvsp_cuda_learned_available() == 1
    m = np.zeros(rv.MLP_FLOATS, np.float32)
    assert L.rvsp_cuda_mlp_get(m.ctypes.data, rv.MLP_FLOATS) == 0
    mean, inv_std, z, params = rv.model_from_vector(m)
    assert np.isfinite(m).all() and (inv_std > 0).all() and 0.0 < z < 10.0
