"""The seeded synthetic inputs stand in for the benchmark configurations: each
generator's output is canonical CSR with the sizes and value distributions the
configurations name (checked here at reduced sizes where the full ones take
long to generate)."""

import numpy as np

from rvsp_b200 import gen


def _canonical(M):
    rp = M.row_ptr.astype(np.int64)
    assert rp[0] == 0 and np.all(np.diff(rp) >= 0) and rp[-1] == M.col_idx.size == M.values.size
    assert M.row_ptr.dtype == np.int32 and M.col_idx.dtype == np.int32 and M.values.dtype == np.float32
    if M.col_idx.size:
        assert M.col_idx.min() >= 0 and M.col_idx.max() < M.cols
        r = np.repeat(np.arange(M.rows), np.diff(rp))
        same_row = r[1:] == r[:-1]
        assert np.all(np.diff(M.col_idx.astype(np.int64))[same_row] > 0)  # strictly ascending


def test_plain_exactly_16_distinct_per_row_seeded():
    A = gen.uniform_fixed()
    _canonical(A)
    assert (A.rows, A.cols) == (4096, 4096)
    assert np.all(A.row_lengths() == 16)
    assert A.values.min() >= -1.0 and A.values.max() < 1.0
    assert gen.products(A, A) == 1_048_576
    B = gen.uniform_fixed()
    assert np.array_equal(A.col_idx, B.col_idx) and np.array_equal(A.values, B.values)


def test_poisson_stencil_sizes_and_values():
    A = gen.poisson2d(1024)
    _canonical(A)
    assert (A.rows, A.nnz) == (1_048_576, 5_238_784)
    assert set(np.unique(A.values).tolist()) == {-1.0, 4.0}
    assert gen.products(A, A) == 26_177_544


def test_rmat_quadrants_and_canonical():
    R = gen.rmat(scale=12, edge_factor=16)
    _canonical(R)
    assert R.rows == R.cols == 4096
    assert 0.7 * 16 * 4096 < R.nnz <= 16 * 4096  # duplicates merged
    # a = 0.57 puts most edges in the top-left quadrant at every level
    half = R.rows // 2
    rows = np.repeat(np.arange(R.rows), R.row_lengths())
    top_left = np.mean((rows < half) & (R.col_idx < half))
    assert 0.45 < top_left < 0.75
    lens = R.row_lengths()
    assert lens.max() > 20 * lens.mean()  # power-law: hub rows


def test_batched_sizes_log_uniform_and_poisson_rows():
    pairs = gen.batched_uneven(count=8, hi=4096)
    assert len(pairs) == 8
    for A, B in pairs:
        _canonical(A)
        _canonical(B)
        assert A.rows == A.cols == B.rows == B.cols
        assert 256 <= A.rows <= 4096
        assert 2.0 <= A.row_lengths().mean() <= 40.0


def test_tall_skinny_shapes_and_row_lengths():
    A, B = gen.tall_skinny(a_rows=200_000, k=20_000, n=20_000, b_max=6000, seed=3)
    _canonical(A)
    _canonical(B)
    assert (A.rows, A.cols, B.rows, B.cols) == (200_000, 20_000, 20_000, 20_000)
    assert 7.0 < A.row_lengths().mean() < 9.0  # geometric, mean 8
    lb = B.row_lengths()
    # power law, mean about 24; the longest row draws b_max columns, of which
    # repeats are merged
    assert 0.8 * 6000 < lb.max() <= 6000 and 15.0 < lb.mean() < 35.0
