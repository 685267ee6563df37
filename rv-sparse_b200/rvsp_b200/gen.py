"""Seeded synthetic CSR generators for the SpGEMM workloads.

All generators return canonical CSR (row_ptr from 0, non-decreasing, columns
strictly ascending within a row, in range) with int32 indices and FP32
values, the input contract of rv-sparse (docs/api_design.md:11-14).

Workloads (sizes are the defaults; every generator takes smaller sizes for
tests):

* ``uniform_fixed``   M x N, exactly ``per_row`` distinct uniform columns per
  row, values U(-1, 1).  4096^2, 16 per row, seed 0 is the plain C = A * A case.
* ``poisson2d``       5-point Laplacian on an n x n grid (4 on the diagonal,
  -1 on the four neighbours), N = n^2.
* ``rmat``            R-MAT graph, 2^scale nodes, ``edge_factor * 2^scale``
  edge samples with quadrant probabilities (a, b, c, d); duplicate edges are
  merged, self loops kept, no noise; values U(-1, 1).
* ``poisson_rows``    nnz per row ~ Poisson(lam) (capped at the column count),
  distinct uniform columns; used for the batched uneven products.
* ``tall_skinny``     A rows with geometric(mean 8) nnz and uniform columns;
  B rows with a truncated power-law length distribution (mean about 24, the
  longest row drawing ``b_max`` columns), uniform columns with repeats merged.

Columns that a row draws twice are merged; rows that must hold an exact count
are topped up until they do.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class CSR:
    rows: int
    cols: int
    row_ptr: np.ndarray  # int32[rows + 1]
    col_idx: np.ndarray  # int32[nnz]
    values: np.ndarray  # float32[nnz]

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1])

    def row_lengths(self) -> np.ndarray:
        return np.diff(self.row_ptr.astype(np.int64))


def from_keys(rows: int, cols: int, keys: np.ndarray, values: np.ndarray | None,
              rng: np.random.Generator | None) -> CSR:
    """Builds CSR from sorted unique int64 keys row * cols + col."""
    r = (keys // cols).astype(np.int64)
    c = (keys % cols).astype(np.int32)
    counts = np.bincount(r, minlength=rows)
    rp = np.zeros(rows + 1, np.int64)
    np.cumsum(counts, out=rp[1:])
    if rp[-1] > np.iinfo(np.int32).max:
        raise ValueError("nnz exceeds int32")
    if values is None:
        values = rng.uniform(-1.0, 1.0, size=keys.size).astype(np.float32)
    return CSR(rows, cols, rp.astype(np.int32), c, values.astype(np.float32))


def _sorted_unique(x: np.ndarray) -> np.ndarray:
    """np.unique(x) by sorting (the same array; numpy's hash-based unique is
    much slower on tens of millions of int64 keys)."""
    x = np.sort(x)
    if x.size > 1:
        keep = np.empty(x.size, bool)
        keep[0] = True
        np.not_equal(x[1:], x[:-1], out=keep[1:])
        x = x[keep]
    return x


def _distinct_rows(counts: np.ndarray, cols: int, rng: np.random.Generator,
                   exact: bool = True) -> np.ndarray:
    """Sorted unique keys row*cols+col with counts[r] distinct uniform columns per row."""
    counts = np.minimum(counts.astype(np.int64), cols)
    rows = counts.size
    keys = np.empty(0, np.int64)
    need = counts.copy()
    for _ in range(64):
        tot = int(need.sum())
        if tot == 0:
            break
        r = np.repeat(np.arange(rows, dtype=np.int64), need)
        new = r * cols + rng.integers(0, cols, size=tot, dtype=np.int64)
        keys = _sorted_unique(np.concatenate([keys, new]))
        if not exact:
            break
        have = np.bincount(keys // cols, minlength=rows)
        need = counts - have
    return keys


def uniform_fixed(rows: int = 4096, cols: int = 4096, per_row: int = 16, seed: int = 0) -> CSR:
    rng = np.random.default_rng(seed)
    keys = _distinct_rows(np.full(rows, per_row), cols, rng)
    return from_keys(rows, cols, keys, None, rng)


def poisson2d(n: int = 1024) -> CSR:
    N = n * n
    idx = np.arange(N, dtype=np.int64)
    i, j = idx // n, idx % n
    parts_c = []
    parts_v = []
    parts_r = []
    for di, dj, val in ((-1, 0, -1.0), (0, -1, -1.0), (0, 0, 4.0), (0, 1, -1.0), (1, 0, -1.0)):
        ok = (i + di >= 0) & (i + di < n) & (j + dj >= 0) & (j + dj < n)
        parts_r.append(idx[ok])
        parts_c.append(idx[ok] + di * n + dj)
        parts_v.append(np.full(int(ok.sum()), val, np.float32))
    keys = np.concatenate(parts_r) * N + np.concatenate(parts_c)
    vals = np.concatenate(parts_v)
    order = np.argsort(keys, kind="stable")
    return from_keys(N, N, keys[order], vals[order], None)


def rmat(scale: int = 20, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
         c: float = 0.19, seed: int = 0) -> CSR:
    rng = np.random.default_rng(seed)
    n = 1 << scale
    E = edge_factor * n
    row = np.zeros(E, np.int64)
    col = np.zeros(E, np.int64)
    chunk = 1 << 22
    for lo in range(0, E, chunk):
        hi = min(E, lo + chunk)
        rr = np.zeros(hi - lo, np.int64)
        cc = np.zeros(hi - lo, np.int64)
        for bit in range(scale):
            u = rng.random(hi - lo)
            rbit = u >= a + b
            cbit = ((u >= a) & (u < a + b)) | (u >= a + b + c)
            rr |= rbit.astype(np.int64) << bit
            cc |= cbit.astype(np.int64) << bit
        row[lo:hi] = rr
        col[lo:hi] = cc
    keys = _sorted_unique(row * n + col)
    return from_keys(n, n, keys, None, rng)


def poisson_rows(rows: int, cols: int, lam: float, rng: np.random.Generator) -> CSR:
    counts = np.minimum(rng.poisson(lam, size=rows), cols)
    keys = _distinct_rows(counts, cols, rng)
    return from_keys(rows, cols, keys, None, rng)


def batched_uneven(count: int = 512, lo: int = 256, hi: int = 65536, lam_lo: float = 4.0,
                   lam_hi: float = 32.0, seed: int = 0):
    """`count` independent (A, B) pairs, M = K = N log-uniform in [lo, hi]."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(lo), math.log(hi), size=count)).astype(np.int64)
    lams = rng.uniform(lam_lo, lam_hi, size=count)
    out = []
    for n, lam in zip(sizes.tolist(), lams.tolist()):
        A = poisson_rows(n, n, lam, rng)
        B = poisson_rows(n, n, lam, rng)
        out.append((A, B))
    return out


def _powerlaw_lengths(rows: int, mean: float, max_len: int, cols: int,
                      rng: np.random.Generator, beta: float = 1.1) -> np.ndarray:
    """Truncated Pareto row lengths, xmin fitted so the mean is about `mean`."""
    u = rng.random(rows)
    lo, hi = 0.01, float(mean)
    for _ in range(60):
        xmin = 0.5 * (lo + hi)
        L = np.clip(np.floor(xmin * u ** (-1.0 / beta)), 1, max_len)
        if L.mean() < mean:
            lo = xmin
        else:
            hi = xmin
    L = np.clip(np.floor(xmin * u ** (-1.0 / beta)), 1, min(max_len, cols)).astype(np.int64)
    L[int(np.argmax(L))] = min(max_len, cols)
    return L


def tall_skinny(a_rows: int = 2_000_000, k: int = 100_000, n: int = 100_000,
                a_mean: float = 8.0, b_mean: float = 24.0, b_max: int = 20_000, seed: int = 0):
    rng = np.random.default_rng(seed)
    a_counts = np.minimum(rng.geometric(1.0 / a_mean, size=a_rows), k)
    A = from_keys(a_rows, k, _distinct_rows(a_counts, k, rng, exact=False), None, rng)
    b_counts = _powerlaw_lengths(k, b_mean, b_max, n, rng)
    B = from_keys(k, n, _distinct_rows(b_counts, n, rng, exact=False), None, rng)
    return A, B


def products(A: CSR, B: CSR) -> int:
    """Intermediate products sum_i sum_{k in A_i} len(B_k) (rv-sparse bench/bench.c:215-240)."""
    blen = np.diff(B.row_ptr.astype(np.int64))
    return int(blen[A.col_idx].sum()) if A.nnz else 0


def row_products(A: CSR, B: CSR) -> np.ndarray:
    blen = np.diff(B.row_ptr.astype(np.int64))
    per = blen[A.col_idx] if A.nnz else np.zeros(0, np.int64)
    if not A.nnz:
        return np.zeros(A.rows, np.int64)
    rows = np.repeat(np.arange(A.rows), np.diff(A.row_ptr.astype(np.int64)))
    return np.bincount(rows, weights=per, minlength=A.rows).astype(np.int64)


def scale_values(M: CSR, rng: np.random.Generator, lo: float = 0.5, hi: float = 1.5) -> CSR:
    """Same pattern, values multiplied entry-wise by U(lo, hi)."""
    s = rng.uniform(lo, hi, size=M.nnz).astype(np.float32)
    return CSR(M.rows, M.cols, M.row_ptr, M.col_idx, (M.values * s).astype(np.float32))
