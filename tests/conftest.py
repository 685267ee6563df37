"""Shared test setup: import paths, the gpu marker, golden fixtures.

Tests marked ``gpu`` need a CUDA device and the built librvsp_b200.so; the
rest run on CPU (oracle checks, host-side logic, symbol exports).
"""

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "rv-sparse_b200"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


class Mat:
    """Plain CSR holder for fixtures (rows, cols, row_ptr, col_idx, values)."""

    def __init__(self, rows, cols, row_ptr, col_idx, values):
        self.rows, self.cols = int(rows), int(cols)
        self.row_ptr = np.ascontiguousarray(row_ptr, np.int32)
        self.col_idx = np.ascontiguousarray(col_idx, np.int32)
        self.values = np.ascontiguousarray(values, np.float32)

    @property
    def nnz(self):
        return int(self.row_ptr[-1])


def load_fixtures():
    """The six hand-computed triples of rv-sparse tests/csr_fixtures.h."""
    with open(os.path.join(GOLDEN, "csr_fixtures.json")) as f:
        data = json.load(f)["pairs"]
    out = []
    for p in data:
        mk = lambda d: Mat(d["rows"], d["cols"], d["row_ptr"], d["col_idx"], d["values"])  # noqa: E731
        out.append((p["name"], mk(p["a"]), mk(p["b"]), mk(p["c"])))
    return out


def load_ref_cases():
    """Seeded products with the reference scalar kernel's outputs."""
    meta = json.load(open(os.path.join(GOLDEN, "ref_outputs.json")))
    z = np.load(os.path.join(GOLDEN, "ref_outputs.npz"))
    out = []
    for name, info in meta["cases"].items():
        A = Mat(info["a"][0], info["a"][1], z[f"{name}.a.row_ptr"], z[f"{name}.a.col_idx"],
                z[f"{name}.a.values"])
        B = Mat(info["b"][0], info["b"][1], z[f"{name}.b.row_ptr"], z[f"{name}.b.col_idx"],
                z[f"{name}.b.values"])
        Cc = (z[f"{name}.c.row_ptr"], z[f"{name}.c.col_idx"], z[f"{name}.c.values"])
        out.append((name, A, B, Cc, z[f"{name}.ops"]))
    return out


def ref_digests():
    return json.load(open(os.path.join(GOLDEN, "ref_outputs.json")))["digests"]


@pytest.fixture(scope="session")
def fixtures():
    return load_fixtures()


@pytest.fixture(scope="session")
def ref_cases():
    return load_ref_cases()


def have_gpu():
    try:
        import rvsp_b200
        return os.path.exists(rvsp_b200.LIB_PATH) and rvsp_b200.device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_lib():
    import rvsp_b200
    if not os.path.exists(rvsp_b200.LIB_PATH):
        pytest.fail("librvsp_b200.so not built (make -C rv-sparse_b200)")
    if rvsp_b200.device_count() == 0:
        pytest.skip("no CUDA device")
    return rvsp_b200


class TypedMat:
    """CSR with values of any dtype (the legacy FP64 / INT8 products)."""

    def __init__(self, rows, cols, row_ptr, col_idx, values):
        self.rows, self.cols = int(rows), int(cols)
        self.row_ptr = np.ascontiguousarray(row_ptr, np.int32)
        self.col_idx = np.ascontiguousarray(col_idx, np.int32)
        self.values = np.ascontiguousarray(values)

    @property
    def nnz(self):
        return int(self.row_ptr[-1])


def typed_pair(A, B, dtype, seed=0):
    """A and B's structure with values drawn from a small set, so that some
    output sums cancel to exactly zero (dtype "f64": +-{0.5, 1, 2}, "i8":
    -3..3 without 0, and a few -128/127 entries)."""
    rng = np.random.default_rng(seed)

    def vals(n):
        if dtype == "f64":
            return rng.choice([-2.0, -1.0, -0.5, 0.5, 1.0, 2.0], n).astype(np.float64)
        v = rng.choice([-3, -2, -1, 1, 2, 3], n).astype(np.int8)
        if n:
            v[rng.integers(0, n, max(1, n // 500))] = rng.choice([-128, 127])
        return v

    return (TypedMat(A.rows, A.cols, A.row_ptr, A.col_idx, vals(A.nnz)),
            TypedMat(B.rows, B.cols, B.row_ptr, B.col_idx, vals(B.nnz)))


def write_mtx(path, rows, cols, entries, field="real", symmetry="general", declared=None):
    """A Matrix Market file; entries are (row, col[, value]) 1-based, value a
    string written as is."""
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate {field} {symmetry}\n")
        f.write("% written by the tests\n%\n")
        f.write(f"{rows} {cols} {len(entries) if declared is None else declared}\n")
        for e in entries:
            f.write(" ".join(str(x) for x in e) + "\n")


def mtx_cases(tmpdir, seed=0):
    """Seeded files: general real with repeated entries (pairs and triples),
    symmetric real, pattern general, and a short file (fewer entries than declared)."""
    rng = np.random.default_rng(seed)
    out = []
    rows, cols = 300, 200
    n = 4000
    r = rng.integers(1, rows + 1, n)
    c = rng.integers(1, cols + 1, n)
    dup = rng.integers(0, n, 300)  # repeat some entries once or twice more
    r = np.concatenate([r, r[dup], r[dup[:100]]])
    c = np.concatenate([c, c[dup], c[dup[:100]]])
    vals = [f"{x:.7g}" for x in rng.uniform(-10, 10, r.size)]
    perm = rng.permutation(r.size)
    ents = [(int(r[i]), int(c[i]), vals[i]) for i in perm]
    p = os.path.join(tmpdir, "general.mtx")
    write_mtx(p, rows, cols, ents)
    out.append(("general", p))
    m = 250
    rr = rng.integers(1, m + 1, 3000)
    cc = rng.integers(1, m + 1, 3000)
    lo, hi = np.minimum(rr, cc), np.maximum(rr, cc)
    ents = [(int(hi[i]), int(lo[i]), f"{rng.uniform(-1, 1):.6e}") for i in range(rr.size)]
    p = os.path.join(tmpdir, "symmetric.mtx")
    write_mtx(p, m, m, ents, symmetry="symmetric")
    out.append(("symmetric", p))
    ents = [(int(rng.integers(1, 120)), int(rng.integers(1, 90))) for _ in range(900)]
    p = os.path.join(tmpdir, "pattern.mtx")
    write_mtx(p, 119, 89, ents, field="pattern")
    out.append(("pattern", p))
    ents = [(1, 1, "2.5"), (3, 2, "-1"), (3, 2, "4")]
    p = os.path.join(tmpdir, "short.mtx")
    write_mtx(p, 3, 3, ents, declared=10)
    out.append(("short", p))
    return out
