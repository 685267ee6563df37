"""The benchmark's roofline arithmetic on CPU: the algorithmic bytes of the
headline product (the per-unit byte formula of the hot path, every operand
array read once and C written once) and the exact sizes of the Poisson 1024^2
product it is quoted on."""

import importlib.util
import os

import numpy as np

from rvsp_b200 import gen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_algorithmic_bytes_of_the_poisson_product():
    bench = _bench()
    A = gen.poisson2d(1024)
    assert (A.rows, A.nnz) == (1_048_576, 5_238_784)
    assert gen.products(A, A) == 26_177_544
    nnz_c = 13_611_012  # nnz(C) of A * A, pinned by the reference's output digest
    b = bench.algorithmic_bytes(A.rows, A.nnz, nnz_c, A.rows, A.nnz)
    assert b == 4 * (A.rows + 1) * 3 + 8 * (2 * A.nnz + nnz_c) == 205_291_564


def test_nnz_of_the_poisson_product_from_the_oracle():
    import oracle
    A = gen.poisson2d(64)
    rp, ci, v = oracle.spgemm_f32(A, A)
    # interior rows of the 5-point stencil squared reach 13 columns
    lens = np.diff(np.asarray(rp, np.int64))
    assert lens.max() == 13 and lens.min() == 6
