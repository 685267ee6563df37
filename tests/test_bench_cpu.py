"""The benchmark's host logic on CPU: the algorithmic bytes of a product
(the per-unit byte formula of the hot path, every operand array read once and
C written once) on the Poisson 1024^2 product, the heavy-row rule behind the
roofline's byte count, the row sample of the CPU baselines, and the reference
arm's JSON line on the R-MAT 2^20 headline product."""

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


def test_reference_arm_prints_one_contract_line():
    """`bench.py --impl reference` times the reference's own CPU numeric pass
    (compiled from its sources) on the headline workload and prints one JSON
    line with the same metric and unit as the CUDA arm."""
    import json
    import subprocess
    import sys

    import oracle
    if not oracle.ref_available():
        import pytest
        pytest.skip("reference library not built")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "3"], capture_output=True, text=True,
                         timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    bench = _bench()
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["higher_is_better"] is True and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    assert d["config"]["workload"] == "rmat_scale20_ef16_c_eq_a_times_a"
    assert d["config"]["products"] == 20_936_185_642


def test_heavy_row_rule_matches_the_bins():
    """bench.heavy_rows restates the library's bin rule (spgemm_types.cuh
    table_bin / bin_of) for the roofline's byte count: a row is heavy when it
    has more products than the tiny bin and its table ub + (ub >> 2) passes
    the 2048-slot warp table."""
    bench = _bench()
    ops = np.array([0, 32, 33, 1638, 1639, 2000, 10**9])
    # ub = min(ops, cols); 1638 + 409 = 2047 fits, 1639 + 409 = 2048 fits,
    # 2000 + 500 > 2048 does not
    assert bench.heavy_rows(ops, 1 << 20).tolist() == [False, False, False, False, False,
                                                       True, True]
    assert bench.heavy_rows(ops, 1000).tolist() == [False] * 7


def test_row_sample_is_a_csr_of_the_sampled_rows():
    bench = _bench()
    A = gen.rmat(scale=10, edge_factor=16, seed=0)
    ops = gen.row_products(A, A)
    S, Ps, rows = bench.row_sample(A, ops, 0.2, 5)
    assert S.rows == rows.size and np.all(np.diff(rows) > 0)
    for i, r in enumerate(rows[:50]):
        a, b = A.row_ptr[r], A.row_ptr[r + 1]
        assert np.array_equal(S.col_idx[S.row_ptr[i]:S.row_ptr[i + 1]], A.col_idx[a:b])
        assert np.array_equal(S.values[S.row_ptr[i]:S.row_ptr[i + 1]], A.values[a:b])
    assert Ps == int(ops[rows].sum())


def test_each_rank_takes_its_own_visible_gpu():
    """Under a launcher (WORLD_SIZE > 1) a rank keeps only the LOCAL_RANK-th
    of the GPUs already visible to it (or GPU LOCAL_RANK when none are
    named), before anything loads CUDA."""
    import subprocess
    import sys
    code = "import os, bench; print(os.environ['CUDA_VISIBLE_DEVICES'])"
    for visible, rank, want in (("4,5", "1", "5"), ("", "1", "1"), ("2,3,6", "0", "2")):
        env = dict(os.environ, WORLD_SIZE="2", RANK=rank, LOCAL_RANK=rank,
                   CUDA_VISIBLE_DEVICES=visible)
        out = subprocess.run([sys.executable, "-c", code], env=env, cwd=ROOT,
                             capture_output=True, text=True, timeout=300)
        assert out.returncode == 0, out.stderr[-500:]
        assert out.stdout.strip().splitlines()[-1] == want
