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


def _e2e_worker(rank, port, world, out_dir):
    """One rank of the end-to-end leg with the library replaced by a stand-in
    that returns a C of 10 entries a panel and takes rank-dependent time."""
    import ctypes as C
    import json
    import time
    import types

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      LOCAL_RANK=str(rank), WORLD_SIZE=str(world))
    import rvsp_b200 as rv
    from rvsp_b200 import ranks
    bench = _bench()
    dist = ranks.init("gloo", timeout_s=120)

    class FakeLib:
        def rvsp_spgemm_csr(self, a, b, c, opts):
            time.sleep(0.01 * (rank + 1))
            c._obj.nnz = 10
            return 0

        def rvsp_csr_destroy(self, c):
            return 0

    fake = FakeLib()
    rvf = types.SimpleNamespace(lib=lambda: fake, csr_struct=rv.csr_struct,
                                SpgemmOptions=rv.SpgemmOptions, CsrMatrix=rv.CsrMatrix,
                                check=rv.check,
                                RVSP_BACKEND_CUDA_LEARNED=rv.RVSP_BACKEND_CUDA_LEARNED,
                                RVSP_DTYPE_FP32=rv.RVSP_DTYPE_FP32)
    A = gen.rmat(scale=12, edge_factor=16, seed=5)
    ops = gen.row_products(A, A)
    panels_all = [(0, 64), (64, 128), (128, 200), (200, A.rows)]
    panels = ranks.shard_panels(panels_all, ops, rank, world)
    args = types.SimpleNamespace(steps=2, e2e_steps=2)
    r = bench.run_rmat_e2e(rvf, A, ops, panels, args, None, dist)
    with open(os.path.join(out_dir, f"e2e_{rank}.json"), "w") as f:
        json.dump({"r": r, "panels": panels}, f)
    ranks.barrier(dist)
    dist.destroy_process_group()


def test_e2e_leg_reports_the_whole_job_over_two_ranks(tmp_path):
    """With two ranks the end-to-end number covers every rank's panels: the
    products and bytes of both, over the slower rank's time, identical on
    both ranks (what rank 0 prints)."""
    import json
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    mp.spawn(_e2e_worker, args=(port, 2, str(tmp_path)), nprocs=2, join=True)
    res = [json.load(open(tmp_path / f"e2e_{r}.json")) for r in range(2)]
    A = gen.rmat(scale=12, edge_factor=16, seed=5)
    ops = gen.row_products(A, A)
    assert res[0]["r"] == res[1]["r"]
    owned = [tuple(p) for x in res for p in x["panels"]]
    assert sorted(owned) == [(0, 64), (64, 128), (128, 200), (200, A.rows)]
    r = res[0]["r"]
    # 10 C entries a panel (8 bytes each) plus each panel's row pointer
    assert r["d2h_bytes_per_step"] == sum(4 * (r1 - r0 + 1) + 80 for r0, r1 in owned)
    h2d = sum(4 * (r1 - r0 + 1 + A.rows + 1) + 8 * (int(A.row_ptr[r1] - A.row_ptr[r0]) + A.nnz)
              for r0, r1 in owned)
    assert r["h2d_bytes_per_step"] == h2d
    # every rank's products over the slower rank's time (20 ms a call on rank 1)
    assert r["ms_per_step"] >= 0.02 * len(res[1]["panels"]) * 1e3
    want = 2.0 * int(ops.sum()) / (r["ms_per_step"] * 1e-3) / 1e9
    assert abs(r["value"] - want) <= 0.01 * want
