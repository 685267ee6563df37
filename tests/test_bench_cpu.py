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
    assert d["config"]["workload"].startswith("poisson2d_1024")
