"""The reference's own C tests and examples, compiled unchanged.

rv-sparse tests/test_spgemm_descr_f32.c (the descriptor contract: 27
checks), tests/test_spgemm_reference_f32.c (every strategy the build
provides on the six fixtures of tests/csr_fixtures.h, exact structure and
values within 1e-5 + 1e-4 |want|) and examples/spgemm_csr_f32.c,
spgemm_csr_descr_f32.c, spgemm_csr_reuse_f32.c are compiled by
oracle/Makefile (`reftests`) twice: against this repository's headers and
librvsp_b200.so (`.ours`, runs on the GPU), and against the reference's own
API sources (`.ref`, its behaviour on the CPU). The programs pass host
arrays and select the reference's default strategy (RVSP_SPGEMM_ALGO_DEFAULT,
RVSP_BACKEND_SCALAR), which this build runs on the CUDA exact path.
"""

import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "bin")
TESTS = ("test_spgemm_descr_f32", "test_spgemm_reference_f32")
EXAMPLES = ("spgemm_csr_f32", "spgemm_csr_descr_f32", "spgemm_csr_reuse_f32")


def _run(name, kind):
    exe = os.path.join(BIN, f"{name}.{kind}")
    if not os.path.exists(exe):
        pytest.skip(f"{exe} is built only next to a reference checkout")
    p = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    return p.returncode, p.stdout


@pytest.mark.parametrize("name", TESTS)
def test_reference_test_programs_pass_on_the_reference_itself(name):
    rc, out = _run(name, "ref")
    assert rc == 0 and "PASS" in out, out


@pytest.mark.gpu
def test_reference_descriptor_contract_program():
    rc, out = _run("test_spgemm_descr_f32", "ours")
    assert rc == 0, out
    assert "test_spgemm_descr_f32: PASS  (27 checks, 0 failed)" in out, out


@pytest.mark.gpu
def test_reference_strategy_program():
    rc, out = _run("test_spgemm_reference_f32", "ours")
    assert rc == 0, out
    # the default (scalar) strategy ran every fixture; the three vector
    # strategies are skipped, as on the reference's own non-vector build
    _, ref_out = _run("test_spgemm_reference_f32", "ref")
    assert out == ref_out, (out, ref_out)
    assert "3 strategies skipped" in out and "0 failed" in out, out
    assert out.count("  scalar ") == 6, out


@pytest.mark.gpu
@pytest.mark.parametrize("name", EXAMPLES)
def test_reference_examples_print_what_the_reference_prints(name):
    rc, out = _run(name, "ours")
    rc_ref, ref_out = _run(name, "ref")
    assert rc == 0 and rc_ref == 0, (out, ref_out)
    assert out == ref_out, (out, ref_out)
