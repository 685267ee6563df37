"""Regenerates the golden fixtures in this directory from the reference.

Run next to a reference checkout named by $RVSP_REFERENCE_DIR:

    RVSP_REFERENCE_DIR=<checkout> python tests/golden/make_golden.py

Writes:

* csr_fixtures.json -- the six hand-computed A, B, C triples of
  rv-sparse tests/csr_fixtures.h:42-153, extracted by compiling a throwaway
  C program against that header and printing its tables.
* ref_outputs.npz / ref_outputs.json -- outputs of the reference's own
  scalar kernel (oracle/_ref/librvsp_ref.so, built from the reference
  sources by oracle/Makefile) on seeded synthetic inputs: small cases are
  stored whole (inputs and outputs), the full 4096^2 plain case and the
  1024^2 Poisson case as SHA-256 digests of the output arrays plus nnz.
"""

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "rv-sparse_b200"))

import oracle  # noqa: E402
from rvsp_b200 import gen  # noqa: E402

REF = os.environ.get("RVSP_REFERENCE_DIR", "")

DUMP_C = r"""
#include <stdio.h>
#include "csr_fixtures.h"
static void arr_i(const char *k, const int32_t *a, int n, int last) {
    printf("\"%s\": [", k);
    for (int i = 0; i < n; i++) printf(i ? ", %d" : "%d", a[i]);
    printf("]%s", last ? "" : ", ");
}
static void arr_f(const char *k, const float *a, int n, int last) {
    printf("\"%s\": [", k);
    for (int i = 0; i < n; i++) printf(i ? ", %.9g" : "%.9g", (double)a[i]);
    printf("]%s", last ? "" : ", ");
}
static void mat(const char *k, const rvsp_fx_csr_t *m, int last) {
    printf("\"%s\": {\"rows\": %d, \"cols\": %d, \"nnz\": %d, ", k, m->rows, m->cols, m->nnz);
    arr_i("row_ptr", m->row_ptr, m->rows + 1, 0);
    arr_i("col_idx", m->col_idx, m->nnz, 0);
    arr_f("values", m->values, m->nnz, 1);
    printf("}%s", last ? "" : ", ");
}
int main(void) {
    const rvsp_fx_pair_t *fx = rvsp_fx_all();
    printf("[");
    for (int i = 0; i < rvsp_fx_count(); i++) {
        printf(i ? ",\n{" : "\n{");
        printf("\"name\": \"%s\", \"targets\": \"%s\", ", fx[i].name, fx[i].targets);
        mat("a", &fx[i].a, 0); mat("b", &fx[i].b, 0); mat("c", &fx[i].c, 1);
        printf("}");
    }
    printf("\n]\n");
    return 0;
}
"""


def dump_fixtures():
    with tempfile.TemporaryDirectory() as td:
        src = os.path.join(td, "dump.c")
        exe = os.path.join(td, "dump")
        with open(src, "w") as f:
            f.write(DUMP_C)
        subprocess.run(["gcc", "-std=c11", "-I", os.path.join(REF, "tests"), "-o", exe, src],
                       check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    data = json.loads(out)
    with open(os.path.join(HERE, "csr_fixtures.json"), "w") as f:
        json.dump({"source": "rv-sparse tests/csr_fixtures.h:42-153", "pairs": data}, f, indent=1)
    return data


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def small_cases():
    """Seeded small products stored whole."""
    cases = {}
    cases["uniform_128x512_16"] = (gen.uniform_fixed(128, 128, 16, seed=1), gen.uniform_fixed(128, 512, 16, seed=2))
    cases["poisson2d_16"] = (gen.poisson2d(16),) * 2
    R = gen.rmat(scale=9, edge_factor=8, seed=3)
    cases["rmat_s9_ef8"] = (R, R)
    rng = np.random.default_rng(5)
    A = gen.poisson_rows(300, 200, 6.0, rng)
    B = gen.poisson_rows(200, 700, 9.0, rng)
    cases["rect_300x200x700"] = (A, B)
    A, B = gen.tall_skinny(a_rows=400, k=2000, n=2000, b_max=600, seed=7)
    cases["tall_skinny_400x2000"] = (A, B)
    return cases


def main():
    if not os.path.isdir(os.path.join(REF, "tests")):
        sys.exit("set RVSP_REFERENCE_DIR to a reference checkout")
    oracle.build(REF)
    dump_fixtures()
    arrays = {}
    meta = {"generator": "tests/golden/make_golden.py",
            "kernel": "reference rvsp_spgemm_scalar_f32 (oracle/_ref/librvsp_ref.so)",
            "cases": {}}
    for name, (A, B) in small_cases().items():
        rp, ci, v, ops, st = oracle.ref_spgemm(A, B)
        assert st == 0, (name, st)
        for tag, M in (("a", A), ("b", B)):
            arrays[f"{name}.{tag}.row_ptr"] = M.row_ptr
            arrays[f"{name}.{tag}.col_idx"] = M.col_idx
            arrays[f"{name}.{tag}.values"] = M.values
        arrays[f"{name}.c.row_ptr"] = rp
        arrays[f"{name}.c.col_idx"] = ci
        arrays[f"{name}.c.values"] = v
        arrays[f"{name}.ops"] = ops
        meta["cases"][name] = {"a": [A.rows, A.cols, A.nnz], "b": [B.rows, B.cols, B.nnz],
                               "c_nnz": int(rp[-1]), "products": int(ops.sum())}
    np.savez_compressed(os.path.join(HERE, "ref_outputs.npz"), **arrays)
    digests = {}
    for name, (A, B) in (("uniform_4096x4096_16_seed0", (gen.uniform_fixed(),) * 2),
                         ("poisson2d_1024", (gen.poisson2d(1024),) * 2)):
        rp, ci, v, ops, st = oracle.ref_spgemm(A, B)
        assert st == 0
        digests[name] = {"c_nnz": int(rp[-1]), "products": int(ops.sum()),
                         "row_ptr_sha256": sha(rp), "col_idx_sha256": sha(ci),
                         "values_sha256": sha(v), "ops_sha256": sha(ops)}
    meta["digests"] = digests
    with open(os.path.join(HERE, "ref_outputs.json"), "w") as f:
        json.dump(meta, f, indent=1)
    print(json.dumps(meta, indent=1))


if __name__ == "__main__":
    main()
