"""One-shot products of the benchmark matrices, for profiling a kernel.

    python -m rvsp_b200.profile_case WORKLOAD [--algo exact|learned]
        [--params tiny,slack,warpmax,cwlog2] [--rows R0:R1] [--steps N]

Run from rv-sparse_b200/ on a machine with a CUDA device. WORKLOAD is
rmatS (R-MAT 2^S vertices, 16 edges per vertex, C = A * A), tall (the 2M x
100k tall-skinny product), plain (4096^2, 16 per row) or poisson (1024^2
5-point Laplacian). --rows restricts A to a row panel (device-resident A with
its row pointer offset into the full arrays), so one kernel of a large
product can be captured on a small case. Each step is one rvsp_cuda_spgemm_f32
call on device operands (C freed after the call); the first step is a
warm-up. Prints the median step time and GFLOP/s (2 x products / time).
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import statistics
import time

import numpy as np

import rvsp_b200 as rv
from rvsp_b200 import gen


class _Dev:
    def __init__(self, M, torch, r0=0, r1=None):
        d = lambda a: torch.from_numpy(np.ascontiguousarray(a if a.size else np.zeros(1, a.dtype))).cuda()  # noqa: E731
        r1 = M.rows if r1 is None else r1
        self.rows, self.cols = r1 - r0, M.cols
        self.full_rp = d(M.row_ptr)
        self.row_ptr = self.full_rp[r0:r1 + 1]
        self.col_idx, self.values = d(M.col_idx), d(M.values)


def _matrices(name: str):
    if name.startswith("rmat"):
        A = gen.rmat(scale=int(name[4:]), edge_factor=16, seed=0)
        return A, A
    if name == "tall":
        return gen.tall_skinny(a_rows=2_000_000)
    if name == "plain":
        A = gen.uniform_fixed()
        return A, A
    if name == "poisson":
        A = gen.poisson2d(1024)
        return A, A
    raise SystemExit(f"unknown workload {name}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("workload")
    ap.add_argument("--algo", default="exact", choices=["exact", "learned"])
    ap.add_argument("--params", default=None)
    ap.add_argument("--rows", default=None)
    ap.add_argument("--steps", type=int, default=2)
    args = ap.parse_args()
    import torch
    torch.zeros(1, device="cuda")
    A, B = _matrices(args.workload)
    r0, r1 = (0, A.rows) if args.rows is None else (int(x) for x in args.rows.split(":"))
    dA, dB = _Dev(A, torch, r0, r1), _Dev(B, torch)
    P = int(gen.row_products(A, B)[r0:r1].sum())
    if args.params:
        rv.check(rv.set_default_params([int(x) for x in args.params.split(",")]), "params")
    algo = rv.RVSP_CUDA_ALGO_EXACT if args.algo == "exact" else rv.RVSP_CUDA_ALGO_LEARNED
    L = rv.lib()
    times = []
    for _ in range(max(args.steps, 1)):
        prp, pci, pv = C.c_void_p(), C.c_void_p(), C.c_void_p()
        nnz = C.c_int32()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = L.rvsp_cuda_spgemm_f32(algo, dA.rows, dA.cols, dB.cols, rv.ptr(dA.row_ptr),
                                    rv.ptr(dA.col_idx), rv.ptr(dA.values), rv.ptr(dB.row_ptr),
                                    rv.ptr(dB.col_idx), rv.ptr(dB.values), C.byref(prp),
                                    C.byref(pci), C.byref(pv), C.byref(nnz), None)
        rv.check(st, "rvsp_cuda_spgemm_f32")
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
        rv.free_device(prp.value, pci.value, pv.value)
    t = statistics.median(times[1:] if len(times) > 1 else times)
    print(json.dumps({"workload": args.workload, "rows": [r0, r1], "algo": args.algo,
                      "params": args.params, "products": P, "nnz_c": nnz.value,
                      "ms": t * 1e3, "gflops": 2 * P / t / 1e9}))


if __name__ == "__main__":
    main()
