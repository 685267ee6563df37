#!/usr/bin/env python
"""FP32 CSR SpGEMM benchmark on B200 (one process per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload poisson_reuse|plain|batched|tall_skinny|rmat|coo]

Default workload (the descriptor-reuse case): C = A * A for the 5-point
Laplacian on a 1024 x 1024 grid (N = 1,048,576, nnz(A) = 5,238,784,
nnz(C) = 13,611,012, 26,177,544 intermediate products). The structure is
analysed once; every step rescales A's values entry-wise by U(0.5, 1.5)
(seeded) and re-executes the numeric phase only, replayed from a CUDA graph.

Printed as one JSON line by rank 0:
  value   GFLOP/s = 2 * products / step time, device-timed with CUDA events on
          the plan's stream, operands resident in HBM, L2 flushed (256 MiB
          write) before every step
  e2e     the same metric through the public C API (rvsp_spgemm_compute) with
          pinned host buffers: the H2D copy of the new values and the D2H copy
          of C inside the timed region (wall clock)
  roofline  algorithmic bytes of one numeric pass / its kernel time vs the
          measured HBM copy bandwidth (MEASURED_PEAKS.json)
  cpu_baseline  the reference's scalar numeric pass (oracle/_ref, compiled
          from the reference sources) on 1 host core, bounded sample
With --impl reference the reference's CPU implementation is timed instead,
on all host cores (row panels), with the same workload, metric and unit.

The other workloads (--workload) print one JSON line of one-shot comparisons:
exact-symbolic vs learned-binned, default vs autotuned bin parameters, and
batched vs sequential products, with the FP32-vs-FP64 error of sampled rows.
rmat is C = A * A for an R-MAT graph of 2^scale vertices (default 20, 16
edges per vertex); its intermediate products exceed the int32 range of one
CSR, so it runs as row panels of at most 2^31 - 1 products each.

N > 1 (torchrun): every rank runs its own full-size product on its own GPU
(independent products, no data-path collective; weak scaling); a gloo
barrier brackets the timed loop and the step time is the max over ranks.
"""

from __future__ import annotations

import argparse
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
RANK = int(os.environ.get("RANK", "0"))
WORLD = int(os.environ.get("WORLD_SIZE", "1"))
LOCAL_RANK = int(os.environ.get("LOCAL_RANK", "0"))
if WORLD > 1:
    # one GPU per process: both this process's CUDA runtimes see it as device 0
    os.environ["CUDA_VISIBLE_DEVICES"] = str(LOCAL_RANK)

sys.path.insert(0, os.path.join(ROOT, "rv-sparse_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

METRIC = "SpGEMM GFLOP/s, HBM % of roofline: learned-binned vs exact-symbolic, 1 B200"
UNIT = "GFLOP/s"


def log(*a):
    if RANK == 0:
        print(*a, file=sys.stderr, flush=True)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self):
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            idx = os.environ.get("CUDA_VISIBLE_DEVICES", "0").split(",")[0]
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={idx}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        rows = []
        with open(self.file.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------

def poisson_workload():
    from rvsp_b200 import gen
    A = gen.poisson2d(1024)
    P = gen.products(A, A)
    return A, P


def algorithmic_bytes(M, nnz_a, nnz_c, b_rows, nnz_b):
    """Compulsory bytes of one product, 4(M+1) + 8 nnzA + 4(K+1) + 8 nnzB +
    4(M+1) + 8 nnzC: every operand array read once (B counted as its own
    operand also when it is A), C's row pointer and col_idx + values once
    (col_idx read and values written on descriptor reuse)."""
    return 4 * (M + 1) + 8 * nnz_a + 4 * (b_rows + 1) + 8 * nnz_b + 4 * (M + 1) + 8 * nnz_c


def run_ours(args):
    import ctypes as C

    import torch

    import rvsp_b200 as rv

    from rvsp_b200 import ranks
    dist = ranks.init("gloo", timeout_s=300)
    torch.cuda.set_device(0)
    torch.zeros(1, device="cuda")  # context current on this thread for both runtimes
    L = rv.lib()

    A, P = poisson_workload()
    M, nnz_a = A.rows, A.nnz
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    drp, dci, dv = dev(A.row_ptr), dev(A.col_idx), dev(A.values.copy())

    plan = C.c_void_p()
    rv.check(L.rvsp_cuda_plan_create(C.byref(plan), rv.RVSP_CUDA_ALGO_EXACT), "plan")
    nnz = C.c_int64()
    wsz = C.c_size_t()
    rv.check(L.rvsp_cuda_symbolic(plan, M, A.cols, nnz_a, drp.data_ptr(), dci.data_ptr(), M,
                                  A.cols, nnz_a, drp.data_ptr(), dci.data_ptr(), C.byref(nnz),
                                  C.byref(wsz)), "symbolic")
    nnz_c = nnz.value
    crp = torch.zeros(M + 1, dtype=torch.int32, device="cuda")
    cci = torch.zeros(nnz_c, dtype=torch.int32, device="cuda")
    cv = torch.zeros(nnz_c, dtype=torch.float32, device="cuda")
    ptrs = lambda: (drp.data_ptr(), dci.data_ptr(), dv.data_ptr(), drp.data_ptr(),  # noqa: E731
                    dci.data_ptr(), dv.data_ptr(), crp.data_ptr(), cci.data_ptr(), cv.data_ptr())
    rv.check(L.rvsp_cuda_numeric(plan, *ptrs(), 1, None), "numeric fill")
    torch.cuda.synchronize()
    # parity of the first pass against the reference kernel's output digests
    parity = None
    gold = os.path.join(ROOT, "tests", "golden", "ref_outputs.json")
    if os.path.exists(gold):
        d = json.load(open(gold))["digests"]["poisson2d_1024"]
        parity = (sha(crp.cpu().numpy()) == d["row_ptr_sha256"] and
                  sha(cci.cpu().numpy()) == d["col_idx_sha256"] and
                  sha(cv.cpu().numpy()) == d["values_sha256"])
    rv.check(L.rvsp_cuda_plan_set_async(plan, 1), "async")
    stream = torch.cuda.ExternalStream(L.rvsp_cuda_plan_stream(plan))

    rng = np.random.default_rng(1000 + RANK)
    R = 4
    variants = [dev((A.values * rng.uniform(0.5, 1.5, nnz_a)).astype(np.float32)) for _ in range(R)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def step(i, ev0=None, ev1=None):
        with torch.cuda.stream(stream):
            dv.copy_(variants[i % R])
            flush.zero_()
            if ev0 is not None:
                ev0.record(stream)
            st = L.rvsp_cuda_numeric(plan, *ptrs(), 0, None)
            if ev1 is not None:
                ev1.record(stream)
        rv.check(st, "numeric reuse")

    sampler = ClockSampler()
    sampler.start()
    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    ranks.barrier(dist)
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    l0 = rv.launch_count()
    for i in range(args.steps):
        step(args.warmup + i, *evs[i])
    torch.cuda.synchronize()
    launches = rv.launch_count() - l0
    ranks.barrier(dist)
    times = [a.elapsed_time(b) for a, b in evs]  # ms
    ms = sum(times) / len(times)
    ms_max = ranks.max_over_ranks(dist, ms)
    value = 2.0 * P * WORLD / (ms_max * 1e-3) / 1e9

    # end to end through the public API with pinned host buffers
    e2e = run_e2e(rv, A, P, args, torch)
    # the one-shot product of the same matrices, exact-symbolic vs learned-binned
    oneshot_cmp = compare_oneshot(rv, A, P, torch, args)
    clocks = sampler.stop()

    rv.check(L.rvsp_cuda_plan_set_async(plan, 0))
    L.rvsp_cuda_plan_destroy(plan)
    ranks.barrier(dist)
    if RANK != 0:
        if dist:
            dist.destroy_process_group()
        return

    hbm, peak_kind = peaks()
    bytes_alg = algorithmic_bytes(M, nnz_a, nnz_c, M, nnz_a)
    bytes_distinct = bytes_alg - (4 * (M + 1) + 8 * nnz_a)  # B's arrays are A's
    achieved = bytes_alg / (ms * 1e-3) / 1e9
    traffic = None
    tr_path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tr_path):
        traffic = json.load(open(tr_path)).get("poisson2d_1024_reuse")
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": WORLD,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_max, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (5-point Laplacian, values rescaled U(0.5,1.5) per step, seeded)",
        "config": {"workload": "poisson2d_1024_descriptor_reuse", "grid": 1024, "rows": M,
                   "nnz_a": nnz_a, "nnz_c": nnz_c, "products": P, "path": "numeric-only, CUDA graph",
                   "l2": "flushed (256 MiB write) before every timed step",
                   "parallelism": f"{WORLD} independent products, one per GPU"},
        "parity_first_pass_vs_reference": parity,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 4), "traffic": traffic,
                     "peak_source": f"{peak_kind} hbm_gbs", "kernel": "k_tiny_reuse_map",
                     "bytes_per_launch": bytes_alg,
                     "frac_distinct_arrays": round(bytes_distinct / (ms * 1e-3) / 1e9 / hbm, 4)},
        "e2e": e2e,
        "oneshot_exact_vs_learned": oneshot_cmp,
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if WORLD == 1:
        out["cpu_baseline"] = cpu_baseline(A, P)
    print(json.dumps(out), flush=True)
    if dist:
        dist.destroy_process_group()


def compare_oneshot(rv, A, P, torch, args):
    """One-shot C = A*A (analysis + C allocation + fill), exact-symbolic vs
    learned-binned, device-resident inputs, median wall time per product."""
    dA = DevMat(A, torch)
    out = {}
    ref = None
    for name, algo in (("exact", rv.RVSP_CUDA_ALGO_EXACT), ("learned", rv.RVSP_CUDA_ALGO_LEARNED)):
        def fn(algo=algo):
            ptrs, n = _oneshot_dev(rv, dA, dA, algo)
            rv.free_device(*ptrs)
        t = _time(fn, max(5, args.steps // 10), args.warmup, torch)
        ptrs, n = _oneshot_dev(rv, dA, dA, algo)
        v = _d2h(ptrs[2], n, np.float32, torch)
        rv.free_device(*ptrs)
        if ref is None:
            ref = v
        out[name + "_gflops"] = round(2.0 * P / t / 1e9, 3)
        out[name + "_ms"] = round(t * 1e3, 4)
    out["learned_over_exact"] = round(out["learned_gflops"] / out["exact_gflops"], 4)
    out["learned_values_bit_identical"] = bool(np.array_equal(ref.view(np.uint32), v.view(np.uint32)))
    return out


def run_e2e(rv, A, P, args, torch):
    import ctypes as C
    L = rv.lib()

    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        return t

    hrp, hci, hv = pinned(A.row_ptr), pinned(A.col_idx), pinned(A.values.copy())
    a = rv.csr_struct(A.rows, A.cols, A.nnz, hrp, hci, hv)
    d = rv.Descriptor(rv.RVSP_SPGEMM_ALGO_CUDA)
    st, ws, nnz = d.work_estimation(a, a)
    rv.check(st, "e2e estimation")
    crp = pinned(np.zeros(A.rows + 1, np.int32))
    cci = pinned(np.zeros(nnz, np.int32))
    cv = pinned(np.zeros(nnz, np.float32))
    wsb = np.zeros(max(ws, 4), np.uint8)
    c = rv.csr_struct(A.rows, A.cols, nnz, crp, cci, cv)
    rv.check(d.compute(a, a, c, wsb), "e2e first compute")
    rng = np.random.default_rng(2000 + RANK)
    variants = [(A.values * rng.uniform(0.5, 1.5, A.nnz)).astype(np.float32) for _ in range(4)]
    hvn = hv.numpy()
    for i in range(args.warmup):
        hvn[:] = variants[i % 4]
        rv.check(d.compute(a, a, c, wsb))
    times = []
    for i in range(args.steps):
        hvn[:] = variants[i % 4]
        t0 = time.perf_counter()
        st = d.compute(a, a, c, wsb)
        times.append(time.perf_counter() - t0)
        rv.check(st, "e2e compute")
    d.close()
    t = sum(times) / len(times)
    return {"value": round(2.0 * P / t / 1e9, 3), "unit": UNIT,
            "h2d_bytes_per_step": int(A.nnz * 4),
            "d2h_bytes_per_step": int(nnz * 4 + (A.rows + 1) * 4),
            "api": "rvsp_spgemm_compute (descriptor reuse), pinned host A/C",
            "ms_per_step": round(t * 1e3, 4)}


def cpu_baseline(A, P, budget_s=10.0):
    """Reference scalar numeric pass (oracle/_ref) on 1 host core, bounded sample."""
    import oracle
    if not oracle.ref_available():
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "unavailable: oracle/_ref not built"}
    rp, ci, _, _, st = oracle.ref_spgemm(A, A)
    cv = np.zeros(max(int(rp[-1]), 1), np.float32)
    t1 = oracle.ref_time_numeric(A, A, rp, ci, cv, nthreads=1, repeats=1)
    reps = max(1, int(budget_s / max(t1, 1e-3)))
    t = oracle.ref_time_numeric(A, A, rp, ci, cv, nthreads=1, repeats=reps)
    return {"value": round(2.0 * P * reps / t / 1e9, 4), "unit": UNIT, "cores": 1,
            "kind": "reference",
            "sample": f"full 1024^2 Poisson numeric pass (rvsp_spgemm_scalar_f32_numeric) x {reps}, "
                      f"{t:.1f} s, 1 thread"}


def run_reference(args):
    """The reference's own CPU numeric pass on all host cores (row panels)."""
    if RANK != 0:
        return
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/librvsp_ref.so not built"}), flush=True)
        return
    A, P = poisson_workload()
    cores = len(os.sched_getaffinity(0))
    rp, ci, _, _, st = oracle.ref_spgemm(A, A)
    cv = np.zeros(max(int(rp[-1]), 1), np.float32)
    rng = np.random.default_rng(1000)
    variants = [(A.values * rng.uniform(0.5, 1.5, A.nnz)).astype(np.float32) for _ in range(4)]
    from rvsp_b200.gen import CSR

    def step(i):
        Ai = CSR(A.rows, A.cols, A.row_ptr, A.col_idx, variants[i % 4])
        return oracle.ref_time_numeric(Ai, Ai, rp, ci, cv, nthreads=cores, repeats=1)

    for i in range(args.warmup):
        step(i)
    times = [step(args.warmup + i) for i in range(args.steps)]
    t = sum(times) / len(times)
    value = 2.0 * P / t / 1e9
    out = {"metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": WORLD,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t * 1e3, 4),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (5-point Laplacian, values rescaled U(0.5,1.5) per step, seeded)",
           "config": {"workload": "poisson2d_1024_descriptor_reuse", "grid": 1024, "rows": A.rows,
                      "products": P, "path": "numeric-only (reference rvsp_spgemm_scalar_f32_numeric)"},
           "impl": "reference",
           "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": cores,
                            "kind": "reference",
                            "sample": f"full numeric pass per step, {cores} threads on row panels"},
           "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# other BASELINE workloads: exact vs learned (and batched vs sequential)
# ---------------------------------------------------------------------------

class DevMat:
    def __init__(self, M, torch):
        self.rows, self.cols, self.nnz = M.rows, M.cols, M.nnz
        d = lambda a: torch.from_numpy(np.ascontiguousarray(a if a.size else np.zeros(1, a.dtype))).cuda()  # noqa: E731
        self.row_ptr, self.col_idx, self.values = d(M.row_ptr), d(M.col_idx), d(M.values)


def _oneshot_dev(rv, A, B, algo):
    import ctypes as C
    L = rv.lib()
    prp, pci, pv = C.c_void_p(), C.c_void_p(), C.c_void_p()
    nnz = C.c_int32()
    st = L.rvsp_cuda_spgemm_f32(algo, A.rows, A.cols, B.cols, A.row_ptr.data_ptr(),
                                A.col_idx.data_ptr(), A.values.data_ptr(), B.row_ptr.data_ptr(),
                                B.col_idx.data_ptr(), B.values.data_ptr(), C.byref(prp),
                                C.byref(pci), C.byref(pv), C.byref(nnz), None)
    rv.check(st, "rvsp_cuda_spgemm_f32")
    return (prp.value, pci.value, pv.value), nnz.value


def _time(fn, steps, warmup, torch):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t0)
    return statistics.median(ts)


def _d2h(ptr_, n, dtype, torch):
    """Copy n elements of a library-owned device array to the host."""
    import ctypes as C
    if n == 0:
        return sha(np.zeros(0, dtype))
    out = np.empty(n, dtype)
    cuda = C.CDLL("libcuda.so.1")
    cuda.cuMemcpyDtoH_v2.argtypes = [C.c_void_p, C.c_uint64, C.c_size_t]
    assert cuda.cuMemcpyDtoH_v2(out.ctypes.data, ptr_, out.nbytes) == 0
    return out


class PanelView:
    """Rows [r0, r1) of a device CSR: the row pointer is a view into the full
    one, so its offsets index the full column and value arrays directly."""

    def __init__(self, M, r0, r1):
        self.rows, self.cols = r1 - r0, M.cols
        self.row_ptr = M.row_ptr[r0:r1 + 1]
        self.col_idx, self.values = M.col_idx, M.values


def run_rmat(args, rv, gen, torch):
    """Power-law C = A * A by row panels: exact vs learned, default vs tuned."""
    import oracle
    from rvsp_b200 import ranks
    dist = ranks.init("gloo", timeout_s=900)
    t0 = time.time()
    A = gen.rmat(scale=args.rmat_scale, edge_factor=16, seed=0)
    ops = gen.row_products(A, A)
    P = int(ops.sum())
    # every rank computes its contiguous group of row panels (strong scaling)
    panels = ranks.shard_panels(ranks.row_panels(ops), ops, RANK, WORLD)
    log(f"rmat scale {args.rmat_scale}: {A.rows} rows, nnz {A.nnz}, {P} products, "
        f"{len(panels)} panels, generated in {time.time() - t0:.1f} s")
    dA = DevMat(A, torch)
    views = [PanelView(dA, r0, r1) for r0, r1 in panels]
    heavy = int(np.argmax([ops[r0:r1].sum() for r0, r1 in panels]))

    def run_all(algo):
        nnz = 0
        for v in views:
            ptrs, n = _oneshot_dev(rv, v, dA, algo)
            rv.free_device(*ptrs)
            nnz += n
        return nnz

    steps = max(1, min(args.steps, 3))
    times = {}
    def timed(algo):
        # all ranks start together; the job's time is the slowest rank's
        ranks.barrier(dist)
        return ranks.max_over_ranks(dist, _time(lambda: run_all(algo), steps, 1, torch))

    nnz_c = ranks.sum_over_ranks(dist, run_all(rv.RVSP_CUDA_ALGO_EXACT))
    for name, algo in (("exact", rv.RVSP_CUDA_ALGO_EXACT), ("learned", rv.RVSP_CUDA_ALGO_LEARNED)):
        times[name] = timed(algo)
    # autotune on the panel with the most products, then every panel under the choice
    plan = rv.Plan()
    st, _, best, trials = plan.autotune(views[heavy], dA, reps=1)
    rv.check(st, "autotune")
    plan.close()
    rv.check(rv.set_default_params(best))
    try:
        for name, algo in (("tuned_exact", rv.RVSP_CUDA_ALGO_EXACT),
                           ("tuned_learned", rv.RVSP_CUDA_ALGO_LEARNED)):
            times[name] = timed(algo)
        # misprediction rate of the learned sizing, measured against the exact recount
        lp = rv.Plan(rv.RVSP_CUDA_ALGO_LEARNED)
        st, lnnz = lp.symbolic(views[heavy], dA)
        rv.check(st, "learned symbolic")
        ls = lp.learned_stats()
        lp.close()
        # parity: sampled rows of the first and the heaviest panel, bit-exact
        rng = np.random.default_rng(1)
        ok, errs = True, []
        for pi in sorted({0, heavy}):
            r0, r1 = panels[pi]
            for algo in (rv.RVSP_CUDA_ALGO_EXACT, rv.RVSP_CUDA_ALGO_LEARNED):
                ptrs, n = _oneshot_dev(rv, views[pi], dA, algo)
                rp = _d2h(ptrs[0], r1 - r0 + 1, np.int32, torch)
                ci = _d2h(ptrs[1], n, np.int32, torch)
                v = _d2h(ptrs[2], n, np.float32, torch)
                rv.free_device(*ptrs)
                for r in np.sort(rng.choice(np.arange(r0, r1), min(100, r1 - r0), replace=False)):
                    srp, sci, sv = oracle.spgemm_f32(A, A, int(r), int(r) + 1)
                    lo, hi = rp[r - r0], rp[r - r0 + 1]
                    ok &= np.array_equal(sci, ci[lo:hi]) and \
                        np.array_equal(sv.view(np.uint32), v[lo:hi].view(np.uint32))
                    if algo == rv.RVSP_CUDA_ALGO_EXACT and sci.size:
                        d = oracle.numeric_f64(A, A, srp, sci, int(r), int(r) + 1)
                        errs.append(np.abs(v[lo:hi] - d) / np.maximum(np.abs(d), 1e-30))
    finally:
        rv.check(rv.set_default_params(None))
    e = np.concatenate(errs) if errs else np.zeros(1)
    g = {k: 2 * P / t / 1e9 for k, t in times.items()}
    return {
        "config": {"workload": f"rmat_scale{args.rmat_scale}_ef16_a0.57_b0.19_c0.19", "rows": A.rows,
                   "nnz_a": A.nnz, "products": P, "nnz_c": nnz_c, "panels_this_rank": len(panels),
                   "max_row_products": int(ops.max())},
        "n_gpus": WORLD, "scaling": "strong",
        "gflops": g, "ms": {k: t * 1e3 for k, t in times.items()},
        "learned_over_exact": times["exact"] / times["learned"],
        "tuned_learned_over_exact": times["exact"] / times["tuned_learned"],
        "tuned_params": list(best),
        "autotune_trials": [[list(p), round(ms, 3)] for p, ms in trials],
        "mispredict": {"panel": heavy, **ls,
                       "rate": ls["underpredicted_rows"] / max(ls["predicted_rows"], 1),
                       "rerun_rate": ls["overflowed_rows"] / max(ls["predicted_rows"], 1)},
        "sampled_rows_bit_exact_vs_oracle": bool(ok),
        "fp32_vs_fp64_rel_err": {"max": float(e.max()), "median": float(np.median(e)),
                                 "p99": float(np.quantile(e, 0.99))},
    }


def run_coo(args, rv, torch):
    """COO -> canonical CSR (the Matrix Market loader's canonicalisation) of an
    R-MAT 2^scale edge list with its repeated edges, device in and out."""
    import ctypes as C
    import oracle
    rng = np.random.default_rng(0)
    scale, ef = args.rmat_scale, 16
    n = ef << scale
    r = np.zeros(n, np.int64)
    c = np.zeros(n, np.int64)
    for bit in range(scale):  # the R-MAT recursion of rvsp_b200.gen.rmat, duplicates kept
        u = rng.random(n)
        r |= (u >= 0.76).astype(np.int64) << bit
        c |= (((u >= 0.57) & (u < 0.76)) | (u >= 0.95)).astype(np.int64) << bit
    r = r.astype(np.int32)
    c = c.astype(np.int32)
    v = rng.uniform(-1, 1, n).astype(np.float32)
    m = 1 << scale
    dr, dc, dv = (torch.from_numpy(x).cuda() for x in (r, c, v))
    L = rv.lib()
    out = {}

    def once():
        prp, pci, pv = C.c_void_p(), C.c_void_p(), C.c_void_p()
        nnz = C.c_int32()
        rv.check(L.rvsp_cuda_coo_to_csr(m, m, n, dr.data_ptr(), dc.data_ptr(), dv.data_ptr(), 0, 1,
                                        C.byref(prp), C.byref(pci), C.byref(pv), C.byref(nnz)),
                 "coo_to_csr")
        out["nnz"] = nnz.value
        out["ptrs"] = (prp.value, pci.value, pv.value)

    def step():
        once()
        rv.free_device(*out["ptrs"])

    t = _time(step, args.steps, args.warmup, torch)
    once()
    rp = _d2h(out["ptrs"][0], m + 1, np.int32, torch)
    ci = _d2h(out["ptrs"][1], out["nnz"], np.int32, torch)
    vv = _d2h(out["ptrs"][2], out["nnz"], np.float32, torch)
    rv.free_device(*out["ptrs"])
    t0 = time.perf_counter()
    wrp, wci, wv = oracle.coo_to_csr(m, m, r, c, v, False)
    t_cpu = time.perf_counter() - t0
    same = (np.array_equal(rp.astype(np.int64), wrp) and np.array_equal(ci, wci) and
            np.array_equal(vv.view(np.uint32), wv.view(np.uint32)))
    bits = 2 * scale
    passes = (bits + 7) // 8
    # per entry: COO in (12 B), keys + payload written (16 B), each radix pass
    # reads and writes them (32 B), the run sums read them (16 B), CSR out (8 B)
    per_entry = 12 + 16 + 32 * passes + 16 + 8
    hbm, kind = peaks()
    return {"config": {"workload": f"coo_to_csr_rmat{scale}_edges_with_repeats", "entries": n,
                       "rows": m, "nnz_out": out["nnz"], "radix_passes": passes},
            "ms": t * 1e3, "entries_per_s": n / t,
            "roofline": {"bound": "hbm", "bytes_per_entry": per_entry,
                         "achieved_gbs": per_entry * n / t / 1e9, "peak": hbm,
                         "frac": per_entry * n / t / 1e9 / hbm, "peak_source": f"{kind} hbm_gbs"},
            "cpu_baseline": {"ms": t_cpu * 1e3, "cores": 1, "kind": "port",
                             "sample": "the oracle's canonicalisation of the same list, once"},
            "bit_exact_vs_oracle": bool(same)}


def run_compare(args):
    """One-shot exact vs learned (and batched vs sequential) on a BASELINE config."""
    import torch

    import rvsp_b200 as rv
    from rvsp_b200 import gen
    torch.zeros(1, device="cuda")
    L = rv.lib()
    res = {}
    if args.workload in ("plain", "tall_skinny"):
        if args.workload == "plain":
            A = gen.uniform_fixed()
            B = A
            cfg = {"workload": "plain_4096x4096_16_per_row", "seed": 0}
        else:
            A, B = gen.tall_skinny(a_rows=args.ts_rows)
            cfg = {"workload": f"tall_skinny_{args.ts_rows}x100000_x_100000^2", "a_rows": A.rows,
                   "nnz_a": A.nnz, "nnz_b": B.nnz}
        P = gen.products(A, B)
        dA, dB = DevMat(A, torch), DevMat(B, torch)
        times = {}
        outs = {}
        for name, algo in (("exact", rv.RVSP_CUDA_ALGO_EXACT), ("learned", rv.RVSP_CUDA_ALGO_LEARNED)):
            def fn(algo=algo):
                ptrs, n = _oneshot_dev(rv, dA, dB, algo)
                rv.free_device(*ptrs)
            times[name] = _time(fn, args.steps, args.warmup, torch)
            ptrs, n = _oneshot_dev(rv, dA, dB, algo)
            outs[name] = (_d2h(ptrs[0], A.rows + 1, np.int32, torch),
                          _d2h(ptrs[1], n, np.int32, torch), _d2h(ptrs[2], n, np.float32, torch))
            rv.free_device(*ptrs)
        same = all(np.array_equal(a, b) for a, b in zip(outs["exact"], outs["learned"]))
        nnz_c = int(outs["exact"][0][-1])
        res["config"] = dict(cfg, rows=A.rows, products=P, nnz_c=nnz_c)
        res["exact_gflops"] = 2 * P / times["exact"] / 1e9
        res["learned_gflops"] = 2 * P / times["learned"] / 1e9
        res["learned_over_exact"] = times["exact"] / times["learned"]
        res["learned_bit_identical_to_exact"] = bool(same)
        res["ms"] = {k: v * 1e3 for k, v in times.items()}
        b_alg = algorithmic_bytes(A.rows, A.nnz, nnz_c, B.rows, B.nnz)
        res["bytes_alg"] = b_alg
        res["hbm_frac_learned"] = b_alg / times["learned"] / 1e9 / peaks()[0]
        # FP64 error of the FP32 result on sampled rows
        import oracle
        rng = np.random.default_rng(0)
        rows = np.sort(rng.choice(A.rows, min(2000, A.rows), replace=False))
        errs = []
        rp, ci, v = outs["exact"]
        for r in rows[:400]:
            srp, sci, sv = oracle.spgemm_f32(A, B, int(r), int(r) + 1)
            d = oracle.numeric_f64(A, B, srp, sci, int(r), int(r) + 1)
            got = v[rp[r]:rp[r + 1]]
            assert np.array_equal(sci, ci[rp[r]:rp[r + 1]])
            errs.append(np.abs(got - d) / np.maximum(np.abs(d), 1e-30))
        e = np.concatenate(errs) if errs else np.zeros(1)
        res["fp32_vs_fp64_rel_err"] = {"max": float(e.max()), "median": float(np.median(e)),
                                       "p99": float(np.quantile(e, 0.99)), "rows_sampled": 400}
    elif args.workload == "rmat":
        res = run_rmat(args, rv, gen, torch)
    elif args.workload == "coo":
        res = run_coo(args, rv, torch)
    elif args.workload == "batched":
        pairs = gen.batched_uneven(count=args.batch_count)
        prods = [gen.products(A, B) for A, B in pairs]
        P = sum(prods)
        dev_pairs = [(DevMat(A, torch), DevMat(B, torch)) for A, B in pairs]
        # one batched call per group whose products (an upper bound on nnz)
        # fit the int32 row pointer of a packed C
        groups, cur, acc = [], [], 0
        for i, p in enumerate(prods):
            if cur and acc + p > (1 << 31) - 1:
                groups.append(cur)
                cur, acc = [], 0
            cur.append(i)
            acc += p
        groups.append(cur)
        def seq():
            for dA, dB in dev_pairs:
                ptrs, n = _oneshot_dev(rv, dA, dB, rv.RVSP_CUDA_ALGO_EXACT)
                rv.free_device(*ptrs)
        times = {"sequential_exact": _time(seq, max(1, args.steps // 10), 1, torch)}
        for name, algo in (("batched_exact", rv.RVSP_CUDA_ALGO_EXACT),
                           ("batched_learned", rv.RVSP_CUDA_ALGO_LEARNED)):
            def fn(algo=algo):
                for g in groups:
                    ptrs, n, offs = rv.spgemm_batched([dev_pairs[i] for i in g], algo)
                    rv.free_device(*ptrs)
            times[name] = _time(fn, args.steps, args.warmup, torch)
        # correctness: the group holding product 0 (and its spot checks)
        g0 = groups[0]
        pairs = [pairs[i] for i in g0]
        ptrs, n, offs = rv.spgemm_batched([dev_pairs[i] for i in g0], rv.RVSP_CUDA_ALGO_LEARNED)
        crp = _d2h(ptrs[0], int(offs[-1]) + 1, np.int32, torch)
        cci = _d2h(ptrs[1], n, np.int32, torch)
        cv = _d2h(ptrs[2], n, np.float32, torch)
        rv.free_device(*ptrs)
        # spot-check three products against the oracle
        import oracle
        ok = True
        for i in (0, len(pairs) // 2, len(pairs) - 1):
            A, B = pairs[i]
            r0, r1 = int(offs[i]), int(offs[i + 1])
            wrp, wci, wv = oracle.spgemm_f32(A, B)
            lrp = crp[r0:r1 + 1] - crp[r0]
            ok &= np.array_equal(lrp, wrp) and np.array_equal(cci[crp[r0]:crp[r1]], wci) and \
                np.array_equal(cv[crp[r0]:crp[r1]].view(np.uint32), wv.view(np.uint32))
        res["config"] = {"workload": f"batched_{len(dev_pairs)}_uneven", "products": P,
                         "groups": len(groups), "group0_rows": int(offs[-1]), "group0_nnz_c": n}
        res["gflops"] = {k: 2 * P / t / 1e9 for k, t in times.items()}
        res["ms"] = {k: t * 1e3 for k, t in times.items()}
        res["batched_learned_over_sequential"] = times["sequential_exact"] / times["batched_learned"]
        res["batched_learned_over_batched_exact"] = times["batched_exact"] / times["batched_learned"]
        res["spot_check_bit_exact_vs_oracle"] = bool(ok)
    if RANK == 0:
        print(json.dumps({"workload": args.workload, **res}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="poisson_reuse",
                    choices=["poisson_reuse", "plain", "batched", "tall_skinny", "rmat", "coo"])
    ap.add_argument("--rmat-scale", type=int, default=20)
    ap.add_argument("--batch-count", type=int, default=512)
    ap.add_argument("--ts-rows", type=int, default=2_000_000)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload != "poisson_reuse":
        run_compare(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
