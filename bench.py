#!/usr/bin/env python
"""FP32 CSR SpGEMM benchmark on B200 (one process per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload rmat|poisson_reuse|plain|batched|tall_skinny|coo|profile]

Default workload (the power-law product the metric is quoted on): C = A * A
for an R-MAT graph of 2^20 vertices, 16 * 2^20 edge samples with
(a, b, c, d) = (0.57, 0.19, 0.19, 0.05), duplicates merged, values U(-1, 1),
seed 0 (nnz(A) = 16,086,301, 2.09e10 intermediate products, nnz(C) = 9.7e9).
Its C is too large for one int32 CSR (the reference refuses such a product,
rvsp_symbolic.c:69), so it runs as A row panels of at most 2^31 - 1 products,
each panel one call of the one-shot entry point on device-resident operands
(the panel's row pointer offset into the full arrays). One step is the whole
product, every panel; the next step starts on a flushed L2.

Printed as one JSON line by rank 0:
  value   learned-binned GFLOP/s = 2 * products / step time (the MLP-sized
          path, RVSP_CUDA_ALGO_LEARNED), device-timed with CUDA events,
          operands resident in HBM; exact_gflops beside it is the
          exact-symbolic path (RVSP_CUDA_ALGO_EXACT) timed the same way
  roofline  the dominant kernel's algorithmic bytes per launch over its mean
          launch duration (per-family CUDA events inside the library, live in
          the timed region) against the measured HBM copy bandwidth
  e2e     the same metric through the public C API (rvsp_spgemm_csr with the
          learned backend) on host buffers: every panel's A upload, B upload
          and C download inside the timed region
  cpu_baseline  the reference's scalar kernel (oracle/_ref, compiled from the
          reference sources) on 1 host core over a seeded sample of A's rows
  parity  sampled rows bit-exact against the oracle, learned C bit-identical
          to exact C over the whole product, FP32-vs-FP64 error
With --impl reference the reference's own CPU implementation is timed on all
host cores over a seeded row sample of the same product, same metric and unit.

The other workloads print one JSON line each: poisson_reuse (descriptor
reuse of the 1024^2 5-point Laplacian, numeric-only, CUDA graph), plain,
tall_skinny, batched (one-shot comparisons: exact vs learned, batched vs
sequential), coo (Matrix Market canonicalisation) and profile (one product of
a named matrix, optionally a row range, for capturing a kernel).

N > 1 (torchrun): the product's panels are dealt to the ranks in contiguous
groups of about equal products (strong scaling; no data-path collective,
output rows are independent); a gloo barrier brackets each timed loop and the
step time is the max over ranks.
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
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
RANK = int(os.environ.get("RANK", "0"))
WORLD = int(os.environ.get("WORLD_SIZE", "1"))
LOCAL_RANK = int(os.environ.get("LOCAL_RANK", "0"))
if WORLD > 1:
    # one GPU per process: both this process's CUDA runtimes see it as device
    # 0 (the LOCAL_RANK-th of the GPUs the launcher made visible, if it chose)
    _visible = [d for d in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if d.strip()]
    os.environ["CUDA_VISIBLE_DEVICES"] = (_visible[LOCAL_RANK] if LOCAL_RANK < len(_visible)
                                          else str(LOCAL_RANK))

sys.path.insert(0, os.path.join(ROOT, "rv-sparse_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

METRIC = "SpGEMM GFLOP/s, HBM % of roofline: learned-binned vs exact-symbolic, 1 B200"
UNIT = "GFLOP/s"
RMAT_DATA = ("synthetic R-MAT (a,b,c,d)=(0.57,0.19,0.19,0.05), 16 edge samples per vertex, "
             "duplicates merged, values U(-1,1), seed 0")
# default bin parameters of the library (tiny_ops, slack_shift, warp_cap_max, heavy_cw_log2)
DEFAULT_PARAMS = (32, 2, 2048, 11)


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
            return
        # nvidia-smi's start-up queries the driver heavily: the timed region
        # begins once its first sample is written
        t0 = time.time()
        while time.time() - t0 < 10 and self.proc.poll() is None:
            if os.path.getsize(self.file.name) > 0:
                break
            time.sleep(0.05)

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


def algorithmic_bytes(M, nnz_a, nnz_c, b_rows, nnz_b):
    """Compulsory bytes of one product, 4(M+1) + 8 nnzA + 4(K+1) + 8 nnzB +
    4(M+1) + 8 nnzC: every operand array read once (B counted as its own
    operand also when it is A), C's row pointer and col_idx + values once
    (col_idx read and values written on descriptor reuse)."""
    return 4 * (M + 1) + 8 * nnz_a + 4 * (b_rows + 1) + 8 * nnz_b + 4 * (M + 1) + 8 * nnz_c


def heavy_rows(ops, b_cols, params=DEFAULT_PARAMS):
    """Rows the library bins as heavy (a warp per column chunk) under the bin
    parameters: more products than the tiny bin and an upper bound
    ub = min(ops, cols) whose table ub + (ub >> slack) passes warp_cap_max."""
    tiny, slack, wmax, _ = params
    ops = np.asarray(ops, np.int64)
    ub = np.minimum(ops, b_cols)
    return (ub > 0) & (ops > tiny) & (ub + (ub >> slack) > wmax)


# ---------------------------------------------------------------------------
# device helpers
# ---------------------------------------------------------------------------

class DevMat:
    def __init__(self, M, torch):
        self.rows, self.cols, self.nnz = M.rows, M.cols, M.nnz
        d = lambda a: torch.from_numpy(np.ascontiguousarray(a if a.size else np.zeros(1, a.dtype))).cuda()  # noqa: E731
        self.row_ptr, self.col_idx, self.values = d(M.row_ptr), d(M.col_idx), d(M.values)


class PanelView:
    """Rows [r0, r1) of a device CSR: the row pointer is a view into the full
    one, so its offsets index the full column and value arrays directly."""

    def __init__(self, M, r0, r1):
        self.rows, self.cols = r1 - r0, M.cols
        self.row_ptr = M.row_ptr[r0:r1 + 1]
        self.col_idx, self.values = M.col_idx, M.values


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


class _DevArray:
    """__cuda_array_interface__ view of a library-owned device array."""

    def __init__(self, p, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (p, False),
                                         "version": 3}


def dev_tensor(torch, p, n, dtype):
    """Zero-copy torch view of n elements at device address p."""
    ts = {np.int32: "<i4", np.float32: "<f4"}[dtype]
    if n == 0:
        return torch.zeros(0, dtype=torch.int32 if dtype == np.int32 else torch.float32,
                           device="cuda")
    return torch.as_tensor(_DevArray(p, n, ts), device="cuda")


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
    if n == 0:
        return np.zeros(0, dtype)
    return dev_tensor(torch, ptr_, n, dtype).cpu().numpy()


def _fp64_errors(oracle, A, B, rows, rp, ci, v, base=0):
    """Per-entry relative error of FP32 C rows against the FP64 oracle, with
    a check that their columns match the oracle's."""
    errs, same = [], True
    for r in rows:
        srp, sci, sv = oracle.spgemm_f32(A, B, int(r), int(r) + 1)
        lo, hi = int(rp[r - base]), int(rp[r - base + 1])
        same &= bool(np.array_equal(sci, ci[lo:hi]) and
                     np.array_equal(sv.view(np.uint32), v[lo:hi].view(np.uint32)))
        if sci.size:
            d = oracle.numeric_f64(A, B, srp, sci, int(r), int(r) + 1)
            errs.append(np.abs(v[lo:hi] - d) / np.maximum(np.abs(d), 1e-30))
    e = np.concatenate(errs) if errs else np.zeros(1)
    return same, {"max": float(e.max()), "median": float(np.median(e)),
                  "p99": float(np.quantile(e, 0.99))}


# ---------------------------------------------------------------------------
# the R-MAT product (headline)
# ---------------------------------------------------------------------------

def rmat_product(scale):
    from rvsp_b200 import gen, ranks
    A = gen.rmat(scale=scale, edge_factor=16, seed=0)
    ops = gen.row_products(A, A)
    return A, ops, ranks.row_panels(ops)


def row_sample(A, ops, frac, seed):
    """A seeded uniform sample of A's rows as its own CSR (rows in order),
    and its product count against B = A."""
    from rvsp_b200.gen import CSR
    rng = np.random.default_rng(seed)
    m = max(1, int(round(A.rows * frac)))
    rows = np.sort(rng.choice(A.rows, m, replace=False))
    lens = np.diff(A.row_ptr.astype(np.int64))[rows]
    rp = np.zeros(m + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    # entry k of the sample is entry k - rp[i] of sampled row i
    idx = np.repeat(A.row_ptr[rows].astype(np.int64) - rp[:-1], lens) + np.arange(rp[-1])
    S = CSR(m, A.cols, rp.astype(np.int32), A.col_idx[idx], A.values[idx])
    return S, int(ops[rows].sum()), rows


def reference_sample_rate(A, ops, threads, target_s, seed):
    """The reference's one-shot kernel over a seeded row sample sized so one
    call takes about target_s on `threads` host threads; (GFLOP/s, sample
    description, seconds per call)."""
    import oracle
    frac = 1.0 / 1024  # pilot
    S, Ps, rows = row_sample(A, ops, frac, seed)
    t = oracle.ref_time_oneshot(S, A, nthreads=threads, repeats=1)
    frac = min(0.25, frac * target_s / max(t, 1e-3))
    S, Ps, rows = row_sample(A, ops, frac, seed)
    t = oracle.ref_time_oneshot(S, A, nthreads=threads, repeats=1)
    if t < 0:
        raise RuntimeError("reference kernel failed on the sample")
    desc = (f"{S.rows} seeded uniform rows of A ({frac:.5f} of {A.rows}) times A, "
            f"{Ps} products, rvsp_spgemm_scalar_f32 one-shot")
    return 2.0 * Ps / t / 1e9, desc, t, S, Ps


def run_headline(args):
    import torch

    import oracle
    import rvsp_b200 as rv
    from rvsp_b200 import ranks

    dist = ranks.init("gloo", timeout_s=1800)
    torch.cuda.set_device(0)
    torch.zeros(1, device="cuda")
    rv.lib()
    t0 = time.time()
    A, ops, panels_all = rmat_product(args.rmat_scale)
    P_all = int(ops.sum())
    panels = ranks.shard_panels(panels_all, ops, RANK, WORLD)
    log(f"rmat 2^{args.rmat_scale}: {A.rows} rows, nnz {A.nnz}, {P_all} products, "
        f"{len(panels_all)} panels ({len(panels)} on this rank), generated in "
        f"{time.time() - t0:.1f} s")
    dA = DevMat(A, torch)
    views = [PanelView(dA, r0, r1) for r0, r1 in panels]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def product(algo):
        for v in views:
            ptrs, n = _oneshot_dev(rv, v, dA, algo)
            rv.free_device(*ptrs)

    def timed(steps, warmup):
        """Learned and exact steps alternate, so both run under the same
        conditions (clock, power, host load); per algorithm: mean device ms
        per step, launches of the learned steps, kernel-family totals."""
        algos = (rv.RVSP_CUDA_ALGO_LEARNED, rv.RVSP_CUDA_ALGO_EXACT)
        for _ in range(warmup):
            for algo in algos:
                product(algo)
        torch.cuda.synchronize()
        ranks.barrier(dist)
        torch.cuda.synchronize()
        evs = {a: [] for a in algos}
        kts = {a: {} for a in algos}
        launches = 0
        for _ in range(steps):
            for algo in algos:
                flush.zero_()
                rv.kernel_timing(True)
                l0 = rv.launch_count()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                product(algo)
                e1.record()
                torch.cuda.synchronize()
                if algo == algos[0]:
                    launches += rv.launch_count() - l0
                for k, (t, n) in rv.kernel_times().items():
                    a = kts[algo].setdefault(k, [0.0, 0])
                    a[0] += t
                    a[1] += n
                rv.kernel_timing(False)
                evs[algo].append(e0.elapsed_time(e1))
        ranks.barrier(dist)
        ms = {a: ranks.max_over_ranks(dist, statistics.mean(evs[a])) for a in algos}
        return ms[algos[0]], ms[algos[1]], launches, kts[algos[0]], kts[algos[1]]

    sampler = ClockSampler()
    sampler.start()
    ms_l, ms_x, launches, kt_l, kt_x = timed(args.steps, args.warmup)
    clocks = sampler.stop()
    value = 2.0 * P_all / (ms_l * 1e-3) / 1e9
    exact_gflops = 2.0 * P_all / (ms_x * 1e-3) / 1e9

    # verification pass (untimed): every panel exact and learned, compared on
    # the device; C's row pointer kept for the byte counts; sampled rows of
    # the first and the heaviest panel against the oracle
    heavy_panel = int(np.argmax([ops[r0:r1].sum() for r0, r1 in panels]))
    rng = np.random.default_rng(1)
    identical = True
    row_nnz = np.zeros(A.rows, np.int64)
    parity_ok, errs = True, []
    for pi, (v, (r0, r1)) in enumerate(zip(views, panels)):
        px, nx = _oneshot_dev(rv, v, dA, rv.RVSP_CUDA_ALGO_EXACT)
        pl, nl = _oneshot_dev(rv, v, dA, rv.RVSP_CUDA_ALGO_LEARNED)
        if pi == heavy_panel:  # the learned sizing of the heaviest panel's one-shot product
            ls = rv.oneshot_learned_stats()
        m = r1 - r0
        same = nx == nl
        if same:
            for k, (dt, n) in enumerate(((np.int32, m + 1), (np.int32, nx), (np.float32, nx))):
                a = dev_tensor(torch, px[k], n, dt)
                b = dev_tensor(torch, pl[k], n, dt)
                same &= bool(torch.equal(a.view(torch.int32), b.view(torch.int32)))
        identical &= same
        rp = _d2h(px[0], m + 1, np.int32, torch).astype(np.int64)
        row_nnz[r0:r1] = np.diff(rp)
        if pi in (0, heavy_panel):
            rows = np.sort(rng.choice(np.arange(r0, r1), min(args.check_rows, m), replace=False))
            ci = _d2h(px[1], nx, np.int32, torch)
            vv = _d2h(px[2], nx, np.float32, torch)
            ok, e = _fp64_errors(oracle, A, A, rows, rp, ci, vv, base=r0)
            parity_ok &= ok
            errs.append(e)
            del ci, vv
        rv.free_device(*px)
        rv.free_device(*pl)
    nnz_c = int(ranks.sum_over_ranks(dist, int(row_nnz.sum())))

    e2e = run_rmat_e2e(rv, A, ops, panels, args, torch, dist)
    if RANK != 0:
        ranks.barrier(dist)
        if dist:
            dist.destroy_process_group()
        return

    # roofline of the dominant kernel (largest share of the exact path's
    # kernel time): algorithmic bytes of the rows it processes per launch
    hbm, peak_kind = peaks()
    fam, (fam_ms, fam_n) = max(kt_x.items(), key=lambda kv: kv[1][0])
    heavy = heavy_rows(ops, A.cols)
    a_len = np.diff(A.row_ptr.astype(np.int64))
    per_panel = []
    for r0, r1 in panels:
        h = heavy[r0:r1]
        per_panel.append(algorithmic_bytes(int(h.sum()), int(a_len[r0:r1][h].sum()),
                                           int(row_nnz[r0:r1][h].sum()), A.rows, A.nnz))
    bytes_heavy = sum(per_panel) / len(per_panel)
    fam_launch_ms = fam_ms / max(fam_n, 1)
    achieved = bytes_heavy / (fam_launch_ms * 1e-3) / 1e9 if fam.startswith("k_heavy") else None
    bytes_product = sum(algorithmic_bytes(r1 - r0, int(a_len[r0:r1].sum()),
                                          int(row_nnz[r0:r1].sum()), A.rows, A.nnz)
                        for r0, r1 in panels)
    steps_k = args.steps
    out = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": WORLD,
        "steps": steps_k, "warmup": args.warmup, "ms_per_step": round(ms_l, 3),
        "higher_is_better": True, "scaling": "strong" if WORLD > 1 else "weak",
        "vs_baseline": None, "dtype": "f32", "data": RMAT_DATA,
        "config": {"workload": f"rmat_scale{args.rmat_scale}_ef16_c_eq_a_times_a",
                   "rows": A.rows, "nnz_a": A.nnz, "products": P_all, "nnz_c": nnz_c,
                   "panels": len(panels_all),
                   "path": "one-shot rvsp_cuda_spgemm_f32 per row panel, device-resident operands",
                   "l2": "flushed (256 MiB write) before every timed step; C (78 GB) >> L2",
                   "parallelism": f"row panels over {WORLD} GPU(s), no data-path collective"},
        "exact_gflops": round(exact_gflops, 3), "exact_ms_per_step": round(ms_x, 3),
        "learned_over_exact": round(ms_x / ms_l, 4),
        "learned_bit_identical_to_exact": bool(identical),
        "parity": {"sampled_rows_bit_exact_vs_oracle": bool(parity_ok),
                   "rows_checked": int(2 * args.check_rows),
                   "fp32_vs_fp64_rel_err": errs},
        "mispredict": {"panel": heavy_panel, **ls,
                       "rate": ls["underpredicted_rows"] / max(ls["predicted_rows"], 1),
                       "refill_rate": ls["overflowed_rows"] / max(ls["predicted_rows"], 1)},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1) if achieved else None,
                     "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 4) if achieved else None,
                     **committed_traffic(fam, bytes_heavy),
                     "peak_source": f"{peak_kind} hbm_gbs", "kernel": fam,
                     "bytes_per_launch": int(bytes_heavy), "launch_ms": round(fam_launch_ms, 3),
                     "whole_product_frac_learned": round(
                         bytes_product / (ms_l * 1e-3) / 1e9 / hbm, 4)},
        "kernel_ms_per_step": {
            "learned": {k: round(v[0] / steps_k, 3) for k, v in kt_l.items() if v[1]},
            "exact": {k: round(v[0] / steps_k, 3) for k, v in kt_x.items() if v[1]}},
        "e2e": e2e,
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if WORLD == 1:
        out["cpu_baseline"] = cpu_baseline_rmat(A, ops)
    if args.extras:
        out["extras"] = run_extras(args, rv, torch)
    print(json.dumps(out), flush=True)
    ranks.barrier(dist)
    if dist:
        dist.destroy_process_group()


def committed_traffic(kernel, bytes_per_launch):
    """DRAM traffic of the dominant kernel from the committed ncu summary
    (profiles/traffic.json: read + write bytes of one captured launch per
    algorithmic byte of that launch, scaled here to this launch's algorithmic
    bytes), labelled as such; None when no capture covers the kernel."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        ratio = json.load(open(path))["rmat"][kernel]["dram_bytes_per_algorithmic_byte"]
    except Exception:
        return {"traffic": None, "traffic_source": "no ncu capture of this kernel committed"}
    return {"traffic": int(ratio * bytes_per_launch),
            "traffic_source": "committed ncu figure (profiles/traffic.json), DRAM bytes per "
                              "algorithmic byte of a captured launch scaled to this launch"}


def run_rmat_e2e(rv, A, ops, panels, args, torch, dist=None):
    """The product through rvsp_spgemm_csr (learned backend) on host CSR:
    each panel's A (its row pointer rebased, its entries a view) and B = A are
    host arrays; the library uploads them and hands C back in host arrays
    (staged through pinned memory), freed by rvsp_csr_destroy. Wall time of
    this rank's panels per step; with several ranks the timed steps start
    after a barrier, the time is the slowest rank's and the products and
    bytes are every rank's (the whole job)."""
    import ctypes as C

    from rvsp_b200 import ranks
    L = rv.lib()
    hb = rv.csr_struct(A.rows, A.cols, A.nnz, A.row_ptr, A.col_idx, A.values)
    pa = []
    for r0, r1 in panels:
        s, e = int(A.row_ptr[r0]), int(A.row_ptr[r1])
        rp = (A.row_ptr[r0:r1 + 1] - A.row_ptr[r0]).astype(np.int32)
        ci, v = A.col_idx[s:e], A.values[s:e]
        pa.append((rp, ci, v, rv.csr_struct(r1 - r0, A.cols, e - s, rp, ci, v)))
    opts = rv.SpgemmOptions(rv.RVSP_BACKEND_CUDA_LEARNED, rv.RVSP_DTYPE_FP32, rv.RVSP_DTYPE_FP32)
    h2d = d2h = 0

    def step():
        nonlocal h2d, d2h
        h2d = d2h = 0
        for (rp, ci, v, a), (r0, r1) in zip(pa, panels):
            c = rv.CsrMatrix()
            rv.check(L.rvsp_spgemm_csr(C.byref(a), C.byref(hb), C.byref(c), C.byref(opts)),
                     "rvsp_spgemm_csr")
            h2d += 4 * (rp.size + A.rows + 1) + 8 * (ci.size + A.nnz)
            d2h += 4 * (r1 - r0 + 1) + 8 * c.nnz
            L.rvsp_csr_destroy(C.byref(c))

    steps = max(1, min(args.steps, args.e2e_steps))
    step()  # warm-up
    ranks.barrier(dist)
    ts = []
    for _ in range(steps):
        t0 = time.perf_counter()
        step()
        ts.append(time.perf_counter() - t0)
    t = ranks.max_over_ranks(dist, statistics.mean(ts))
    P = ranks.sum_over_ranks(dist, int(sum(ops[r0:r1].sum() for r0, r1 in panels)))
    h2d = ranks.sum_over_ranks(dist, h2d)
    d2h = ranks.sum_over_ranks(dist, d2h)
    return {"value": round(2.0 * P / t / 1e9, 3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "steps": steps,
            "api": "rvsp_spgemm_csr (RVSP_BACKEND_CUDA_LEARNED) per row panel, host A/B/C",
            "ms_per_step": round(t * 1e3, 1)}


def cpu_baseline_rmat(A, ops):
    """Reference scalar one-shot (oracle/_ref) on 1 host core, seeded row sample."""
    import oracle
    if not oracle.ref_available():
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                "sample": "unavailable: oracle/_ref not built"}
    g, desc, t, _, _ = reference_sample_rate(A, ops, 1, 12.0, seed=7)
    return {"value": round(g, 4), "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"{desc}, {t:.1f} s, 1 thread"}


def run_reference(args):
    """The reference's own CPU kernel on all host cores (rank 0 only)."""
    if RANK != 0:
        return
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/librvsp_ref.so not built"}), flush=True)
        return
    if args.workload == "poisson_reuse":
        return run_reference_poisson(args)
    cores = len(os.sched_getaffinity(0))
    A, ops, _ = rmat_product(args.rmat_scale)
    _, desc, _, S, Ps = reference_sample_rate(A, ops, cores, 1.5, seed=11)
    for _ in range(args.warmup):
        oracle.ref_time_oneshot(S, A, nthreads=cores, repeats=1)
    times = [oracle.ref_time_oneshot(S, A, nthreads=cores, repeats=1) for _ in range(args.steps)]
    t = sum(times) / len(times)
    value = 2.0 * Ps / t / 1e9
    out = {"metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": WORLD,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t * 1e3, 3),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": RMAT_DATA,
           "config": {"workload": f"rmat_scale{args.rmat_scale}_ef16_c_eq_a_times_a",
                      "rows": A.rows, "nnz_a": A.nnz, "products": int(ops.sum()),
                      "path": "reference rvsp_spgemm_scalar_f32 one-shot, row sample"},
           "impl": "reference",
           "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": cores,
                            "kind": "reference",
                            "sample": f"{desc}, {cores} threads on row panels per step"},
           "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# descriptor reuse of the Poisson product
# ---------------------------------------------------------------------------

def poisson_workload():
    from rvsp_b200 import gen
    A = gen.poisson2d(1024)
    P = gen.products(A, A)
    return A, P


def poisson_reuse(args, rv, torch, steps, warmup):
    """Numeric-only reuse of the 1024^2 Poisson product (graph replay): device
    time per step, roofline of the map-replay kernel, parity of the first fill
    against the reference's output digests."""
    import ctypes as C
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

    for i in range(warmup):
        step(i)
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(steps)]
    l0 = rv.launch_count()
    for i in range(steps):
        step(warmup + i, *evs[i])
    torch.cuda.synchronize()
    launches = rv.launch_count() - l0
    ms = sum(a.elapsed_time(b) for a, b in evs) / steps
    rv.check(L.rvsp_cuda_plan_set_async(plan, 0))
    L.rvsp_cuda_plan_destroy(plan)
    hbm, peak_kind = peaks()
    bytes_alg = algorithmic_bytes(M, nnz_a, nnz_c, M, nnz_a)
    bytes_distinct = bytes_alg - (4 * (M + 1) + 8 * nnz_a)  # B's arrays are A's
    achieved = bytes_alg / (ms * 1e-3) / 1e9
    return {"gflops": round(2.0 * P / (ms * 1e-3) / 1e9, 3), "ms_per_step": round(ms, 5),
            "steps": steps, "gpu_launches": int(launches),
            "config": {"workload": "poisson2d_1024_descriptor_reuse", "rows": M, "nnz_a": nnz_a,
                       "nnz_c": nnz_c, "products": P, "path": "numeric-only, CUDA graph",
                       "l2": "flushed (256 MiB write) before every timed step"},
            "parity_first_pass_vs_reference": parity,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm,
                         "unit": "GB/s", "frac": round(achieved / hbm, 4),
                         "peak_source": f"{peak_kind} hbm_gbs", "kernel": "k_tiny_reuse_map",
                         "bytes_per_launch": bytes_alg,
                         "frac_distinct_arrays": round(
                             bytes_distinct / (ms * 1e-3) / 1e9 / hbm, 4)}}


def poisson_e2e(rv, A, P, steps, warmup):
    """rvsp_spgemm_compute (descriptor reuse) with pinned host A and C."""
    import torch

    def pinned(a):
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()

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
    for i in range(warmup):
        hvn[:] = variants[i % 4]
        rv.check(d.compute(a, a, c, wsb))
    times = []
    for i in range(steps):
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


def run_poisson_line(args):
    """--workload poisson_reuse: the descriptor-reuse product as its own line."""
    import torch

    import rvsp_b200 as rv
    from rvsp_b200 import ranks
    dist = ranks.init("gloo", timeout_s=300)
    torch.cuda.set_device(0)
    torch.zeros(1, device="cuda")
    sampler = ClockSampler()
    sampler.start()
    ranks.barrier(dist)
    r = poisson_reuse(args, rv, torch, args.steps, args.warmup)
    ms_max = ranks.max_over_ranks(dist, r["ms_per_step"])
    A, P = poisson_workload()
    e2e = poisson_e2e(rv, A, P, args.steps, args.warmup)
    clocks = sampler.stop()
    ranks.barrier(dist)
    if RANK == 0:
        out = {"metric": METRIC, "value": round(2.0 * P * WORLD / (ms_max * 1e-3) / 1e9, 3),
               "unit": UNIT, "n_gpus": WORLD, "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32",
               "data": "synthetic (5-point Laplacian, values rescaled U(0.5,1.5) per step, seeded)",
               "config": dict(r["config"], parallelism=f"{WORLD} independent products, one per GPU"),
               "parity_first_pass_vs_reference": r["parity_first_pass_vs_reference"],
               "roofline": r["roofline"], "e2e": e2e, "gpu_launches": r["gpu_launches"],
               "clocks": clocks}
        if WORLD == 1:
            out["cpu_baseline"] = cpu_baseline_poisson(A, P)
        print(json.dumps(out), flush=True)
    if dist:
        dist.destroy_process_group()


def cpu_baseline_poisson(A, P, budget_s=10.0):
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


def run_reference_poisson(args):
    import oracle
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
# the other configurations: exact vs learned, batched vs sequential
# ---------------------------------------------------------------------------

def compare_plain(rv, torch, steps, warmup, which="plain", ts_rows=2_000_000, fp64_rows=400):
    """One-shot product of the plain or tall-skinny configuration, exact vs
    learned, device-resident operands, median wall time per product."""
    import oracle
    from rvsp_b200 import gen
    if which == "plain":
        A = gen.uniform_fixed()
        B = A
        cfg = {"workload": "plain_4096x4096_16_per_row", "seed": 0}
    else:
        A, B = gen.tall_skinny(a_rows=ts_rows)
        cfg = {"workload": f"tall_skinny_{ts_rows}x100000_x_100000^2", "a_rows": A.rows,
               "nnz_a": A.nnz, "nnz_b": B.nnz}
    P = gen.products(A, B)
    dA, dB = DevMat(A, torch), DevMat(B, torch)
    times, outs = {}, {}
    for name, algo in (("exact", rv.RVSP_CUDA_ALGO_EXACT), ("learned", rv.RVSP_CUDA_ALGO_LEARNED)):
        def fn(algo=algo):
            ptrs, n = _oneshot_dev(rv, dA, dB, algo)
            rv.free_device(*ptrs)
        times[name] = _time(fn, steps, warmup, torch)
        ptrs, n = _oneshot_dev(rv, dA, dB, algo)
        outs[name] = (_d2h(ptrs[0], A.rows + 1, np.int32, torch),
                      _d2h(ptrs[1], n, np.int32, torch), _d2h(ptrs[2], n, np.float32, torch))
        rv.free_device(*ptrs)
    same = all(np.array_equal(a, b) for a, b in zip(outs["exact"], outs["learned"]))
    nnz_c = int(outs["exact"][0][-1])
    res = {"config": dict(cfg, rows=A.rows, products=P, nnz_c=nnz_c),
           "exact_gflops": 2 * P / times["exact"] / 1e9,
           "learned_gflops": 2 * P / times["learned"] / 1e9,
           "learned_over_exact": times["exact"] / times["learned"],
           "learned_bit_identical_to_exact": bool(same),
           "ms": {k: v * 1e3 for k, v in times.items()}}
    b_alg = algorithmic_bytes(A.rows, A.nnz, nnz_c, B.rows, B.nnz)
    res["bytes_alg"] = b_alg
    res["hbm_frac_exact"] = b_alg / times["exact"] / 1e9 / peaks()[0]
    rng = np.random.default_rng(0)
    rows = np.sort(rng.choice(A.rows, min(fp64_rows, A.rows), replace=False))
    rp, ci, v = outs["exact"]
    ok, e = _fp64_errors(oracle, A, B, rows, rp.astype(np.int64), ci, v)
    res["sampled_rows_bit_exact_vs_oracle"] = bool(ok)
    res["fp32_vs_fp64_rel_err"] = dict(e, rows_sampled=int(rows.size))
    return res


def compare_batched(rv, torch, steps, warmup, count=512):
    """512 uneven products: 512 sequential one-shot calls vs the batched
    entry point (exact and learned), spot-checked against the oracle."""
    import oracle
    from rvsp_b200 import gen
    pairs = gen.batched_uneven(count=count)
    prods = [gen.products(A, B) for A, B in pairs]
    P = sum(prods)
    dev_pairs = [(DevMat(A, torch), DevMat(B, torch)) for A, B in pairs]

    def seq():
        for dA, dB in dev_pairs:
            ptrs, n = _oneshot_dev(rv, dA, dB, rv.RVSP_CUDA_ALGO_EXACT)
            rv.free_device(*ptrs)
    times = {"sequential_exact": _time(seq, max(1, steps // 3), 1, torch)}
    for name, algo in (("batched_exact", rv.RVSP_CUDA_ALGO_EXACT),
                       ("batched_learned", rv.RVSP_CUDA_ALGO_LEARNED)):
        def fn(algo=algo):
            ptrs, n, offs, coffs = rv.spgemm_batched(dev_pairs, algo)
            rv.free_device(*ptrs)
        times[name] = _time(fn, steps, warmup, torch)
    torch.cuda.synchronize()
    rv.kernel_timing(True)
    ptrs, n, offs, coffs = rv.spgemm_batched(dev_pairs, rv.RVSP_CUDA_ALGO_LEARNED)
    torch.cuda.synchronize()
    kt = {k: round(v[0], 3) for k, v in rv.kernel_times().items() if v[1]}
    rv.kernel_timing(False)
    total_rows = int(offs[-1])
    crp = _d2h(ptrs[0], total_rows + len(pairs), np.int32, torch).astype(np.int64)
    ok = True
    order = np.argsort(prods)
    check = sorted({int(order[-1]), int(order[0]), 0, len(pairs) // 2, len(pairs) - 1})
    for i in check:
        A, B = pairs[i]
        r0 = int(offs[i]) + i
        e0, e1 = int(coffs[i]), int(coffs[i + 1])
        wrp, wci, wv = oracle.spgemm_f32(A, B)
        ci = _d2h(ptrs[1] + 4 * e0, e1 - e0, np.int32, torch)
        v = _d2h(ptrs[2] + 4 * e0, e1 - e0, np.float32, torch)
        ok &= bool(np.array_equal(crp[r0:r0 + A.rows + 1], wrp) and np.array_equal(ci, wci) and
                   np.array_equal(v.view(np.uint32), wv.view(np.uint32)))
    rv.free_device(*ptrs)
    return {"config": {"workload": f"batched_{len(dev_pairs)}_uneven", "products": P,
                       "rows": total_rows, "nnz_c": int(n), "calls": 1},
            "gflops": {k: 2 * P / t / 1e9 for k, t in times.items()},
            "ms": {k: t * 1e3 for k, t in times.items()},
            "batched_learned_over_sequential": times["sequential_exact"] / times["batched_learned"],
            "batched_learned_over_batched_exact": times["batched_exact"] / times["batched_learned"],
            "products_checked_vs_oracle": check,
            "spot_check_bit_exact_vs_oracle": bool(ok),
            "kernel_ms_batched_learned": kt}


def run_extras(args, rv, torch):
    """The other configurations' headline numbers, briefly: descriptor reuse
    (Poisson), batched vs sequential, plain 4096^2."""
    out = {}
    try:
        out["poisson_reuse"] = poisson_reuse(args, rv, torch, 20, 5)
        out["plain_4096"] = compare_plain(rv, torch, 10, 3, "plain", fp64_rows=100)
        out["batched_512"] = compare_batched(rv, torch, 3, 1)
    except Exception as e:  # an extra never hides the headline
        out["error"] = repr(e)
    return out


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
    passes = (2 * scale + 7) // 8
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


def profile_matrices(name):
    from rvsp_b200 import gen
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
    raise SystemExit(f"unknown matrix {name}")


def run_profile(args, rv, torch):
    """One-shot products of a named matrix (rmatS, tall, plain, poisson),
    optionally a row range of A (a device panel), for capturing one kernel:
    the first step is a warm-up; prints the median time and the per-family
    kernel times of the timed steps."""
    from rvsp_b200 import gen
    A, B = profile_matrices(args.case)
    r0, r1 = (0, A.rows) if args.rows is None else (int(x) for x in args.rows.split(":"))
    dA, dB = DevMat(A, torch), DevMat(B, torch)
    view = PanelView(dA, r0, r1)
    P = int(gen.row_products(A, B)[r0:r1].sum())
    if args.params:
        rv.check(rv.set_default_params([int(x) for x in args.params.split(",")]), "params")
    algo = rv.RVSP_CUDA_ALGO_EXACT if args.algo == "exact" else rv.RVSP_CUDA_ALGO_LEARNED
    times = []
    nnz = 0
    for i in range(max(args.steps, 1)):
        if i == 1:
            rv.kernel_timing(True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ptrs, nnz = _oneshot_dev(rv, view, dB, algo)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
        rv.free_device(*ptrs)
    kt = rv.kernel_times()
    rv.kernel_timing(False)
    timed = times[1:] if len(times) > 1 else times
    t = statistics.median(timed)
    return {"case": args.case, "rows": [r0, r1], "algo": args.algo, "params": args.params,
            "products": P, "nnz_c": nnz, "ms": t * 1e3, "gflops": 2 * P / t / 1e9,
            "kernel_ms_per_step": {k: round(v[0] / len(timed), 3) for k, v in kt.items() if v[1]}}


def run_compare(args):
    import torch

    import rvsp_b200 as rv
    torch.zeros(1, device="cuda")
    rv.lib()
    if args.workload in ("plain", "tall_skinny"):
        res = compare_plain(rv, torch, args.steps, args.warmup,
                            "plain" if args.workload == "plain" else "tall", args.ts_rows)
    elif args.workload == "batched":
        res = compare_batched(rv, torch, args.steps, args.warmup, args.batch_count)
    elif args.workload == "coo":
        res = run_coo(args, rv, torch)
    else:
        res = run_profile(args, rv, torch)
    if RANK == 0:
        print(json.dumps({"workload": args.workload, **res}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rmat",
                    choices=["rmat", "poisson_reuse", "plain", "batched", "tall_skinny", "coo",
                             "profile"])
    ap.add_argument("--rmat-scale", type=int, default=20)
    ap.add_argument("--check-rows", type=int, default=100,
                    help="rmat: rows of two panels checked against the oracle")
    ap.add_argument("--e2e-steps", type=int, default=2, help="rmat: timed e2e steps (host API)")
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="rmat: skip the other configurations' numbers")
    ap.add_argument("--batch-count", type=int, default=512)
    ap.add_argument("--ts-rows", type=int, default=2_000_000)
    ap.add_argument("--case", default="rmat18", help="profile: rmatS, tall, plain, poisson")
    ap.add_argument("--rows", default=None, help="profile: row range R0:R1 of A")
    ap.add_argument("--algo", default="exact", choices=["exact", "learned"])
    ap.add_argument("--params", default=None, help="profile: tiny,slack,warpmax,cwlog2")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "rmat":
        run_headline(args)
    elif args.workload == "poisson_reuse":
        run_poisson_line(args)
    else:
        run_compare(args)


if __name__ == "__main__":
    main()
