"""Train the row-size predictor of the learned SpGEMM path.

    python -m rvsp_b200.train --out weights/row_mlp_v1.bin [--epochs 40]

Run from rv-sparse_b200/ on a machine with a CUDA device. Steps:

1. Corpus: seeded synthetic products of several families -- fixed-degree
   uniform, Poisson-degree uniform (the batched-product family), R-MAT graphs
   (several skews), tall-skinny products with power-law B rows, banded
   matrices. Each is analysed by the library's exact path (rvsp_cuda_symbolic
   with features on), which returns every row's features and exact nnz.
2. Rows whose upper bound exceeds the tiny bin (the only rows the learned
   path predicts) are kept; features enter as log2(1 + f), standardised with
   the training mean and std; the target is log2(1 + nnz).
3. rvsp_cuda_mlp_train fits the 4-32-32-2 network on the GPU (Gaussian NLL,
   Adam). Families held out from training (a different seed set) choose the
   safety quantile z so that about --overflow of their rows would outgrow the
   capacity 2^(mu + z sigma) - 1.
4. The checkpoint (magic, version, model, checksum) is written with
   rvsp_cuda_mlp_save, and a JSON report beside it records the loss curve,
   the held-out overflow rate, and how much capacity the prediction saves
   against the upper bound the exact path uses.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import gen
import rvsp_b200 as rv

TINY_OPS = 32


def corpus(seed: int, scale: float = 1.0):
    """(name, A, B) products of every family, seeded."""
    rng = np.random.default_rng(seed)
    s = lambda n: max(64, int(n * scale))  # noqa: E731
    out = []
    for cols in (512, 4096, 65536):
        for per in (8, 16, 32, 64):
            A = gen.uniform_fixed(s(3000), s(3000), per, seed=int(rng.integers(1 << 30)))
            B = gen.uniform_fixed(s(3000), cols, per, seed=int(rng.integers(1 << 30)))
            out.append((f"uniform_c{cols}_k{per}", A, B))
    for lam in (4.0, 8.0, 16.0, 24.0, 32.0):
        for n in (300, 3000, 30000):
            A = gen.poisson_rows(s(n), s(n), lam, rng)
            B = gen.poisson_rows(s(n), s(n), lam, rng)
            out.append((f"poisson_n{n}_l{lam:g}", A, B))
    # power-law graphs up to 2^18 vertices: their heavy rows (a warp per
    # column chunk) are sized by the prediction too
    for sc, (a, b, c) in ((12, (0.57, 0.19, 0.19)), (13, (0.45, 0.22, 0.22)),
                          (14, (0.57, 0.19, 0.19)), (13, (0.65, 0.15, 0.15)),
                          (16, (0.57, 0.19, 0.19)), (17, (0.57, 0.19, 0.19)),
                          (18, (0.57, 0.19, 0.19)), (16, (0.45, 0.22, 0.22))):
        R = gen.rmat(scale=sc, edge_factor=16, a=a, b=b, c=c, seed=int(rng.integers(1 << 30)))
        out.append((f"rmat_s{sc}_a{a}", R, R))
    for bmax in (500, 4000):
        A, B = gen.tall_skinny(a_rows=s(40000), k=s(8000), n=s(8000), b_max=bmax,
                               seed=int(rng.integers(1 << 30)))
        out.append((f"tall_bmax{bmax}", A, B))
    for bw in (8, 64, 512):  # banded: column j in [i - bw, i + bw]
        n = s(20000)
        rows = np.repeat(np.arange(n), 12)
        cols = np.clip(rows + rng.integers(-bw, bw + 1, rows.size), 0, n - 1)
        keys = np.unique(rows.astype(np.int64) * n + cols)
        M = gen.from_keys(n, n, keys, None, rng)
        out.append((f"band{bw}", M, M))
    return out


def collect(A, B):
    """Features, exact nnz and upper bounds of every row of A * B (exact path)."""
    plan = rv.Plan(rv.RVSP_CUDA_ALGO_EXACT, features=True)
    st, nnz = plan.symbolic(A, B)
    rv.check(st, "symbolic")
    feat, cnt, ub = plan.row_stats()
    plan.close()
    return feat, cnt, ub


def dataset(seed: int, scale: float, max_rows_per_product: int = 60000):
    X, Y, U, names = [], [], [], []
    rng = np.random.default_rng(seed + 17)
    ops_all = []
    for name, A, B in corpus(seed, scale):
        feat, cnt, ub = collect(A, B)
        keep = np.nonzero(feat[:, 1] > TINY_OPS)[0]
        if keep.size > max_rows_per_product:
            keep = np.sort(rng.choice(keep, max_rows_per_product, replace=False))
        X.append(feat[keep])
        Y.append(cnt[keep])
        U.append(ub[keep])
        names += [name] * keep.size
        ops_all.append(feat[keep, 1])
    return (np.concatenate(X).astype(np.float32), np.concatenate(Y).astype(np.float32),
            np.concatenate(U).astype(np.int32), np.array(names))


def he_init(rng):
    p = {}
    p["W1"] = rng.normal(0, math.sqrt(2 / 4), (32, 4))
    p["b1"] = np.zeros(32)
    p["W2"] = rng.normal(0, math.sqrt(2 / 32), (32, 32))
    p["b2"] = np.zeros(32)
    p["W3"] = rng.normal(0, math.sqrt(1 / 32), (2, 32))
    p["b3"] = np.array([6.0, 0.0])
    return rv.pack_params(p).astype(np.float32)


def train(args):
    t0 = time.time()
    Xr, cnt, ub, names = dataset(args.seed, args.scale)
    Xh, cnth, ubh, namesh = dataset(args.seed + 1000, args.scale)
    t_data = time.time() - t0
    L = rv.lib()
    logx = np.log2(1.0 + Xr)
    mean = logx.mean(0).astype(np.float32)
    std = np.maximum(logx.std(0), 1e-3).astype(np.float32)
    inv_std = (1.0 / std).astype(np.float32)
    X = ((logx - mean) * inv_std).astype(np.float32)
    y = np.log2(1.0 + cnt).astype(np.float32)
    params = he_init(np.random.default_rng(args.seed))
    losses = np.zeros(args.epochs, np.float32)
    t1 = time.time()
    rv.check(L.rvsp_cuda_mlp_train(params.ctypes.data, X.ctypes.data, y.ctypes.data, None,
                                   X.shape[0], args.epochs, args.batch, args.lr, args.seed,
                                   losses.ctypes.data), "mlp_train")
    t_train = time.time() - t1
    # choose z on held-out products
    model = rv.model_to_vector(mean, inv_std, 0.0, params)
    mu = np.zeros(Xh.shape[0], np.float32)
    sig = np.zeros(Xh.shape[0], np.float32)
    cap = np.zeros(Xh.shape[0], np.int32)
    rv.check(L.rvsp_cuda_mlp_infer(model.ctypes.data, rv.MLP_FLOATS, Xh.ctypes.data,
                                   ubh.ctypes.data, Xh.shape[0], mu.ctypes.data, sig.ctypes.data,
                                   cap.ctypes.data), "mlp_infer")
    yh = np.log2(1.0 + cnth)
    zneed = (yh - mu) / sig
    z = float(np.quantile(zneed, 1.0 - args.overflow))
    model = rv.model_to_vector(mean, inv_std, z, params)
    rv.check(L.rvsp_cuda_mlp_infer(model.ctypes.data, rv.MLP_FLOATS, Xh.ctypes.data,
                                   ubh.ctypes.data, Xh.shape[0], mu.ctypes.data, sig.ctypes.data,
                                   cap.ctypes.data), "mlp_infer")
    over = cap < cnth
    per_family = {}
    for fam in sorted(set(n.split("_")[0] for n in namesh)):
        m = np.array([n.split("_")[0] == fam for n in namesh])
        per_family[fam] = {"rows": int(m.sum()), "overflow_rate": float(over[m].mean()),
                           "capacity_over_nnz": float(cap[m].sum() / max(cnth[m].sum(), 1)),
                           "ub_over_nnz": float(ubh[m].sum() / max(cnth[m].sum(), 1))}
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    rv.check(L.rvsp_cuda_mlp_save(args.out.encode(), model.ctypes.data, rv.MLP_FLOATS), "save")
    report = {
        "checkpoint": os.path.basename(args.out),
        "train_rows": int(X.shape[0]), "heldout_rows": int(Xh.shape[0]),
        "epochs": args.epochs, "batch": args.batch, "lr": args.lr, "seed": args.seed,
        "feature_mean_log2": mean.tolist(), "feature_std_log2": std.tolist(), "z": z,
        "loss_first_last": [float(losses[0]), float(losses[-1])],
        "loss_curve": [round(float(v), 5) for v in losses],
        "heldout_overflow_rate": float(over.mean()),
        "heldout_capacity_over_nnz": float(cap.sum() / max(cnth.sum(), 1)),
        "heldout_ub_over_nnz": float(ubh.sum() / max(cnth.sum(), 1)),
        "per_family": per_family,
        "seconds": {"data": round(t_data, 2), "train_gpu": round(t_train, 2)},
    }
    with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
        json.dump(report, f, indent=1)
    print(json.dumps({k: v for k, v in report.items() if k != "loss_curve"}, indent=1))
    return report


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(rv.PKG_DIR, "weights", "row_mlp_v1.bin"))
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--overflow", type=float, default=0.02)
    train(ap.parse_args())


if __name__ == "__main__":
    main()
