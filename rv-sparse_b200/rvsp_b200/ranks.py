"""Host-side logic of runs over several GPUs, one process per GPU.

Output rows of C = A * B are independent, so nothing in the product needs a
collective: a product larger than one GPU is split into row panels
(contiguous row ranges, each holding at most 2^31 - 1 intermediate products
so its nnz fits an int32 row pointer), and the panels are dealt to the ranks
in contiguous groups of about equal products. B is read whole by every rank:
each rank loads it, or one rank broadcasts it (broadcast_operand). The only
other collectives are the timing ones (a barrier around the timed region, the
maximum of the per-rank times, the sum of the per-rank output sizes) and, to
place each rank's C rows in one global C, an exclusive scan of the per-rank
nnz built from one gathered int64 per rank (c_offsets).
"""

from __future__ import annotations

import datetime
import os

import numpy as np

PANEL_LIMIT = (1 << 31) - 1


def row_panels(ops, limit: int = PANEL_LIMIT):
    """Contiguous row ranges [r0, r1) whose products stay within limit.

    ops: per-row intermediate products (int64). A single row above the limit
    still gets a panel of its own (its nnz is bounded by cols(B))."""
    ops = np.asarray(ops, np.int64)
    cum = np.cumsum(ops)
    out, r0, base = [], 0, 0
    n = len(ops)
    while r0 < n:
        r1 = int(np.searchsorted(cum, base + limit, side="right"))
        r1 = max(r1, r0 + 1)
        out.append((r0, r1))
        base = int(cum[r1 - 1])
        r0 = r1
    return out


def shard_panels(panels, ops, rank: int, world: int):
    """The contiguous group of panels that rank `rank` of `world` computes:
    panel i goes to the rank whose share of the cumulative products holds the
    panel's midpoint, so every panel has exactly one owner."""
    if world <= 1:
        return list(panels)
    ops = np.asarray(ops, np.int64)
    w = np.array([ops[r0:r1].sum() for r0, r1 in panels], np.float64)
    cum = np.concatenate([[0.0], np.cumsum(w)])
    mid = (cum[:-1] + cum[1:]) / 2
    owner = np.minimum((mid * world / max(cum[-1], 1.0)).astype(np.int64), world - 1)
    return [p for p, o in zip(panels, owner) if o == rank]


def init(backend: str = "gloo", timeout_s: int = 300):
    """torch.distributed over the launcher's environment (RANK, WORLD_SIZE,
    MASTER_ADDR, MASTER_PORT), or None for a single process."""
    if int(os.environ.get("WORLD_SIZE", "1")) <= 1:
        return None
    import torch.distributed as dist
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(dist, value: float) -> float:
    """The maximum of value over all ranks (value itself without dist)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t[0])


def sum_over_ranks(dist, value: int) -> int:
    """The sum of an integer over all ranks (value itself without dist)."""
    if dist is None:
        return int(value)
    import torch
    t = torch.tensor([int(value)], dtype=torch.int64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return int(t[0])


def barrier(dist) -> None:
    if dist is not None:
        dist.barrier()


def broadcast_operand(dist, t, src: int = 0):
    """Replicates rank src's tensor t (one of B's arrays) on every rank, in
    place: an NCCL broadcast over NVLink between GPUs (t on the device), a
    gloo broadcast on CPU. Returns t."""
    if dist is not None:
        dist.broadcast(t, src=src)
    return t


def c_offsets(dist, local_nnz: int, device: str = "cpu"):
    """(first, total): where this rank's C entries start in the global C (the
    exclusive scan of the ranks' nnz, in rank order, which is row order since
    ranks own contiguous panel groups) and the global nnz. One int64 per rank
    is gathered; device is where the gathered tensors live (the GPU under
    NCCL)."""
    if dist is None:
        return 0, int(local_nnz)
    import torch
    t = torch.tensor([int(local_nnz)], dtype=torch.int64, device=device)
    parts = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(dist.get_world_size())]
    dist.all_gather(parts, t)
    sizes = [int(p[0]) for p in parts]
    return sum(sizes[:dist.get_rank()]), sum(sizes)

