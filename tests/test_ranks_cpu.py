"""Multi-rank host logic on CPU: two gloo ranks on 127.0.0.1.

Over several GPUs a product is split into row panels and each rank computes
its own contiguous group of panels (rvsp_b200.ranks). B is broadcast from rank
0; the collectives are that broadcast, the timing barrier, the max of the
per-rank times, the sum of the per-rank nnz and the gather of one int64 a rank
that places each rank's C in the global C. Here each rank computes its panels
with the oracle instead of a GPU, and rank 0 checks that the gathered panels,
put at their global offsets, are exactly the whole product.
"""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

WORLD = 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _product():
    from rvsp_b200 import gen
    A = gen.rmat(scale=10, edge_factor=8, seed=3)
    return A, A


def _worker(rank, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(WORLD))
    import oracle
    from rvsp_b200 import gen, ranks
    dist = ranks.init("gloo", timeout_s=60)
    try:
        assert ranks.max_over_ranks(dist, rank + 1.5) == WORLD + 0.5
        assert ranks.sum_over_ranks(dist, rank + 1) == WORLD * (WORLD + 1) // 2
        A, B = _product()
        # B's arrays from rank 0: the other ranks start from zeros
        import torch
        b_arrays = [torch.from_numpy(np.ascontiguousarray(a)) for a in (B.row_ptr, B.col_idx, B.values)]
        got = [a.clone() if rank == 0 else torch.zeros_like(a) for a in b_arrays]
        for t in got:
            ranks.broadcast_operand(dist, t, src=0)
        assert all(torch.equal(g, a) for g, a in zip(got, b_arrays))
        ops = gen.row_products(A, B)
        panels = ranks.row_panels(ops, limit=max(1, int(ops.sum()) // 7))
        mine = ranks.shard_panels(panels, ops, rank, WORLD)
        parts = []
        for r0, r1 in mine:
            rp, ci, v = oracle.spgemm_f32(A, B, r0, r1)
            parts.append((r0, r1, rp, ci, v))
        local = sum(int(p[2][-1]) for p in parts)
        nnz = ranks.sum_over_ranks(dist, local)
        first, total = ranks.c_offsets(dist, local)
        assert total == nnz
        gathered = [None] * WORLD
        import torch.distributed as td
        td.all_gather_object(gathered, (first, parts))
        ranks.barrier(dist)
        if rank == 0:
            allp = sorted((p for g in gathered for p in g[1]), key=lambda p: p[0])
            assert [(p[0], p[1]) for p in allp] == panels  # every panel exactly once
            w_rp, w_ci, w_v = oracle.spgemm_f32(A, B)
            assert nnz == w_ci.size
            # each rank's C entries start at its exclusive-scan offset
            for first_r, parts_r in gathered:
                if parts_r:
                    assert first_r == int(w_rp[parts_r[0][0]])
            ci = np.concatenate([p[3] for p in allp])
            v = np.concatenate([p[4] for p in allp])
            rp, off = [np.zeros(1, np.int64)], 0
            for p in allp:  # panel row pointers start at 0: shift by the entries before
                rp.append(p[2][1:] + off)
                off += int(p[2][-1])
            rp = np.concatenate(rp)
            assert np.array_equal(rp, w_rp)
            assert np.array_equal(ci, w_ci)
            assert np.array_equal(v.view(np.uint32), w_v.view(np.uint32))
    finally:
        import torch.distributed as td
        td.destroy_process_group()


def test_row_panels_cover_rows_within_limit():
    from rvsp_b200 import ranks
    rng = np.random.default_rng(0)
    ops = rng.integers(0, 1000, 5000)
    ops[17] = 50_000  # a row above the limit gets a panel of its own
    panels = ranks.row_panels(ops, limit=20_000)
    assert panels[0][0] == 0 and panels[-1][1] == len(ops)
    assert all(a[1] == b[0] for a, b in zip(panels, panels[1:]))
    for r0, r1 in panels:
        assert r1 - r0 == 1 or ops[r0:r1].sum() <= 20_000
    for world in (1, 2, 3, 8):
        owned = [ranks.shard_panels(panels, ops, r, world) for r in range(world)]
        flat = [p for o in owned for p in o]
        assert sorted(flat) == panels
        for o in owned:  # contiguous groups
            idx = [panels.index(p) for p in o]
            assert idx == list(range(idx[0], idx[0] + len(idx))) if idx else True


@pytest.mark.timeout(300)
def test_two_gloo_ranks_compute_the_product_by_panels():
    mp.spawn(_worker, args=(_free_port(),), nprocs=WORLD, join=True)
