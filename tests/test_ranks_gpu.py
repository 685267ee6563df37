"""Multi-rank product on the CUDA path: two gloo ranks on 127.0.0.1.

The row-panel sharding of rvsp_b200.ranks with each rank computing its own
contiguous group of panels through the library (device-resident A panels whose
row pointer is offset into the full arrays, rvsp_cuda_spgemm_f32; rank 0 on
the exact path, rank 1 on the learned path). Both ranks use the one visible
GPU: their kernels never wait on each other, only the host collectives (gloo)
do. Rank 0 places the gathered panels at the offsets from ranks.c_offsets and
checks the whole C bit for bit against the oracle.
"""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

WORLD = 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, port):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(WORLD))
    import ctypes as C

    import torch
    import torch.distributed as td

    import oracle
    import rvsp_b200 as rv
    from gpu_util import DevCSR, d2h
    from rvsp_b200 import gen, ranks
    dist = ranks.init("gloo", timeout_s=120)
    try:
        torch.cuda.set_device(0)
        L = rv.lib()
        A = gen.rmat(scale=14, edge_factor=16, seed=6)
        ops = gen.row_products(A, A)
        panels = ranks.row_panels(ops, limit=max(1, int(ops.sum()) // 6))
        mine = ranks.shard_panels(panels, ops, rank, WORLD)
        algo = rv.RVSP_CUDA_ALGO_EXACT if rank == 0 else rv.RVSP_CUDA_ALGO_LEARNED
        dA = DevCSR(A)
        parts = []
        for r0, r1 in mine:
            prp, pci, pv = C.c_void_p(), C.c_void_p(), C.c_void_p()
            nnz = C.c_int32()
            rv.check(L.rvsp_cuda_spgemm_f32(algo, r1 - r0, A.cols, A.cols,
                                            rv.ptr(dA.row_ptr[r0:r1 + 1]), rv.ptr(dA.col_idx),
                                            rv.ptr(dA.values), rv.ptr(dA.row_ptr),
                                            rv.ptr(dA.col_idx), rv.ptr(dA.values), C.byref(prp),
                                            C.byref(pci), C.byref(pv), C.byref(nnz), None), "panel")
            n = nnz.value
            parts.append((r0, r1, d2h(prp.value, r1 - r0 + 1, np.int32),
                          d2h(pci.value, n, np.int32), d2h(pv.value, n, np.float32)))
            for p in (prp, pci, pv):
                L.rvsp_cuda_free(p)
        local = sum(int(p[2][-1]) for p in parts)
        first, total = ranks.c_offsets(dist, local)
        gathered = [None] * WORLD
        td.all_gather_object(gathered, (first, parts))
        ranks.barrier(dist)
        if rank == 0:
            allp = sorted((p for g in gathered for p in g[1]), key=lambda p: p[0])
            assert [(p[0], p[1]) for p in allp] == panels  # every panel exactly once
            w_rp, w_ci, w_v = oracle.spgemm_f32(A, A)
            assert total == w_ci.size
            for first_r, parts_r in gathered:
                if parts_r:
                    assert first_r == int(w_rp[parts_r[0][0]])
            rp, off = [np.zeros(1, np.int64)], 0
            for p in allp:
                rp.append(p[2][1:].astype(np.int64) + off)
                off += int(p[2][-1])
            assert np.array_equal(np.concatenate(rp), w_rp)
            assert np.array_equal(np.concatenate([p[3] for p in allp]), w_ci)
            v = np.concatenate([p[4] for p in allp])
            assert np.array_equal(v.view(np.uint32), w_v.view(np.uint32))
    finally:
        td.destroy_process_group()


@pytest.mark.timeout(600)
def test_two_ranks_compute_the_product_by_panels_on_the_gpu(gpu_lib):
    mp.spawn(_worker, args=(_free_port(),), nprocs=WORLD, join=True)
