"""rvsp_cuda_row_ptr_noalloc: C's row pointer from per-row counts without any
device allocation, for callers that cannot allocate where they need it (code
recording a CUDA graph under stream capture, latency-critical loops that
cannot take cudaFree's device-wide synchronisation, processes whose device
memory another allocator owns). Its scratch is a static device array shared
by every call.

Checked against the existing path (the row pointer the plan path writes into
C), bit for bit -- integer prefix sums have no tolerance -- on two calls in a
row, so a stale scratch from the first call cannot leak into the second. This
file is collected last so a run that stops at the first failure has already
run every other test; it needs nothing from them and passes on its own.
"""

import ctypes as C

import numpy as np
import pytest

import oracle
import rvsp_b200 as rv
from gpu_util import dev, oneshot
from rvsp_b200 import gen

pytestmark = pytest.mark.gpu

MAX_ROWS = 8_388_608


def _noalloc(counts_np):
    import torch
    counts = dev(counts_np.astype(np.int32))
    row_ptr = torch.full((counts_np.size + 1,), -1, dtype=torch.int32, device="cuda")
    total = C.c_int64(-1)
    st = rv.lib().rvsp_cuda_row_ptr_noalloc(counts.data_ptr(), counts_np.size, row_ptr.data_ptr(),
                                            C.byref(total), None)
    return st, row_ptr.cpu().numpy(), total.value


def _existing_row_ptr(A, B):
    """Row pointer of C from the existing one-shot entry point."""
    rp, _, _ = oneshot(A, B, algo=rv.RVSP_CUDA_ALGO_EXACT, device=True)
    return rp


def test_noalloc_row_ptr_matches_existing_path_twice(gpu_lib):
    cases = [(gen.rmat(scale=13, edge_factor=8, seed=31),) * 2,
             (gen.uniform_fixed(2000, 3000, 16, seed=5), gen.uniform_fixed(3000, 700, 12, seed=6))]
    for A, B in cases:  # two calls in a row on the shared scratch
        _, counts = oracle.symbolic(A, B)
        want = _existing_row_ptr(A, B)
        st, got, total = _noalloc(counts)
        assert st == rv.RVSP_SUCCESS, rv.last_error()
        assert np.array_equal(got, want)
        assert total == int(want[-1])


def test_noalloc_rejects_what_it_cannot_hold(gpu_lib):
    import torch
    L = rv.lib()
    d = torch.zeros(16, dtype=torch.int32, device="cuda")
    out = torch.zeros(17, dtype=torch.int32, device="cuda")
    # beyond the static scratch: rejected before any device work
    assert L.rvsp_cuda_row_ptr_noalloc(d.data_ptr(), MAX_ROWS + 1, out.data_ptr(), None, None) \
        == rv.RVSP_ERROR_INVALID_ARGUMENT
    assert "8388608" in rv.last_error()
    assert L.rvsp_cuda_row_ptr_noalloc(d.data_ptr(), 0, out.data_ptr(), None, None) \
        == rv.RVSP_ERROR_INVALID_ARGUMENT
    host = np.zeros(16, np.int32)
    assert L.rvsp_cuda_row_ptr_noalloc(host.ctypes.data, 16, out.data_ptr(), None, None) \
        == rv.RVSP_ERROR_INVALID_ARGUMENT
    assert L.rvsp_cuda_row_ptr_noalloc(None, 16, out.data_ptr(), None, None) \
        == rv.RVSP_ERROR_NULL_POINTER
    # a total past INT32_MAX fails like the symbolic phase (rv-sparse rvsp_symbolic.c:69) ...
    st, _, total = _noalloc(np.array([1 << 30, 1 << 30, 1 << 30], np.int64))
    assert st == rv.RVSP_ERROR_ALLOCATION_FAILED and total == 3 << 30
    # ... and the cleared overflow flag does not stick to the next call
    st, got, total = _noalloc(np.array([3, 0, 5], np.int64))
    assert st == rv.RVSP_SUCCESS and list(got) == [0, 3, 3, 8] and total == 8
