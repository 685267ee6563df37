"""Device-memory helpers for the GPU tests (torch supplies the allocations;
every product is computed by librvsp_b200.so through its C ABI)."""

import ctypes as C

import numpy as np

import rvsp_b200 as rv


def torch():
    import torch as T
    return T


def dev(a):
    """numpy -> CUDA tensor (same dtype)."""
    T = torch()
    a = np.ascontiguousarray(a)
    if a.size == 0:
        a = np.zeros(1, a.dtype)
    return T.from_numpy(a.copy()).to("cuda")


class DevCSR:
    def __init__(self, M):
        self.rows, self.cols = M.rows, M.cols
        self.nnz = int(M.row_ptr[-1])
        self.row_ptr = dev(M.row_ptr)
        self.col_idx = dev(M.col_idx)
        self.values = dev(M.values)

    def struct(self):
        return rv.csr_struct(self.rows, self.cols, self.nnz, self.row_ptr, self.col_idx,
                             self.values)


_cuda = None


def _driver():
    """libcuda (driver API) for reading back library-owned device buffers."""
    global _cuda
    if _cuda is None:
        _cuda = C.CDLL("libcuda.so.1")
        _cuda.cuMemcpyDtoH_v2.argtypes = [C.c_void_p, C.c_uint64, C.c_size_t]
        _cuda.cuMemcpyDtoH_v2.restype = C.c_int
    return _cuda


def d2h(p, n, np_dtype):
    out = np.empty(n, np_dtype)
    if n:
        st = _driver().cuMemcpyDtoH_v2(out.ctypes.data, p, out.nbytes)
        assert st == 0, f"cuMemcpyDtoH failed: {st}"
    return out


def _to_np(p, n, ctype, np_dtype, device):
    if n == 0:
        return np.zeros(0, np_dtype)
    if device:
        return d2h(p, n, np_dtype)
    return np.ctypeslib.as_array(C.cast(p, C.POINTER(ctype)), (n,)).copy()


def oneshot(A, B, algo=rv.RVSP_CUDA_ALGO_EXACT, device=True, want_ops=False):
    """rvsp_cuda_spgemm_f32 on device (or host) operands; returns numpy (rp, ci, v[, ops])."""
    L = rv.lib()
    if device:
        dA, dB = DevCSR(A), DevCSR(B)
        args = (dA.row_ptr, dA.col_idx, dA.values, dB.row_ptr, dB.col_idx, dB.values)
    else:
        args = (A.row_ptr, A.col_idx, A.values, B.row_ptr, B.col_idx, B.values)
    prp, pci, pv = C.c_void_p(), C.c_void_p(), C.c_void_p()
    nnz = C.c_int32()
    ops = np.zeros(max(A.rows, 1), np.int64)
    st = L.rvsp_cuda_spgemm_f32(algo, A.rows, A.cols, B.cols, *[rv.ptr(x) for x in args],
                                C.byref(prp), C.byref(pci), C.byref(pv), C.byref(nnz),
                                rv.ptr(ops) if want_ops else None)
    rv.check(st, "rvsp_cuda_spgemm_f32")
    n = nnz.value
    rp = _to_np(prp.value, A.rows + 1, C.c_int32, np.int32, device)
    ci = _to_np(pci.value, n, C.c_int32, np.int32, device)
    v = _to_np(pv.value, n, C.c_float, np.float32, device)
    if device:
        for p in (prp, pci, pv):
            L.rvsp_cuda_free(p)
    else:
        libc = C.CDLL(None)
        libc.free.argtypes = [C.c_void_p]
        for p in (prp, pci, pv):
            libc.free(p)
    if want_ops:
        return rp, ci, v, ops[: A.rows]
    return rp, ci, v


def bits(v):
    return np.ascontiguousarray(v, np.float32).view(np.uint32)
