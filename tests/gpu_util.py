"""Helpers for the GPU parity tests: move host matrices to the device and
build handles through the public binding."""
import numpy as np


def dev(a, torch):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def make_handle(A, torch, csc=True, hola=True):
    from spmx import SpmspvHandle
    h = SpmspvHandle(A.m, A.n, A.nnz)
    rp, cl = dev(A.rowptr, torch), dev(A.col, torch)
    vl = dev(A.val, torch) if A.val is not None else None
    h.InputCSR(A.nnz, rp, cl, vl)
    if csc:
        h.ToCSC()
    if hola and A.val is not None:
        h.holaPreprocess()
    return h


def set_sparse(h, key, val, torch):
    k = dev(key.astype(np.int32), torch)
    v = dev(val.astype(np.float32), torch)
    h.set_sparse_x(k, v, len(key))
    return k, v
