"""Matrix files: MatrixMarket and the reference's binary CSR cache.

read_mtx parses on the host cores (libspmx's spmx_mtx_read) and returns the
COO in file order; the (row, col) sort runs on the GPU in
SpmspvHandle.InputCOO (or load_mtx, which does both).  store_csr / load_csr
read and write the reference's ``.csr`` cache (INC/mtx.hpp:706-808), so files
written here load in the reference's drivers and the other way round.
"""
import ctypes
import os

import numpy as np

from ._lib import lib, check, c_int, c_ll, c_void_p
from .gen import Csr, _take

FIELDS = ("real", "integer", "pattern", "complex")
SYMMETRIES = ("general", "symmetric", "skew-symmetric", "hermitian")


class Coo:
    """A host COO matrix, 0-based, entries in file order."""

    def __init__(self, m, n, row, col, val, field="real", symmetry="general"):
        self.m, self.n = int(m), int(n)
        self.row = np.ascontiguousarray(row, dtype=np.int32)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        self.val = np.ascontiguousarray(val, dtype=np.float32)
        self.field, self.symmetry = field, symmetry

    @property
    def nnz(self):
        return int(self.row.shape[0])


def _path(p):
    return os.fsencode(os.fspath(p))


def read_mtx(path):
    """MatrixMarket coordinate file -> Coo (symmetric files expanded, each
    mirror right after its entry; duplicates kept)."""
    m, n, nnz = c_int(), c_int(), c_ll()
    rp, cp, vp = c_void_p(), c_void_p(), c_void_p()
    info = (c_int * 2)()
    check(lib.spmx_mtx_read(_path(path), ctypes.byref(m), ctypes.byref(n), ctypes.byref(nnz),
                            ctypes.byref(rp), ctypes.byref(cp), ctypes.byref(vp), info),
          "read_mtx")
    k = nnz.value
    return Coo(m.value, n.value, _take(rp, k, np.int32), _take(cp, k, np.int32),
               _take(vp, k, np.float32), FIELDS[info[0]], SYMMETRIES[info[1]])


def write_mtx(path, A, symmetry="general"):
    """Write a Coo or Csr as a MatrixMarket coordinate file ("real", or
    "pattern" without values).  symmetry "symmetric" only labels the file:
    pass one triangle.  Values are written as the shortest text that reads
    back to the same float32."""
    if symmetry not in ("general", "symmetric"):
        raise ValueError("symmetry must be 'general' or 'symmetric'")
    if isinstance(A, Csr):
        row = np.repeat(np.arange(A.m, dtype=np.int32), np.diff(A.rowptr))
        col, val = A.col, A.val
    else:
        row, col, val = A.row, A.col, A.val
    row = np.ascontiguousarray(row, np.int32)
    col = np.ascontiguousarray(col, np.int32)
    val = None if val is None else np.ascontiguousarray(val, np.float32)
    check(lib.spmx_mtx_write(_path(path), A.m, A.n, len(row), row.ctypes.data, col.ctypes.data,
                             None if val is None else val.ctypes.data,
                             int(symmetry == "symmetric")), "write_mtx")


def store_csr(path, A):
    """Write a host Csr in the reference's binary cache layout."""
    val = A.val if A.val is not None else np.ones(A.nnz, np.float32)
    check(lib.spmx_csr_store(_path(path), A.m, A.n, A.nnz, A.rowptr.ctypes.data,
                             A.col.ctypes.data, val.ctypes.data), "store_csr")


def load_csr(path):
    """Read a binary CSR cache file into a host Csr."""
    m, n, nnz = c_int(), c_int(), c_int()
    check(lib.spmx_csr_load_header(_path(path), ctypes.byref(m), ctypes.byref(n),
                                   ctypes.byref(nnz)), "load_csr header")
    rowptr = np.empty(m.value + 1, np.int32)
    col = np.empty(max(nnz.value, 1), np.int32)
    val = np.empty(max(nnz.value, 1), np.float32)
    check(lib.spmx_csr_load(_path(path), m.value, n.value, nnz.value, rowptr.ctypes.data,
                            col.ctypes.data, val.ctypes.data), "load_csr")
    return Csr(m.value, n.value, rowptr, col[:nnz.value], val[:nnz.value])


def load_mtx(path, stream=None):
    """MatrixMarket file -> SpmspvHandle holding the device CSR (host parse,
    one host-to-device copy of the COO, GPU sort)."""
    import torch
    from .handle import SpmspvHandle
    A = read_mtx(path)
    h = SpmspvHandle(A.m, A.n, A.nnz, stream=stream)
    pinned = [torch.from_numpy(a).pin_memory() for a in (A.row, A.col, A.val)]
    row, col, val = (t.to("cuda", non_blocking=True) for t in pinned)
    torch.cuda.current_stream().synchronize()
    h.InputCOO(A.nnz, row, col, val)
    return h
