"""Synthetic inputs (host arrays, numpy) from the deterministic C generators.

The generators run on the host cores (OpenMP) with a counter-based RNG, so
their output depends only on the arguments.  The configurations of the
benchmark suite are named here with their sizes.
"""
import ctypes

import numpy as np

from ._lib import lib, check, c_int, c_ll, c_void_p


def _take(ptr, count, dtype):
    """Copy a malloc'ed C array into numpy and release it."""
    if count == 0:
        out = np.zeros(0, dtype=dtype)
    else:
        ct = {np.int32: ctypes.c_int32, np.float32: ctypes.c_float}[dtype]
        buf = (ct * count).from_address(ptr.value)
        out = np.frombuffer(buf, dtype=dtype).copy()
    if ptr.value:
        lib.spmx_host_free(ptr)
    return out


class Csr:
    """A host CSR matrix (int32 row pointer / columns, float32 values)."""

    def __init__(self, m, n, rowptr, col, val):
        self.m, self.n = int(m), int(n)
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        self.val = None if val is None else np.ascontiguousarray(val, dtype=np.float32)

    @property
    def nnz(self):
        return int(self.rowptr[-1])

    def to_csc(self):
        """Stable host transpose: (colptr, row, val) with rows sorted per column."""
        colptr = np.zeros(self.n + 1, dtype=np.int32)
        row = np.zeros(max(self.nnz, 1), dtype=np.int32)
        cval = np.zeros(max(self.nnz, 1), dtype=np.float32) if self.val is not None else None
        check(lib.spmx_host_csr2csc(
            self.m, self.n, self.rowptr.ctypes.data, self.col.ctypes.data,
            None if self.val is None else self.val.ctypes.data,
            colptr.ctypes.data, row.ctypes.data,
            None if cval is None else cval.ctypes.data), "host csr2csc")
        row = row[:self.nnz]
        if cval is not None:
            cval = cval[:self.nnz]
        return colptr, row, cval


def rmat(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=1):
    """Symmetric R-MAT graph (pattern only): self-loops and duplicates removed."""
    m = c_int()
    nnz = c_ll()
    rp, cp = c_void_p(), c_void_p()
    check(lib.spmx_gen_rmat(scale, edge_factor, a, b, c, seed, ctypes.byref(m),
                            ctypes.byref(nnz), ctypes.byref(rp), ctypes.byref(cp)), "rmat")
    rowptr = _take(rp, m.value + 1, np.int32)
    col = _take(cp, nnz.value, np.int32)
    return Csr(m.value, m.value, rowptr, col, None)


def zipf_rows(m, s=1.5, mean=16, maxlen=10000, seed=2):
    """m x m matrix with Zipf(s) row lengths (mean `mean`, cap `maxlen`),
    uniform distinct columns, values U(-1, 1)."""
    nnz = c_ll()
    rp, cp, vp = c_void_p(), c_void_p(), c_void_p()
    check(lib.spmx_gen_zipf_rows(m, s, mean, maxlen, seed, ctypes.byref(nnz),
                                 ctypes.byref(rp), ctypes.byref(cp), ctypes.byref(vp)), "zipf")
    return Csr(m, m, _take(rp, m + 1, np.int32), _take(cp, nnz.value, np.int32),
               _take(vp, nnz.value, np.float32))


def chung_lu(n, gamma=2.1, avg=32.0, seed=5):
    """Chung-Lu power-law graph with N(0,1) values (symmetric pattern)."""
    nnz = c_ll()
    rp, cp, vp = c_void_p(), c_void_p(), c_void_p()
    check(lib.spmx_gen_chung_lu(n, gamma, avg, seed, ctypes.byref(nnz), ctypes.byref(rp),
                                ctypes.byref(cp), ctypes.byref(vp)), "chung-lu")
    return Csr(n, n, _take(rp, n + 1, np.int32), _take(cp, nnz.value, np.int32),
               _take(vp, nnz.value, np.float32))


def laplacian(g, sigma=0.01, seed=4):
    """5-point Laplacian on a g x g grid, off-diagonals -1 + N(0, sigma^2)."""
    nnz = c_ll()
    rp, cp, vp = c_void_p(), c_void_p(), c_void_p()
    check(lib.spmx_gen_laplacian(g, sigma, seed, ctypes.byref(nnz), ctypes.byref(rp),
                                 ctypes.byref(cp), ctypes.byref(vp)), "laplacian")
    n = g * g
    return Csr(n, n, _take(rp, n + 1, np.int32), _take(cp, nnz.value, np.int32),
               _take(vp, nnz.value, np.float32))


def sparse_vector(n, k, dist="uniform", seed=7):
    """k distinct sorted positions in [0, n) with U(-1,1) or N(0,1) values."""
    key = np.zeros(max(k, 1), dtype=np.int32)
    val = np.zeros(max(k, 1), dtype=np.float32)
    check(lib.spmx_gen_sparse_vector(n, k, 0 if dist == "uniform" else 1, seed,
                                     key.ctypes.data, val.ctypes.data), "sparse vector")
    return key[:k], val[:k]


def density_nnz(n, d):
    """x_nnz = ceil(d * n) for the density sweep."""
    import math
    return min(n, int(math.ceil(d * n)))


# the benchmark configurations, by what they are
C2_DENSITIES = (1e-5, 1e-4, 1e-3, 1e-2, 1e-1, 1.0)


def zipf_1m(seed=2):
    """1,048,576 x 1,048,576, Zipf(1.5) rows, mean 16, max 10,000."""
    return zipf_rows(1 << 20, 1.5, 16, 10000, seed)
