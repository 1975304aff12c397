"""Python face of the CPU oracle (spmx_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product.  See spmx_oracle.c for the
reference routine each function restates.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")


def build():
    """Compile liboracle.so with gcc (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


if not os.path.exists(_SO):
    build()
_lib = ctypes.CDLL(_SO)

_P = ctypes.c_void_p
_i, _d, _f = ctypes.c_int, ctypes.c_double, ctypes.c_float
_sigs = {
    "oracle_serialspmv_f32": (None, [_i, _P, _P, _P, _P, _P, _f]),
    "oracle_spmv_f64": (None, [_i, _P, _P, _P, _P, _P, _d, _P, _P]),
    "oracle_spmspv_csc_f64": (None, [_i, _P, _P, _P, _i, _P, _P, _d, _P, _P, _P]),
    "oracle_sparse_output_flt_eps": (_i, [_i, _P, _P, _P]),
    "oracle_sparse2dense_bits": (None, [_i, _i, _P, _P, _P, _P]),
    "oracle_dense2sparse": (_i, [_i, _P, _P, _P]),
    "oracle_dense2bitarray": (None, [_i, _P, _P]),
    "oracle_mat_features": (None, [_i, _i, _i, _P, _P]),
    "oracle_mat_features_faithful": (None, [_i, _i, _i, _P, _P]),
    "oracle_std_row_intmean": (_d, [_i, _i, _P]),
    "oracle_std_row_intmean_faithful": (_f, [_i, _i, _P]),
    "oracle_vec_features": (None, [_P, _i, _P, _P]),
    "oracle_gm": (None, [_i, _i, _i, ctypes.c_longlong, _P]),
    "oracle_csr5_sigma": (_i, [_i, _i]),
    "oracle_bfs_spmspv": (_i, [_i, _P, _P, _i, _P]),
    "oracle_bfs_queue": (_i, [_i, _P, _P, _i, _P]),
    "oracle_spmv_t_f64": (None, [_i, _i, _P, _P, _P, _P, _P, _P]),
    "oracle_dvals_f64": (None, [_i, _P, _P, _P, _P, _P]),
    "cpu_spmv_serial": (None, [_i, _P, _P, _P, _P, _P, _f]),
    "cpu_spmv_omp": (None, [_i, _P, _P, _P, _P, _P, _f]),
    "cpu_spmspv_csc_serial": (None, [_i, _P, _P, _P, _i, _P, _P, _P]),
    "cpu_spmspv_csc_omp": (None, [_i, _P, _P, _P, _i, _P, _P, _P]),
    "cpu_threads": (_i, []),
    "oracle_free": (None, [_P]),
    "oracle_coo2hybrid": (_i, [_i, _i, _P, _P, _P]),
    "oracle_mtx_read": (_i, [ctypes.c_char_p, _P, _P, _P, _P, _P, _P]),
    "oracle_spmspv_csc_host_faithful": (_i, [_i, _P, _P, _P, _i, _P, _P, _P, _P]),
    "oracle_csr2csc": (_i, [_i, _i, _P, _P, _P, _P, _P, _P]),
    "oracle_gen_zipf_rows": (_i, [_i, _d, _i, _i, ctypes.c_uint64, _P, _P, _P]),
    "oracle_gen_sparse_vector": (_i, [_i, _i, _i, ctypes.c_uint64, _P, _P]),
}
for _n, (_r, _a) in _sigs.items():
    _fn = getattr(_lib, _n)
    _fn.restype = _r
    _fn.argtypes = _a

raw = _lib


def _a(x, dt):
    return np.ascontiguousarray(x, dtype=dt)


def _p(x):
    return None if x is None else x.ctypes.data


def spmv_f64(rowptr, col, val, x, alpha=1.0, bits=None):
    """y = alpha*A*x in FP64 plus sum |a_ij x_j| per row (serialspmv)."""
    rowptr, col, val, x = _a(rowptr, np.int32), _a(col, np.int32), _a(val, np.float32), _a(x, np.float32)
    m = len(rowptr) - 1
    y = np.zeros(m, np.float64)
    ay = np.zeros(m, np.float64)
    b = None if bits is None else _a(bits, np.int32)
    _lib.oracle_spmv_f64(m, _p(rowptr), _p(col), _p(val), _p(x), _p(b), alpha, _p(y), _p(ay))
    return y, ay


def serialspmv_f32(rowptr, col, val, x, alpha=1.0):
    rowptr, col, val, x = _a(rowptr, np.int32), _a(col, np.int32), _a(val, np.float32), _a(x, np.float32)
    m = len(rowptr) - 1
    y = np.zeros(m, np.float32)
    _lib.oracle_serialspmv_f32(m, _p(rowptr), _p(col), _p(val), _p(x), _p(y), alpha)
    return y


def spmspv_csc_f64(m, colptr, row, val, x_key, x_val, alpha=1.0):
    """(y, |y| magnitude, touched rows) of y = alpha*A*x for sparse x (SpmSpvCSCHost)."""
    colptr, row, val = _a(colptr, np.int32), _a(row, np.int32), _a(val, np.float32)
    x_key, x_val = _a(x_key, np.int32), _a(x_val, np.float32)
    y = np.zeros(m, np.float64)
    ay = np.zeros(m, np.float64)
    t = np.zeros(m, np.uint8)
    _lib.oracle_spmspv_csc_f64(m, _p(colptr), _p(row), _p(val), len(x_key), _p(x_key), _p(x_val),
                               alpha, _p(y), _p(ay), _p(t))
    return y, ay, t.astype(bool)


def sparse2dense_bits(n, key, val):
    key = _a(key, np.int32)
    val = None if val is None else _a(val, np.float32)
    dense = np.zeros(n, np.float32)
    bits = np.zeros((n + 31) // 32, np.uint32)
    _lib.oracle_sparse2dense_bits(n, len(key), _p(key), _p(val), _p(dense), _p(bits))
    return dense, bits


def dense2sparse(dense):
    dense = _a(dense, np.float32)
    key = np.zeros(max(len(dense), 1), np.int32)
    val = np.zeros(max(len(dense), 1), np.float32)
    k = _lib.oracle_dense2sparse(len(dense), _p(dense), _p(key), _p(val))
    return key[:k], val[:k]


def dense2bitarray(dense):
    dense = _a(dense, np.float32)
    bits = np.zeros((len(dense) + 31) // 32, np.uint32)
    _lib.oracle_dense2bitarray(len(dense), _p(dense), _p(bits))
    return bits


def mat_features(n, rowptr):
    rowptr = _a(rowptr, np.int32)
    m = len(rowptr) - 1
    out = np.zeros(10, np.float64)
    _lib.oracle_mat_features(m, n, int(rowptr[-1]), _p(rowptr), _p(out))
    return out


def mat_features_faithful(n, rowptr):
    rowptr = _a(rowptr, np.int32)
    m = len(rowptr) - 1
    out = np.zeros(7, np.float32)
    _lib.oracle_mat_features_faithful(m, n, int(rowptr[-1]), _p(rowptr), _p(out))
    return out


def std_row_intmean(rowptr):
    rowptr = _a(rowptr, np.int32)
    return _lib.oracle_std_row_intmean(len(rowptr) - 1, int(rowptr[-1]), _p(rowptr))


def std_row_intmean_faithful(rowptr):
    rowptr = _a(rowptr, np.int32)
    return _lib.oracle_std_row_intmean_faithful(len(rowptr) - 1, int(rowptr[-1]), _p(rowptr))


def vec_features(colptr, x_key):
    colptr, x_key = _a(colptr, np.int32), _a(x_key, np.int32)
    out = np.zeros(3, np.int64)
    _lib.oracle_vec_features(_p(colptr), len(x_key), _p(x_key), _p(out))
    return out


def gm(m, nnz, x_nnz, bin_len):
    out = np.zeros(3, np.float64)
    _lib.oracle_gm(m, nnz, x_nnz, bin_len, _p(out))
    return out


def csr5_sigma(m, nnz):
    return _lib.oracle_csr5_sigma(m, nnz)


def bfs_spmspv(n, colptr, row, src):
    colptr, row = _a(colptr, np.int32), _a(row, np.int32)
    lv = np.zeros(n, np.int32)
    d = _lib.oracle_bfs_spmspv(n, _p(colptr), _p(row), src, _p(lv))
    return lv, d


def bfs_queue(n, rowptr, col, src):
    rowptr, col = _a(rowptr, np.int32), _a(col, np.int32)
    lv = np.zeros(n, np.int32)
    d = _lib.oracle_bfs_queue(n, _p(rowptr), _p(col), src, _p(lv))
    return lv, d


def spmv_t_f64(n, rowptr, col, val, dy):
    rowptr, col, val, dy = _a(rowptr, np.int32), _a(col, np.int32), _a(val, np.float32), _a(dy, np.float32)
    dx = np.zeros(n, np.float64)
    adx = np.zeros(n, np.float64)
    _lib.oracle_spmv_t_f64(len(rowptr) - 1, n, _p(rowptr), _p(col), _p(val), _p(dy), _p(dx), _p(adx))
    return dx, adx


def dvals_f64(rowptr, col, dy, x):
    rowptr, col, dy, x = _a(rowptr, np.int32), _a(col, np.int32), _a(dy, np.float32), _a(x, np.float32)
    out = np.zeros(int(rowptr[-1]), np.float64)
    _lib.oracle_dvals_f64(len(rowptr) - 1, _p(rowptr), _p(col), _p(dy), _p(x), _p(out))
    return out


def within_tol(y32, y64, mag, rtol=1e-5):
    """Per-element |y32 - y64| <= rtol * max(|y64|, sum |a_ij x_j|)."""
    y32 = np.asarray(y32, np.float64)
    bound = rtol * np.maximum(np.abs(y64), mag)
    ok = np.abs(y32 - y64) <= bound
    return bool(ok.all()), ok


def max_scaled_err(y32, y64, mag):
    y32 = np.asarray(y32, np.float64)
    den = np.maximum(np.maximum(np.abs(y64), mag), 1e-300)
    return float(np.max(np.abs(y32 - y64) / den)) if len(y64) else 0.0


def mtx_read_sorted(path):
    """ReadMTX restated: (m, n, row, col, val) sorted by (row, col), stable."""
    m, n, nnz = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    rp, cp, vp = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    rc = _lib.oracle_mtx_read(os.fsencode(path), ctypes.byref(m), ctypes.byref(n),
                              ctypes.byref(nnz), ctypes.byref(rp), ctypes.byref(cp),
                              ctypes.byref(vp))
    if rc != 0:
        raise ValueError(f"oracle_mtx_read({path}) = {rc}")
    k = nnz.value
    out = []
    for ptr, ct, dt in ((rp, ctypes.c_int32, np.int32), (cp, ctypes.c_int32, np.int32),
                        (vp, ctypes.c_float, np.float32)):
        a = np.frombuffer((ct * k).from_address(ptr.value), dtype=dt).copy() if k else \
            np.zeros(0, dt)
        _lib.oracle_free(ptr)
        out.append(a)
    return (m.value, n.value, *out)


def coo2hybrid(n, rowptr, col):
    """COO2Hybrid (row priority) restated: (csr_nnz, to_csr flags in CSR order)."""
    rowptr, col = _a(rowptr, np.int32), _a(col, np.int32)
    flags = np.zeros(max(len(col), 1), np.uint8)
    k = _lib.oracle_coo2hybrid(len(rowptr) - 1, n, _p(rowptr), _p(col), _p(flags))
    return k, flags[:len(col)].astype(bool)


def spmspv_csc_host_faithful(m, colptr, row, val, x_key, x_val):
    """SpmSpvCSCHost as written (x truncated to int, FP32, IS_FLOAT_ZERO
    output filter): (y_key, y_val)."""
    colptr, row, val = _a(colptr, np.int32), _a(row, np.int32), _a(val, np.float32)
    x_key, x_val = _a(x_key, np.int32), _a(x_val, np.float32)
    key = np.zeros(max(m, 1), np.int32)
    v = np.zeros(max(m, 1), np.float32)
    k = _lib.oracle_spmspv_csc_host_faithful(m, _p(colptr), _p(row), _p(val), len(x_key), _p(x_key),
                                             _p(x_val), _p(key), _p(v))
    return key[:k], v[:k]


def csr2csc(m, n, rowptr, col, val=None):
    """Stable CSR -> CSC transpose: (colptr, row, cval)."""
    rowptr, col = _a(rowptr, np.int32), _a(col, np.int32)
    val = None if val is None else _a(val, np.float32)
    nnz = int(rowptr[-1])
    colptr = np.zeros(n + 1, np.int32)
    row = np.zeros(max(nnz, 1), np.int32)
    cval = None if val is None else np.zeros(max(nnz, 1), np.float32)
    if _lib.oracle_csr2csc(m, n, _p(rowptr), _p(col), _p(val), _p(colptr), _p(row), _p(cval)):
        raise ValueError("column index out of range")
    return colptr, row[:nnz], None if cval is None else cval[:nnz]


class HostCsr:
    """A host CSR (int32 row pointer / columns, float32 values)."""

    def __init__(self, m, n, rowptr, col, val):
        self.m, self.n = int(m), int(n)
        self.rowptr, self.col, self.val = rowptr, col, val

    @property
    def nnz(self):
        return int(self.rowptr[-1])

    def to_csc(self):
        return csr2csc(self.m, self.n, self.rowptr, self.col, self.val)


def gen_zipf_rows(m, s=1.5, mean=16, maxlen=10000, seed=2):
    """The benchmark's Zipf-row matrix (restated generator, see spmx_oracle.c)."""
    rowptr = np.zeros(m + 1, np.int32)
    col = np.zeros(max(mean * m, 1), np.int32)
    val = np.zeros(max(mean * m, 1), np.float32)
    if _lib.oracle_gen_zipf_rows(m, s, mean, maxlen, seed, _p(rowptr), _p(col), _p(val)):
        raise ValueError("zipf arguments out of range")
    return HostCsr(m, m, rowptr, col[:mean * m], val[:mean * m])


def gen_zipf_1m(seed=2):
    """1,048,576 x 1,048,576, Zipf(1.5) rows, mean 16, max 10,000."""
    return gen_zipf_rows(1 << 20, 1.5, 16, 10000, seed)


def gen_sparse_vector(n, k, dist="uniform", seed=7):
    """k distinct sorted positions in [0, n), U(-1,1) or N(0,1) values."""
    key = np.zeros(max(k, 1), np.int32)
    val = np.zeros(max(k, 1), np.float32)
    if _lib.oracle_gen_sparse_vector(n, k, 0 if dist == "uniform" else 1, seed, _p(key), _p(val)):
        raise ValueError("k out of range")
    return key[:k], val[:k]


def density_nnz(n, d):
    """x_nnz = ceil(d * n) for the density sweep."""
    import math
    return min(n, int(math.ceil(d * n)))
