"""Pin the oracle against the reference's own serial routines, compiled from
its sources by oracle/build_ref.sh into oracle/_ref/libref_host.so and
oracle/_ref/libref_csc.so (built by __graft_entry__.build() wherever the
reference tree is present).

  serialspmv (test/test_application.cu:107-116)       == oracle_serialspmv_f32, bit for bit
  computeMatFeture_serial (spmspv.h:2275-2335)        == oracle_mat_features_faithful, bit for bit
  extractMatFeature (spmspv.h:423-447)                == oracle_std_row_intmean_faithful, bit for bit
  SpmSpvCSCHost (test/test_sort_spmspv.cu:330-375)    == oracle_spmspv_csc_host_faithful, bit for bit
SpmSpvCSCHost reads x into an int; on integer-valued x that changes nothing,
and there the FP64 CSC oracle the GPU tests use agrees with it within FP32
accumulation error.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import rand_csr
import oracle.oracle as orc

SO = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                  "libref_host.so")
SO_CSC = os.path.join(os.path.dirname(SO), "libref_csc.so")


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(SO):
        pytest.skip("oracle/_ref/libref_host.so not built (no reference tree on this machine)")
    lib = ctypes.CDLL(SO)
    P = ctypes.c_void_p
    lib.ref_serialspmv.argtypes = [ctypes.c_int] * 3 + [P] * 5 + [ctypes.c_float]
    lib.ref_serialspmv.restype = None
    lib.ref_mat_features.argtypes = [ctypes.c_int] * 3 + [P, P]
    lib.ref_mat_features.restype = None
    lib.ref_std_row.argtypes = [ctypes.c_int] * 3 + [P]
    lib.ref_std_row.restype = ctypes.c_float
    return lib


def _mats():
    from spmx import gen
    rng = np.random.default_rng(5)
    yield rand_csr(500, 400, density=0.03, seed=1)
    yield rand_csr(3000, 3000, lens=np.minimum(rng.zipf(1.4, 3000), 2500), seed=2)
    yield gen.zipf_rows(1 << 16, 1.5, 16, 10000, seed=2)
    yield gen.laplacian(64, 0.01, seed=4)


@pytest.mark.parametrize("idx", range(4))
@pytest.mark.parametrize("alpha", [1.0, 0.375])
def test_serialspmv_bit_exact(ref, idx, alpha):
    A = list(_mats())[idx]
    x = np.random.default_rng(idx).uniform(-1, 1, A.n).astype(np.float32)
    y_ref = np.zeros(A.m, np.float32)
    rp, cl, vl = (np.ascontiguousarray(a) for a in (A.rowptr, A.col, A.val))
    ref.ref_serialspmv(A.m, A.n, A.nnz, rp.ctypes.data, cl.ctypes.data, vl.ctypes.data,
                       x.ctypes.data, y_ref.ctypes.data, alpha)
    y_orc = orc.serialspmv_f32(A.rowptr, A.col, A.val, x, alpha=alpha)
    assert np.array_equal(y_ref.view(np.uint32), y_orc.view(np.uint32))
    # and the FP64 oracle agrees with it within FP32 accumulation error
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, x, alpha=alpha)
    assert orc.within_tol(y_ref, y64, mag, 1e-4)[0]


@pytest.mark.parametrize("idx", range(4))
def test_matrix_features_bit_exact(ref, idx):
    A = list(_mats())[idx]
    out = np.zeros(7, np.float32)
    rp = np.ascontiguousarray(A.rowptr)
    ref.ref_mat_features(A.m, A.n, A.nnz, rp.ctypes.data, out.ctypes.data)
    mine = orc.mat_features_faithful(A.n, A.rowptr)
    assert np.array_equal(out.view(np.uint32), mine.view(np.uint32)), (out, mine)
    exact = orc.mat_features(A.n, A.rowptr)
    # the exact (FP64) features the engine reports stay close to the float ones
    assert exact[3] == out[0] and exact[4] == out[1]
    assert np.allclose(exact[[5, 6, 7, 8, 9]], out[[2, 3, 4, 5, 6]], rtol=2e-3)


@pytest.mark.parametrize("idx", range(4))
def test_std_row_intmean(ref, idx):
    A = list(_mats())[idx]
    rp = np.ascontiguousarray(A.rowptr)
    r = np.float32(ref.ref_std_row(A.m, A.n, A.nnz, rp.ctypes.data))
    assert r == np.float32(orc.std_row_intmean_faithful(A.rowptr))
    # the exact (FP64) value the engine reports differs only by float drift
    assert float(r) == pytest.approx(orc.std_row_intmean(A.rowptr), rel=1e-3)


@pytest.mark.parametrize("idx", range(3))
def test_coo2hybrid_split_matches_reference(ref, idx):
    """The oracle's COO2Hybrid restatement (row priority) against the
    reference's own COO2Hybrid: the same CSR-part count, the same CSR part in
    (row, column) order and the same CSC part in (column, row) order.  The
    reference sizes its count arrays by nnz, so every case has
    nnz >= max(m, n)."""
    from spmx import gen
    rng = np.random.default_rng(11)
    A = [rand_csr(600, 500, density=0.02, seed=12),
         rand_csr(3000, 2000, lens=np.minimum(rng.zipf(1.4, 3000), 1500) + 1, seed=13),
         gen.laplacian(40, 0.01, seed=4)][idx]
    assert A.nnz >= max(A.m, A.n)
    ref.ref_coo2hybrid.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p] * 4
    ref.ref_coo2hybrid.restype = None
    row = np.repeat(np.arange(A.m, dtype=np.int32), np.diff(A.rowptr))
    col, val = A.col.copy(), A.val.copy()
    k = ctypes.c_int()
    ref.ref_coo2hybrid(A.m, A.n, A.nnz, row.ctypes.data, col.ctypes.data, val.ctypes.data,
                       ctypes.byref(k))
    kk, flags = orc.coo2hybrid(A.n, A.rowptr, A.col)
    assert kk == k.value
    r0 = np.repeat(np.arange(A.m, dtype=np.int32), np.diff(A.rowptr))
    assert np.array_equal(row[:kk], r0[flags]) and np.array_equal(col[:kk], A.col[flags])
    assert np.array_equal(val[:kk].view(np.uint32), A.val[flags].view(np.uint32))
    o = np.lexsort((r0[~flags], A.col[~flags]))
    assert np.array_equal(row[kk:], r0[~flags][o]) and np.array_equal(col[kk:], A.col[~flags][o])
    assert np.array_equal(val[kk:].view(np.uint32), A.val[~flags][o].view(np.uint32))


@pytest.fixture(scope="module")
def ref_csc():
    if not os.path.exists(SO_CSC):
        pytest.skip("oracle/_ref/libref_csc.so not built (no reference tree on this machine)")
    lib = ctypes.CDLL(SO_CSC)
    P = ctypes.c_void_p
    lib.ref_spmspv_csc_host.argtypes = [ctypes.c_int] * 3 + [P] * 3 + [ctypes.c_int] + [P] * 5
    lib.ref_spmspv_csc_host.restype = None
    return lib


def _ref_csc_call(lib, A, csc, key, xv):
    colptr, row, cval = (np.ascontiguousarray(a) for a in csc)
    key, xv = np.ascontiguousarray(key, np.int32), np.ascontiguousarray(xv, np.float32)
    yn = ctypes.c_int()
    yk = np.zeros(max(A.m, 1), np.int32)
    yv = np.zeros(max(A.m, 1), np.float32)
    lib.ref_spmspv_csc_host(A.m, A.n, A.nnz, row.ctypes.data, colptr.ctypes.data, cval.ctypes.data,
                            len(key), key.ctypes.data, xv.ctypes.data, ctypes.byref(yn),
                            yk.ctypes.data, yv.ctypes.data)
    return yk[:yn.value], yv[:yn.value]


@pytest.mark.parametrize("idx", range(4))
@pytest.mark.parametrize("xkind", ["integer", "uniform", "mixed"])
def test_spmspv_csc_host_bit_exact(ref_csc, idx, xkind):
    """The reference's SpmSpvCSCHost against the oracle's faithful form, bit
    for bit: integer-valued x (the int read keeps it), U(-1,1) x (the int read
    makes every product 0 and the output empty) and values in (-4, 4) (the
    read truncates toward zero)."""
    A = list(_mats())[idx]
    csc = A.to_csc()
    rng = np.random.default_rng(100 + idx)
    k = max(1, A.n // 7)
    key = np.sort(rng.choice(A.n, k, replace=False)).astype(np.int32)
    if xkind == "integer":
        xv = rng.integers(-3, 4, k).astype(np.float32)
    elif xkind == "uniform":
        xv = rng.uniform(-1, 1, k).astype(np.float32)
    else:
        xv = rng.uniform(-4, 4, k).astype(np.float32)
    rk, rv = _ref_csc_call(ref_csc, A, csc, key, xv)
    ok, ov = orc.spmspv_csc_host_faithful(A.m, *csc, key, xv)
    assert np.array_equal(rk, ok)
    assert np.array_equal(rv.view(np.uint32), ov.view(np.uint32))
    if xkind == "uniform":
        assert len(rk) == 0
    if xkind == "integer":
        # the FP64 oracle of the GPU tests agrees with the reference's output
        y64, mag, _ = orc.spmspv_csc_f64(A.m, *csc, key, xv)
        dense = np.zeros(A.m, np.float32)
        dense[rk] = rv
        _, good = orc.within_tol(dense, y64, mag, 1e-4)
        # entries the reference drops as IS_FLOAT_ZERO are within FLT_EPSILON of 0
        assert (good | (np.abs(y64) < 2 * np.finfo(np.float32).eps)).all()


def test_spmspv_csc_host_edge_cases(ref_csc):
    """Empty x, a column without nonzeros and an exactly cancelling row."""
    from spmx.gen import Csr
    # column 1 is empty; row 0 gets 0.5*2 + (-1)*1 = 0 exactly
    A = Csr(3, 3, np.array([0, 2, 3, 4], np.int32), np.array([0, 2, 0, 2], np.int32),
            np.array([0.5, -1.0, 0.25, 3.0], np.float32))
    csc = A.to_csc()
    for key, xv in ((np.zeros(0, np.int32), np.zeros(0, np.float32)),
                    (np.array([1], np.int32), np.array([2.0], np.float32)),
                    (np.array([0, 1, 2], np.int32), np.array([2.0, 5.0, 1.0], np.float32))):
        rk, rv = _ref_csc_call(ref_csc, A, csc, key, xv)
        ok, ov = orc.spmspv_csc_host_faithful(A.m, *csc, key, xv)
        assert np.array_equal(rk, ok) and np.array_equal(rv.view(np.uint32), ov.view(np.uint32))
    assert list(rk) == [1, 2]  # row 0 cancelled to exactly 0 and is dropped
