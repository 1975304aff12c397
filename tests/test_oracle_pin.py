"""Pin the oracle against the reference's own serial routines, compiled from
its sources by oracle/build_ref.sh into oracle/_ref/libref_host.so (built by
__graft_entry__.build() wherever the reference tree is present).

  serialspmv (test/test_application.cu:107-116)       == oracle_serialspmv_f32, bit for bit
  computeMatFeture_serial (spmspv.h:2275-2335)        == oracle_mat_features_faithful, bit for bit
  extractMatFeature (spmspv.h:423-447)                == oracle_std_row_intmean_faithful, bit for bit
SpmSpvCSCHost (test/test_sort_spmspv.cu:330-375) lives in a driver that no
longer compiles against the reference's own handle API, so it is not pinned
here; the oracle checks its CSC restatement against serialspmv instead
(tests/test_oracle.py).
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import rand_csr
import oracle.oracle as orc

SO = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                  "libref_host.so")


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
