"""Generators: determinism and the structural properties of each workload."""
import numpy as np
import pytest

from spmx import gen


def _check_csr(A, symmetric=False):
    d = np.diff(A.rowptr)
    assert (d >= 0).all() and A.rowptr[0] == 0 and A.rowptr[-1] == len(A.col)
    for i in range(A.m):
        c = A.col[A.rowptr[i]:A.rowptr[i + 1]]
        assert (np.diff(c) > 0).all(), "columns sorted and distinct"
        assert (c >= 0).all() and (c < A.n).all()
    if symmetric:
        colptr, row, _ = A.to_csc()
        assert np.array_equal(colptr, A.rowptr) and np.array_equal(row, A.col)


def test_rmat_small_properties_and_determinism():
    A = gen.rmat(10, 16, seed=1)
    B = gen.rmat(10, 16, seed=1)
    assert np.array_equal(A.rowptr, B.rowptr) and np.array_equal(A.col, B.col)
    _check_csr(A, symmetric=True)
    for i in range(A.m):
        assert i not in set(A.col[A.rowptr[i]:A.rowptr[i + 1]]), "no self loops"
    C = gen.rmat(10, 16, seed=2)
    assert not np.array_equal(A.col[:100], C.col[:100])


def test_rmat_scale14_size():
    A = gen.rmat(14, 16, seed=1)
    assert A.m == 16384
    assert 300_000 < A.nnz <= 2 * 16 * 16384


def test_zipf_rows_exact_total_and_cap():
    A = gen.zipf_rows(20000, 1.5, 16, 10000, seed=2)
    assert A.nnz == 16 * 20000
    d = np.diff(A.rowptr)
    assert d.max() <= 10000 and d.min() >= 0
    assert (A.val >= -1).all() and (A.val <= 1).all()
    _check_csr(A)


def test_laplacian_structure():
    g = 16
    A = gen.laplacian(g, 0.01, seed=4)
    assert A.nnz == 5 * g * g - 4 * g
    _check_csr(A, symmetric=True)
    diag = [A.val[A.rowptr[i] + list(A.col[A.rowptr[i]:A.rowptr[i + 1]]).index(i)] for i in range(A.m)]
    assert np.all(np.array(diag) == 4.0)
    off = A.val[A.val != 4.0]
    assert abs(off.mean() + 1) < 0.01 and 0.005 < off.std() < 0.02


def test_chung_lu_small():
    A = gen.chung_lu(5000, 2.1, 32.0, seed=5)
    _check_csr(A)
    d = np.diff(A.rowptr)
    assert 15 < d.mean() < 40 and d.max() > 10 * d.mean()


@pytest.mark.parametrize("n,k", [(1000, 0), (1000, 1), (1000, 999), (1000, 1000), (10**6, 105)])
def test_sparse_vector(n, k):
    key, val = gen.sparse_vector(n, k, seed=3)
    assert len(key) == k and len(np.unique(key)) == k
    assert (np.diff(key) > 0).all() if k > 1 else True
    if k:
        assert key.min() >= 0 and key.max() < n and (np.abs(val) <= 1).all()


def test_oracle_generators_equal_product_generators():
    """The oracle's restatement of the benchmark's generators (used by the
    CPU reference arm, which loads nothing from the product) produces the
    same bits as the product's generators."""
    import oracle.oracle as orc
    for m, seed in ((20000, 2), (4096, 9)):
        A = gen.zipf_rows(m, 1.5, 16, min(10000, m), seed=seed)
        B = orc.gen_zipf_rows(m, 1.5, 16, min(10000, m), seed=seed)
        assert np.array_equal(A.rowptr, B.rowptr) and np.array_equal(A.col, B.col)
        assert np.array_equal(A.val.view(np.uint32), B.val.view(np.uint32))
        assert all(np.array_equal(x, y) for x, y in zip(A.to_csc(), B.to_csc()))
    for n, k, dist in ((10**6, 11, "uniform"), (10**6, 105, "normal"), (3000, 1000, "uniform"),
                       (3000, 2999, "normal"), (3000, 3000, "uniform"), (50, 0, "uniform")):
        a, b = gen.sparse_vector(n, k, dist=dist, seed=k + 1), orc.gen_sparse_vector(n, k, dist, k + 1)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))
