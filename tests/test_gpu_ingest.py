"""Device COO -> CSR (spmx_input_coo) against the oracle's stable host sort.

Bit-exact: the row pointer, the columns and the values (as bit patterns) must
equal a stable (row, col) sort of the same COO, duplicates in input order.
Inputs cover every sort path (shuffled, already (row, col) ordered,
column-major), duplicates, empty rows at both ends, nnz 0, a single row or
column, an out-of-range index (rejected, handle unchanged), and the whole
file -> handle path (spmx.io.load_mtx) followed by a SpMV and a CSC SpMSpV
checked against the oracle."""
import numpy as np
import pytest

from conftest import rand_csr
from gpu_util import dev
import oracle.oracle as orc

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _csr_of(m, row, col, val):
    """Stable (row, col) sort on the host (the oracle's order) and its rowptr."""
    order = np.lexsort((col, row))
    rowptr = np.zeros(m + 1, np.int32)
    np.cumsum(np.bincount(row, minlength=m), out=rowptr[1:])
    return rowptr, col[order], None if val is None else val[order]


def _ingest(torch, m, n, row, col, val):
    from spmx import SpmspvHandle
    h = SpmspvHandle(m, n, len(row))
    h.InputCOO(len(row), dev(row, torch), dev(col, torch), None if val is None else dev(val, torch))
    return h


def _check(torch, m, n, row, col, val):
    h = _ingest(torch, m, n, row, col, val)
    rp, cl, vl = h.get_csr()
    erp, ecl, evl = _csr_of(m, row, col, val)
    assert np.array_equal(rp.cpu().numpy(), erp)
    assert np.array_equal(cl.cpu().numpy(), ecl)
    if val is not None:
        assert np.array_equal(vl.cpu().numpy().view(np.uint32), evl.view(np.uint32))
    return h


def _coo(A):
    row = np.repeat(np.arange(A.m, dtype=np.int32), np.diff(A.rowptr))
    return row, A.col.copy(), A.val.copy()


@pytest.mark.parametrize("order", ["shuffled", "row_major", "col_major", "reversed"])
def test_input_coo_orders(torch_cuda, order):
    torch = torch_cuda
    A = rand_csr(3000, 2500, lens=np.minimum(np.random.default_rng(1).zipf(1.5, 3000), 2000), seed=3)
    row, col, val = _coo(A)
    rng = np.random.default_rng(7)
    if order == "shuffled":
        p = rng.permutation(len(row))
    elif order == "row_major":
        p = np.arange(len(row))
    elif order == "col_major":
        p = np.lexsort((row, col))
    else:
        p = np.arange(len(row))[::-1]
    _check(torch, A.m, A.n, row[p], col[p], val[p])


def test_input_coo_duplicates_and_empty_rows(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(11)
    m, n, k = 5000, 300, 40000
    row = rng.integers(100, m - 100, k).astype(np.int32)   # empty rows at both ends
    col = rng.integers(0, 40, k).astype(np.int32)          # many duplicates
    val = rng.standard_normal(k).astype(np.float32)
    _check(torch, m, n, row, col, val)


def test_input_coo_pattern_only(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(12)
    row = rng.integers(0, 2000, 9000).astype(np.int32)
    col = rng.integers(0, 70000, 9000).astype(np.int32)
    _check(torch, 2000, 70000, row, col, None)


@pytest.mark.parametrize("shape", [(1, 4000), (4000, 1), (1, 1)])
def test_input_coo_thin(torch_cuda, shape):
    torch = torch_cuda
    m, n = shape
    rng = np.random.default_rng(13)
    k = 3000
    row = rng.integers(0, m, k).astype(np.int32)
    col = rng.integers(0, n, k).astype(np.int32)
    val = rng.uniform(-1, 1, k).astype(np.float32)
    _check(torch, m, n, row, col, val)


def test_input_coo_empty(torch_cuda):
    torch = torch_cuda
    from spmx import SpmspvHandle
    h = SpmspvHandle(17, 9, 0)
    z = torch.empty(0, dtype=torch.int32, device="cuda")
    h.InputCOO(0, z, z, torch.empty(0, device="cuda"))
    rp, _, _ = h.get_csr()
    assert np.array_equal(rp.cpu().numpy(), np.zeros(18, np.int32))


def test_input_coo_out_of_range(torch_cuda):
    torch = torch_cuda
    from spmx import SpmspvHandle, SpmxError
    A = rand_csr(400, 300, density=0.02, seed=14)
    row, col, val = _coo(A)
    h = _check(torch, A.m, A.n, row, col, val)
    bad = col.copy()
    bad[len(bad) // 2] = A.n  # one column past the end
    with pytest.raises(SpmxError):
        h.InputCOO(len(row), dev(row, torch), dev(bad, torch), dev(val, torch))
    rp, cl, _ = h.get_csr()  # the handle keeps the previous CSR
    assert np.array_equal(rp.cpu().numpy(), A.rowptr) and np.array_equal(cl.cpu().numpy(), A.col)
    neg = row.copy()
    neg[0] = -1
    with pytest.raises(SpmxError):
        h.InputCOO(len(row), dev(neg, torch), dev(col, torch), dev(val, torch))
    h2 = SpmspvHandle(A.m, A.n, A.nnz)
    with pytest.raises(SpmxError):
        h2.InputCOO(A.nnz - 1, dev(row, torch), dev(col, torch), dev(val, torch))


def test_input_coo_large(torch_cuda):
    """The 1M-row Zipf matrix, shuffled: every radix pass of both sorts."""
    torch = torch_cuda
    from spmx import gen
    A = gen.zipf_1m()
    row, col, val = _coo(A)
    p = np.random.default_rng(15).permutation(len(row))
    h = _ingest(torch, A.m, A.n, row[p], col[p], val[p])
    rp, cl, vl = h.get_csr()
    # the generator's CSR has sorted distinct columns per row: it is the answer
    assert np.array_equal(rp.cpu().numpy(), A.rowptr)
    assert np.array_equal(cl.cpu().numpy(), A.col)
    assert np.array_equal(vl.cpu().numpy().view(np.uint32), A.val.view(np.uint32))


def test_load_mtx_then_kernels(torch_cuda, tmp_path):
    """File -> handle (host parse, GPU sort) -> SpMV and CSC SpMSpV."""
    torch = torch_cuda
    from spmx import gen, io
    A = gen.chung_lu(30000, 2.1, 12.0, seed=16)
    # lower triangle as a symmetric MatrixMarket file, rows shuffled
    row, col, val = _coo(A)
    keep = row >= col
    Lr, Lc, Lv = row[keep], col[keep], val[keep]
    p = np.random.default_rng(17).permutation(len(Lr))
    path = str(tmp_path / "cl.mtx")
    io.write_mtx(path, io.Coo(A.m, A.n, Lr[p], Lc[p], Lv[p]), symmetry="symmetric")
    h = io.load_mtx(path)
    rp, cl, vl = h.get_csr()
    m, n, orow, ocol, oval = orc.mtx_read_sorted(path)
    orp = np.zeros(m + 1, np.int32)
    np.cumsum(np.bincount(orow, minlength=m), out=orp[1:])
    assert np.array_equal(rp.cpu().numpy(), orp)
    assert np.array_equal(cl.cpu().numpy(), ocol)
    assert np.array_equal(vl.cpu().numpy().view(np.uint32), oval.view(np.uint32))
    # the loaded matrix drives the kernels
    x = np.random.default_rng(18).uniform(-1, 1, n).astype(np.float32)
    xd = dev(x, torch)
    y = torch.empty(m, device="cuda")
    h.holaPreprocess()
    h.set_x(xd)
    h.spmv(1.0, y)
    y64, mag = orc.spmv_f64(orp, ocol, oval, x)
    assert orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)[0]
    h.ToCSC()
    key = np.sort(np.random.default_rng(19).choice(n, 500, replace=False)).astype(np.int32)
    xv = np.random.default_rng(20).uniform(-1, 1, 500).astype(np.float32)
    h.set_sparse_x(dev(key, torch), dev(xv, torch), 500)
    z = torch.empty(m, device="cuda")
    h.spmspv_csc(0, 0, 1.0, z)
    colptr = np.zeros(n + 1, np.int32)
    np.cumsum(np.bincount(ocol, minlength=n), out=colptr[1:])
    t = np.lexsort((orow, ocol))
    z64, zmag, _ = orc.spmspv_csc_f64(m, colptr, orow[t], oval[t], key, xv)
    assert orc.within_tol(z.cpu().numpy(), z64, zmag, RTOL)[0]
    h.check_device_error()


def test_feature_dump_and_collect_from_files(torch_cuda, tmp_path):
    """The training-data tools on MatrixMarket files: the feature dump matches
    the oracle's matrix features, and collect writes one timed record per
    density with a valid best kernel."""
    import json
    from spmx import gen, io, selector_train
    A = gen.zipf_rows(1 << 14, 1.5, 16, 2000, seed=31)
    p = str(tmp_path / "z.mtx")
    io.write_mtx(p, A)
    out = str(tmp_path / "f.jsonl")
    selector_train.dump_features(out, [p])
    rec = json.loads(open(out).read().splitlines()[0])
    want = orc.mat_features(A.n, A.rowptr)
    got = [rec[k] for k in selector_train.MAT_FEATURES]
    assert rec["matrix"] == "z.mtx" and rec["nnz"] == A.nnz and rec["m"] == A.m
    assert np.allclose(got, want, rtol=1e-9, atol=1e-12)
    data = str(tmp_path / "c.jsonl")
    old = selector_train.DENSITIES
    selector_train.DENSITIES = [1e-3, 1.0]
    try:
        selector_train.collect(data, reps=2, paths=[p])
    finally:
        selector_train.DENSITIES = old
    recs = [json.loads(ln) for ln in open(data)]
    assert [r["density"] for r in recs] == [1e-3, 1.0]
    for r in recs:
        assert len(r["us"]) == 8 and r["best"] == int(np.argmin(r["us"])) and min(r["us"]) > 0
