"""CSC SpMSpV (every work distribution x write-back), the device transpose,
vector conversions and features on the GPU against the oracle."""
import numpy as np
import pytest

from conftest import rand_csr
from gpu_util import dev, make_handle, set_sparse
import oracle.oracle as orc

pytestmark = pytest.mark.gpu
RTOL = 1e-5

VARIANTS = [("naive", 0), ("merge", 1), ("twolayer", 2)]


def _matrix(kind):
    rng = np.random.default_rng(42)
    if kind == "uniform":
        return rand_csr(4000, 3000, density=0.005, seed=7)
    if kind == "skewed":
        # power-law-ish columns: column 17 appears in a third of the rows and
        # column 4000 in a tenth (long CSC columns), plus many empty columns
        from spmx.gen import Csr
        m, n = 6000, 5000
        rows = []
        for i in range(m):
            c = set(rng.choice(n, int(rng.integers(0, 6)), replace=False).tolist())
            if i % 3 == 0:
                c.add(17)
            if i % 10 == 0:
                c.add(4000)
            c = {j for j in c if j % 97 != 5}
            rows.append(sorted(c))
        rowptr = np.zeros(m + 1, np.int32)
        rowptr[1:] = np.cumsum([len(r) for r in rows])
        col = np.array([j for r in rows for j in r], np.int32)
        return Csr(m, n, rowptr, col, rng.uniform(-1, 1, len(col)).astype(np.float32))
    if kind == "long-col":
        lens = np.zeros(300, np.int64)
        lens[:] = 40
        A = rand_csr(300, 20000, lens=lens, seed=9)
        return A
    raise ValueError(kind)


def _x(n, k, seed):
    rng = np.random.default_rng(seed)
    key = np.sort(rng.choice(n, k, replace=False)).astype(np.int32)
    return key, rng.uniform(-1, 1, k).astype(np.float32)


@pytest.mark.parametrize("mat", ["uniform", "skewed", "long-col"])
@pytest.mark.parametrize("vname,variant", VARIANTS)
@pytest.mark.parametrize("frac", [0.0005, 0.02, 0.5, 1.0])
def test_csc_atomic(torch_cuda, mat, vname, variant, frac):
    torch = torch_cuda
    A = _matrix(mat)
    h = make_handle(A, torch, hola=False)
    k = max(1, int(frac * A.n))
    key, val = _x(A.n, k, 3)
    set_sparse(h, key, val, torch)
    y = torch.full((A.m,), 3.0, device="cuda")
    yk = torch.empty(A.m, dtype=torch.int32, device="cuda")
    yv = torch.empty(A.m, device="cuda")
    ynnz = h.spmspv_csc(variant, 0, 1.5, y, yk, yv)
    h.check_device_error()
    colptr, row, cval = A.to_csc()
    y64, mag, touched = orc.spmspv_csc_f64(A.m, colptr, row, cval, key, val, alpha=1.5)
    yh = y.cpu().numpy()
    ok, _ = orc.within_tol(yh, y64, mag, RTOL)
    assert ok, orc.max_scaled_err(yh, y64, mag)
    # keyval = the nonzeros of the dense result, in row order
    ek, ev = orc.dense2sparse(yh)
    assert ynnz == len(ek)
    assert np.array_equal(yk[:ynnz].cpu().numpy(), ek)
    assert np.array_equal(yv[:ynnz].cpu().numpy(), ev)


@pytest.mark.parametrize("k", [50_000, 200_000])
def test_csc_naive_several_entries_per_lane_group(torch_cuda, k):
    """An x large enough that the naive scatter gives each lane group two
    (k = 50,000) or four (k = 200,000) entries, on the 1M-row Zipf matrix."""
    torch = torch_cuda
    from spmx import gen
    A = gen.zipf_1m()
    h = make_handle(A, torch, hola=False)
    key, val = _x(A.n, k, 5)
    set_sparse(h, key, val, torch)
    y = torch.full((A.m,), 3.0, device="cuda")
    h.spmspv_csc(0, 0, 1.5, y, sync=False)
    h.check_device_error()
    colptr, row, cval = A.to_csc()
    y64, mag, _ = orc.spmspv_csc_f64(A.m, colptr, row, cval, key, val, alpha=1.5)
    yh = y.cpu().numpy()
    ok, _ = orc.within_tol(yh, y64, mag, RTOL)
    assert ok, orc.max_scaled_err(yh, y64, mag)


@pytest.mark.parametrize("lanes", [1, 4, 32])
def test_csc_naive_lanes_setter(torch_cuda, lanes):
    """The naive CSC scatter with its lanes per column set through
    spmx_set_naive_lanes, on the skewed matrix (columns far longer than the
    lane groups) and x of 1 and 33 entries, against the FP64 oracle."""
    torch = torch_cuda
    A = _matrix("skewed")
    h = make_handle(A, torch, hola=False)
    h.set_naive_lanes(0, lanes)
    colptr, row, cval = A.to_csc()
    for key in (np.array([17], np.int32), np.unique(np.r_[_x(A.n, 31, 11)[0], 17, 4000]).astype(np.int32)):
        val = np.random.default_rng(3).uniform(-1, 1, len(key)).astype(np.float32)
        set_sparse(h, key, val, torch)
        y = torch.full((A.m,), 3.0, device="cuda")
        h.spmspv_csc(0, 0, 1.5, y)
        h.check_device_error()
        y64, mag, _ = orc.spmspv_csc_f64(A.m, colptr, row, cval, key, val, alpha=1.5)
        ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
        assert ok


def test_naive_lanes_setter_rejects_bad_values(torch_cuda):
    torch = torch_cuda
    from spmx import SpmxError
    h = make_handle(_matrix("uniform"), torch, hola=False)
    for rl, cl in [(3, 0), (0, 48), (64, 0), (0, 64), (-1, 0)]:
        with pytest.raises(SpmxError):
            h.set_naive_lanes(rl, cl)
    h.set_naive_lanes(8, 32)


@pytest.mark.parametrize("mat", ["uniform", "skewed"])
@pytest.mark.parametrize("vname,variant", VARIANTS)
@pytest.mark.parametrize("frac", [0.001, 0.1, 1.0])
def test_csc_sort(torch_cuda, mat, vname, variant, frac):
    torch = torch_cuda
    A = _matrix(mat)
    h = make_handle(A, torch, hola=False)
    k = max(1, int(frac * A.n))
    key, val = _x(A.n, k, 4)
    set_sparse(h, key, val, torch)
    yk = torch.empty(A.m, dtype=torch.int32, device="cuda")
    yv = torch.empty(A.m, device="cuda")
    y = torch.empty(A.m, device="cuda")
    ynnz = h.spmspv_csc(variant, 1, -2.0, y, yk, yv)
    h.check_device_error()
    colptr, row, cval = A.to_csc()
    y64, mag, touched = orc.spmspv_csc_f64(A.m, colptr, row, cval, key, val, alpha=-2.0)
    rows = np.nonzero(touched)[0]
    # reduce_by_key semantics: every touched row, sorted, zeros kept
    assert ynnz == len(rows)
    assert np.array_equal(yk[:ynnz].cpu().numpy(), rows)
    ok, _ = orc.within_tol(yv[:ynnz].cpu().numpy(), y64[rows], mag[rows], RTOL)
    assert ok
    ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
    assert ok


def test_csc_empty_x_and_reference_names(torch_cuda):
    torch = torch_cuda
    A = _matrix("uniform")
    h = make_handle(A, torch, hola=False)
    empty_k = torch.empty(0, dtype=torch.int32, device="cuda")
    empty_v = torch.empty(0, device="cuda")
    h.set_sparse_x(empty_k, empty_v, 0)
    y = torch.full((A.m,), 5.0, device="cuda")
    assert h.CscBasedNoSortNaiveSpmspv(1.0, y) == 0
    assert float(y.abs().sum()) == 0.0
    key, val = _x(A.n, 50, 9)
    set_sparse(h, key, val, torch)
    yk = torch.empty(A.m, dtype=torch.int32, device="cuda")
    yv = torch.empty(A.m, device="cuda")
    n1 = h.CscBasedNoSortMergeSpmspv_keyval(True, 1.0, y, yk, yv)
    a = (yk[:n1].cpu().numpy().copy(), yv[:n1].cpu().numpy().copy())
    n2 = h.CscBasedMyNoSortSpmspv_keyval(True, 1.0, y, yk, yv)
    assert n1 == n2 and np.array_equal(a[0], yk[:n2].cpu().numpy())
    n3 = h.CscBasedSortNaiveSpmspv(1.0, yk, yv)
    n4 = h.CscBasedSortMergeSpmspv(False, 1.0, y, yk, yv)
    n5 = h.CscBasedSortMySpmspv(False, 1.0, y, yk, yv)
    assert n3 == n4 == n5 >= n1


def test_csc_bad_key_reports_oob(torch_cuda):
    """An out-of-range x key is skipped and reported, never dereferenced."""
    torch = torch_cuda
    A = _matrix("uniform")
    h = make_handle(A, torch, hola=False)
    key = np.array([1, 2, A.n + 5], np.int32)
    val = np.ones(3, np.float32)
    set_sparse(h, key, val, torch)
    y = torch.empty(A.m, device="cuda")
    h.spmspv_csc(1, 0, 1.0, y)
    from spmx import SpmxError
    with pytest.raises(SpmxError) as e:
        h.check_device_error()
    assert e.value.code == -23


def test_device_transpose_matches_host(torch_cuda):
    torch = torch_cuda
    for A in (_matrix("uniform"), _matrix("skewed"), _matrix("long-col")):
        h = make_handle(A, torch, hola=False)
        row, colptr, val = h.get_csc()
        ecolptr, erow, eval_ = A.to_csc()
        assert np.array_equal(colptr.cpu().numpy(), ecolptr)
        assert np.array_equal(row.cpu().numpy(), erow)
        assert np.array_equal(val.cpu().numpy(), eval_)


def test_vector_conversions(torch_cuda):
    torch = torch_cuda
    A = _matrix("uniform")
    h = make_handle(A, torch, hola=False)
    key, val = _x(A.n, 300, 1)
    kd, vd = set_sparse(h, key, val, torch)
    xd = torch.full((A.n,), 9.0, device="cuda")
    bits = torch.full(((A.n + 31) // 32,), -1, dtype=torch.int32, device="cuda")
    h.set_x(xd)
    h.set_bitvector(bits, (A.n + 31) // 32)
    h.sparse2bitarray()
    ed, eb = orc.sparse2dense_bits(A.n, key, val)
    assert np.array_equal(xd.cpu().numpy(), ed)
    assert np.array_equal(bits.cpu().numpy().view(np.uint32), eb)
    bits.fill_(0)
    h.dense2bitarray()
    assert np.array_equal(bits.cpu().numpy().view(np.uint32), orc.dense2bitarray(ed))
    h.sparse2dense()
    assert np.array_equal(xd.cpu().numpy(), ed)
    kd.fill_(-1)
    vd.fill_(0)
    assert h.dense2sparse() == 300
    assert np.array_equal(kd.cpu().numpy(), key) and np.array_equal(vd.cpu().numpy(), val)
    # outer forms on a longer vector spanning many tiles
    d = np.random.default_rng(2).uniform(-1, 1, 70000).astype(np.float32)
    d[np.random.default_rng(3).random(70000) < 0.9] = 0
    dk = torch.empty(70000, dtype=torch.int32, device="cuda")
    dv = torch.empty(70000, device="cuda")
    cnt = h.dense2sparse_outer(70000, dev(d, torch), dk, dv)
    ek, ev = orc.dense2sparse(d)
    assert cnt == len(ek) and np.array_equal(dk[:cnt].cpu().numpy(), ek)
    back = torch.empty(70000, device="cuda")
    h.sparse2dense_outer(cnt, dk, dv, 70000, back)
    assert np.array_equal(back.cpu().numpy(), d)
    # the same compaction written straight into pinned host memory, twice in a
    # row on the handle's stream (no synchronisation inside the call)
    hk = torch.full((70000,), -1, dtype=torch.int32).pin_memory()
    hv = torch.zeros(70000).pin_memory()
    hc = torch.full((1,), -1, dtype=torch.int32).pin_memory()
    for dd in (d, np.where(np.arange(70000) % 3 == 0, d, 0).astype(np.float32)):
        dd_d = dev(dd, torch)
        h.dense2sparse_to_host(70000, dd_d, hk, hv, hc)
        torch.cuda.synchronize()
        ek, ev = orc.dense2sparse(dd)
        c = int(hc[0])
        assert c == len(ek)
        assert np.array_equal(hk[:c].numpy(), ek) and np.array_equal(hv[:c].numpy(), ev)
    with pytest.raises(ValueError):
        h.dense2sparse_to_host(70000, dd_d, dk.cpu(), hv, hc)  # not pinned


@pytest.mark.parametrize("length,frac", [(1, 1.0), (2047, 0.5), (2048, 0.0), (2049, 1.0), (2_097_152, 0.01),
                                         (2_097_153, 0.3), (5_000_001, 0.05)])
def test_compaction_lengths(torch_cuda, length, frac):
    """Dense -> (key, value) of the nonzeros, to device buffers and straight
    into pinned host memory, against numpy: ragged last ranges, no nonzeros,
    every element nonzero, and vectors longer than 1,024 ranges of 2,048
    elements (each CTA then compacts several sub-tiles in turn)."""
    torch = torch_cuda
    h = make_handle(rand_csr(64, 64, density=0.1, seed=3), torch, hola=False)
    rng = np.random.default_rng(length)
    d = rng.uniform(-1, 1, length).astype(np.float32)
    d[rng.random(length) >= frac] = 0
    ek, ev = orc.dense2sparse(d)
    dd = dev(d, torch)
    dk = torch.full((length,), -1, dtype=torch.int32, device="cuda")
    dv = torch.zeros(length, device="cuda")
    cnt = h.dense2sparse_outer(length, dd, dk, dv)
    assert cnt == len(ek)
    assert np.array_equal(dk[:cnt].cpu().numpy(), ek) and np.array_equal(dv[:cnt].cpu().numpy(), ev)
    hk = torch.full((length,), -1, dtype=torch.int32).pin_memory()
    hv = torch.zeros(length).pin_memory()
    hc = torch.full((1,), -1, dtype=torch.int32).pin_memory()
    h.dense2sparse_to_host(length, dd, hk, hv, hc)
    torch.cuda.synchronize()
    c = int(hc[0])
    assert c == len(ek)
    assert np.array_equal(hk[:c].numpy(), ek) and np.array_equal(hv[:c].numpy(), ev)
    h.check_device_error()


def test_compaction_on_read_back_stream(torch_cuda):
    """The e2e pattern: SpMSpV calls on one stream, each result compacted into
    pinned host memory on a second stream (the handle switched to it for that
    call) while the next calls run; every host result against the oracle."""
    torch = torch_cuda
    from spmx import gen
    A = gen.zipf_rows(200_000, 1.5, 16, 2000, seed=4)
    h = make_handle(A, torch, hola=False)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    h.set_stream(s1)
    colptr, row, cval = A.to_csc()
    xs = [_x(A.n, k, 20 + k) for k in (3, 200, 5_000, 60_000)]
    keys = [dev(k, torch) for k, _ in xs]
    vals = [dev(v, torch) for _, v in xs]
    ys = [torch.empty(A.m, device="cuda") for _ in xs]
    hk = [torch.empty(A.m, dtype=torch.int32).pin_memory() for _ in xs]
    hv = [torch.empty(A.m).pin_memory() for _ in xs]
    hc = torch.full((len(xs),), -1, dtype=torch.int32).pin_memory()
    evs = [torch.cuda.Event() for _ in xs]
    for rep in range(2):
        for i in range(len(xs)):
            h.set_sparse_x(keys[i], vals[i], len(xs[i][0]))
            h.spmspv_csc(0, 0, 1.0, ys[i], sync=False)
            evs[i].record(s1)
            s2.wait_event(evs[i])
            h.set_stream(s2)
            h.dense2sparse_to_host(A.m, ys[i], hk[i], hv[i], hc[i:i + 1])
            h.set_stream(s1)
        torch.cuda.synchronize()
        h.check_device_error()
        for i, (key, val) in enumerate(xs):
            y64, mag, _ = orc.spmspv_csc_f64(A.m, colptr, row, cval, key, val)
            got = np.zeros(A.m)
            c = int(hc[i])
            got[hk[i][:c].numpy()] = hv[i][:c].numpy()
            ok, _ = orc.within_tol(got, y64, mag, RTOL)
            assert ok, (rep, i)


def test_features(torch_cuda):
    torch = torch_cuda
    from spmx import gen
    for A in (_matrix("skewed"), gen.zipf_rows(50000, 1.5, 16, 10000, seed=2)):
        h = make_handle(A, torch, hola=False)
        f = h.computeMatFeture()
        e = orc.mat_features(A.n, A.rowptr)
        assert np.allclose(f, e, rtol=1e-9, atol=1e-12)
        assert h.extractMatFeatureParallel() == pytest.approx(orc.std_row_intmean(A.rowptr), rel=1e-6)
        key, val = _x(A.n, 1000, 5)
        set_sparse(h, key, val, torch)
        colptr, _, _ = A.to_csc()
        assert list(h.computeVecFeture()) == orc.vec_features(colptr, key).tolist()
        b = h.computeBinlenVer2()
        assert h.computeGM() == pytest.approx(orc.gm(A.m, A.nnz, 1000, b).tolist())
        feats = h.features()
        assert feats["bin_len"] == b and feats["x_nnz"] == 1000


@pytest.mark.parametrize("mat", ["uniform", "skewed", "long-col"])
@pytest.mark.parametrize("frac", [0.0005, 0.05, 1.0])
@pytest.mark.parametrize("buckets", [0, 3, 64])
def test_csc_bucket(torch_cuda, mat, frac, buckets):
    """Bucket write-back: dense y and the sorted touched rows (no global atomics)."""
    torch = torch_cuda
    A = _matrix(mat)
    h = make_handle(A, torch, hola=False)
    k = max(1, int(frac * A.n))
    key, val = _x(A.n, k, 6)
    set_sparse(h, key, val, torch)
    y = torch.full((A.m,), 4.0, device="cuda")
    yk = torch.empty(A.m, dtype=torch.int32, device="cuda")
    yv = torch.empty(A.m, device="cuda")
    ynnz = h.CscBasedBucketSpmspv(0.5, y, yk, yv, buckets)
    h.check_device_error()
    colptr, row, cval = A.to_csc()
    y64, mag, touched = orc.spmspv_csc_f64(A.m, colptr, row, cval, key, val, alpha=0.5)
    ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
    assert ok
    rows = np.nonzero(touched)[0]
    assert ynnz == len(rows)
    assert np.array_equal(yk[:ynnz].cpu().numpy(), rows)
    assert np.array_equal(yv[:ynnz].cpu().numpy(), y.cpu().numpy()[rows])
