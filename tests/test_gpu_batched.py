"""Batched SpMSpV forward and adjoint on the GPU against FP64 references.

Y and dY are m x nvec, row-major (Y[i, v] = (A x_v)[i]).

Forward: every vector of the batch against the oracle's SpmSpvCSCHost
restatement, |y32 - y64| <= 1e-5 * max(|y64|, sum |a_ij x_j|).  Backward:
dxval and dvals against FP64 sums of the same products, with the bound
1e-5 * (sum of |terms|) + 1e-30.  CUDA-graph replay of forward + backward
must reproduce the direct calls within the same bounds."""
import numpy as np
import pytest

from gpu_util import dev, make_handle
import oracle.oracle as orc

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _batch(n, nvec, seed, lo=1, hi=2000, with_empty=True):
    """nvec sparse vectors with log-uniform nnz, concatenated; one empty."""
    from spmx import gen
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), nvec)).astype(np.int64)
    if with_empty:
        sizes[nvec // 3] = 0
    keys, vals = [], []
    for v, k in enumerate(sizes):
        kk, vv = gen.sparse_vector(n, int(k), dist="normal", seed=seed * 1000 + v)
        keys.append(kk)
        vals.append(vv)
    xptr = np.zeros(nvec + 1, np.int32)
    xptr[1:] = np.cumsum(sizes)
    return xptr, np.concatenate(keys).astype(np.int32), np.concatenate(vals).astype(np.float32)


def _refs(A, xptr, xkey, xval, dY, alpha):
    """FP64 dxval, dvals (CSR order) and their magnitude bounds."""
    colptr, row, cval = A.to_csc()
    # CSR index of each CSC position: stable transpose of the CSR positions
    order = np.argsort(A.col, kind="stable").astype(np.int64)
    nvec = len(xptr) - 1
    dx = np.zeros(len(xkey))
    dxm = np.zeros(len(xkey))
    dv = np.zeros(A.nnz)
    dvm = np.zeros(A.nnz)
    for v in range(nvec):
        for e in range(xptr[v], xptr[v + 1]):
            j = xkey[e]
            ks = np.arange(colptr[j], colptr[j + 1])
            g = dY[row[ks], v].astype(np.float64)
            a = cval[ks].astype(np.float64)
            dx[e] = alpha * np.sum(a * g)
            dxm[e] = abs(alpha) * np.sum(np.abs(a * g))
            t = alpha * float(xval[e]) * g
            np.add.at(dv, order[ks], t)
            np.add.at(dvm, order[ks], np.abs(t))
    return dx, dxm, dv, dvm


@pytest.fixture(scope="module")
def problem(torch_cuda):
    from spmx import gen
    A = gen.chung_lu(20000, 2.1, 16.0, seed=5)
    xptr, xkey, xval = _batch(A.n, 24, seed=3)
    return A, xptr, xkey, xval


def _check_forward(A, xptr, xkey, xval, Y, alpha):
    colptr, row, cval = A.to_csc()
    for v in range(len(xptr) - 1):
        k, x = xkey[xptr[v]:xptr[v + 1]], xval[xptr[v]:xptr[v + 1]]
        y64, mag, _ = orc.spmspv_csc_f64(A.m, colptr, row, cval, k, x, alpha=alpha)
        ok, _ = orc.within_tol(Y[:, v], y64, mag, RTOL)
        assert ok, (v, orc.max_scaled_err(Y[:, v], y64, mag))


def _close(got, ref, mag):
    return np.all(np.abs(np.asarray(got, np.float64) - ref) <= RTOL * mag + 1e-30)


@pytest.mark.parametrize("alpha", [1.0, -0.5])
def test_batched_forward(torch_cuda, problem, alpha):
    torch = torch_cuda
    A, xptr, xkey, xval = problem
    h = make_handle(A, torch, hola=False)
    Y = torch.full((A.m, len(xptr) - 1), 5.0, device="cuda")
    h.spmspv_batched(dev(xptr, torch), dev(xkey, torch), dev(xval, torch), alpha, Y)
    h.check_device_error()
    _check_forward(A, xptr, xkey, xval, Y.cpu().numpy(), alpha)


def test_batched_backward(torch_cuda, problem):
    torch = torch_cuda
    A, xptr, xkey, xval = problem
    alpha = 0.75
    h = make_handle(A, torch, hola=False)
    nvec = len(xptr) - 1
    dY = np.random.default_rng(9).standard_normal((A.m, nvec)).astype(np.float32)
    dxval = torch.full((len(xkey),), 7.0, device="cuda")
    dvals = torch.full((A.nnz,), 7.0, device="cuda")
    h.spmspv_batched_backward(dev(xptr, torch), dev(xkey, torch), dev(xval, torch), alpha,
                              dev(dY, torch), dxval, dvals)
    h.check_device_error()
    dx, dxm, dv, dvm = _refs(A, xptr, xkey, xval, dY, alpha)
    assert _close(dxval.cpu().numpy(), dx, dxm)
    assert _close(dvals.cpu().numpy(), dv, dvm)


def test_batched_graph_replay(torch_cuda, problem):
    """Forward + backward captured once in a CUDA graph, replayed twice."""
    torch = torch_cuda
    A, xptr, xkey, xval = problem
    h = make_handle(A, torch, hola=False)
    nvec = len(xptr) - 1
    xp, xk, xv = dev(xptr, torch), dev(xkey, torch), dev(xval, torch)
    dY = dev(np.random.default_rng(4).standard_normal((A.m, nvec)).astype(np.float32), torch)
    Y = torch.empty((A.m, nvec), device="cuda")
    dxval = torch.empty(len(xkey), device="cuda")
    dvals = torch.empty(A.nnz, device="cuda")
    tot = int(xptr[-1])  # host-side entry count: nothing is read back during capture
    s = torch.cuda.Stream()
    h.set_stream(s)
    with torch.cuda.stream(s):
        # first calls outside capture allocate the handle's scratch
        h.spmspv_batched(xp, xk, xv, 1.0, Y, x_total=tot)
        h.spmspv_batched_backward(xp, xk, xv, 1.0, dY, dxval, dvals, x_total=tot)
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        h.spmspv_batched(xp, xk, xv, 1.0, Y, x_total=tot)
        h.spmspv_batched_backward(xp, xk, xv, 1.0, dY, dxval, dvals, x_total=tot)
    for _ in range(2):
        Y.fill_(3.0)
        dxval.fill_(3.0)
        dvals.fill_(3.0)
        g.replay()
        torch.cuda.synchronize()
        h.check_device_error()
        _check_forward(A, xptr, xkey, xval, Y.cpu().numpy(), 1.0)
        dx, dxm, dv, dvm = _refs(A, xptr, xkey, xval, dY.cpu().numpy(), 1.0)
        assert _close(dxval.cpu().numpy(), dx, dxm)
        assert _close(dvals.cpu().numpy(), dv, dvm)
    del g


def test_batched_matches_single_calls(torch_cuda, problem):
    """nvec = 1 calls, one per vector, give the rows of the batched result."""
    torch = torch_cuda
    A, xptr, xkey, xval = problem
    h = make_handle(A, torch, hola=False)
    nvec = len(xptr) - 1
    Yb = torch.empty((A.m, nvec), device="cuda")
    h.spmspv_batched(dev(xptr, torch), dev(xkey, torch), dev(xval, torch), 1.0, Yb)
    Ybh = Yb.cpu().numpy()
    colptr, row, cval = A.to_csc()
    for v in range(nvec):
        a, b = xptr[v], xptr[v + 1]
        y1 = torch.empty((A.m, 1), device="cuda")
        h.spmspv_batched(dev(np.array([0, b - a], np.int32), torch), dev(xkey[a:b], torch),
                         dev(xval[a:b], torch), 1.0, y1)
        y64, mag, _ = orc.spmspv_csc_f64(A.m, colptr, row, cval, xkey[a:b], xval[a:b])
        ok, _ = orc.within_tol(y1.cpu().numpy()[:, 0], y64, mag, RTOL)
        assert ok
        ok, _ = orc.within_tol(Ybh[:, v], y64, mag, RTOL)
        assert ok


def test_batched_out_of_range_key(torch_cuda):
    from spmx import gen, SpmxError
    torch = torch_cuda
    A = gen.chung_lu(2000, 2.1, 8.0, seed=6)
    h = make_handle(A, torch, hola=False)
    xptr = np.array([0, 2], np.int32)
    xkey = np.array([3, A.n], np.int32)  # second key is out of range
    xval = np.ones(2, np.float32)
    Y = torch.empty((A.m, 1), device="cuda")
    h.spmspv_batched(dev(xptr, torch), dev(xkey, torch), dev(xval, torch), 1.0, Y)
    with pytest.raises(SpmxError):
        h.check_device_error()


def test_batched_deterministic(torch_cuda, problem):
    """Backward results are bit-identical across calls (no atomics)."""
    torch = torch_cuda
    A, xptr, xkey, xval = problem
    h = make_handle(A, torch, hola=False)
    nvec = len(xptr) - 1
    dY = dev(np.random.default_rng(8).standard_normal((A.m, nvec)).astype(np.float32), torch)
    xp, xk, xv = dev(xptr, torch), dev(xkey, torch), dev(xval, torch)
    outs = []
    for _ in range(2):
        dxval = torch.empty(len(xkey), device="cuda")
        dvals = torch.empty(A.nnz, device="cuda")
        h.spmspv_batched_backward(xp, xk, xv, 1.0, dY, dxval, dvals)
        outs.append((dxval.cpu().numpy(), dvals.cpu().numpy()))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


@pytest.mark.parametrize("graph", [False, True])
def test_batched_options_reuse_and_fused(torch_cuda, problem, graph):
    """With SPMX_BATCH_REUSE_INVERSION | SPMX_BATCH_FUSED_DXVAL the backward
    reuses the forward's inversion and accumulates dxval in the dvals pass;
    results stay within the same bounds, directly and replayed from a graph.
    A backward on another batch (other pointers) inverts again."""
    torch = torch_cuda
    from spmx import abi
    A, xptr, xkey, xval = problem
    h = make_handle(A, torch, hola=False)
    h.set_batch_options(abi.BATCH_REUSE_INVERSION | abi.BATCH_FUSED_DXVAL)
    nvec = len(xptr) - 1
    xp, xk, xv = dev(xptr, torch), dev(xkey, torch), dev(xval, torch)
    dYh = np.random.default_rng(12).standard_normal((A.m, nvec)).astype(np.float32)
    dY = dev(dYh, torch)
    Y = torch.empty((A.m, nvec), device="cuda")
    dxval = torch.full((len(xkey),), 7.0, device="cuda")
    dvals = torch.full((A.nnz,), 7.0, device="cuda")
    tot = int(xptr[-1])
    s = torch.cuda.Stream()
    h.set_stream(s)

    def work():
        h.spmspv_batched(xp, xk, xv, 0.5, Y, x_total=tot)
        h.spmspv_batched_backward(xp, xk, xv, 0.5, dY, dxval, dvals, x_total=tot)

    with torch.cuda.stream(s):
        work()
    s.synchronize()
    if graph:
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            work()
        for t in (Y, dxval, dvals):
            t.fill_(3.0)
        g.replay()
        s.synchronize()
    h.check_device_error()
    _check_forward(A, xptr, xkey, xval, Y.cpu().numpy(), 0.5)
    dx, dxm, dv, dvm = _refs(A, xptr, xkey, xval, dYh, 0.5)
    assert _close(dxval.cpu().numpy(), dx, dxm)
    assert _close(dvals.cpu().numpy(), dv, dvm)
    # another batch: the backward must not reuse the first batch's inversion
    xptr2, xkey2, xval2 = _batch(A.n, 5, seed=21, with_empty=False)
    xp2, xk2, xv2 = dev(xptr2, torch), dev(xkey2, torch), dev(xval2, torch)
    dY2h = dYh[:, :5].copy()
    dxval2 = torch.empty(len(xkey2), device="cuda")
    dvals2 = torch.empty(A.nnz, device="cuda")
    with torch.cuda.stream(s):
        h.spmspv_batched_backward(xp2, xk2, xv2, 1.0, dev(dY2h, torch), dxval2, dvals2)
    s.synchronize()
    h.check_device_error()
    dx, dxm, dv, dvm = _refs(A, xptr2, xkey2, xval2, dY2h, 1.0)
    assert _close(dxval2.cpu().numpy(), dx, dxm)
    assert _close(dvals2.cpu().numpy(), dv, dvm)


def test_batched_rows_heavier_than_a_chunk(torch_cuda):
    """A row of 9,000 nonzeros spans several row chunks (the chunks whose
    weight boundaries fall inside it are empty and must be skipped), between
    empty rows and short ones; forward and fused backward against FP64."""
    torch = torch_cuda
    from conftest import rand_csr
    rng = np.random.default_rng(61)
    lens = rng.integers(0, 8, 3000)
    lens[rng.choice(3000, 400, replace=False)] = 0
    lens[7] = 9000
    lens[2999] = 5000
    A = rand_csr(3000, 12000, lens=lens, seed=62)
    xptr, xkey, xval = _batch(A.n, 8, seed=63, lo=50, hi=3000)
    h = make_handle(A, torch, hola=False)
    h.set_batch_options(3)
    nvec, tot = len(xptr) - 1, int(xptr[-1])
    Y = torch.empty((A.m, nvec), device="cuda")
    xp, xk, xv = dev(xptr, torch), dev(xkey, torch), dev(xval, torch)
    h.spmspv_batched(xp, xk, xv, 1.25, Y, x_total=tot)
    dY = np.random.default_rng(64).standard_normal((A.m, nvec)).astype(np.float32)
    dxval = torch.empty(tot, device="cuda")
    dvals = torch.empty(A.nnz, device="cuda")
    h.spmspv_batched_backward(xp, xk, xv, 1.25, dev(dY, torch), dxval, dvals, x_total=tot)
    h.check_device_error()
    _check_forward(A, xptr, xkey, xval, Y.cpu().numpy(), 1.25)
    dx, dxm, dv, dvm = _refs(A, xptr, xkey, xval, dY, 1.25)
    assert _close(dxval.cpu().numpy(), dx, dxm)
    assert _close(dvals.cpu().numpy(), dv, dvm)


def test_batched_unaligned_outputs(torch_cuda, problem):
    """Y and dY that start 4 bytes past a 16-byte boundary take the scalar
    row stores / loads (nvec is a multiple of 4 here)."""
    torch = torch_cuda
    A, xptr, xkey, xval = problem
    nvec = len(xptr) - 1
    assert nvec % 4 == 0
    h = make_handle(A, torch, hola=False)
    xp, xk, xv = dev(xptr, torch), dev(xkey, torch), dev(xval, torch)
    Ybuf = torch.full((A.m * nvec + 1,), 5.0, device="cuda")
    Y = Ybuf[1:].view(A.m, nvec)
    assert Y.data_ptr() % 16 == 4
    h.spmspv_batched(xp, xk, xv, 1.0, Y)
    h.check_device_error()
    _check_forward(A, xptr, xkey, xval, Y.cpu().numpy(), 1.0)
    dYh = np.random.default_rng(13).standard_normal((A.m, nvec)).astype(np.float32)
    dYbuf = torch.empty(A.m * nvec + 1, device="cuda")
    dYbuf[1:].copy_(torch.from_numpy(dYh.ravel()))
    dY = dYbuf[1:].view(A.m, nvec)
    dxval = torch.empty(len(xkey), device="cuda")
    dvals = torch.empty(A.nnz, device="cuda")
    h.spmspv_batched_backward(xp, xk, xv, 1.0, dY, dxval, dvals)
    h.check_device_error()
    dx, dxm, dv, dvm = _refs(A, xptr, xkey, xval, dYh, 1.0)
    assert _close(dxval.cpu().numpy(), dx, dxm)
    assert _close(dvals.cpu().numpy(), dv, dvm)
