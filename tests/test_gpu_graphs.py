"""Entry points without host round trips can be recorded in a CUDA graph.

After one call outside capture (which sizes the handle's scratch), these are
captured on the handle's stream and replayed:
- the dispatched SpMV (tiled back-end);
- the CSC SpMSpV with atomic write-back, naive and merge-path;
- the adaptive call (selector on host-known features + chosen kernel);
- a whole BFS traversal (one cooperative launch).
Replays must match the oracle like direct calls do."""
import numpy as np
import pytest

from conftest import rand_csr
from gpu_util import dev, make_handle
import oracle.oracle as orc

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _capture(torch, h, fn):
    s = torch.cuda.Stream()
    h.set_stream(s)
    with torch.cuda.stream(s):
        fn()  # outside capture: scratch allocation, preprocessing caches
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        fn()
    return g, s


def test_graph_spmv_and_csc_spmspv(torch_cuda):
    torch = torch_cuda
    A = rand_csr(6000, 5000, density=0.003, seed=21)
    h = make_handle(A, torch)
    h.tiledPreprocess()
    h.set_spmv_type(2)
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, A.n).astype(np.float32)
    k = 400
    key = np.sort(rng.choice(A.n, k, replace=False)).astype(np.int32)
    val = rng.uniform(-1, 1, k).astype(np.float32)
    xd, kd, vd = dev(x, torch), dev(key, torch), dev(val, torch)
    y0 = torch.empty(A.m, device="cuda")
    y1 = torch.empty(A.m, device="cuda")
    y2 = torch.empty(A.m, device="cuda")

    def work():
        h.set_x(xd)
        h.spmv(1.0, y0)
        h.set_sparse_x(kd, vd, k)
        h.spmspv_csc(0, 0, 1.0, y1, sync=False)  # naive, atomic
        h.spmspv_csc(1, 0, 1.0, y2, sync=False)  # merge-path, atomic

    g, s = _capture(torch, h, work)
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, x)
    colptr, row, cval = A.to_csc()
    z64, zmag, _ = orc.spmspv_csc_f64(A.m, colptr, row, cval, key, val)
    for _ in range(2):
        for t in (y0, y1, y2):
            t.fill_(9.0)
        g.replay()
        s.synchronize()
        h.check_device_error()
        assert orc.within_tol(y0.cpu().numpy(), y64, mag, RTOL)[0]
        assert orc.within_tol(y1.cpu().numpy(), z64, zmag, RTOL)[0]
        assert orc.within_tol(y2.cpu().numpy(), z64, zmag, RTOL)[0]
    del g


def test_graph_adaptive(torch_cuda):
    torch = torch_cuda
    A = rand_csr(8000, 8000, density=0.002, seed=22)
    h = make_handle(A, torch)
    h.allocPreBuffer()
    rng = np.random.default_rng(4)
    k = 80
    key = np.sort(rng.choice(A.n, k, replace=False)).astype(np.int32)
    val = rng.uniform(-1, 1, k).astype(np.float32)
    kd, vd = dev(key, torch), dev(val, torch)
    y = torch.empty(A.m, device="cuda")
    h.set_sparse_x(kd, vd, k)
    chosen = h.select()
    # the sort write-back reads its pair count back, so it is not capturable
    assert chosen not in (0, 2), "expected an atomic CSC kernel for this tiny x"

    def work():
        h.run_adaptive(1.0, y)

    g, s = _capture(torch, h, work)
    colptr, row, cval = A.to_csc()
    z64, zmag, _ = orc.spmspv_csc_f64(A.m, colptr, row, cval, key, val)
    y.fill_(5.0)
    g.replay()
    s.synchronize()
    h.check_device_error()
    assert orc.within_tol(y.cpu().numpy(), z64, zmag, RTOL)[0], chosen
    del g


def test_graph_bfs(torch_cuda):
    torch = torch_cuda
    from spmx import gen, SpmspvHandle
    g = gen.rmat(13, 8, seed=23)
    n = g.n
    h = SpmspvHandle(n, n, g.nnz)
    rp, cl = dev(g.rowptr, torch), dev(g.col, torch)
    h.InputCSR(g.nnz, rp, cl, None)
    lv = torch.empty(n, dtype=torch.int32, device="cuda")
    ref, _ = orc.bfs_queue(n, g.rowptr, g.col, 7)

    def work():
        h.bfs(7, lv, sync=False)

    graph, s = _capture(torch, h, work)
    for _ in range(2):
        lv.fill_(-5)
        graph.replay()
        s.synchronize()
        h.check_device_error()
        assert np.array_equal(lv.cpu().numpy(), ref)
    del graph


@pytest.mark.parametrize("parts", [1, 2])
def test_graph_round_spmv_chain(torch_cuda, parts):
    """The round back-end launched as the dependent of the sparse-to-dense
    scatter (cluster and programmatic-dependent-launch attributes) replays
    from a graph: sparse x -> dense x -> SpMV, and the gated form; one CTA
    per row block and 2-CTA clusters."""
    torch = torch_cuda
    from spmx import gen
    A = gen.zipf_rows(1 << 15, 1.5, 16, 3000, seed=24)
    h = make_handle(A, torch, csc=False, hola=False)
    h.roundPreprocess(0, parts)
    h.set_spmv_type(3)
    rng = np.random.default_rng(25)
    k = A.n // 3
    key = np.sort(rng.choice(A.n, k, replace=False)).astype(np.int32)
    val = rng.uniform(-1, 1, k).astype(np.float32)
    kd, vd = dev(key, torch), dev(val, torch)
    xdense = torch.zeros(A.n, device="cuda")
    bits = torch.zeros((A.n + 31) // 32, dtype=torch.int32, device="cuda")
    h.set_x(xdense)
    h.set_bitvector(bits, (A.n + 31) // 32)
    y0 = torch.empty(A.m, device="cuda")
    y1 = torch.empty(A.m, device="cuda")

    def work():
        h.set_sparse_x(kd, vd, k)
        h.sparse2dense()
        h.spmv(1.0, y0)
        h.sparse2bitarray()
        h.spmspv(2.0, y1)

    g, s = _capture(torch, h, work)
    xd, bm = orc.sparse2dense_bits(A.n, key, val)
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, xd)
    z64, zmag = orc.spmv_f64(A.rowptr, A.col, A.val, xd, alpha=2.0, bits=bm.view(np.int32))
    for _ in range(2):
        y0.fill_(9.0)
        y1.fill_(9.0)
        xdense.fill_(5.0)  # the replayed scatter rebuilds x from the sparse vector
        g.replay()
        s.synchronize()
        h.check_device_error()
        assert orc.within_tol(y0.cpu().numpy(), y64, mag, RTOL)[0]
        assert orc.within_tol(y1.cpu().numpy(), z64, zmag, RTOL)[0]
    del g


def test_graph_replay_after_keys_change(torch_cuda):
    """A captured load-balanced CSC SpMSpV (look-back scan + merge-path pass)
    replayed after x's keys and values change in place: every replay scans
    with a fresh look-back epoch (kept in device memory), so no tile can take
    a prefix left by the previous replay.  x spans many scan tiles."""
    torch = torch_cuda
    A = rand_csr(30000, 40000, density=0.0008, seed=23)
    h = make_handle(A, torch, hola=False)
    rng = np.random.default_rng(5)
    k = 20000
    keys = [np.sort(rng.choice(A.n, k, replace=False)).astype(np.int32) for _ in range(3)]
    vals = [rng.uniform(-1, 1, k).astype(np.float32) for _ in range(3)]
    kd, vd = dev(keys[0], torch), dev(vals[0], torch)
    y = torch.empty(A.m, device="cuda")

    def work():
        h.set_sparse_x(kd, vd, k)
        h.spmspv_csc(1, 0, 1.0, y, sync=False)  # merge-path, atomic

    g, s = _capture(torch, h, work)
    colptr, row, cval = A.to_csc()
    for rep in range(6):
        i = rep % 3
        with torch.cuda.stream(s):
            kd.copy_(torch.from_numpy(keys[i]))
            vd.copy_(torch.from_numpy(vals[i]))
            y.fill_(9.0)
        g.replay()
        s.synchronize()
        h.check_device_error()
        y64, mag, _ = orc.spmspv_csc_f64(A.m, colptr, row, cval, keys[i], vals[i])
        assert orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)[0], f"replay {rep}"
    del g
