"""BFS levels on the GPU are bit-exact against the oracle's level-synchronous
Boolean SpMSpV BFS."""
import numpy as np
import pytest

from conftest import sym_graph
from gpu_util import make_handle
import oracle.oracle as orc

pytestmark = pytest.mark.gpu


def _bfs(h, src, n, torch):
    lv = torch.empty(n, dtype=torch.int32, device="cuda")
    d = h.bfs(src, lv)
    h.check_device_error()
    return lv.cpu().numpy(), d


def test_bfs_rmat_scale14(torch_cuda):
    """R-MAT scale 14, edge factor 16, seed 1, source 0."""
    torch = torch_cuda
    from spmx import gen
    g = gen.rmat(14, 16, seed=1)
    h = make_handle(g, torch, csc=False, hola=False)
    for src in (0, 1, 77, 16383):
        lv, d = _bfs(h, src, g.n, torch)
        colptr, row, _ = g.to_csc()
        e, ed = orc.bfs_spmspv(g.n, colptr, row, src)
        assert np.array_equal(lv, e), src
        assert d == ed


def test_bfs_small_graphs(torch_cuda):
    torch = torch_cuda
    cases = [
        (7, [(0, 1), (0, 2), (1, 3), (2, 3), (3, 4), (5, 6)], 0),
        (1, [], 0),
        (5, [], 3),
        (200, [(i, i + 1) for i in range(199)], 0),              # path: 200 levels
        (300, [(0, i) for i in range(1, 300)], 5),               # star from a leaf
    ]
    for n, edges, src in cases:
        g = sym_graph(n, edges)
        h = make_handle(g, torch, csc=False, hola=False)
        lv, d = _bfs(h, src, n, torch)
        e, ed = orc.bfs_queue(n, g.rowptr, g.col, src)
        assert np.array_equal(lv, e) and d == ed, (n, src)


def test_bfs_rmat_larger_both_directions(torch_cuda):
    """Scale 18 exercises push and pull levels."""
    torch = torch_cuda
    from spmx import gen
    g = gen.rmat(18, 16, seed=3)
    h = make_handle(g, torch, csc=False, hola=False)
    lv, d = _bfs(h, 0, g.n, torch)
    e, ed = orc.bfs_queue(g.n, g.rowptr, g.col, 0)
    assert np.array_equal(lv, e) and d == ed


def test_bfs_level_stepped_mode(torch_cuda):
    torch = torch_cuda
    from spmx import gen
    g = gen.rmat(14, 16, seed=1)
    h = make_handle(g, torch, csc=False, hola=False)
    h.set_bfs_mode(1)
    lv, d = _bfs(h, 0, g.n, torch)
    e, ed = orc.bfs_queue(g.n, g.rowptr, g.col, 0)
    assert np.array_equal(lv, e) and d == ed


@pytest.mark.parametrize("layout", [0, 1])
def test_batched_bfs_matches_plain_runs(torch_cuda, layout):
    """64 sources in one launch == 64 single-source traversals, bit for bit."""
    torch = torch_cuda
    from spmx import gen
    g = gen.rmat(14, 16, seed=1)
    h = make_handle(g, torch, csc=False, hola=False)
    rng = np.random.default_rng(3)
    deg = np.diff(g.rowptr)
    srcs = rng.choice(np.nonzero(deg > 0)[0], 64, replace=False).tolist()
    srcs[5] = srcs[4]  # a repeated source shares its frontier word
    srcs[63] = int(np.nonzero(deg == 0)[0][0]) if (deg == 0).any() else srcs[63]
    lv = torch.empty(64 * g.n, dtype=torch.int32, device="cuda")
    depth = h.bfs_batched(srcs, lv, layout=layout)
    h.check_device_error()
    got = lv.cpu().numpy().reshape((64, g.n) if layout == 1 else (g.n, 64))
    if layout == 0:
        got = got.T
    dmax = 0
    for s, src in enumerate(srcs):
        e, ed = orc.bfs_queue(g.n, g.rowptr, g.col, src)
        assert np.array_equal(got[s], e), s
        dmax = max(dmax, ed)
    assert depth == dmax


def test_batched_bfs_small_graphs(torch_cuda):
    torch = torch_cuda
    g = sym_graph(300, [(i, i + 1) for i in range(299)] + [(0, 150)])
    h = make_handle(g, torch, csc=False, hola=False)
    srcs = [0, 299, 150, 77]
    lv = torch.empty(len(srcs) * g.n, dtype=torch.int32, device="cuda")
    h.bfs_batched(srcs, lv, layout=1)
    got = lv.cpu().numpy().reshape(len(srcs), g.n)
    for s, src in enumerate(srcs):
        e, _ = orc.bfs_queue(g.n, g.rowptr, g.col, src)
        assert np.array_equal(got[s], e)
