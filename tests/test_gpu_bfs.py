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
