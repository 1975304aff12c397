"""Shared test set-up: import paths, the `gpu` marker, common fixtures.

Tests marked `gpu` run the CUDA library on a real B200 and compare it with the
CPU oracle; everything else runs on the CPU (oracle, generators, host logic,
ABI surface).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "spmspv-adaptive_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libspmx.so")


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    return torch


def rand_csr(m, n, density=None, lens=None, seed=0, val=True):
    """Random CSR with sorted distinct columns; `lens` overrides row lengths."""
    from spmx.gen import Csr
    rng = np.random.default_rng(seed)
    if lens is None:
        lens = rng.binomial(n, density, size=m)
    lens = np.minimum(np.asarray(lens, dtype=np.int64), n)
    rowptr = np.zeros(m + 1, np.int64)
    rowptr[1:] = np.cumsum(lens)
    col = np.empty(int(rowptr[-1]), np.int32)
    for i in range(m):
        if lens[i]:
            col[rowptr[i]:rowptr[i + 1]] = np.sort(rng.choice(n, size=int(lens[i]), replace=False))
    v = rng.uniform(-1, 1, size=len(col)).astype(np.float32) if val else None
    return Csr(m, n, rowptr.astype(np.int32), col, v)


def sym_graph(n, edges):
    """Symmetric CSR pattern from an undirected edge list (no self loops)."""
    from spmx.gen import Csr
    adj = [set() for _ in range(n)]
    for u, v in edges:
        if u != v:
            adj[u].add(v)
            adj[v].add(u)
    rowptr = np.zeros(n + 1, np.int32)
    cols = []
    for i in range(n):
        s = sorted(adj[i])
        cols.extend(s)
        rowptr[i + 1] = rowptr[i] + len(s)
    return Csr(n, n, rowptr, np.array(cols, np.int32), None)
