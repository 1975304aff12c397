"""The per-matrix autotuner: it picks a back-end and launch parameters that
still give correct results, stores them in its cache file, and a second
handle on the same matrix applies the cached choice (including cache lines
written before the CSR5 sigma was tuned, which have one field fewer)."""
import numpy as np
import pytest

from conftest import rand_csr
from gpu_util import dev, make_handle, set_sparse
import oracle.oracle as orc

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _spmv_ok(h, A, torch):
    x = np.random.default_rng(3).uniform(-1, 1, A.n).astype(np.float32)
    h.set_x(dev(x, torch))
    y = torch.full((A.m,), 7.0, device="cuda")
    h.spmv(1.0, y)
    h.check_device_error()
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, x)
    return orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)[0]


def test_autotune_cache_round_trip(torch_cuda, tmp_path):
    torch = torch_cuda
    A = rand_csr(20000, 15000, lens=np.minimum(np.random.default_rng(1).zipf(1.5, 20000), 3000), seed=2)
    cache = str(tmp_path / "tune.txt")
    h = make_handle(A, torch)
    h.allocPreBuffer()
    backend = h.autotune(cache)
    assert backend in (0, 1, 2, 3)
    assert _spmv_ok(h, A, torch)
    lines = open(cache).read().split()
    assert len(lines) == 10  # fingerprint + 9 parameters
    # a fresh handle reads the cache instead of timing
    h2 = make_handle(A, torch)
    assert h2.autotune(cache) == backend
    assert _spmv_ok(h2, A, torch)
    # the naive CSC kernel with the tuned lanes per column still matches
    key = np.sort(np.random.default_rng(4).choice(A.n, 300, replace=False)).astype(np.int32)
    val = np.random.default_rng(5).uniform(-1, 1, 300).astype(np.float32)
    set_sparse(h2, key, val, torch)
    y = torch.empty(A.m, device="cuda")
    h2.spmspv_csc(0, 0, 1.0, y)
    colptr, row, cval = A.to_csc()
    y64, mag, _ = orc.spmspv_csc_f64(A.m, colptr, row, cval, key, val)
    assert orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)[0]


def test_autotune_reads_nine_field_cache_lines(torch_cuda, tmp_path):
    torch = torch_cuda
    A = rand_csr(8000, 8000, density=0.002, seed=6)
    cache = str(tmp_path / "tune.txt")
    h = make_handle(A, torch)
    backend = h.autotune(cache)
    fields = open(cache).read().split()
    with open(cache, "w") as f:
        f.write(" ".join(fields[:9]) + "\n")  # drop the CSR5 sigma field
    h2 = make_handle(A, torch)
    assert h2.autotune(cache) == backend
    assert _spmv_ok(h2, A, torch)
