"""SpMV and bitmap-gated CSR SpMSpV on the GPU against the FP64 oracle.

Tolerance (FP32 vs FP64, per row): |y32 - y64| <= 1e-5 * max(|y64|,
sum_j |a_ij x_j|).  Untouched rows must be exactly 0."""
import numpy as np
import pytest

from conftest import rand_csr
from gpu_util import dev, make_handle
import oracle.oracle as orc

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _cases():
    rng = np.random.default_rng(0)
    yield "uniform", rand_csr(3000, 2500, density=0.004, seed=1)
    # long rows spanning many 2048-nnz chunks, empty rows, trailing empty rows
    lens = np.zeros(5000, np.int64)
    lens[7] = 9000
    lens[8] = 1
    lens[100:4000] = rng.integers(0, 40, 3900)
    lens[4001] = 4096
    yield "long-rows", rand_csr(5000, 12000, lens=lens, seed=2)
    yield "one-row", rand_csr(1, 50000, lens=[30000], seed=3)
    yield "all-empty", rand_csr(100, 100, lens=np.zeros(100, int), seed=4)
    lens = np.zeros(3000, np.int64)
    lens[0] = 2048
    lens[1] = 2048
    lens[2] = 4095
    yield "chunk-aligned", rand_csr(3000, 5000, lens=lens, seed=5)


CASES = list(_cases())


@pytest.mark.parametrize("name,A", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("kind", ["naive", "hola"])
@pytest.mark.parametrize("alpha", [1.0, -0.75])
def test_spmv(torch_cuda, name, A, kind, alpha):
    torch = torch_cuda
    h = make_handle(A, torch, csc=False)
    x = np.random.default_rng(11).uniform(-1, 1, A.n).astype(np.float32)
    xd = dev(x, torch)
    h.set_x(xd)
    y = torch.full((A.m,), 7.0, device="cuda")
    getattr(h, kind + "spmv")(alpha, y)
    h.check_device_error()
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, x, alpha=alpha)
    ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
    assert ok, orc.max_scaled_err(y.cpu().numpy(), y64, mag)


@pytest.mark.parametrize("name,A", CASES[:3], ids=[c[0] for c in CASES[:3]])
@pytest.mark.parametrize("kind", ["naive", "hola"])
def test_spmspv_gated(torch_cuda, name, A, kind):
    torch = torch_cuda
    h = make_handle(A, torch, csc=False)
    rng = np.random.default_rng(5)
    k = max(1, A.n // 50)
    key = np.sort(rng.choice(A.n, k, replace=False)).astype(np.int32)
    val = rng.uniform(-1, 1, k).astype(np.float32)
    kd, vd = dev(key, torch), dev(val, torch)
    h.set_sparse_x(kd, vd, k)
    h.sparse2bitarray()
    y = torch.zeros(A.m, device="cuda")
    getattr(h, kind + "spmspv")(1.0, y)
    h.check_device_error()
    xd, bits = orc.sparse2dense_bits(A.n, key, val)
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, xd, bits=bits.view(np.int32))
    ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
    assert ok


def test_hola_repeated_calls_deterministic(torch_cuda):
    """The split-row counters reset themselves: repeated calls agree bitwise."""
    torch = torch_cuda
    A = CASES[1][1]
    h = make_handle(A, torch, csc=False)
    x = dev(np.random.default_rng(3).uniform(-1, 1, A.n).astype(np.float32), torch)
    h.set_x(x)
    ys = []
    for _ in range(4):
        y = torch.empty(A.m, device="cuda")
        h.holaspmv(1.0, y)
        ys.append(y.cpu().numpy())
    for y in ys[1:]:
        assert np.array_equal(y, ys[0])


def test_spmv_full_size_zipf(torch_cuda):
    """The 1M-row Zipf matrix at full size against the FP64 oracle."""
    torch = torch_cuda
    from spmx import gen
    A = gen.zipf_1m()
    h = make_handle(A, torch, csc=False)
    x = np.random.default_rng(2).uniform(-1, 1, A.n).astype(np.float32)
    h.set_x(dev(x, torch))
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, x)
    for kind in ("naive", "hola"):
        y = torch.empty(A.m, device="cuda")
        getattr(h, kind + "spmv")(1.0, y)
        h.check_device_error()
        ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
        assert ok, kind


@pytest.mark.parametrize("name,A", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("sigma", [-1, 4, 12, 32])
def test_csr5_spmv(torch_cuda, name, A, sigma):
    torch = torch_cuda
    h = make_handle(A, torch, csc=False, hola=False)
    h.setSigma(sigma)
    h.CSR5Preprocess()
    x = np.random.default_rng(13).uniform(-1, 1, A.n).astype(np.float32)
    h.set_x(dev(x, torch))
    for rep in range(2):  # the second call checks the self-resetting counters
        y = torch.full((A.m,), 7.0, device="cuda")
        h.csr5spmv(1.25, y)
        h.check_device_error()
        y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, x, alpha=1.25)
        ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
        assert ok, orc.max_scaled_err(y.cpu().numpy(), y64, mag)


@pytest.mark.parametrize("name,A", CASES[:3], ids=[c[0] for c in CASES[:3]])
def test_csr5_spmspv_gated(torch_cuda, name, A):
    torch = torch_cuda
    h = make_handle(A, torch, csc=False, hola=False)
    h.CSR5Preprocess()
    rng = np.random.default_rng(8)
    k = max(1, A.n // 40)
    key = np.sort(rng.choice(A.n, k, replace=False)).astype(np.int32)
    val = rng.uniform(-1, 1, k).astype(np.float32)
    kd, vd = dev(key, torch), dev(val, torch)
    h.set_sparse_x(kd, vd, k)
    h.sparse2bitarray()
    y = torch.zeros(A.m, device="cuda")
    h.csr5spmspv(1.0, y)
    h.check_device_error()
    xd, bits = orc.sparse2dense_bits(A.n, key, val)
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, xd, bits=bits.view(np.int32))
    ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
    assert ok


def test_csr5_zipf_full_size(torch_cuda):
    torch = torch_cuda
    from spmx import gen
    A = gen.zipf_1m()
    h = make_handle(A, torch, csc=False, hola=False)
    h.CSR5Preprocess()
    x = np.random.default_rng(2).uniform(-1, 1, A.n).astype(np.float32)
    h.set_x(dev(x, torch))
    y = torch.empty(A.m, device="cuda")
    h.csr5spmv(1.0, y)
    h.check_device_error()
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, x)
    ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
    assert ok


@pytest.mark.parametrize("name,A", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("rb,win,chunk,warps", [(256, 512, 300, 8), (1024, 256, 64, 16), (0, 0, 0, 0),
                                               (0, 8192, 4096, 4)])
def test_tiled_spmv(torch_cuda, name, A, rb, win, chunk, warps):
    torch = torch_cuda
    h = make_handle(A, torch, csc=False, hola=False)
    h.tiledPreprocess(rb, win, chunk, warps)
    x = np.random.default_rng(17).uniform(-1, 1, A.n).astype(np.float32)
    h.set_x(dev(x, torch))
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, x, alpha=-1.5)
    for rep in range(2):
        y = torch.full((A.m,), 3.0, device="cuda")
        h.tiledspmv(-1.5, y)
        h.check_device_error()
        ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
        assert ok, orc.max_scaled_err(y.cpu().numpy(), y64, mag)
    # bitmap-gated form through the dispatcher
    h.set_spmv_type(2)
    rng = np.random.default_rng(2)
    k = max(1, A.n // 30)
    key = np.sort(rng.choice(A.n, k, replace=False)).astype(np.int32)
    val = rng.uniform(-1, 1, k).astype(np.float32)
    kd, vd = dev(key, torch), dev(val, torch)
    h.set_sparse_x(kd, vd, k)
    h.sparse2bitarray()
    y = torch.empty(A.m, device="cuda")
    h.spmspv(1.0, y)
    xd, bits = orc.sparse2dense_bits(A.n, key, val)
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, xd, bits=bits.view(np.int32))
    ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
    assert ok


def test_tiled_zipf_full_size(torch_cuda):
    torch = torch_cuda
    from spmx import gen
    A = gen.zipf_1m()
    h = make_handle(A, torch, csc=False, hola=False)
    h.tiledPreprocess()
    x = np.random.default_rng(2).uniform(-1, 1, A.n).astype(np.float32)
    h.set_x(dev(x, torch))
    y = torch.empty(A.m, device="cuda")
    h.tiledspmv(1.0, y)
    h.check_device_error()
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, x)
    ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
    assert ok
