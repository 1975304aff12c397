"""Hybrid CSR/CSC split SpMV against the oracle.

The device split (spmx_hybrid_preprocess) must equal the oracle's COO2Hybrid
restatement bit for bit (CSR part in CSR order, CSC part by column then row),
and y = alpha * (A_csr x + A_csc x) must satisfy the FP32 bound against the
FP64 product of the whole matrix."""
import numpy as np
import pytest

from conftest import rand_csr
from gpu_util import dev, make_handle
import oracle.oracle as orc

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _mats():
    from spmx import gen
    rng = np.random.default_rng(21)
    return {
        "uniform": rand_csr(4000, 3000, density=0.004, seed=22),
        "skewed": rand_csr(5000, 5000, lens=np.minimum(rng.zipf(1.5, 5000), 4000), seed=23),
        "empty-rows": rand_csr(3000, 6000, lens=np.where(rng.random(3000) < 0.4, 0,
                                                         rng.integers(1, 40, 3000)), seed=24),
        "laplacian": gen.laplacian(96, 0.01, seed=4),
        "chung-lu": gen.chung_lu(20000, 2.1, 16.0, seed=25),
    }


@pytest.mark.parametrize("name", list(_mats()))
@pytest.mark.parametrize("alpha", [1.0, -0.75])
def test_hybrid_split_and_spmv(torch_cuda, name, alpha):
    torch = torch_cuda
    A = _mats()[name]
    h = make_handle(A, torch, csc=False, hola=False)
    h.hybridPreprocess()
    k, flags = orc.coo2hybrid(A.n, A.rowptr, A.col)
    a, b = h.hybrid_info()
    assert (a, b) == (k, A.nnz - k)
    (rp, cl, vl), (cp, rw, cv) = h.hybrid_parts()
    row = np.repeat(np.arange(A.m, dtype=np.int32), np.diff(A.rowptr))
    erp = np.zeros(A.m + 1, np.int32)
    np.cumsum(np.bincount(row[flags], minlength=A.m), out=erp[1:])
    assert np.array_equal(rp.cpu().numpy(), erp)
    assert np.array_equal(cl.cpu().numpy(), A.col[flags])
    assert np.array_equal(vl.cpu().numpy().view(np.uint32), A.val[flags].view(np.uint32))
    o = np.lexsort((row[~flags], A.col[~flags]))
    ecp = np.zeros(A.n + 1, np.int32)
    np.cumsum(np.bincount(A.col[~flags], minlength=A.n), out=ecp[1:])
    assert np.array_equal(cp.cpu().numpy(), ecp)
    assert np.array_equal(rw.cpu().numpy(), row[~flags][o])
    assert np.array_equal(cv.cpu().numpy().view(np.uint32), A.val[~flags][o].view(np.uint32))
    x = np.random.default_rng(26).uniform(-1, 1, A.n).astype(np.float32)
    x[::7] = 0.0
    h.set_x(dev(x, torch))
    y = torch.full((A.m,), 9.0, device="cuda")
    h.hybridspmv(alpha, y)
    h.check_device_error()
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, x, alpha=alpha)
    ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
    assert ok, orc.max_scaled_err(y.cpu().numpy(), y64, mag)


def test_hybrid_needs_preprocess(torch_cuda):
    torch = torch_cuda
    from spmx import SpmxError
    A = rand_csr(300, 200, density=0.05, seed=27)
    h = make_handle(A, torch, csc=False, hola=False)
    h.set_x(dev(np.ones(A.n, np.float32), torch))
    with pytest.raises(SpmxError):
        h.hybridspmv(1.0, torch.empty(A.m, device="cuda"))
