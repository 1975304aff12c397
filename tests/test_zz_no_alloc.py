"""The allocation-free CSC SpMSpV entry point (spmx_spmspv_csc_noalloc).

It exists for callers that cannot let the library allocate device memory:
a host framework that manages the device heap with its own allocator, or a
latency-critical loop in which cudaMalloc / cudaFree could synchronise the
device.  Its scratch is one fixed device array shared by all calls, so this
test calls it through the C ABI twice in a row (the second call must not see
the first call's leftovers) and compares each result with the handle-based
merge-path CSC SpMSpV, within the tolerance of the other parity tests.  This
file is collected last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from conftest import rand_csr
from gpu_util import dev, make_handle, set_sparse
import oracle.oracle as orc

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _noalloc(abi, torch, A, colptr_d, row_d, val_d, key_d, xv_d, k, alpha, y):
    stream = torch.cuda.current_stream().cuda_stream
    rc = abi.lib.spmx_spmspv_csc_noalloc(A.m, A.n, A.nnz, row_d.data_ptr(), colptr_d.data_ptr(),
                                         val_d.data_ptr(), k, key_d.data_ptr(), xv_d.data_ptr(),
                                         ctypes.c_float(alpha), y.data_ptr(), stream)
    assert rc == 0, abi.last_error()
    torch.cuda.synchronize()


def test_noalloc_matches_handle_entry_point(torch_cuda):
    torch = torch_cuda
    from spmx import abi
    A = rand_csr(6000, 5000, density=0.004, seed=21)
    colptr, row, cval = A.to_csc()
    colptr_d, row_d, val_d = dev(colptr, torch), dev(row, torch), dev(cval, torch)
    h = make_handle(A, torch, hola=False)
    rng = np.random.default_rng(4)
    for call, (k, alpha) in enumerate([(2500, 1.0), (37, -0.5)]):  # two calls in a row
        key = np.sort(rng.choice(A.n, k, replace=False)).astype(np.int32)
        xv = rng.uniform(-1, 1, k).astype(np.float32)
        key_d, xv_d = dev(key, torch), dev(xv, torch)
        y_na = torch.full((A.m,), 9.0, device="cuda")
        _noalloc(abi, torch, A, colptr_d, row_d, val_d, key_d, xv_d, k, alpha, y_na)
        set_sparse(h, key, xv, torch)
        y_ref = torch.empty(A.m, device="cuda")
        h.spmspv_csc(1, 0, alpha, y_ref)
        h.check_device_error()
        _, mag, _ = orc.spmspv_csc_f64(A.m, colptr, row, cval, key, xv, alpha=alpha)
        ok, _ = orc.within_tol(y_na.cpu().numpy(), y_ref.cpu().numpy().astype(np.float64), mag, RTOL)
        assert ok, f"call {call}"


def test_noalloc_rejects_oversized_x(torch_cuda):
    torch = torch_cuda
    from spmx import abi
    n = (1 << 20) + 10
    y = torch.empty(4, device="cuda")
    one = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = abi.lib.spmx_spmspv_csc_noalloc(4, n, 1, one.data_ptr(), one.data_ptr(),
                                         y.data_ptr(), (1 << 20) + 1, one.data_ptr(),
                                         y.data_ptr(), ctypes.c_float(1.0), y.data_ptr(), None)
    assert rc == abi.ERR_INVALID_VALUE
    assert "exceeds the fixed scratch limit" in abi.last_error()
