"""The allocation-free CSC SpMSpV entry point (spmx_spmspv_csc_noalloc).

It exists for callers that cannot let the library allocate device memory:
a host framework that manages the device heap with its own allocator, or a
latency-critical loop in which cudaMalloc / cudaFree could synchronise the
device.  Its scratch is one fixed device array shared by all calls, so this
test calls it through the C ABI twice in a row (the second call must not see
the first call's leftovers) and checks each result against the FP64 oracle
and against the handle-based merge-path CSC SpMSpV, within the tolerance of
the other parity tests.  It also checks the documented limits and the error
word read back by spmx_spmspv_csc_noalloc_check.  This file is collected last
so that a run stopping at the first failure has already run every other test;
it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from conftest import rand_csr
from gpu_util import dev, make_handle, set_sparse
import oracle.oracle as orc

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _call(abi, torch, m, n, nnz, row_ptr, colptr_ptr, val_ptr, k, key_ptr, xv_ptr, alpha, y_ptr):
    stream = torch.cuda.current_stream().cuda_stream
    return abi.lib.spmx_spmspv_csc_noalloc(m, n, nnz, row_ptr, colptr_ptr, val_ptr, k, key_ptr,
                                           xv_ptr, ctypes.c_float(alpha), y_ptr, stream)


def _check(abi, torch):
    return abi.lib.spmx_spmspv_csc_noalloc_check(torch.cuda.current_stream().cuda_stream)


def test_noalloc_matches_oracle_and_handle(torch_cuda):
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
        rc = _call(abi, torch, A.m, A.n, A.nnz, row_d.data_ptr(), colptr_d.data_ptr(),
                   val_d.data_ptr(), k, key_d.data_ptr(), xv_d.data_ptr(), alpha, y_na.data_ptr())
        assert rc == 0, abi.last_error()
        assert _check(abi, torch) == 0, abi.last_error()
        y64, mag, _ = orc.spmspv_csc_f64(A.m, colptr, row, cval, key, xv, alpha=alpha)
        got = y_na.cpu().numpy()
        assert orc.within_tol(got, y64, mag, RTOL)[0], f"call {call} vs the FP64 oracle"
        set_sparse(h, key, xv, torch)
        y_ref = torch.empty(A.m, device="cuda")
        h.spmspv_csc(1, 0, alpha, y_ref)
        h.check_device_error()
        assert orc.within_tol(got, y_ref.cpu().numpy().astype(np.float64), mag, RTOL)[0], \
            f"call {call} vs the handle entry point"


def test_noalloc_empty_x_zeroes_y(torch_cuda):
    torch = torch_cuda
    from spmx import abi
    A = rand_csr(300, 200, density=0.05, seed=3)
    colptr, row, cval = A.to_csc()
    colptr_d, row_d, val_d = dev(colptr, torch), dev(row, torch), dev(cval, torch)
    y = torch.full((A.m,), 5.0, device="cuda")
    rc = _call(abi, torch, A.m, A.n, A.nnz, row_d.data_ptr(), colptr_d.data_ptr(), val_d.data_ptr(),
               0, 0, 0, 1.0, y.data_ptr())
    assert rc == 0, abi.last_error()
    torch.cuda.synchronize()
    assert bool((y == 0).all())


def test_noalloc_reports_out_of_range_key(torch_cuda):
    """A key outside [0, n) is skipped by the kernels and reported by the
    check call; the next good call reports success again."""
    torch = torch_cuda
    from spmx import abi
    A = rand_csr(400, 300, density=0.05, seed=5)
    colptr, row, cval = A.to_csc()
    colptr_d, row_d, val_d = dev(colptr, torch), dev(row, torch), dev(cval, torch)
    key = np.array([3, 17, A.n + 5], np.int32)
    xv = np.array([1.0, -2.0, 0.5], np.float32)
    key_d, xv_d = dev(key, torch), dev(xv, torch)
    y = torch.empty(A.m, device="cuda")
    rc = _call(abi, torch, A.m, A.n, A.nnz, row_d.data_ptr(), colptr_d.data_ptr(), val_d.data_ptr(),
               3, key_d.data_ptr(), xv_d.data_ptr(), 1.0, y.data_ptr())
    assert rc == 0, abi.last_error()
    assert _check(abi, torch) == abi.ERR_OOB
    good = dev(key[:2], torch)
    rc = _call(abi, torch, A.m, A.n, A.nnz, row_d.data_ptr(), colptr_d.data_ptr(), val_d.data_ptr(),
               2, good.data_ptr(), xv_d.data_ptr(), 1.0, y.data_ptr())
    assert rc == 0 and _check(abi, torch) == 0, abi.last_error()
    y64, mag, _ = orc.spmspv_csc_f64(A.m, colptr, row, cval, key[:2], xv[:2])
    assert orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)[0]


def test_noalloc_rejects_oversized_and_null(torch_cuda):
    torch = torch_cuda
    from spmx import abi
    y = torch.empty(4, device="cuda")
    one = torch.zeros(1, dtype=torch.int32, device="cuda")
    n = (1 << 20) + 10
    rc = _call(abi, torch, 4, n, 1, one.data_ptr(), one.data_ptr(), y.data_ptr(), (1 << 20) + 1,
               one.data_ptr(), y.data_ptr(), 1.0, y.data_ptr())
    assert rc == abi.ERR_INVALID_VALUE
    assert "exceeds the fixed scratch limit" in abi.last_error()
    # nnz + x_nnz above 2^27
    rc = _call(abi, torch, 4, 1 << 20, (1 << 27) - 5, one.data_ptr(), one.data_ptr(), y.data_ptr(),
               10, one.data_ptr(), y.data_ptr(), 1.0, y.data_ptr())
    assert rc == abi.ERR_INVALID_VALUE and "nnz + x_nnz" in abi.last_error()
    # NULL pointers
    rc = _call(abi, torch, 4, 4, 1, one.data_ptr(), 0, y.data_ptr(), 1, one.data_ptr(),
               y.data_ptr(), 1.0, y.data_ptr())
    assert rc == abi.ERR_INVALID_VALUE and "NULL" in abi.last_error()
    rc = _call(abi, torch, 4, 4, 1, one.data_ptr(), one.data_ptr(), y.data_ptr(), 1, one.data_ptr(),
               y.data_ptr(), 1.0, 0)
    assert rc == abi.ERR_INVALID_VALUE and "NULL" in abi.last_error()
