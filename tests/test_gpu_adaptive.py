"""The eight kernels run by id, the selector and the adaptive iteration on the
1M-row Zipf matrix and on a small matrix, against the FP64 oracle."""
import numpy as np
import pytest

from conftest import rand_csr
from gpu_util import dev, make_handle, set_sparse
import oracle.oracle as orc

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _check_all(h, A, key, val, torch):
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, orc.sparse2dense_bits(A.n, key, val)[0])
    for kid in range(8):
        y = torch.full((A.m,), 1.0, device="cuda")
        h.run_kernel(kid, 1.0, y)
        h.check_device_error()
        ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
        assert ok, kid
    y = torch.empty(A.m, device="cuda")
    kid = h.run_adaptive(1.0, y)
    assert 0 <= kid < 8
    ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
    assert ok


def test_all_kernels_small(torch_cuda):
    torch = torch_cuda
    A = rand_csr(3000, 3000, density=0.003, seed=12)
    h = make_handle(A, torch)
    rng = np.random.default_rng(1)
    for k in (1, 30, 3000):
        key = np.sort(rng.choice(A.n, k, replace=False)).astype(np.int32)
        val = rng.uniform(-1, 1, k).astype(np.float32)
        set_sparse(h, key, val, torch)
        _check_all(h, A, key, val, torch)


def test_all_kernels_zipf_1m_density_sweep(torch_cuda):
    torch = torch_cuda
    from spmx import gen
    A = gen.zipf_1m()
    h = make_handle(A, torch)
    h.allocPreBuffer()
    for d in gen.C2_DENSITIES:
        k = gen.density_nnz(A.n, d)
        key, val = gen.sparse_vector(A.n, k, seed=100 + k)
        set_sparse(h, key, val, torch)
        _check_all(h, A, key, val, torch)


def test_selector_host_only_matches_handle(torch_cuda):
    torch = torch_cuda
    import ctypes
    from spmx import abi
    A = rand_csr(2000, 2000, density=0.01, seed=3)
    h = make_handle(A, torch)
    key, val = np.arange(0, 2000, 7, dtype=np.int32), np.ones(286, np.float32)
    set_sparse(h, key, val, torch)
    k1 = h.select()
    f = h.features()
    est = dict(f)
    est["bin_len"] = 286 * A.nnz / A.n
    arr = (ctypes.c_double * 23)(*[est[n] for n in abi.FEATURE_NAMES])
    # the handle's selector uses the estimated bin_len and no column extremes
    arr[12] = 0
    arr[13] = 0
    for i, name in enumerate(abi.FEATURE_NAMES):
        if name in ("bin_len/nnz",):
            arr[i] = est["bin_len"] / A.nnz
    k2 = ctypes.c_int()
    assert abi.lib.spmx_select_features(arr, ctypes.byref(k2)) == 0
    assert 0 <= k1 < 8 and 0 <= k2.value < 8


def test_chained_adaptive_calls_share_y(torch_cuda):
    """Adaptive calls back to back on one stream into the SAME y, each followed
    by a compaction of y into its own pinned host buffers, one synchronisation
    at the end: every call's first kernel starts before the previous grid ends
    (programmatic dependent launch), so it must wait both for the previous
    call's writes to y and for the compaction still reading y.  Densities from
    1e-5 to 1.0 (the dense x takes the sparse-to-dense conversion and the
    autotuned SpMV back-end), twice, every result against the FP64 oracle."""
    torch = torch_cuda
    from spmx import gen
    A = gen.zipf_rows(1 << 18, 1.5, 16, 3000, seed=9)
    h = make_handle(A, torch)
    h.allocPreBuffer()
    h.autotune()
    h.set_x(torch.zeros(A.n, device="cuda"))
    h.set_bitvector(torch.zeros((A.n + 31) // 32, dtype=torch.int32, device="cuda"), (A.n + 31) // 32)
    dens = [1e-5, 1e-2, 1.0, 1e-3, 0.1, 1e-4, 1.0, 0.5]
    xs = []
    for i, d in enumerate(dens):
        k = gen.density_nnz(A.n, d)
        key, val = gen.sparse_vector(A.n, k, seed=300 + i)
        xs.append((key, val, dev(key.astype(np.int32), torch), dev(val.astype(np.float32), torch)))
    y = torch.empty(A.m, device="cuda")
    hk = [torch.empty(A.m, dtype=torch.int32).pin_memory() for _ in dens]
    hv = [torch.empty(A.m).pin_memory() for _ in dens]
    hc = torch.full((len(dens),), -1, dtype=torch.int32).pin_memory()
    for rep in range(2):
        for i, (key, val, kd, vd) in enumerate(xs):
            h.set_sparse_x(kd, vd, len(key))
            h.run_adaptive(1.0, y)
            h.dense2sparse_to_host(A.m, y, hk[i], hv[i], hc[i:i + 1])
        torch.cuda.synchronize()
        h.check_device_error()
        for i, (key, val, _, _) in enumerate(xs):
            y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, orc.sparse2dense_bits(A.n, key, val)[0])
            got = np.zeros(A.m)
            c = int(hc[i])
            got[hk[i][:c].numpy()] = hv[i][:c].numpy()
            ok, _ = orc.within_tol(got, y64, mag, RTOL)
            assert ok, (rep, dens[i])
