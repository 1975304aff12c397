"""Round SpMV / bitmap-gated SpMSpV (spmv_type 3) against the FP64 oracle.

Tolerance (FP32 vs FP64, per row): |y32 - y64| <= 1e-5 * max(|y64|,
sum_j |a_ij x_j|).  Cases: the SpMV suite's matrices (long rows spanning many
rounds, empty and trailing empty rows, a single row whose accumulators fill
whole rounds, all rows empty), hub rows with thousands of accumulators, row
blocks capped small enough that
the grid runs in several waves, a tall thin matrix, the 1M-row Zipf matrix;
alpha values; the gated form through the dispatcher; determinism (bitwise
equal results of repeated calls); matrices whose 128 consecutive nonzeros of a
row block span 2^16 columns or more (the build pads every 2^16-column segment
to a chunk boundary); and the preprocessing's refusal of a column out of
range, after which the handle still serves the other back-ends."""
import numpy as np
import pytest

from conftest import rand_csr
from gpu_util import dev, make_handle
import oracle.oracle as orc
from test_gpu_spmv import CASES

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _extra():
    rng = np.random.default_rng(40)
    # hub rows of 20,000 nonzeros: thousands of accumulators each
    lens = rng.integers(0, 12, 30000)
    lens[[5, 17, 29000]] = 20000
    yield "hubs", rand_csr(30000, 40000, lens=lens, seed=41)
    yield "tall-thin", rand_csr(200000, 3, density=0.4, seed=42)
    from spmx import gen
    yield "zipf-64k", gen.zipf_rows(1 << 16, 1.5, 16, 5000, seed=43)
    # power-law rows and columns (hub rows fill whole rounds) and a stencil
    # (neighbouring columns: several slots per row): both need the retry with
    # shorter row blocks
    yield "chung-lu-64k", gen.chung_lu(1 << 16, 2.1, 16.0, seed=46)
    g = gen.rmat(15, 16, seed=47)
    g.val = np.random.default_rng(48).uniform(-1, 1, g.nnz).astype(np.float32)
    yield "rmat-15", g
    yield "laplacian-512", gen.laplacian(512)
    # chunks spanning 2^16 columns or more: 24,000 nonzeros over 16M columns,
    # and an R-MAT graph with 131,072 columns (two segments)
    yield "span-16M", rand_csr(4, 1 << 24, lens=[6000, 6000, 6000, 6000], seed=45)
    g = gen.rmat(17, 16, seed=49)
    g.val = np.random.default_rng(50).uniform(-1, 1, g.nnz).astype(np.float32)
    yield "rmat-17", g


EXTRA = list(_extra())
ALL = CASES + EXTRA


def _check_spmv(torch, h, A, alpha, x):
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, x, alpha=alpha)
    outs = []
    for _ in range(2):
        y = torch.full((A.m,), 3.0, device="cuda")
        h.roundspmv(alpha, y)
        h.check_device_error()
        yh = y.cpu().numpy()
        ok, _ = orc.within_tol(yh, y64, mag, RTOL)
        assert ok, orc.max_scaled_err(yh, y64, mag)
        outs.append(yh)
    assert np.array_equal(outs[0].view(np.uint32), outs[1].view(np.uint32))  # deterministic


@pytest.mark.parametrize("name,A", ALL, ids=[c[0] for c in ALL])
@pytest.mark.parametrize("rb", [0, 64])
@pytest.mark.parametrize("parts", [1, 2, 4])
def test_round_spmv(torch_cuda, name, A, rb, parts):
    torch = torch_cuda
    h = make_handle(A, torch, csc=False, hola=False)
    h.roundPreprocess(rb, parts)
    info = h.round_info()
    assert info["parts"] == parts and info["round"] == 4096
    assert info["grid"] == parts * info["row_blocks"]
    assert info["rounds"] >= (A.nnz + 4095) // 4096
    # every row with a nonzero has an accumulator; the 32 padding slots follow
    assert info["slots"] >= 32 + min(A.m, np.count_nonzero(np.diff(A.rowptr))) // max(1, info["row_blocks"])
    if rb:
        assert info["rmax"] <= 64
    x = np.random.default_rng(17).uniform(-1, 1, A.n).astype(np.float32)
    h.set_x(dev(x, torch))
    _check_spmv(torch, h, A, -1.5 if rb else 1.0, x)
    # bitmap-gated form through the dispatcher
    h.set_spmv_type(3)
    rng = np.random.default_rng(2)
    k = max(1, A.n // 30)
    key = np.sort(rng.choice(A.n, k, replace=False)).astype(np.int32)
    val = rng.uniform(-1, 1, k).astype(np.float32)
    h.set_sparse_x(dev(key, torch), dev(val, torch), k)
    h.sparse2bitarray()
    y = torch.empty(A.m, device="cuda")
    h.spmspv(1.0, y)
    h.check_device_error()
    xd, bits = orc.sparse2dense_bits(A.n, key, val)
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, xd, bits=bits.view(np.int32))
    ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
    assert ok
    # dense x through the dispatcher
    h.set_x(dev(x, torch))
    y = torch.empty(A.m, device="cuda")
    h.spmv(0.5, y)
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, x, alpha=0.5)
    assert orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)[0]
    h.roundPostprocess()


@pytest.mark.parametrize("parts", [1, 2, 4])
def test_round_zipf_full_size(torch_cuda, parts):
    torch = torch_cuda
    from spmx import gen
    A = gen.zipf_1m()
    h = make_handle(A, torch, csc=False, hola=False)
    h.roundPreprocess(0, parts)
    info = h.round_info()
    assert info["row_blocks"] == 148 // parts and info["grid"] == 148
    x = np.random.default_rng(2).uniform(-1, 1, A.n).astype(np.float32)
    h.set_x(dev(x, torch))
    _check_spmv(torch, h, A, 1.0, x)


@pytest.mark.parametrize("parts", [1, 2])
@pytest.mark.parametrize("offset", [0, 1])
def test_round_ragged_rows_and_unaligned_y(torch_cuda, parts, offset):
    """m not a multiple of 4 (the last row block ends off a 4-row group) and,
    with offset 1, a y that is not 16-byte aligned (the one-CTA fold's scalar
    stores)."""
    torch = torch_cuda
    A = rand_csr(10003, 5000, density=0.004, seed=51)
    h = make_handle(A, torch, csc=False, hola=False)
    h.roundPreprocess(0, parts)
    x = np.random.default_rng(52).uniform(-1, 1, A.n).astype(np.float32)
    h.set_x(dev(x, torch))
    ybuf = torch.full((A.m + 1,), 7.0, device="cuda")
    y = ybuf[offset:offset + A.m]
    h.roundspmv(-0.5, y)
    h.check_device_error()
    y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, x, alpha=-0.5)
    ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
    assert ok
    edge = ybuf[A.m] if offset == 0 else ybuf[0]
    assert float(edge) == 7.0  # nothing written outside y


def test_round_refusals_keep_handle_usable(torch_cuda):
    torch = torch_cuda
    from spmx import SpmxError
    # a column outside [0, n)
    A = rand_csr(500, 400, density=0.02, seed=44)
    bad = A.col.copy()
    bad[len(bad) // 2] = A.n
    from spmx import SpmspvHandle
    h = SpmspvHandle(A.m, A.n, A.nnz)
    h.InputCSR(A.nnz, dev(A.rowptr, torch), dev(bad, torch), dev(A.val, torch))
    with pytest.raises(SpmxError):
        h.roundPreprocess()
    with pytest.raises(SpmxError):
        h.round_info()  # nothing kept
    # the other back-ends still serve the handle
    x = np.random.default_rng(3).uniform(-1, 1, A.n).astype(np.float32)
    h.set_x(dev(x, torch))
    h.holaPreprocess()
    y = torch.empty(A.m, device="cuda")
    h.holaspmv(1.0, y)
    with pytest.raises(SpmxError):
        h.check_device_error()  # Hola skips the bad column and reports it
    ok = bad < A.n
    y64, mag = orc.spmv_f64(A.rowptr, np.where(ok, bad, 0), np.where(ok, A.val, 0), x)
    assert orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)[0]


def test_two_handles_with_different_shared_memory(torch_cuda):
    """A kernel's dynamic shared-memory limit belongs to the function, not to
    a handle: a handle whose format needs more shared memory than the format
    built last (by another handle) still launches, for the round and the tiled
    back-ends, and both results match the FP64 oracle."""
    torch = torch_cuda
    big = dict(EXTRA)["hubs"]
    small = rand_csr(2000, 1500, density=0.004, seed=61)
    hb, hs = make_handle(big, torch, hola=False), make_handle(small, torch, hola=False)
    hb.roundPreprocess(0, 1)
    hs.roundPreprocess(0, 1)
    assert hb.round_info()["smem"] > hs.round_info()["smem"]
    hb.tiledPreprocess()
    hs.tiledPreprocess(rb_rows=256)
    assert hb.tiled_info()["smem"] > hs.tiled_info()["smem"]
    for h, A in ((hb, big), (hs, small), (hb, big)):
        x = np.random.default_rng(A.m).uniform(-1, 1, A.n).astype(np.float32)
        h.set_x(dev(x, torch))
        y64, mag = orc.spmv_f64(A.rowptr, A.col, A.val, x)
        for run in (h.roundspmv, h.tiledspmv):
            y = torch.full((A.m,), 3.0, device="cuda")
            run(1.0, y)
            h.check_device_error()
            ok, _ = orc.within_tol(y.cpu().numpy(), y64, mag, RTOL)
            assert ok, run.__name__
