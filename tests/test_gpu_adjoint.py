"""Adjoint of y = A x on the GPU: dx = A^T dy and dvals = dy[row]*x[col]
against the FP64 oracle, the autograd binding against a dense FP64 gradient,
and FP64 central finite differences on sampled coordinates.

Tolerance (FP32 vs FP64): |g32 - g64| <= 1e-5 * max(|g64|, sum of |terms|)."""
import numpy as np
import pytest

from conftest import rand_csr
from gpu_util import dev, make_handle
import oracle.oracle as orc

pytestmark = pytest.mark.gpu
RTOL = 1e-5


@pytest.mark.parametrize("csc", [False, True])
@pytest.mark.parametrize("kind", ["zipf", "laplacian"])
def test_backward_dense_and_sparse_dy(torch_cuda, kind, csc):
    """Dense dy goes through the one-pass atomic kernel without a CSC and
    through the CSC gather + CSR dvals pass with one."""
    torch = torch_cuda
    from spmx import gen
    A = rand_csr(5000, 4000, lens=np.minimum(np.random.default_rng(1).zipf(1.6, 5000), 3000),
                 seed=2) if kind == "zipf" else gen.laplacian(64, 0.01, seed=4)
    h = make_handle(A, torch, csc=csc)
    rng = np.random.default_rng(7)
    x = rng.normal(size=A.n).astype(np.float32)
    dy = rng.normal(size=A.m).astype(np.float32)
    for sparse in (False, True):
        if sparse:
            mask = rng.random(A.m) < 0.01
            dy = np.where(mask, dy, 0).astype(np.float32)
        dx = torch.empty(A.n, device="cuda")
        dv = torch.empty(A.nnz, device="cuda")
        if sparse:
            key = np.nonzero(dy)[0].astype(np.int32)
            h.spmv_backward_sparse(dev(x, torch), dev(key, torch), dev(dy[key], torch), len(key), dx, dv)
        else:
            h.spmv_backward(dev(x, torch), dev(dy, torch), dx, dv)
        h.check_device_error()
        edx, mdx = orc.spmv_t_f64(A.n, A.rowptr, A.col, A.val, dy)
        ok, _ = orc.within_tol(dx.cpu().numpy(), edx, mdx, RTOL)
        assert ok, (kind, sparse, orc.max_scaled_err(dx.cpu().numpy(), edx, mdx))
        edv = orc.dvals_f64(A.rowptr, A.col, dy, x)
        ok, _ = orc.within_tol(dv.cpu().numpy(), edv, np.abs(edv), RTOL)
        assert ok, (kind, sparse)


@pytest.mark.parametrize("g,masked", [(128, False), (128, True), (2048, False), (2048, True)])
def test_autograd_laplacian_fd_and_dense(torch_cuda, g, masked):
    """2-D 5-point Laplacian (g x g grid, off-diagonals -1 + N(0, 0.01^2)),
    loss = 0.5 ||A x - t||^2, optionally with the residual masked to 1 % of the
    rows.  Gradients vs a dense FP64 gradient and FP64 central differences
    (h = 1e-6) on 1,000 sampled coordinates of x and of vals."""
    torch = torch_cuda
    from spmx import gen
    from spmx.autograd import SparseMatrix
    A = gen.laplacian(g, 0.01, seed=4)
    rng = np.random.default_rng(11)
    x = rng.normal(size=A.n).astype(np.float32)
    t = rng.normal(size=A.m).astype(np.float32)
    mask = (rng.random(A.m) < 0.01) if masked else np.ones(A.m, bool)
    op = SparseMatrix(A.m, A.n, dev(A.rowptr, torch), dev(A.col, torch))
    vals_t = dev(A.val, torch).requires_grad_(True)
    x_t = dev(x, torch).requires_grad_(True)
    m_t = dev(mask.astype(np.float32), torch)
    y = op(vals_t, x_t)
    loss = 0.5 * (((y - dev(t, torch)) * m_t) ** 2).sum()
    gv, gx = torch.autograd.grad(loss, [vals_t, x_t])
    gv, gx = gv.cpu().numpy(), gx.cpu().numpy()
    # dense FP64 gradient of the masked loss
    yy, magy = orc.spmv_f64(A.rowptr, A.col, A.val, x)
    r = (yy - t) * mask
    rows = np.repeat(np.arange(A.m), np.diff(A.rowptr))
    a64 = A.val.astype(np.float64)
    ex = np.zeros(A.n)
    np.add.at(ex, A.col, a64 * r[rows])
    ev = r[rows] * x.astype(np.float64)[A.col]
    # error budget: the FP32 forward gives r with |r32 - r64| <= rb (the
    # forward's own 1e-5 tolerance plus one rounding of the subtraction),
    # which the backward carries through its products and sums
    rb = (1e-5 * magy + 1e-6 * np.abs(r)) * mask
    tol_v = np.abs(x.astype(np.float64))[A.col] * rb[rows] + 1e-5 * np.abs(ev)
    tol_x = np.zeros(A.n)
    np.add.at(tol_x, A.col, np.abs(a64) * rb[rows] + 1e-5 * np.abs(a64 * r[rows]))
    assert np.all(np.abs(gv - ev) <= tol_v + 1e-30)
    assert np.all(np.abs(gx - ex) <= tol_x + 1e-30)
    # central differences in FP64, evaluated incrementally (a coordinate of x
    # touches one column, a value touches one row)
    h = 1e-6
    cscp, cscr, cscv = A.to_csc()

    def loss_rows(rows_idx, yrows):
        rr = (yrows - t[rows_idx]) * mask[rows_idx]
        return 0.5 * float(rr @ rr)

    for j in rng.choice(A.n, 1000, replace=False):
        rs = cscr[cscp[j]:cscp[j + 1]]
        a = cscv[cscp[j]:cscp[j + 1]].astype(np.float64)
        base = yy[rs]
        fd = (loss_rows(rs, base + a * h) - loss_rows(rs, base - a * h)) / (2 * h)
        assert abs(fd - gx[j]) <= 2 * tol_x[j] + 1e-6, (j, fd, gx[j])
    for k in rng.choice(A.nnz, 1000, replace=False):
        r0 = rows[k]
        d = x[A.col[k]] * h
        fd = (loss_rows(np.array([r0]), np.array([yy[r0] + d])) -
              loss_rows(np.array([r0]), np.array([yy[r0] - d]))) / (2 * h)
        assert abs(fd - gv[k]) <= 2 * tol_v[k] + 1e-6, (k, fd, gv[k])


def test_backward_with_csc_is_deterministic(torch_cuda):
    """With a CSC the dense-dy backward has no atomics: repeated calls are
    bit-identical, and an empty column gives dx exactly 0."""
    torch = torch_cuda
    A = rand_csr(3000, 2500, lens=np.minimum(np.random.default_rng(3).zipf(1.5, 3000), 2000), seed=4)
    A.col[A.col == 7] = 8  # column 7 empty (duplicates are allowed)
    h = make_handle(A, torch, csc=True)
    rng = np.random.default_rng(9)
    x = dev(rng.normal(size=A.n).astype(np.float32), torch)
    dy = dev(rng.normal(size=A.m).astype(np.float32), torch)
    outs = []
    for _ in range(2):
        dx = torch.full((A.n,), 5.0, device="cuda")
        dv = torch.full((A.nnz,), 5.0, device="cuda")
        h.spmv_backward(x, dy, dx, dv)
        outs.append((dx.cpu().numpy(), dv.cpu().numpy()))
    h.check_device_error()
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    assert outs[0][0][7] == 0.0
