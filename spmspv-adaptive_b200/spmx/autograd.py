"""Differentiable FP32 SpMV: y = A(vals) x as a torch.autograd.Function.

The sparsity pattern (CSR row pointer and columns) is fixed per operator; the
values `vals` (one per nonzero, CSR order) and the dense `x` are
differentiable.  Forward is the Hola SpMV kernel; backward is the fused
adjoint pass of the library (spmx_spmv_backward): dx = A^T dy and
dvals[k] = dy[row_k] * x[col_k] from one sweep over the matrix.  When dy is
mostly zeros (a masked loss) the sparse-dy adjoint runs instead: only the rows
in dy's support are touched (the CSC SpMSpV of A^T).

No reference counterpart: the reference has no differentiation.
"""
import torch

from .handle import SpmspvHandle


class SparseMatrix:
    """A CSR pattern on the GPU with a handle bound to it.

    rowptr: int32 [m+1], col: int32 [nnz] (CUDA tensors).  `sparse_grad`:
    "auto" compacts dy on the device and takes the sparse adjoint when fewer
    than `sparse_threshold` * m rows are nonzero (this reads one count back to
    the host); "dense" / "sparse" force a path.
    """

    def __init__(self, m, n, rowptr, col, sparse_grad="auto", sparse_threshold=0.05):
        if rowptr.dtype != torch.int32 or col.dtype != torch.int32:
            raise TypeError("rowptr and col must be int32")
        self.m, self.n, self.nnz = int(m), int(n), int(col.numel())
        self.rowptr, self.col = rowptr.contiguous(), col.contiguous()
        self.h = SpmspvHandle(self.m, self.n, self.nnz)
        self._vals = None
        self.sparse_grad = sparse_grad
        self.sparse_threshold = sparse_threshold
        self._bind(torch.zeros(self.nnz, dtype=torch.float32, device=col.device))
        self.h.holaPreprocess()

    def _bind(self, vals):
        if self._vals is not vals:
            self.h.InputCSR(self.nnz, self.rowptr, self.col, vals)
            self._vals = vals

    def __call__(self, vals, x):
        return SpMVFunction.apply(vals, x, self)


class SpMVFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vals, x, op):
        vals = vals.contiguous()
        x = x.contiguous()
        if vals.dtype != torch.float32 or x.dtype != torch.float32:
            raise TypeError("vals and x must be float32")
        op._bind(vals)
        op.h.set_x(x)
        y = torch.empty(op.m, dtype=torch.float32, device=x.device)
        op.h.holaspmv(1.0, y)
        ctx.save_for_backward(vals, x)
        ctx.op = op
        return y

    @staticmethod
    def backward(ctx, dy):
        vals, x = ctx.saved_tensors
        op = ctx.op
        dy = dy.contiguous().float()
        op._bind(vals)
        need_vals, need_x = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        dvals = torch.empty_like(vals) if need_vals else None
        dx = torch.empty_like(x) if need_x else None
        mode = op.sparse_grad
        if mode != "dense":
            key = torch.empty(op.m, dtype=torch.int32, device=dy.device)
            val = torch.empty(op.m, dtype=torch.float32, device=dy.device)
            cnt = op.h.dense2sparse_outer(op.m, dy, key, val)
            if mode == "sparse" or cnt < op.sparse_threshold * op.m:
                op.h.spmv_backward_sparse(x, key, val, cnt, dx, dvals)
                return dvals, dx, None
        op.h.spmv_backward(x, dy, dx, dvals)
        return dvals, dx, None
