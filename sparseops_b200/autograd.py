"""Differentiable SpMV: a torch.autograd.Function over the C ABI.

    y = alpha * A(values) @ x

forward   spops_spmv   (the CSR kernel)
backward  grad_x      = alpha * A^T g   spops_spmv_t (device-built transpose, no atomics)
          grad_values = alpha * g_i x_j spops_sddmm  (on A's pattern)

The pattern (row offsets, column indices) is analysed once and kept in a
``SparsePattern``; the values tensor may change between calls (optimizer
steps, new tensors): it is re-pointed with spops_csr_set_values, which keeps
the analysis and marks the transpose's values stale.  FP64 and FP32 values
are supported (FP32 accumulates in FP32).

No reference counterpart: the reference has no differentiation; its
transpose (include/sparse_conversion.h:2066) is the oracle for grad_x.
"""
from __future__ import annotations

import torch

from ._lib import call, dbl, vp
from .spops import CSR_Matrix, default_context


class SparsePattern:
    """A fixed CSR pattern on the device (row_offset, col_index tensors)."""

    def __init__(self, num_rows: int, num_cols: int, row_offset: torch.Tensor, col_index: torch.Tensor,
                 values: torch.Tensor):
        if not (row_offset.is_cuda and col_index.is_cuda and values.is_cuda):
            raise ValueError("SparsePattern arrays must be CUDA tensors")
        self.num_rows, self.num_cols = int(num_rows), int(num_cols)
        self.row_offset, self.col_index = row_offset, col_index
        self.dtype = values.dtype
        self._csr = CSR_Matrix(num_rows, num_cols, row_offset, col_index, values.detach())
        self.handle = self._csr.device(default_context(values.device.index))
        self._values_ptr = values.data_ptr()
        self._keep = values

    def bind(self, values: torch.Tensor) -> None:
        """Point the handle at `values` (same length and dtype)."""
        if values.dtype != self.dtype or values.numel() != self.col_index.numel():
            raise ValueError("values must match the pattern's length and dtype")
        values = values.contiguous()
        if values.data_ptr() != self._values_ptr:
            call("spops_csr_set_values", self.handle.handle, vp(values.data_ptr()))
            self._values_ptr = values.data_ptr()
        else:
            call("spops_matrix_touch", self.handle.handle)  # same buffer, possibly new contents
        self._keep = values

    def ctx(self):
        return self.handle.ctx.follow_torch()


class SpMVFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values: torch.Tensor, x: torch.Tensor, pattern: SparsePattern, alpha: float = 1.0):
        values = values.contiguous()
        x = x.contiguous()
        pattern.bind(values)
        c = pattern.ctx()
        y = torch.empty(pattern.num_rows, dtype=values.dtype, device=values.device)
        call("spops_spmv", c.handle, dbl(alpha), pattern.handle.handle, vp(x.data_ptr()), dbl(0.0),
             vp(y.data_ptr()))
        ctx.save_for_backward(values, x)
        ctx.pattern, ctx.alpha = pattern, alpha
        return y

    @staticmethod
    def backward(ctx, g: torch.Tensor):
        values, x = ctx.saved_tensors
        pattern, alpha = ctx.pattern, ctx.alpha
        g = g.contiguous()
        pattern.bind(values)
        c = pattern.ctx()
        grad_values = grad_x = None
        if ctx.needs_input_grad[0]:
            grad_values = torch.empty_like(values)
            call("spops_sddmm", c.handle, dbl(alpha), pattern.handle.handle, vp(g.data_ptr()), vp(x.data_ptr()),
                 vp(grad_values.data_ptr()))
        if ctx.needs_input_grad[1]:
            grad_x = torch.empty(pattern.num_cols, dtype=values.dtype, device=values.device)
            call("spops_spmv_t", c.handle, dbl(alpha), pattern.handle.handle, vp(g.data_ptr()), dbl(0.0),
                 vp(grad_x.data_ptr()))
        return grad_values, grad_x, None, None


def spmv(values: torch.Tensor, x: torch.Tensor, pattern: SparsePattern, alpha: float = 1.0) -> torch.Tensor:
    """Differentiable y = alpha * A(values) @ x."""
    return SpMVFunction.apply(values, x, pattern, alpha)


class SparseLinear(torch.nn.Module):
    """y = A(values) @ x with the stored values as a trainable parameter."""

    def __init__(self, num_rows, num_cols, row_offset, col_index, values):
        super().__init__()
        self.values = torch.nn.Parameter(values.detach().clone())
        self.pattern = SparsePattern(num_rows, num_cols, row_offset, col_index, self.values.data)

    def forward(self, x):
        return spmv(self.values, x, self.pattern)
