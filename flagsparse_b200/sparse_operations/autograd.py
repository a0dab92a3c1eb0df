"""Differentiable CSR SpMM  Y = A X  on the native kernels.

FlagSparse has no autograd for its CSR operators; this module provides the
backward pass a training loop needs around ``flagsparse_spmm_csr``:

  dX    = A^T dY   over the transposed pattern, built once (stable native
                      transpose) and reused; A's values are read through the
                      transpose permutation each backward, so they may change
                      between steps
  dvals = SDDMM(dY, X) on A's pattern: dvals[p] = <dY[row(p)], X[col(p)]>

Both come from one launch of fsb_spmm_csr_backward, which gathers each dY row
once for the two sums.  Where that kernel does not apply (rows wider than 512
bytes, unaligned rows) the backward runs fsb_gather_values + fsb_spmm_csr for
dX and fsb_sddmm_csr for dvals.

Values and dense operands may be float16, bfloat16, float32 or float64; all
products accumulate in fp32 (fp64 for float64).
"""

import torch

from . import _csr
from .sddmm_csr import _build_row_ids, _native_sddmm
from .spmm_csr import _native_spmm_into, _prepare_spmm_csr_matrix

SUPPORTED_AUTOGRAD_DTYPES = (torch.float16, torch.bfloat16, torch.float32, torch.float64)


class PreparedCsrSpmmAutograd:
    """A's pattern with everything forward and backward need, built once."""

    __slots__ = ("indices", "indptr", "shape", "n_rows", "n_cols", "nnz", "dtype", "_row_ids", "t_indices",
                 "t_indptr", "perm", "perm32", "plan", "t_plan")

    def __init__(self, indices, indptr, shape, dtype):
        self.indices = indices
        self.indptr = indptr
        self.shape = (int(shape[0]), int(shape[1]))
        self.n_rows, self.n_cols = self.shape
        self.nnz = int(indices.numel())
        self.dtype = dtype
        self._row_ids = None
        if self.nnz > 0:
            self.t_indices, self.t_indptr, self.perm = _csr.transpose_pattern(indices, indptr, self.shape,
                                                                              torch.int32, torch.int64)
        else:
            self.t_indices = torch.empty(0, dtype=torch.int32, device=indices.device)
            self.t_indptr = torch.zeros(self.n_cols + 1, dtype=torch.int64, device=indices.device)
            self.perm = torch.empty(0, dtype=torch.int64, device=indices.device)
        # the one-launch backward reads A's values through an int32 permutation
        self.perm32 = self.perm.to(torch.int32) if 0 < self.nnz < 2**31 else None
        self.plan = _csr.SpmmPlan(indptr, self.n_rows, dtype)
        self.t_plan = _csr.SpmmPlan(self.t_indptr, self.n_cols, dtype)

    @property
    def row_ids(self):
        """Row of every nonzero (int32), built on first use: only the separate SDDMM needs it."""
        if self._row_ids is None:
            self._row_ids = _build_row_ids(self.indptr)
        return self._row_ids


def prepare_spmm_csr_autograd(data, indices, indptr, shape):
    """Validate A (the SpMM checks and messages) and build its autograd state."""
    if data.dtype not in SUPPORTED_AUTOGRAD_DTYPES:
        raise TypeError("autograd SpMM supports float16, bfloat16, float32 and float64 values")
    _data, kernel_indices, kernel_indptr, _m, _n, _rl, _mx = _prepare_spmm_csr_matrix(data, indices, indptr, shape)
    return PreparedCsrSpmmAutograd(kernel_indices, kernel_indptr, shape, data.dtype)


def _spmm(prepared, vals, X, transpose=False):
    if transpose:
        vt = _csr.gather_values(vals, prepared.perm) if prepared.nnz > 0 else vals
        out = torch.empty((prepared.n_cols, X.shape[1]), dtype=X.dtype, device=X.device)
        return _native_spmm_into(vt, prepared.t_indices, prepared.t_indptr, prepared.n_cols, prepared.n_rows, X,
                                 prepared.t_plan, out)
    out = torch.empty((prepared.n_rows, X.shape[1]), dtype=X.dtype, device=X.device)
    return _native_spmm_into(vals, prepared.indices, prepared.indptr, prepared.n_rows, prepared.n_cols, X,
                             prepared.plan, out)


class CsrSpmmFunction(torch.autograd.Function):
    """Y = A(vals) @ X with gradients for vals and X."""

    @staticmethod
    def forward(ctx, vals, X, prepared):
        vals = vals.contiguous()
        X = X.contiguous()
        ctx.prepared = prepared
        ctx.save_for_backward(vals, X)
        return _spmm(prepared, vals, X)

    @staticmethod
    def backward(ctx, dY):
        vals, X = ctx.saved_tensors
        p = ctx.prepared
        dY = dY.contiguous()
        d_vals = d_X = None
        if ctx.needs_input_grad[1] and p.perm32 is not None:
            d_X = torch.empty((p.n_cols, X.shape[1]), dtype=X.dtype, device=X.device)
            d_vals = torch.empty_like(vals) if ctx.needs_input_grad[0] else None
            if _csr.spmm_backward(vals, p.perm32, p.t_indices, p.t_indptr, p.n_rows, p.n_cols, dY,
                                  X if d_vals is not None else None, d_X, d_vals, p.t_plan):
                return d_vals, d_X, None
            d_vals = d_X = None
        if ctx.needs_input_grad[1]:
            d_X = _spmm(p, vals, dY, transpose=True)
        if ctx.needs_input_grad[0]:
            d_vals = torch.empty_like(vals)
            _native_sddmm(p.row_ids, p.indices, dY, X, None, 1.0, 0.0, d_vals)
        return d_vals, d_X, None


def flagsparse_spmm_csr_autograd(data, X, prepared=None, indices=None, indptr=None, shape=None):
    """Differentiable ``A @ X``; pass ``prepared`` (from prepare_spmm_csr_autograd) to reuse A's pattern."""
    if prepared is None:
        if any(v is None for v in (indices, indptr, shape)):
            raise ValueError("indices, indptr, and shape are required when prepared is not provided")
        prepared = prepare_spmm_csr_autograd(data, indices, indptr, shape)
    elif not isinstance(prepared, PreparedCsrSpmmAutograd):
        raise TypeError("prepared must be a PreparedCsrSpmmAutograd instance")
    if X.ndim != 2 or X.shape[0] != prepared.n_cols:
        raise ValueError(f"X must be 2D with X.shape[0] == n_cols={prepared.n_cols}")
    if data.dtype != prepared.dtype or X.dtype != prepared.dtype:
        raise TypeError("data and X dtype must match the prepared dtype")
    if data.numel() != prepared.nnz:
        raise ValueError("data length must equal nnz of the prepared pattern")
    return CsrSpmmFunction.apply(data, X, prepared)
