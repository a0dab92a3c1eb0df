"""CSR SpMV host code over the sm_100a native kernel.

Drop-in mirror of FlagSparse ``sparse_operations/spmv_csr.py``: same public
functions, signatures, defaults, op handling (``:32-66``), validation
messages (``:539-611``), int64 -> int32 fallback policy (``:749-834``),
``PreparedCsrSpmv`` slots (``:69-144``) and return/meta contract
(``:837-945``).  The compute is ``fsb_spmv_csr`` (one launch, compensated
accumulation) instead of the Triton kernels; the prepared object caches the
native unit plan so steady-state calls do no host synchronisation.
"""

import time

import torch

from .. import _native as nat
from . import _csr
from ._common import (
    SUPPORTED_INDEX_DTYPES,
    _INDEX_LIMIT_INT32,
    _is_complex_dtype,
)

SUPPORTED_SPMV_VALUE_DTYPES = (
    torch.float16,
    torch.bfloat16,
    torch.float32,
    torch.float64,
    torch.complex64,
    torch.complex128,
)

SPMV_OP_NON = 0
SPMV_OP_TRANS = 1
SPMV_OP_CONJ_TRANS = 2
SPMV_OP_NAMES = {SPMV_OP_NON: "non", SPMV_OP_TRANS: "trans", SPMV_OP_CONJ_TRANS: "conj"}
_SPMV_OP_NAME_TO_CODE = {name: code for code, name in SPMV_OP_NAMES.items()}
_OP_ERROR = "op must be one of: 0=non, 1=trans, 2=conj"

# Row-length buckets of FlagSparse's CSR-vector path (spmv_csr.py:150-175).
# The native kernel does not launch per bucket; the bucket row lists are built
# (stable, natively) for ``use_opt=True`` calls so ``bucket_count`` and
# ``prepared.opt_buckets`` keep their meaning.
_SPMV_OPT_BUCKET_CONFIGS = (
    {"max_row_nnz": 64, "block_size": 32, "num_warps": 1, "num_stages": 2, "batch_rows": 16},
    {"max_row_nnz": 512, "block_size": 256, "num_warps": 8, "num_stages": 2},
    {"max_row_nnz": 4096, "block_size": 512, "num_warps": 16, "num_stages": 2},
    {"max_row_nnz": None, "block_size": 1024, "num_warps": 32, "num_stages": 3},
)
_SPMV_OPT_BUCKET_CONFIGS_FP64 = (
    {"max_row_nnz": 64, "block_size": 32, "num_warps": 1, "num_stages": 2, "batch_rows": 4},
    {"max_row_nnz": 256, "block_size": 64, "num_warps": 2, "num_stages": 2},
    {"max_row_nnz": 2048, "block_size": 128, "num_warps": 4, "num_stages": 2},
    {"max_row_nnz": 8192, "block_size": 256, "num_warps": 8, "num_stages": 2},
    {"max_row_nnz": None, "block_size": 512, "num_warps": 16, "num_stages": 1},
)


def _normalize_spmv_op(op=None, transpose=False):
    if op is None:
        return SPMV_OP_TRANS if bool(transpose) else SPMV_OP_NON
    if isinstance(op, str):
        code = _SPMV_OP_NAME_TO_CODE.get(op.strip().lower())
        if code is None:
            raise ValueError(_OP_ERROR)
        return code
    try:
        code = int(op)
    except (TypeError, ValueError) as exc:
        raise ValueError(_OP_ERROR) from exc
    if code not in SPMV_OP_NAMES:
        raise ValueError(_OP_ERROR)
    return code


def _spmv_op_to_name(op):
    return SPMV_OP_NAMES[_normalize_spmv_op(op)]


def _spmv_op_transposes(op):
    return _normalize_spmv_op(op) in (SPMV_OP_TRANS, SPMV_OP_CONJ_TRANS)


class PreparedCsrSpmv:
    """Cached CSR metadata (and the native launch plan) for repeated SpMV calls."""

    __slots__ = (
        "data",
        "kernel_indices",
        "kernel_indptr",
        "shape",
        "n_rows",
        "n_cols",
        "block_nnz",
        "max_segments",
        "opt_max_segments",
        "row_lengths",
        "max_row_nnz",
        "opt_buckets",
        "supports_opt",
        "transpose",
        "op",
        "index_fallback_policy",
        "index_fallback_applied",
        "index_fallback_reason",
        "_baseline_compute_dtype",
        "_baseline_data",
        "_native_plan",
    )

    def __init__(
        self,
        data,
        kernel_indices,
        kernel_indptr,
        shape,
        n_rows,
        n_cols,
        block_nnz,
        max_segments,
        max_row_nnz,
        opt_buckets=None,
        opt_max_segments=None,
        row_lengths=None,
        transpose=False,
        op=None,
        index_fallback_policy="auto",
        index_fallback_applied=False,
        index_fallback_reason=None,
    ):
        self.data = data
        self.kernel_indices = kernel_indices
        self.kernel_indptr = kernel_indptr
        self.shape = (int(shape[0]), int(shape[1]))
        self.n_rows = n_rows
        self.n_cols = n_cols
        self.block_nnz = block_nnz
        self.max_segments = max_segments
        self.opt_max_segments = opt_max_segments
        if row_lengths is None:
            row_lengths = kernel_indptr[1:] - kernel_indptr[:-1]
        self.row_lengths = row_lengths
        self.max_row_nnz = max_row_nnz
        self.opt_buckets = [] if opt_buckets is None else opt_buckets
        self.supports_opt = data.dtype in (torch.float32, torch.float64) and kernel_indices.dtype == torch.int32
        self.op = _normalize_spmv_op(op, transpose=transpose)
        self.transpose = _spmv_op_transposes(self.op)
        self.index_fallback_policy = str(index_fallback_policy).lower()
        self.index_fallback_applied = bool(index_fallback_applied)
        self.index_fallback_reason = index_fallback_reason
        # The reference upcasts fp32 -> fp64 and f16/bf16 -> fp32 for its
        # baseline kernel; the native kernel reads the stored dtype and
        # accumulates with compensation, so no upcast copy is ever made.
        if data.dtype in (torch.float16, torch.bfloat16):
            self._baseline_compute_dtype = torch.float32
        elif data.dtype == torch.float32:
            self._baseline_compute_dtype = torch.float64
        else:
            self._baseline_compute_dtype = data.dtype
        self._baseline_data = None
        self._native_plan = None

    def native_plan(self):
        """The native unit plan, built on first use and cached."""
        if self._native_plan is None:
            self._native_plan = _csr.NativeSpmvPlan(self.kernel_indptr, self.n_rows, self.data.dtype)
        return self._native_plan


def _build_spmv_opt_buckets(kernel_indptr, n_rows, max_row_nnz, row_index_dtype, max_segments=None, fp64=False):
    """Bucket row lists with FlagSparse's thresholds (spmv_csr.py:371-417), built natively and stably."""
    configs = _SPMV_OPT_BUCKET_CONFIGS_FP64 if fp64 else _SPMV_OPT_BUCKET_CONFIGS
    lists = _csr.bucketize_rows(kernel_indptr, n_rows, [spec["max_row_nnz"] for spec in configs])
    buckets = []
    for spec, rows in zip(configs, lists):
        if rows.numel() == 0:
            continue
        bound = max_row_nnz if spec["max_row_nnz"] is None else spec["max_row_nnz"]
        max_segs = max((bound + spec["block_size"] - 1) // spec["block_size"], 1) if max_segments is None else max_segments
        buckets.append(
            {
                "rows": rows.to(row_index_dtype),
                "block_size": spec["block_size"],
                "max_segs": max_segs,
                "num_warps": spec["num_warps"],
                "num_stages": spec["num_stages"],
                "batch_rows": int(spec.get("batch_rows", 1)),
            }
        )
    return buckets


def _build_spmv_opt_runtime_buckets(prepared):
    row_index_dtype = torch.int32 if prepared.n_rows <= _INDEX_LIMIT_INT32 else torch.int64
    return _build_spmv_opt_buckets(
        prepared.kernel_indptr,
        prepared.n_rows,
        prepared.max_row_nnz,
        row_index_dtype,
        max_segments=prepared.opt_max_segments,
        fp64=prepared.data.dtype == torch.float64,
    )


def _normalize_spmv_index_fallback_policy(index_fallback_policy):
    policy = str(index_fallback_policy).lower()
    if policy not in ("auto", "strict"):
        raise ValueError("index_fallback_policy must be 'auto' or 'strict'")
    return policy


def _spmv_dtype_error_message():
    return "data dtype must be one of: " + ", ".join(
        str(dtype).replace("torch.", "") for dtype in SUPPORTED_SPMV_VALUE_DTYPES
    )


def _transpose_csr_for_spmv(data, indices, indptr, shape):
    """CSR of A^T with the reference's index-dtype rules (spmv_csr.py:498-536)."""
    n_rows, n_cols = int(shape[0]), int(shape[1])
    nnz = data.numel()
    out_index_dtype = indices.dtype if n_rows <= _INDEX_LIMIT_INT32 else torch.int64
    out_indptr_dtype = indptr.dtype if nnz <= _INDEX_LIMIT_INT32 else torch.int64
    if nnz == 0:
        return (
            data,
            torch.empty(0, dtype=out_index_dtype, device=data.device),
            torch.zeros(n_cols + 1, dtype=out_indptr_dtype, device=data.device),
            (n_cols, n_rows),
        )
    t_indices, t_indptr, perm = _csr.transpose_pattern(indices, indptr, shape, out_index_dtype, out_indptr_dtype)
    return _csr.gather_values(data, perm), t_indices, t_indptr, (n_cols, n_rows)


def _prepare_spmv_csr_matrix(data, indices, indptr, shape, index_fallback_policy="auto"):
    _normalize_spmv_index_fallback_policy(index_fallback_policy)
    if not all(torch.is_tensor(t) for t in (data, indices, indptr)):
        raise TypeError("data, indices, indptr must all be torch.Tensor")
    if data.ndim != 1 or indices.ndim != 1 or indptr.ndim != 1:
        raise ValueError("data, indices, indptr must be 1D tensors")
    n_rows, n_cols = int(shape[0]), int(shape[1])
    if indptr.numel() != n_rows + 1:
        raise ValueError(f"indptr length must be n_rows+1={n_rows + 1}, got {indptr.numel()}")
    if data.numel() != indices.numel():
        raise ValueError("data and indices must have the same length (nnz)")
    if not all(t.is_cuda for t in (data, indices, indptr)):
        raise ValueError("data, indices, indptr must be CUDA tensors")
    if not all(t.device == data.device for t in (indices, indptr)):
        raise ValueError("data, indices, indptr must be on the same CUDA device")
    if data.dtype not in SUPPORTED_SPMV_VALUE_DTYPES:
        raise TypeError(_spmv_dtype_error_message())
    if indices.dtype not in SUPPORTED_INDEX_DTYPES:
        raise TypeError("indices dtype must be torch.int32 or torch.int64")
    if indptr.dtype not in SUPPORTED_INDEX_DTYPES:
        raise TypeError("indptr dtype must be torch.int32 or torch.int64")

    data = data.contiguous()
    indices = indices.contiguous()
    indptr = indptr.contiguous()
    nnz = data.numel()
    facts = _csr.inspect_csr(indices, indptr, n_rows, nnz)
    if facts["first"] != 0:
        raise ValueError("indptr must start at zero")
    if facts["last"] != nnz:
        raise ValueError("indptr[-1] must equal nnz")
    if facts["decreasing"]:
        raise ValueError("indptr must be non-decreasing")
    if nnz > 0 and (facts["min_col"] < 0 or facts["max_col"] >= n_cols):
        raise IndexError("indices out of range for n_cols")
    row_lengths = indptr[1:] - indptr[:-1]
    return data, indices, indptr, n_rows, n_cols, row_lengths, int(facts["max_row_nnz"])


def _validate_spmv_x(x, prepared):
    if x is None or not torch.is_tensor(x):
        raise TypeError("x must be a torch.Tensor")
    if x.ndim != 1:
        raise ValueError("x must be a 1D tensor")
    if not x.is_cuda:
        raise ValueError("x must be a CUDA tensor")
    if x.dtype != prepared.data.dtype:
        raise TypeError("x dtype must match sparse matrix dtype")
    if x.numel() != prepared.n_cols:
        raise ValueError(f"x length must be n_cols={prepared.n_cols}, got {x.numel()}")
    if x.device != prepared.data.device:
        raise ValueError("x must be on the same device as sparse matrix data")
    return x.contiguous()


def prepare_spmv_csr(
    data,
    indices,
    indptr,
    shape,
    block_nnz=256,
    max_segments=None,
    transpose=False,
    op=None,
    index_fallback_policy="auto",
):
    index_fallback_policy = _normalize_spmv_index_fallback_policy(index_fallback_policy)
    op_code = _normalize_spmv_op(op, transpose=transpose)
    if op is not None and bool(transpose) and op_code == SPMV_OP_NON:
        raise ValueError("transpose=True conflicts with op=non")
    transpose = _spmv_op_transposes(op_code)
    if transpose:
        data, indices, indptr, *_ = _prepare_spmv_csr_matrix(
            data, indices, indptr, shape, index_fallback_policy=index_fallback_policy
        )
        n_rows = int(shape[0])
        nnz = data.numel()
        out_index_dtype = indices.dtype if n_rows <= _INDEX_LIMIT_INT32 else torch.int64
        out_indptr_dtype = indptr.dtype if nnz <= _INDEX_LIMIT_INT32 else torch.int64
        if nnz == 0:
            indices = torch.empty(0, dtype=out_index_dtype, device=data.device)
            indptr = torch.zeros(int(shape[1]) + 1, dtype=out_indptr_dtype, device=data.device)
        else:
            indices, indptr, perm = _csr.transpose_pattern(indices, indptr, shape, out_index_dtype, out_indptr_dtype)
            conj = op_code == SPMV_OP_CONJ_TRANS and _is_complex_dtype(data.dtype)
            data = _csr.gather_values(data, perm, conj=conj)
        shape = (int(shape[1]), int(shape[0]))
    (data, kernel_indices, kernel_indptr, n_rows, n_cols, row_lengths, max_row_nnz) = _prepare_spmv_csr_matrix(
        data, indices, indptr, shape, index_fallback_policy=index_fallback_policy
    )
    block_nnz_use = block_nnz
    if max_segments is None:
        max_segments_use = max((max_row_nnz + block_nnz_use - 1) // block_nnz_use, 1)
        while max_segments_use > 2048 and block_nnz_use < 65536:
            block_nnz_use *= 2
            max_segments_use = max((max_row_nnz + block_nnz_use - 1) // block_nnz_use, 1)
    else:
        max_segments_use = max_segments
    prepared = PreparedCsrSpmv(
        data=data,
        kernel_indices=kernel_indices,
        kernel_indptr=kernel_indptr,
        shape=shape,
        n_rows=n_rows,
        n_cols=n_cols,
        block_nnz=block_nnz_use,
        max_segments=max_segments_use,
        opt_max_segments=max_segments,
        row_lengths=row_lengths,
        max_row_nnz=max_row_nnz,
        opt_buckets=None,
        transpose=transpose,
        op=op_code,
        index_fallback_policy=index_fallback_policy,
    )
    prepared.native_plan()
    return prepared


def _native_spmv_csr_impl_prepared(prepared, x, out=None):
    """One native SpMV launch: y = A x for the prepared (already op-applied) matrix."""
    y = out if out is not None else torch.empty(prepared.n_rows, dtype=prepared.data.dtype, device=prepared.data.device)
    if prepared.n_rows == 0:
        return y
    plan = prepared.native_plan()
    nat.check(
        nat.lib().fsb_spmv_csr(
            nat.dtype_code(prepared.data.dtype),
            nat.ptr(prepared.data),
            nat.ptr(prepared.kernel_indices),
            nat.is64(prepared.kernel_indices),
            nat.ptr(prepared.kernel_indptr),
            nat.is64(prepared.kernel_indptr),
            prepared.n_rows,
            prepared.n_cols,
            nat.ptr(x),
            nat.ptr(y),
            plan.struct_ref(),
            nat.stream_of(y.device),
        ),
        "fsb_spmv_csr",
    )
    return y


def _spmv_uses_int64_indices(prepared):
    return prepared.kernel_indices.dtype == torch.int64 or prepared.kernel_indptr.dtype == torch.int64


def _spmv_int32_fallback_blocker(prepared):
    if prepared.kernel_indices.dtype == torch.int64 and prepared.kernel_indices.numel() > 0:
        facts = _csr.inspect_csr(prepared.kernel_indices, prepared.kernel_indptr, prepared.n_rows,
                                 prepared.kernel_indices.numel())
        min_index, max_index = int(facts["min_col"]), int(facts["max_col"])
        if min_index < 0 or max_index > _INDEX_LIMIT_INT32:
            return (
                f"column index range [{min_index}, {max_index}] cannot fit int32 "
                f"for shape={prepared.shape}"
            )
    if prepared.kernel_indptr.dtype == torch.int64 and prepared.kernel_indptr.numel() > 0:
        max_offset = int(prepared.kernel_indptr[-1].item())
        if max_offset > _INDEX_LIMIT_INT32:
            return f"CSR nnz offset {max_offset} cannot fit int32 for shape={prepared.shape}"
    if prepared.n_rows > _INDEX_LIMIT_INT32:
        return f"row count {prepared.n_rows} cannot fit int32 row metadata"
    return None


def _spmv_prepared_with_int32_indices(prepared, reason):
    blocker = _spmv_int32_fallback_blocker(prepared)
    if blocker is not None:
        raise RuntimeError(f"native int64 CSR SpMV failed and int32 fallback is unsafe: {blocker}")
    kernel_indices = prepared.kernel_indices.to(torch.int32)
    kernel_indptr = prepared.kernel_indptr.to(torch.int32)
    row_lengths = kernel_indptr[1:] - kernel_indptr[:-1]
    return PreparedCsrSpmv(
        data=prepared.data,
        kernel_indices=kernel_indices,
        kernel_indptr=kernel_indptr,
        shape=prepared.shape,
        n_rows=prepared.n_rows,
        n_cols=prepared.n_cols,
        block_nnz=prepared.block_nnz,
        max_segments=prepared.max_segments,
        opt_max_segments=prepared.opt_max_segments,
        row_lengths=row_lengths,
        max_row_nnz=prepared.max_row_nnz,
        opt_buckets=None,
        transpose=prepared.transpose,
        op=prepared.op,
        index_fallback_policy=prepared.index_fallback_policy,
        index_fallback_applied=True,
        index_fallback_reason=str(reason),
    )


def _run_spmv_prepared(prepared, x, use_opt=False, opt_buckets=None, out=None):
    # Both reference paths (baseline and bucketed) map to the same native
    # kernel; ``use_opt`` only decides whether bucket lists are reported.
    return _native_spmv_csr_impl_prepared(prepared, x, out=out)


def _run_spmv_prepared_with_fallback(prepared, x, use_opt=False, opt_buckets=None, out=None):
    try:
        return _run_spmv_prepared(prepared, x, use_opt=use_opt, opt_buckets=opt_buckets, out=out)
    except Exception as exc:
        if prepared.index_fallback_policy != "auto" or not _spmv_uses_int64_indices(prepared):
            raise
        fallback_prepared = _spmv_prepared_with_int32_indices(prepared, exc)
        return _run_spmv_prepared(fallback_prepared, x, use_opt=use_opt, opt_buckets=None, out=out)


def flagsparse_spmv_csr(
    data=None,
    indices=None,
    indptr=None,
    x=None,
    shape=None,
    block_nnz=256,
    max_segments=None,
    out=None,
    return_time=False,
    return_meta=False,
    use_opt=False,
    prepared=None,
    transpose=None,
    op=None,
    index_fallback_policy="auto",
):
    """CSR SpMV on the sm_100a native kernel.

    data, indices, indptr: CSR arrays; x: dense vector; shape: (n_rows, n_cols).
    prepared: cached state from prepare_spmv_csr for steady-state calls.
    op: 0/'non' for A @ x, 1/'trans' for A.T @ x, 2/'conj' for A.conj().T @ x.
    use_opt: also build FlagSparse's row-length bucket lists (reported in meta);
    the native kernel is the same either way.
    """
    op_explicit = op is not None
    op_code = _normalize_spmv_op(op, transpose=False if transpose is None else bool(transpose))
    if op_explicit and transpose is not None and bool(transpose) != _spmv_op_transposes(op_code):
        raise ValueError("transpose conflicts with op")
    if prepared is None:
        if any(arg is None for arg in (data, indices, indptr, shape)):
            raise ValueError("data, indices, indptr, and shape are required when prepared is not provided")
        prepared = prepare_spmv_csr(
            data,
            indices,
            indptr,
            shape,
            block_nnz=block_nnz,
            max_segments=max_segments,
            op=op_code,
            index_fallback_policy=index_fallback_policy,
        )
    else:
        if op_explicit and op_code != prepared.op:
            raise ValueError(
                f"op={_spmv_op_to_name(op_code)} does not match prepared.op={_spmv_op_to_name(prepared.op)}"
            )
        if not op_explicit and transpose is not None and bool(transpose) != prepared.transpose:
            raise ValueError(
                f"transpose={bool(transpose)} does not match prepared.transpose={prepared.transpose}"
            )
    x = _validate_spmv_x(x, prepared)
    if out is not None:
        if not out.is_cuda:
            raise ValueError("out must be a CUDA tensor")
        if out.device != prepared.data.device:
            raise ValueError("out must be on the same CUDA device as the result")
        if out.shape != (prepared.n_rows,) or out.dtype != prepared.data.dtype:
            raise ValueError("out shape/dtype must match result")
    direct_out = out if (out is not None and out.is_contiguous()) else None

    do_timing = bool(return_time or return_meta)
    symbolic_ms = 0.0 if do_timing else None
    compute_ms = None
    op_total_ms = None
    opt_buckets = None
    if do_timing:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
    if use_opt and prepared.supports_opt:
        opt_buckets = _build_spmv_opt_runtime_buckets(prepared)
    if do_timing:
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        symbolic_ms = (t1 - t0) * 1000.0 if use_opt and prepared.supports_opt else 0.0
    y = _run_spmv_prepared_with_fallback(prepared, x, use_opt=use_opt, opt_buckets=opt_buckets, out=direct_out)
    if do_timing:
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        compute_ms = (t2 - t1) * 1000.0
        op_total_ms = symbolic_ms + compute_ms
    if out is not None and y is not out:
        out.copy_(y)
        y = out
    if return_meta:
        meta = {
            "symbolic_ms": symbolic_ms,
            "compute_ms": compute_ms,
            "op_total_ms": op_total_ms,
            "bucket_count": int(len(opt_buckets)) if opt_buckets is not None else 0,
        }
        if return_time:
            return y, op_total_ms, meta
        return y, meta
    if return_time:
        return y, op_total_ms
    return y


# ---------------------------------------------------------------------------
# COO input: conversion to CSR feeding the CSR SpMV
# (sparse_operations/spmv_csr.py:948-1091 of flagos-ai/FlagSparse).
# ---------------------------------------------------------------------------
def _coo_index(t):
    """int32 / int64 index tensors pass through; other integer dtypes widen to int64."""
    return t if t.dtype in (torch.int32, torch.int64) else t.to(torch.int64)


def _coo_is_sorted_lex(row, col, n_cols):
    """True iff the COO pairs are in non-decreasing (row, col) order."""
    if row.numel() <= 1:
        return True
    unsorted, _, _ = _csr.coo_inspect(_coo_index(row).contiguous(), _coo_index(col).contiguous(), 2**31 - 1,
                                      max(1, int(n_cols)))
    return unsorted == 0


def coo_to_csr_for_spmv(data, row, col, shape, assume_sorted=False):
    """Convert COO to CSR triple (data, csr_col_indices, indptr) for SpMV.

    Returns values in CSR order (``data`` itself when the pairs are already in
    (row, col) order), int32 column indices and int64 row pointers.  The order
    and the index ranges are checked natively in one pass; unordered input is
    sorted even when ``assume_sorted`` is set.  Repeated (row, col) pairs are
    kept as separate entries in their input order.
    """
    n_rows, n_cols = int(shape[0]), int(shape[1])
    row = _coo_index(row).contiguous()
    col = _coo_index(col).contiguous()
    if row.numel() == 0:
        indptr = torch.zeros(n_rows + 1, dtype=torch.int64, device=data.device)
        return data, col.to(torch.int32), indptr
    unsorted, bad_rows, bad_cols = _csr.coo_inspect(row, col, n_rows, n_cols)
    if bad_rows:
        raise RuntimeError(f"row indices out of range for n_rows={n_rows}")
    if bad_cols:
        raise IndexError("indices out of range for n_cols")
    ordered = unsorted == 0
    indices, indptr, perm = _csr.coo_to_csr(row, col, n_rows, n_cols, ordered)
    data_s = data if ordered else _csr.gather_values(data.contiguous(), perm)
    return data_s, indices, indptr


def prepare_spmv_coo_tocsr(
    data,
    row,
    col,
    shape,
    block_nnz=256,
    max_segments=None,
    assume_sorted=False,
):
    """One-time COO -> CSR + plan; use with ``flagsparse_spmv_coo_tocsr(..., prepared=p)``."""
    if not all(torch.is_tensor(t) for t in (data, row, col)):
        raise TypeError("data, row, col must all be torch.Tensor")
    if not all(t.is_cuda for t in (data, row, col)):
        raise ValueError("data, row, col must all be CUDA tensors")
    if data.ndim != 1 or row.ndim != 1 or col.ndim != 1:
        raise ValueError("data, row, col must all be 1D tensors")
    if data.dtype not in SUPPORTED_SPMV_VALUE_DTYPES:
        raise TypeError(_spmv_dtype_error_message())
    if row.numel() != col.numel() or data.numel() != row.numel():
        raise ValueError("data, row, col must have the same length")
    data_s, indices, indptr = coo_to_csr_for_spmv(data, row, col, shape, assume_sorted=assume_sorted)
    return prepare_spmv_csr(
        data_s,
        indices,
        indptr,
        shape,
        block_nnz=block_nnz,
        max_segments=max_segments,
    )


def flagsparse_spmv_coo_tocsr(
    data=None,
    row=None,
    col=None,
    x=None,
    shape=None,
    block_nnz=256,
    max_segments=None,
    out=None,
    return_time=False,
    use_opt=True,
    prepared=None,
    assume_sorted=False,
):
    """COO SpMV via CSR conversion: y = A @ x.

    Steady state: ``p = prepare_spmv_coo_tocsr(data, row, col, shape)`` then
    call with ``prepared=p`` (``data`` / ``row`` / ``col`` may be omitted).
    ``use_opt`` is forwarded to flagsparse_spmv_csr (bucket lists in meta);
    the native kernel is the same either way.
    """
    if prepared is not None:
        if x is None:
            raise TypeError("x is required")
        if shape is None:
            shape = prepared.shape
        sh = (int(shape[0]), int(shape[1]))
        if sh != prepared.shape:
            raise ValueError(f"shape {sh} does not match prepared.shape {prepared.shape}")
        return flagsparse_spmv_csr(
            x=x,
            shape=shape,
            block_nnz=block_nnz,
            max_segments=max_segments,
            out=out,
            return_time=return_time,
            use_opt=use_opt,
            prepared=prepared,
        )

    if not all(torch.is_tensor(t) for t in (data, row, col, x)):
        raise TypeError("data, row, col, x must all be torch.Tensor")
    if not all(t.is_cuda for t in (data, row, col, x)):
        raise ValueError("data, row, col, x must all be CUDA tensors")
    if data.ndim != 1 or row.ndim != 1 or col.ndim != 1 or x.ndim != 1:
        raise ValueError("data, row, col, x must all be 1D tensors")
    if data.dtype not in SUPPORTED_SPMV_VALUE_DTYPES:
        raise TypeError(_spmv_dtype_error_message())
    if x.dtype != data.dtype:
        raise TypeError("x dtype must match data dtype")

    data_s, indices, indptr = coo_to_csr_for_spmv(data, row, col, shape, assume_sorted=assume_sorted)
    return flagsparse_spmv_csr(
        data_s,
        indices,
        indptr,
        x,
        shape,
        block_nnz=block_nnz,
        max_segments=max_segments,
        out=out,
        return_time=return_time,
        use_opt=use_opt,
    )
