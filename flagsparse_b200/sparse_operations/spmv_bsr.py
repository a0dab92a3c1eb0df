"""BSR SpMV on the sm_100a native kernel (``fsb_bsr_spmv``).

Mirrors FlagSparse's ``sparse_operations/spmv_bsr.py`` (``flagsparse_spmv_bsr``
``:895-1024``, ``prepare_spmv_bsr`` ``:510-571``, ``PreparedBsrSpmv``
``:109-180``): the same names, signatures, op handling (non / trans / conj),
algorithm names (``base``, ``blockrow_reduce``), padded result lengths,
validation messages and meta keys.

Both algorithms run the one native kernel: a thread per padded row walks the
blocks of its block row with compensated sums in block order, so results are
deterministic (FlagSparse adds per-segment partial sums with atomics).  For
``trans`` / ``conj`` the prepare step transposes the block matrix once (block
pattern by the stable CSR transpose, each block transposed and, for conj,
conjugated) and the kernel runs on it.  ``blockrow_reduce`` additionally
reports FlagSparse's block-row-length buckets in meta.
"""

import time

import torch

from .. import _native as nat
from . import _csr
from ._common import SUPPORTED_INDEX_DTYPES

SUPPORTED_SPMV_BSR_VALUE_DTYPES = (
    torch.float32,
    torch.float64,
    torch.complex64,
    torch.complex128,
)

SPMV_BSR_OP_NON = 0
SPMV_BSR_OP_TRANS = 1
SPMV_BSR_OP_CONJ_TRANS = 2
SPMV_BSR_OP_NAMES = {
    SPMV_BSR_OP_NON: "non",
    SPMV_BSR_OP_TRANS: "trans",
    SPMV_BSR_OP_CONJ_TRANS: "conj",
}
SPMV_BSR_SUPPORTED_OP_NAMES = ("non", "trans", "conj")
_SPMV_BSR_OP_NAME_TO_CODE = {name: code for code, name in SPMV_BSR_OP_NAMES.items()}
SPMV_BSR_ALG_BASE = "base"
SPMV_BSR_ALG_BLOCKROW_REDUCE = "blockrow_reduce"
SPMV_BSR_SUPPORTED_ALGORITHMS = (SPMV_BSR_ALG_BASE, SPMV_BSR_ALG_BLOCKROW_REDUCE)

# (label, low, high, block_nnz, direct_store) -- spmv_bsr.py:674-681
_BLOCKROW_REDUCE_BUCKETS = (
    ("le1", 0, 1, 1, True),
    ("le4", 2, 4, 4, True),
    ("le16", 5, 16, 16, True),
    ("le64", 17, 64, 64, True),
    ("gt64", 65, None, 128, False),
)


def _spmv_bsr_dtype_error_message():
    return "BSR SpMV supports float32, float64, complex64, and complex128"


def _normalize_spmv_bsr_op(op=None, transpose=False):
    if op is None:
        return SPMV_BSR_OP_TRANS if bool(transpose) else SPMV_BSR_OP_NON
    if isinstance(op, str):
        token = op.strip().lower()
        if token not in _SPMV_BSR_OP_NAME_TO_CODE:
            raise ValueError("op must be one of: 0=non, 1=trans, 2=conj")
        return _SPMV_BSR_OP_NAME_TO_CODE[token]
    try:
        op_code = int(op)
    except (TypeError, ValueError) as exc:
        raise ValueError("op must be one of: 0=non, 1=trans, 2=conj") from exc
    if op_code not in SPMV_BSR_OP_NAMES:
        raise ValueError("op must be one of: 0=non, 1=trans, 2=conj")
    return op_code


def _spmv_bsr_op_to_name(op):
    return SPMV_BSR_OP_NAMES[_normalize_spmv_bsr_op(op)]


def _spmv_bsr_op_transposes(op):
    return _normalize_spmv_bsr_op(op) in (SPMV_BSR_OP_TRANS, SPMV_BSR_OP_CONJ_TRANS)


def _normalize_spmv_bsr_algorithm(use_opt=False):
    if isinstance(use_opt, str):
        token = use_opt.strip().lower().replace("-", "_")
        if token in ("false", "0", "no", "base", "spmv_bsr_base"):
            return SPMV_BSR_ALG_BASE
        if token in ("true", "1", "yes", "opt", "auto", "blockrow_reduce", "spmv_bsr_blockrow_reduce"):
            return SPMV_BSR_ALG_BLOCKROW_REDUCE
        raise ValueError("use_opt must be False, True, 'base', 'auto', or 'blockrow_reduce'")
    return SPMV_BSR_ALG_BLOCKROW_REDUCE if bool(use_opt) else SPMV_BSR_ALG_BASE


def _normalize_spmv_bsr_index_fallback_policy(index_fallback_policy):
    policy = str(index_fallback_policy).lower()
    if policy not in ("auto", "strict"):
        raise ValueError("index_fallback_policy must be 'auto' or 'strict'")
    return policy


class PreparedBsrSpmv:
    """Prepared BSR metadata for repeated SpMV calls (and, for trans / conj, A^T)."""

    __slots__ = (
        "data",
        "kernel_indices",
        "kernel_indptr",
        "shape",
        "n_rows",
        "n_cols",
        "padded_n_rows",
        "padded_n_cols",
        "block_dim",
        "n_block_rows",
        "n_block_cols",
        "nnzb",
        "stored_nnz",
        "block_row_lengths",
        "max_block_row_nnz",
        "block_nnz",
        "max_segments",
        "op",
        "transpose",
        "index_fallback_policy",
        "index_fallback_applied",
        "index_fallback_reason",
        "_t_data",
        "_t_indices",
        "_t_indptr",
    )

    def __init__(
        self,
        data,
        kernel_indices,
        kernel_indptr,
        shape,
        block_dim,
        n_block_rows,
        n_block_cols,
        block_nnz,
        max_segments,
        max_block_row_nnz,
        block_row_lengths=None,
        op=None,
        transpose=False,
        index_fallback_policy="auto",
        index_fallback_applied=False,
        index_fallback_reason=None,
    ):
        self.data = data
        self.kernel_indices = kernel_indices
        self.kernel_indptr = kernel_indptr
        self.shape = (int(shape[0]), int(shape[1]))
        self.n_rows = int(shape[0])
        self.n_cols = int(shape[1])
        self.block_dim = int(block_dim)
        self.n_block_rows = int(n_block_rows)
        self.n_block_cols = int(n_block_cols)
        self.padded_n_rows = self.n_block_rows * self.block_dim
        self.padded_n_cols = self.n_block_cols * self.block_dim
        self.nnzb = int(data.shape[0])
        self.stored_nnz = int(data.numel())
        if block_row_lengths is None:
            block_row_lengths = kernel_indptr[1:] - kernel_indptr[:-1]
        self.block_row_lengths = block_row_lengths
        self.max_block_row_nnz = int(max_block_row_nnz)
        self.block_nnz = int(block_nnz)
        self.max_segments = int(max_segments)
        self.op = _normalize_spmv_bsr_op(op, transpose=transpose)
        self.transpose = _spmv_bsr_op_transposes(self.op)
        self.index_fallback_policy = str(index_fallback_policy).lower()
        self.index_fallback_applied = bool(index_fallback_applied)
        self.index_fallback_reason = index_fallback_reason
        self._t_data = self._t_indices = self._t_indptr = None

    def transposed(self, op_code):
        """A^T (conjugated for conj) as (blocks, indices int32, indptr int64), built once."""
        conj = op_code == SPMV_BSR_OP_CONJ_TRANS and self.data.is_complex()
        key = "conj" if conj else "trans"
        if self._t_data is None or self._t_data[0] != key:
            t_idx, t_ptr, perm = _csr.transpose_pattern(
                self.kernel_indices, self.kernel_indptr, (self.n_block_rows, self.n_block_cols),
                torch.int32, torch.int64,
            )
            blocks = torch.empty_like(self.data)
            nat.check(
                nat.lib().fsb_bsr_transpose_values(
                    nat.dtype_code(self.data.dtype), nat.ptr(self.data), nat.ptr(perm), self.nnzb, self.block_dim,
                    1 if conj else 0, nat.ptr(blocks), nat.stream_of(self.data.device),
                ),
                "fsb_bsr_transpose_values",
            )
            self._t_data = (key, blocks)
            self._t_indices = t_idx
            self._t_indptr = t_ptr
        return self._t_data[1], self._t_indices, self._t_indptr


def _prepare_spmv_bsr_matrix(data, indices, indptr, shape, block_dim):
    if not all(torch.is_tensor(t) for t in (data, indices, indptr)):
        raise TypeError("data, indices, indptr must all be torch.Tensor")
    if data.ndim != 3:
        raise ValueError("data must have shape (nnzb, block_dim, block_dim)")
    if indices.ndim != 1 or indptr.ndim != 1:
        raise ValueError("indices and indptr must be 1D tensors")
    n_rows, n_cols = int(shape[0]), int(shape[1])
    block_dim = int(block_dim)
    if block_dim <= 1:
        raise ValueError("block_dim must be greater than 1 for BSR SpMV")
    if data.shape[1] != block_dim or data.shape[2] != block_dim:
        raise ValueError("data block dimensions must match block_dim")
    n_block_rows = (n_rows + block_dim - 1) // block_dim
    n_block_cols = (n_cols + block_dim - 1) // block_dim
    if indptr.numel() != n_block_rows + 1:
        raise ValueError(f"indptr length must be n_block_rows+1={n_block_rows + 1}, got {indptr.numel()}")
    if data.shape[0] != indices.numel():
        raise ValueError("data.shape[0] and indices length must both equal nnzb")
    if not all(t.is_cuda for t in (data, indices, indptr)):
        raise ValueError("data, indices, indptr must be CUDA tensors")
    if not all(t.device == data.device for t in (indices, indptr)):
        raise ValueError("data, indices, indptr must be on the same CUDA device")
    if data.dtype not in SUPPORTED_SPMV_BSR_VALUE_DTYPES:
        raise TypeError(_spmv_bsr_dtype_error_message())
    if indices.dtype not in SUPPORTED_INDEX_DTYPES:
        raise TypeError("indices dtype must be torch.int32 or torch.int64")
    if indptr.dtype not in SUPPORTED_INDEX_DTYPES:
        raise TypeError("indptr dtype must be torch.int32 or torch.int64")
    data = data.contiguous()
    indices = indices.contiguous()
    indptr = indptr.contiguous()
    facts = _csr.inspect_csr(indices, indptr, n_block_rows, indices.numel())
    if facts["first"] != 0:
        raise ValueError("indptr must start at zero")
    if facts["last"] != data.shape[0]:
        raise ValueError("indptr[-1] must equal nnzb")
    if facts["decreasing"]:
        raise ValueError("indptr must be non-decreasing")
    if indices.numel() > 0 and (facts["min_col"] < 0 or facts["max_col"] >= n_block_cols):
        raise IndexError("indices out of range for n_block_cols")
    block_row_lengths = indptr[1:] - indptr[:-1]
    return (data, indices, indptr, n_rows, n_cols, n_block_rows, n_block_cols, block_row_lengths,
            int(facts["max_row_nnz"]))


def prepare_spmv_bsr(
    data,
    indices,
    indptr,
    shape,
    block_dim,
    block_nnz=128,
    max_segments=None,
    transpose=False,
    op=None,
    use_opt=False,
    index_fallback_policy="auto",
):
    index_fallback_policy = _normalize_spmv_bsr_index_fallback_policy(index_fallback_policy)
    op_code = _normalize_spmv_bsr_op(op, transpose=transpose)
    algorithm = _normalize_spmv_bsr_algorithm(use_opt)
    if algorithm == SPMV_BSR_ALG_BLOCKROW_REDUCE and op_code != SPMV_BSR_OP_NON:
        raise ValueError("spmv_bsr_blockrow_reduce only supports op='non'")
    if algorithm == SPMV_BSR_ALG_BLOCKROW_REDUCE and int(block_dim) not in (2, 4, 8, 16):
        raise ValueError("spmv_bsr_blockrow_reduce supports block_dim values 2, 4, 8, and 16")
    (data, indices, indptr, n_rows, n_cols, n_block_rows, n_block_cols, block_row_lengths,
     max_block_row_nnz) = _prepare_spmv_bsr_matrix(data, indices, indptr, shape, block_dim)
    block_nnz_use = int(block_nnz)
    if block_nnz_use <= 0:
        raise ValueError("block_nnz must be positive")
    if max_segments is None:
        max_segments_use = max((max_block_row_nnz + block_nnz_use - 1) // block_nnz_use, 1)
        while max_segments_use > 2048 and block_nnz_use < 65536:
            block_nnz_use *= 2
            max_segments_use = max((max_block_row_nnz + block_nnz_use - 1) // block_nnz_use, 1)
    else:
        max_segments_use = max(1, int(max_segments))
    prepared = PreparedBsrSpmv(
        data=data,
        kernel_indices=indices,
        kernel_indptr=indptr,
        shape=shape,
        block_dim=block_dim,
        n_block_rows=n_block_rows,
        n_block_cols=n_block_cols,
        block_nnz=block_nnz_use,
        max_segments=max_segments_use,
        max_block_row_nnz=max_block_row_nnz,
        block_row_lengths=block_row_lengths,
        op=op_code,
        index_fallback_policy=index_fallback_policy,
    )
    if _spmv_bsr_op_transposes(op_code):
        prepared.transposed(op_code)
    return prepared


def _validate_spmv_bsr_x(x, prepared, op_code):
    if x is None or not torch.is_tensor(x):
        raise TypeError("x must be a torch.Tensor")
    if x.ndim != 1:
        raise ValueError("x must be a 1D tensor")
    if not x.is_cuda:
        raise ValueError("x must be a CUDA tensor")
    if x.dtype != prepared.data.dtype:
        raise TypeError("x dtype must match sparse matrix dtype")
    logical_expected = prepared.n_rows if _spmv_bsr_op_transposes(op_code) else prepared.n_cols
    padded_expected = prepared.padded_n_rows if _spmv_bsr_op_transposes(op_code) else prepared.padded_n_cols
    if x.numel() not in (logical_expected, padded_expected):
        raise ValueError(
            f"x length must be {logical_expected} or padded length {padded_expected}, got {x.numel()}"
        )
    if x.device != prepared.data.device:
        raise ValueError("x must be on the same device as sparse matrix data")
    x = x.contiguous()
    if x.numel() == padded_expected:
        return x
    padded = torch.zeros(padded_expected, dtype=x.dtype, device=x.device)
    padded[: x.numel()].copy_(x)
    return padded


def _native_spmv_bsr(prepared, x, op_code, out=None):
    """One native launch; returns y of the padded output length."""
    if _spmv_bsr_op_transposes(op_code):
        blocks, indices, indptr = prepared.transposed(op_code)
        n_brows, n_bcols = prepared.n_block_cols, prepared.n_block_rows
    else:
        blocks, indices, indptr = prepared.data, prepared.kernel_indices, prepared.kernel_indptr
        n_brows, n_bcols = prepared.n_block_rows, prepared.n_block_cols
    y = out if out is not None else torch.empty(n_brows * prepared.block_dim, dtype=prepared.data.dtype,
                                                device=prepared.data.device)
    nat.check(
        nat.lib().fsb_bsr_spmv(
            nat.dtype_code(prepared.data.dtype), nat.ptr(blocks), nat.ptr(indices), nat.is64(indices),
            nat.ptr(indptr), nat.is64(indptr), n_brows, n_bcols, prepared.block_dim, nat.ptr(x), nat.ptr(y),
            nat.stream_of(prepared.data.device),
        ),
        "fsb_bsr_spmv",
    )
    return y


def _blockrow_reduce_buckets(prepared):
    """FlagSparse's block-row-length buckets (spmv_bsr.py:684-705), computed natively."""
    rows = _csr.bucketize_rows(prepared.kernel_indptr, prepared.n_block_rows,
                               [high for _, _, high, _, _ in _BLOCKROW_REDUCE_BUCKETS])
    buckets = []
    for (label, _, _, block_nnz, direct), r in zip(_BLOCKROW_REDUCE_BUCKETS, rows):
        if r.numel() == 0:
            continue
        segments = 1 if direct else max(1, (prepared.max_block_row_nnz + block_nnz - 1) // block_nnz)
        buckets.append({"label": label, "rows": r, "block_nnz": block_nnz, "segments": segments,
                        "direct_store": direct})
    return buckets


def _run_spmv_bsr_algorithm(prepared, x, op_code, algorithm, collect_timing=False, out=None):
    empty = {"process_cpu_ms": 0.0, "process_gpu_ms": None, "compute_ms": None, "bucket_counts": None,
             "launch_configs": None}
    if algorithm == SPMV_BSR_ALG_BLOCKROW_REDUCE and op_code != SPMV_BSR_OP_NON:
        raise ValueError("spmv_bsr_blockrow_reduce only supports op='non'")
    if not collect_timing:
        return _native_spmv_bsr(prepared, x, op_code, out=out), empty
    torch.cuda.synchronize()
    process_gpu_ms = 0.0
    buckets = None
    if algorithm == SPMV_BSR_ALG_BLOCKROW_REDUCE:
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record()
        buckets = _blockrow_reduce_buckets(prepared)
        p1.record()
        torch.cuda.synchronize()
        process_gpu_ms = p0.elapsed_time(p1)
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record()
    y = _native_spmv_bsr(prepared, x, op_code, out=out)
    c1.record()
    torch.cuda.synchronize()
    timing = {
        "process_cpu_ms": 0.0,
        "process_gpu_ms": process_gpu_ms,
        "compute_ms": c0.elapsed_time(c1),
        "bucket_counts": None,
        "launch_configs": None,
    }
    if buckets is not None:
        timing["bucket_counts"] = [{"bucket": b["label"], "rows": int(b["rows"].numel())} for b in buckets]
        timing["launch_configs"] = [{"bucket": b["label"], "block_nnz": b["block_nnz"], "segments": b["segments"],
                                     "direct_store": b["direct_store"]} for b in buckets]
    return y, timing


def flagsparse_spmv_bsr(
    data=None,
    indices=None,
    indptr=None,
    x=None,
    shape=None,
    block_dim=None,
    block_nnz=128,
    max_segments=None,
    out=None,
    return_time=False,
    return_meta=False,
    prepared=None,
    transpose=None,
    op=None,
    use_opt=False,
    index_fallback_policy="auto",
):
    """BSR SpMV on the native kernel; returns y of the padded length
    (n_block_rows * block_dim, or n_block_cols * block_dim for trans / conj)."""
    op_explicit = op is not None
    op_code = _normalize_spmv_bsr_op(op, transpose=False if transpose is None else bool(transpose))
    if op_explicit and transpose is not None and bool(transpose) != _spmv_bsr_op_transposes(op_code):
        raise ValueError("transpose conflicts with op")
    algorithm = _normalize_spmv_bsr_algorithm(use_opt)
    if algorithm == SPMV_BSR_ALG_BLOCKROW_REDUCE and op_code != SPMV_BSR_OP_NON:
        raise ValueError("spmv_bsr_blockrow_reduce only supports op='non'")
    if prepared is None:
        if any(arg is None for arg in (data, indices, indptr, shape, block_dim)):
            raise ValueError(
                "data, indices, indptr, shape, and block_dim are required when prepared is not provided"
            )
        prepared = prepare_spmv_bsr(
            data, indices, indptr, shape, block_dim, block_nnz=block_nnz, max_segments=max_segments, op=op_code,
            use_opt=algorithm, index_fallback_policy=index_fallback_policy,
        )
    else:
        if op_explicit and op_code != prepared.op:
            raise ValueError(
                f"op={_spmv_bsr_op_to_name(op_code)} does not match prepared.op={_spmv_bsr_op_to_name(prepared.op)}"
            )
        if not op_explicit and transpose is not None and bool(transpose) != prepared.transpose:
            raise ValueError(
                f"transpose={bool(transpose)} does not match prepared.transpose={prepared.transpose}"
            )
        if not op_explicit:
            op_code = prepared.op
    if algorithm == SPMV_BSR_ALG_BLOCKROW_REDUCE and op_code != SPMV_BSR_OP_NON:
        raise ValueError("spmv_bsr_blockrow_reduce only supports op='non'")
    if algorithm == SPMV_BSR_ALG_BLOCKROW_REDUCE and prepared.block_dim not in (2, 4, 8, 16):
        raise ValueError("spmv_bsr_blockrow_reduce supports block_dim values 2, 4, 8, and 16")
    x = _validate_spmv_bsr_x(x, prepared, op_code)
    out_len = (prepared.padded_n_cols if _spmv_bsr_op_transposes(op_code) else prepared.padded_n_rows)
    if out is not None:
        if not out.is_cuda:
            raise ValueError("out must be a CUDA tensor")
        if out.device != prepared.data.device:
            raise ValueError("out must be on the same CUDA device as the result")
        if out.shape != (out_len,) or out.dtype != prepared.data.dtype:
            raise ValueError("out shape/dtype must match result")
    direct_out = out if (out is not None and out.is_contiguous()) else None
    do_timing = bool(return_time or return_meta)
    if do_timing:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
    y, alg_timing = _run_spmv_bsr_algorithm(prepared, x, op_code, algorithm, collect_timing=do_timing,
                                            out=direct_out)
    if do_timing:
        torch.cuda.synchronize()
        wall_total_ms = (time.perf_counter() - t0) * 1000.0
        compute_ms = alg_timing["compute_ms"]
        process_cpu_ms = alg_timing["process_cpu_ms"]
        process_gpu_ms = alg_timing["process_gpu_ms"]
        op_total_ms = (process_cpu_ms + process_gpu_ms + compute_ms
                       if process_gpu_ms is not None and compute_ms is not None else wall_total_ms)
    else:
        compute_ms = process_cpu_ms = process_gpu_ms = op_total_ms = None
    if out is not None and y is not out:
        out.copy_(y)
        y = out
    if return_meta:
        meta = {
            "algorithm": algorithm,
            "op": _spmv_bsr_op_to_name(op_code),
            "block_dim": prepared.block_dim,
            "logical_shape": prepared.shape,
            "padded_shape": (prepared.padded_n_rows, prepared.padded_n_cols),
            "n_block_rows": prepared.n_block_rows,
            "n_block_cols": prepared.n_block_cols,
            "nnzb": prepared.nnzb,
            "stored_nnz": prepared.stored_nnz,
            "symbolic_ms": (process_cpu_ms or 0.0) + (process_gpu_ms or 0.0) if do_timing else None,
            "process_cpu_ms": process_cpu_ms,
            "process_gpu_ms": process_gpu_ms,
            "compute_ms": compute_ms,
            "op_total_ms": op_total_ms,
            "bucket_counts": alg_timing["bucket_counts"],
            "launch_configs": alg_timing["launch_configs"],
            "index_fallback_applied": prepared.index_fallback_applied,
            "index_fallback_reason": prepared.index_fallback_reason,
        }
        if return_time:
            return y, op_total_ms, meta
        return y, meta
    if return_time:
        return y, op_total_ms
    return y
