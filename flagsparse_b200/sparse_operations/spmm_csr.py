"""CSR SpMM host code over the sm_100a native kernel.

Drop-in mirror of FlagSparse ``sparse_operations/spmm_csr.py``: the same op
handling (``:23-58``), tolerance and error-metric helpers (``:61-141``),
validation messages (``:342-482``), launch-configuration helpers kept for
their meta / diagnostics (``:485-616``), the route registry and run API
(``:619-1000``, ``:2452-2717``), ``flagsparse_spmm_csr`` (``:3981-4137``) and
the ``spmm_csr_opt`` / ``_opt_alg1`` entry points (``:2720-2830``,
``:3156-3249``, ``:4137-4301``).  Every route computes with ``fsb_spmm_csr``:
one launch over the cached unit plan, fp32 accumulation for half / bfloat16 /
fp32 (no upcast copies), Dot2 compensated sums for the accuracy routes.
"""

import time
from dataclasses import dataclass

import torch

from . import _csr
from ._common import (
    SUPPORTED_INDEX_DTYPES,
    SUPPORTED_VALUE_DTYPES,
    _INDEX_LIMIT_INT32,
    _is_complex_dtype,
    _tolerance_for_dtype,
)

SUPPORTED_SPMM_VALUE_DTYPES = SUPPORTED_VALUE_DTYPES

SPMM_OP_NON = 0
SPMM_OP_TRANS = 1
SPMM_OP_CONJ_TRANS = 2
SPMM_OP_NAMES = {SPMM_OP_NON: "non", SPMM_OP_TRANS: "trans", SPMM_OP_CONJ_TRANS: "conj"}
_SPMM_OP_NAME_TO_CODE = {name: code for code, name in SPMM_OP_NAMES.items()}
_OP_ERROR = "op must be one of: 0=non, 1=trans, 2=conj"


def _normalize_spmm_op(op=None, transpose=False):
    if op is None:
        return SPMM_OP_TRANS if bool(transpose) else SPMM_OP_NON
    if isinstance(op, str):
        code = _SPMM_OP_NAME_TO_CODE.get(op.strip().lower())
        if code is None:
            raise ValueError(_OP_ERROR)
        return code
    try:
        code = int(op)
    except (TypeError, ValueError) as exc:
        raise ValueError(_OP_ERROR) from exc
    if code not in SPMM_OP_NAMES:
        raise ValueError(_OP_ERROR)
    return code


def _spmm_op_to_name(op):
    return SPMM_OP_NAMES[_normalize_spmm_op(op)]


def _spmm_op_transposes(op):
    return _normalize_spmm_op(op) in (SPMM_OP_TRANS, SPMM_OP_CONJ_TRANS)


# ---------------------------------------------------------------- tolerances / metrics

def _spmm_relative_threshold(value_dtype):
    """Max-relative-error threshold per dtype (spmm_csr.py:61-70)."""
    if value_dtype == torch.float16:
        return 5e-3
    if value_dtype == torch.bfloat16:
        return 1e-2
    if value_dtype in (torch.float32, torch.complex64):
        return 1e-6
    if value_dtype in (torch.float64, torch.complex128):
        return 1e-12
    return 1e-6


def _spmm_coo_reference_tolerance(value_dtype):
    """(atol, rtol) of the COO-reference comparison (spmm_csr.py:73-82)."""
    if value_dtype == torch.float16:
        return 1e-3, 2e-3
    if value_dtype == torch.bfloat16:
        return 0.016, 1e-1
    if value_dtype in (torch.float32, torch.complex64):
        return 1.3e-6, 1e-3
    if value_dtype in (torch.float64, torch.complex128):
        return 1e-7, 1e-5
    return 1e-6, 1e-5


def _spmm_error_metrics(candidate, reference):
    """Max / sum absolute and relative errors (spmm_csr.py:85-124)."""
    if candidate.shape != reference.shape:
        raise ValueError(
            f"candidate and reference must have the same shape, got {candidate.shape} vs {reference.shape}"
        )
    if candidate.numel() == 0:
        return {
            "max_abs_error": 0.0,
            "max_relative_error": 0.0,
            "sum_relative_error": 0.0,
            "reference_max_magnitude": 0.0,
            "reference_sum_magnitude": 0.0,
        }
    ref_mag = torch.abs(reference)
    diff = torch.abs(candidate - reference)
    max_abs = float(torch.max(diff).item())
    ref_max = float(torch.max(ref_mag).item())
    sum_abs = float(torch.sum(diff).item())
    ref_sum = float(torch.sum(ref_mag).item())
    if ref_max == 0.0:
        max_rel = 0.0 if max_abs == 0.0 else float("inf")
    else:
        max_rel = max_abs / ref_max
    if ref_sum == 0.0:
        sum_rel = 0.0 if sum_abs == 0.0 else float("inf")
    else:
        sum_rel = sum_abs / ref_sum
    return {
        "max_abs_error": max_abs,
        "max_relative_error": max_rel,
        "sum_relative_error": sum_rel,
        "reference_max_magnitude": ref_max,
        "reference_sum_magnitude": ref_sum,
    }


def _spmm_validation_metrics(candidate, reference):
    """Error metrics plus the threshold verdicts (spmm_csr.py:127-141)."""
    metrics = _spmm_error_metrics(candidate, reference)
    threshold = _spmm_relative_threshold(reference.dtype)
    atol, rtol = _tolerance_for_dtype(reference.dtype)
    metrics.update(
        {
            "relative_threshold": threshold,
            "matches_threshold": metrics["max_relative_error"] <= threshold,
            "strict_allclose_match": torch.allclose(candidate, reference, atol=atol, rtol=rtol),
        }
    )
    return metrics


def _spmm_opt_reference_error(candidate, reference, value_dtype):
    atol, rtol = _spmm_coo_reference_tolerance(value_dtype)
    if candidate.numel() == 0:
        return 0.0
    diff = torch.abs(candidate - reference)
    return float(torch.max(diff / (atol + rtol * torch.abs(reference))).item())


# ---------------------------------------------------------------- validation / transpose

def _prepare_spmm_csr_matrix(data, indices, indptr, shape):
    """Validation with the reference's messages (spmm_csr.py:342-404).

    One native inspection pass replaces the reference's chain of ``.item()``
    reductions.  Returns int32 kernel indices and int64 kernel row pointers.
    """
    if len(shape) != 2:
        raise ValueError("shape must be a 2-tuple: (n_rows, n_cols)")
    if data.ndim != 1 or indices.ndim != 1 or indptr.ndim != 1:
        raise ValueError("data, indices, and indptr must be 1D tensors")
    n_rows, n_cols = int(shape[0]), int(shape[1])
    if n_rows < 0 or n_cols < 0:
        raise ValueError("shape dimensions must be non-negative")
    if indptr.numel() != n_rows + 1:
        raise ValueError(f"indptr length must be n_rows+1={n_rows + 1}, got {indptr.numel()}")
    if data.numel() != indices.numel():
        raise ValueError("data and indices must have the same length (nnz)")
    if not all(t.is_cuda for t in (data, indices, indptr)):
        raise ValueError("data, indices, and indptr must be CUDA tensors")
    if not all(t.device == data.device for t in (indices, indptr)):
        raise ValueError("data, indices, and indptr must be on the same CUDA device")
    if data.dtype not in SUPPORTED_SPMM_VALUE_DTYPES:
        raise TypeError("data dtype must be one of: float16, bfloat16, float32, float64, complex64, complex128")
    if indices.dtype not in SUPPORTED_INDEX_DTYPES:
        raise TypeError("indices dtype must be torch.int32 or torch.int64")
    if indptr.dtype not in SUPPORTED_INDEX_DTYPES:
        raise TypeError("indptr dtype must be torch.int32 or torch.int64")

    nnz = data.numel()
    data = data.contiguous()
    indices = indices.contiguous()
    indptr = indptr.contiguous()
    facts = _csr.inspect_csr(indices, indptr, n_rows, nnz)
    if facts["first"] != 0:
        raise ValueError("indptr[0] must be 0")
    if facts["last"] != nnz:
        raise ValueError(f"indptr[-1] must equal nnz={nnz}, got {int(facts['last'])}")
    if facts["decreasing"]:
        raise ValueError("indptr must be nondecreasing")
    if nnz > 0:
        if facts["min_col"] < 0 or facts["max_col"] >= n_cols:
            raise IndexError("indices out of range for n_cols")
        if facts["max_col"] > _INDEX_LIMIT_INT32:
            raise ValueError("column indices exceed the int32 range supported by the Triton kernel")
    kernel_indices = indices.to(torch.int32) if indices.dtype == torch.int64 else indices
    kernel_indptr = indptr.to(torch.int64)
    row_lengths = kernel_indptr[1:] - kernel_indptr[:-1] if n_rows > 0 else kernel_indptr.new_empty((0,))
    return data, kernel_indices, kernel_indptr, n_rows, n_cols, row_lengths, int(facts["max_row_nnz"])


def _transpose_csr_for_spmm(data, indices, indptr, shape):
    """CSR of A^T with the reference's index-dtype rules (spmm_csr.py:407-445),
    computed by the native stable transpose (bit-identical)."""
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


def _materialize_spmm_csr_op(data, indices, indptr, shape, op_code):
    """CSR of op(A) (spmm_csr.py:448-457); conj folds into the native gather."""
    if op_code == SPMM_OP_NON:
        return data, indices, indptr, shape
    n_rows, n_cols = int(shape[0]), int(shape[1])
    nnz = data.numel()
    if nnz == 0:
        return _transpose_csr_for_spmm(data, indices, indptr, shape)
    out_index_dtype = indices.dtype if n_rows <= _INDEX_LIMIT_INT32 else torch.int64
    out_indptr_dtype = indptr.dtype if nnz <= _INDEX_LIMIT_INT32 else torch.int64
    t_indices, t_indptr, perm = _csr.transpose_pattern(indices, indptr, shape, out_index_dtype, out_indptr_dtype)
    conj = op_code == SPMM_OP_CONJ_TRANS and _is_complex_dtype(data.dtype)
    return _csr.gather_values(data, perm, conj=conj), t_indices, t_indptr, (n_cols, n_rows)


def _prepare_spmm_csr_inputs(data, indices, indptr, B, shape):
    """Matrix and dense-operand validation (spmm_csr.py:460-482)."""
    if B.ndim != 2:
        raise ValueError("B must be a 2D dense tensor")
    data, kernel_indices, kernel_indptr, n_rows, n_cols, _rl, _mx = _prepare_spmm_csr_matrix(
        data, indices, indptr, shape
    )
    if B.shape[0] != n_cols:
        raise ValueError(f"B.shape[0] must be n_cols={n_cols}, got {B.shape[0]}")
    if not B.is_cuda:
        raise ValueError("B must be a CUDA tensor")
    if B.device != data.device:
        raise ValueError("B must be on the same CUDA device as the sparse matrix")
    if B.dtype != data.dtype:
        raise TypeError("B dtype must match data dtype")
    B = B.contiguous()
    return data, kernel_indices, kernel_indptr, B, n_rows, n_cols, int(B.shape[1])


# ---------------------------------------------------------------- launch configuration
# The native kernel picks its own launch shape; these restate the reference's
# tile choices (spmm_csr.py:485-616, _alpha_spmm_alg1_common.py:20-37) because
# their overrides are validated and their values are reported in meta.

def _select_spmm_alg1_warp_and_factor(n_dense_cols):
    n = int(n_dense_cols)
    if n > 64:
        return 32, 4
    if n > 32:
        return 32, 2
    if n > 16:
        return 32, 1
    if n > 8:
        return 16, 1
    if n > 4:
        return 8, 1
    return 4, 1


def _resolve_spmm_alg1_launch_config(n_dense_cols, max_row_nnz, block_n=None, block_nnz=None, max_segments=None):
    warp_size, factor = _select_spmm_alg1_warp_and_factor(n_dense_cols)
    if block_n is None:
        block_n = warp_size * factor
    if block_nnz is None:
        block_nnz = warp_size
    if block_n <= 0 or block_nnz <= 0:
        raise ValueError("block_n and block_nnz must be positive when provided")
    if max_segments is not None and max_segments <= 0:
        raise ValueError("max_segments must be positive when provided")
    required = -(-int(max_row_nnz) // int(block_nnz)) if max_row_nnz > 0 else 0
    if max_segments is not None and required > int(max_segments):
        raise ValueError(
            "row nnz requires more CSR segments than the explicit max_segments override allows: "
            f"required {required}, provided {int(max_segments)}"
        )
    return {
        "block_n": int(block_n),
        "block_nnz": int(block_nnz),
        "max_segments": None if max_segments is None else int(max_segments),
        "required_segments": int(required),
        "warp_size": int(warp_size),
        "factor": int(factor),
        "max_row_nnz": int(max_row_nnz),
        "auto_max_segments": max_segments is None,
    }


def _normalize_spmm_base_device_props(device):
    props = torch.cuda.get_device_properties(device)
    return {
        "warp_size": max(1, int(getattr(props, "warp_size", 32) or 32)),
        "max_threads_per_block": max(32, int(getattr(props, "max_threads_per_block", 1024) or 1024)),
        "max_threads_per_mp": max(32, int(getattr(props, "max_threads_per_multi_processor", 2048) or 2048)),
    }


def _clip_spmm_base_num_warps(desired, device_props):
    warp = int(device_props["warp_size"])
    max_supported = min(16, max(1, int(device_props["max_threads_per_block"]) // warp),
                        max(1, int(device_props["max_threads_per_mp"]) // warp))
    supported = [v for v in (1, 2, 4, 8, 16) if v <= max_supported]
    if not supported:
        return 1
    desired = max(1, int(desired))
    for v in reversed(supported):
        if v <= desired:
            return v
    return supported[0]


def _resolve_spmm_base_triton_launch(dtype, n_dense_cols, max_row_nnz, block_n=None, block_nnz=None,
                                     max_segments=None, device_props=None):
    launch = _resolve_spmm_alg1_launch_config(n_dense_cols, max_row_nnz, block_n=block_n, block_nnz=block_nnz,
                                              max_segments=max_segments)
    if device_props is None:
        return {**launch, "num_warps": 1, "num_stages": 2}
    n, mx, bn = int(n_dense_cols), int(max_row_nnz), int(launch["block_n"])
    if n <= 16:
        warps = 1
    elif n <= 32:
        warps = 2
    elif n <= 64:
        warps = 4
    else:
        warps = 8 if mx >= 512 else 4
    if bn >= 128:
        warps = max(warps, 4)
    if mx >= 1024 and n > 32:
        warps = max(warps, 8)
    warps = min(warps, 8 if dtype in (torch.float64, torch.complex128) else 16)
    num_warps = _clip_spmm_base_num_warps(warps, device_props)
    if n > 64 or bn >= 128:
        stages = 1
    elif dtype in (torch.float64, torch.complex128) and mx >= 512:
        stages = 1
    else:
        stages = 2
    return {**launch, "num_warps": int(num_warps), "num_stages": int(stages)}


# ---------------------------------------------------------------- native compute

def _native_spmm_into(data, kernel_indices, kernel_indptr, n_rows, n_cols, B, plan, out, compensated=False):
    """out = A @ B on the native kernel; B, out row-major with unit column stride."""
    if n_rows == 0 or out.shape[1] == 0:
        return out
    return _csr.spmm(data, kernel_indices, kernel_indptr, n_rows, n_cols, B, plan, out, compensated=compensated)


def _spmm_plan(kernel_indptr, n_rows, dtype):
    return _csr.SpmmPlan(kernel_indptr, n_rows, dtype)


def _row_major_out(out, n_rows, n, dtype, device):
    """Output buffer the kernel can write: ``out`` itself when row-major, else a temporary."""
    if out is not None and out.is_contiguous():
        return out, False
    return torch.empty((n_rows, n), dtype=dtype, device=device), out is not None


def flagsparse_spmm_csr(
    data,
    indices,
    indptr,
    B,
    shape,
    block_n=None,
    block_nnz=None,
    max_segments=None,
    out=None,
    return_time=False,
    transpose=None,
    op=None,
    return_meta=False,
):
    """CSR SpMM on the sm_100a native kernel.

    op: 0/'non' for A @ B, 1/'trans' for A.T @ B, 2/'conj' for A.conj().T @ B.
    Same signature, checks, returns and meta as FlagSparse
    ``flagsparse_spmm_csr`` (spmm_csr.py:3981-4137).
    """
    op_explicit = op is not None
    op_code = _normalize_spmm_op(op, transpose=False if transpose is None else bool(transpose))
    if op_explicit and transpose is not None and bool(transpose) != _spmm_op_transposes(op_code):
        raise ValueError("transpose conflicts with op")
    if block_n is not None and block_n <= 0:
        raise ValueError("block_n must be positive when provided")
    if block_nnz is not None and block_nnz <= 0:
        raise ValueError("block_nnz must be positive when provided")
    if max_segments is not None and max_segments <= 0:
        raise ValueError("max_segments must be positive when provided")

    data, kernel_indices, kernel_indptr, n_rows, n_cols, _rl, max_row_nnz = _prepare_spmm_csr_matrix(
        data, indices, indptr, shape
    )
    if B.ndim != 2:
        raise ValueError("B must be a 2D dense tensor")
    eff_rows, eff_cols = (n_cols, n_rows) if _spmm_op_transposes(op_code) else (n_rows, n_cols)
    if B.shape[0] != eff_cols:
        raise ValueError(f"B.shape[0] must be n_cols={eff_cols}, got {B.shape[0]}")
    if not B.is_cuda:
        raise ValueError("B must be a CUDA tensor")
    if B.device != data.device:
        raise ValueError("B must be on the same CUDA device as the sparse matrix")
    if B.dtype != data.dtype:
        raise TypeError("B dtype must match data dtype")
    B = B.contiguous()
    n_dense = int(B.shape[1])
    if out is not None:
        if not out.is_cuda:
            raise ValueError("out must be a CUDA tensor")
        if out.device != data.device:
            raise ValueError("out must be on the same CUDA device as the inputs")
        if out.shape != (eff_rows, n_dense) or out.dtype != data.dtype:
            raise ValueError("out shape/dtype must match result")

    do_timing = bool(return_time or return_meta)
    symbolic_ms = 0.0 if do_timing else None
    compute_ms = None
    op_total_ms = None
    if do_timing:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
    if _spmm_op_transposes(op_code):
        data, kernel_indices, kernel_indptr, shape = _materialize_spmm_csr_op(
            data, kernel_indices, kernel_indptr, shape, op_code
        )
        n_rows, n_cols = int(shape[0]), int(shape[1])
        kernel_indices = kernel_indices.to(torch.int32)
        kernel_indptr = kernel_indptr.to(torch.int64)
        max_row_nnz = None
    if do_timing:
        torch.cuda.synchronize()
        if _spmm_op_transposes(op_code):
            symbolic_ms = (time.perf_counter() - t0) * 1000.0
    plan = _spmm_plan(kernel_indptr, n_rows, data.dtype)
    if max_segments is not None or block_nnz is not None:
        if max_row_nnz is None:
            max_row_nnz = int((kernel_indptr[1:] - kernel_indptr[:-1]).max().item()) if n_rows > 0 else 0
        _resolve_spmm_alg1_launch_config(n_dense, max_row_nnz, block_n=block_n, block_nnz=block_nnz,
                                         max_segments=max_segments)
    if do_timing:
        torch.cuda.synchronize()
        t1 = time.perf_counter()
    C, copy_back = _row_major_out(out, n_rows, n_dense, data.dtype, data.device)
    _native_spmm_into(data, kernel_indices, kernel_indptr, n_rows, n_cols, B, plan, C)
    if copy_back:
        out.copy_(C)
        C = out
    if do_timing:
        torch.cuda.synchronize()
        compute_ms = (time.perf_counter() - t1) * 1000.0
        op_total_ms = symbolic_ms + compute_ms
    if return_meta:
        meta = {
            "symbolic_ms": symbolic_ms,
            "compute_ms": compute_ms,
            "op_total_ms": op_total_ms,
            "op": _spmm_op_to_name(op_code),
        }
        if return_time:
            return C, op_total_ms, meta
        return C, meta
    if return_time:
        return C, op_total_ms
    return C


# ---------------------------------------------------------------- route API

@dataclass(frozen=True)
class SpmmCsrAlgorithm:
    """Registered CSR SpMM route (spmm_csr.py:619-628)."""

    name: str
    display_name: str
    supported_ops: tuple
    supported_dtypes: tuple
    run: object


class SpmmCsrAlgorithmUnavailable(RuntimeError):
    """Raised when a registered SpMM CSR route is unavailable in this runtime."""


class PreparedCsrSpmmRoute:
    """Matrix-level CSR SpMM route preparation (spmm_csr.py:631-677), plus the
    cached native plan of each materialised op."""

    __slots__ = (
        "data",
        "kernel_indices",
        "kernel_indptr",
        "shape",
        "n_rows",
        "n_cols",
        "row_lengths",
        "max_row_nnz",
        "nnz",
        "avg_nnz_per_row",
        "op",
        "alg",
        "_native",
    )

    def __init__(self, data, kernel_indices, kernel_indptr, shape, n_rows, n_cols, row_lengths, max_row_nnz, op,
                 alg):
        self.data = data
        self.kernel_indices = kernel_indices
        self.kernel_indptr = kernel_indptr
        self.shape = (int(shape[0]), int(shape[1]))
        self.n_rows = int(n_rows)
        self.n_cols = int(n_cols)
        self.row_lengths = row_lengths
        self.max_row_nnz = int(max_row_nnz)
        self.nnz = int(data.numel())
        self.avg_nnz_per_row = float(self.nnz) / float(max(1, self.n_rows))
        self.op = str(op)
        self.alg = str(alg)
        self._native = {}  # op name -> (materialised route, SpmmPlan)


def _normalize_spmm_csr_alg(alg):
    token = "auto" if alg is None else str(alg).strip().lower()
    if token in ("base", "csr", "csr_base"):
        return "csr_base"
    if token in ("base_accuracy", "csr_base_accuracy"):
        return "csr_base_accuracy"
    if token in ("alg1", "csr_alg1", "spmm_csr_alg1"):
        return "spmm_csr_alg1"
    if token in ("alg2", "csr_alg2", "spmm_csr_alg2"):
        return "spmm_csr_alg2"
    if token in ("alg2_accuracy", "csr_alg2_accuracy", "spmm_csr_alg2_accuracy"):
        return "spmm_csr_alg2_accuracy"
    if token in ("alg2_accuracy_hp", "csr_alg2_accuracy_hp", "spmm_csr_alg2_accuracy_hp"):
        return "spmm_csr_alg2_accuracy_hp"
    return token


def _normalize_dense_layout(layout):
    token = "row" if layout is None else str(layout).strip().lower()
    if token in ("auto", "default", "row", "row_major", "row-major", "c", "c_order"):
        return "row"
    if token in ("col", "column", "col_major", "column_major", "col-major", "column-major", "f", "fortran"):
        return "col"
    raise ValueError("dense_layout must be one of: auto, row, col")


def _is_col_major_2d(tensor):
    return (
        torch.is_tensor(tensor)
        and tensor.ndim == 2
        and tensor.stride(0) == 1
        and tensor.stride(1) >= max(1, int(tensor.shape[0]))
    )


def _dense_layout_name(tensor):
    if not torch.is_tensor(tensor) or tensor.ndim != 2:
        return "unknown"
    if tensor.is_contiguous():
        return "row"
    if _is_col_major_2d(tensor):
        return "col"
    return "strided"


def _empty_dense_layout(shape, dtype, device, layout):
    layout = _normalize_dense_layout(layout)
    rows, cols = int(shape[0]), int(shape[1])
    if layout == "col":
        return torch.empty_strided((rows, cols), (1, max(1, rows)), dtype=dtype, device=device)
    return torch.empty((rows, cols), dtype=dtype, device=device)


def _zeros_dense_layout(shape, dtype, device, layout):
    out = _empty_dense_layout(shape, dtype, device, layout)
    out.zero_()
    return out


def _materialize_dense_layout(tensor, layout):
    layout = _normalize_dense_layout(layout)
    if tensor.ndim != 2:
        raise ValueError("dense layout materialization expects a 2D tensor")
    if layout == "row":
        return tensor.contiguous()
    if _is_col_major_2d(tensor):
        return tensor
    out = _empty_dense_layout(tensor.shape, tensor.dtype, tensor.device, layout)
    out.copy_(tensor)
    return out


def _validate_spmm_route_runtime_inputs(prepared, B):
    if not isinstance(prepared, PreparedCsrSpmmRoute):
        raise TypeError("prepared must be a PreparedCsrSpmmRoute instance")
    if B is None:
        raise ValueError("B is required")
    if B.ndim != 2:
        raise ValueError("B must be a 2D dense tensor")
    if not B.is_cuda:
        raise ValueError("B must be a CUDA tensor")
    if B.device != prepared.data.device:
        raise ValueError("B must be on the same CUDA device as sparse matrix data")
    if B.dtype != prepared.data.dtype:
        raise TypeError("B dtype must match sparse matrix dtype")
    if B.shape[0] != prepared.n_cols:
        raise ValueError(f"B.shape[0] must be n_cols={prepared.n_cols}, got {B.shape[0]}")
    return B


def _spmm_csr_route_from_materialized(prepared, data, indices, indptr, shape, op_name):
    kernel_indptr = indptr.to(torch.int64)
    n_rows = int(shape[0])
    row_lengths = kernel_indptr[1:] - kernel_indptr[:-1] if n_rows > 0 else kernel_indptr.new_empty((0,))
    max_row_nnz = int(row_lengths.max().item()) if n_rows > 0 else 0
    kernel_indices = indices.to(torch.int32) if indices.dtype == torch.int64 else indices
    return PreparedCsrSpmmRoute(
        data=data.contiguous(), kernel_indices=kernel_indices.contiguous(), kernel_indptr=kernel_indptr.contiguous(),
        shape=shape, n_rows=n_rows, n_cols=int(shape[1]), row_lengths=row_lengths, max_row_nnz=max_row_nnz,
        op=op_name, alg=prepared.alg,
    )


def _route_native(prepared, op_name, timing=False):
    """(materialised route, native plan) for ``op_name``, cached on ``prepared``.

    The reference re-transposes on every trans / conj run (spmm_csr.py:815-842);
    the transpose and plan are built once here.  Returns the op-processing GPU
    time when ``timing`` (0.0 once cached).
    """
    hit = prepared._native.get(op_name)
    if hit is not None:
        return hit[0], hit[1], (0.0 if timing else None)
    start = end = None
    if timing:
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
    if op_name == "non":
        route = prepared
    else:
        data, indices, indptr, shape = _materialize_spmm_csr_op(
            prepared.data, prepared.kernel_indices, prepared.kernel_indptr, prepared.shape,
            _normalize_spmm_op(op_name),
        )
        route = _spmm_csr_route_from_materialized(prepared, data, indices, indptr, shape, op_name)
    plan = _spmm_plan(route.kernel_indptr, route.n_rows, route.data.dtype)
    prepared._native[op_name] = (route, plan)
    ms = None
    if timing:
        end.record()
        torch.cuda.synchronize()
        ms = start.elapsed_time(end)
    return route, plan, ms


def _run_native_route(route, plan, B, *, route_name, display_name, compensated, timing=False, diagnostics=False,
                      dense_layout="row", launch_version="native_v1"):
    B = _validate_spmm_route_runtime_inputs(route, B)
    dense_layout = _normalize_dense_layout(dense_layout)
    B_k = B.contiguous()
    n = int(B_k.shape[1])
    C_out = _empty_dense_layout((route.n_rows, n), route.data.dtype, route.data.device, dense_layout)
    compute_ms = None
    if timing:
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
    C_k, copy_back = _row_major_out(C_out, route.n_rows, n, route.data.dtype, route.data.device)
    _native_spmm_into(route.data, route.kernel_indices, route.kernel_indptr, route.n_rows, route.n_cols, B_k, plan,
                      C_k, compensated=compensated)
    if copy_back:
        C_out.copy_(C_k)
    C = C_out
    if timing:
        end.record()
        torch.cuda.synchronize()
        compute_ms = start.elapsed_time(end)
    B_rep = _materialize_dense_layout(B, dense_layout) if dense_layout == "col" else B_k
    meta = {
        "alg": route_name,
        "display_name": display_name,
        "op": route.op,
        "process_cpu_ms": 0.0,
        "process_gpu_ms": 0.0 if timing else None,
        "compute_ms": compute_ms,
        "dense_layout": dense_layout,
        "b_stride": tuple(int(v) for v in B_rep.stride()),
        "c_stride": tuple(int(v) for v in C.stride()),
        "output_layout": _dense_layout_name(C),
    }
    if diagnostics:
        launch = _resolve_spmm_base_triton_launch(route.data.dtype, n, route.max_row_nnz)
        meta["diagnostics"] = {
            "launch_config_scope": "matrix",
            "launch_config_count": 1,
            "bucket_count": 0,
            "long_row_count": 0,
            "launch_version": launch_version,
            "block_n": launch["block_n"],
            "block_nnz": launch["block_nnz"],
            "num_warps": 8,
            "num_stages": 1,
            "required_segments": launch["required_segments"],
            "warp_size": launch["warp_size"],
            "factor": launch["factor"],
            "native_units": int(plan.n_units),
            "native_long_row_slots": int(plan.n_slots),
            "compensated": bool(compensated),
            "dense_layout": dense_layout,
            "b_stride": meta["b_stride"],
            "c_stride": meta["c_stride"],
            "output_layout": meta["output_layout"],
        }
    return C, meta


def _route_runner(route_name, display_name, compensated):
    def run(route, plan, B, *, timing=False, diagnostics=False, dense_layout="row"):
        return _run_native_route(route, plan, B, route_name=route_name, display_name=display_name,
                                 compensated=compensated, timing=timing, diagnostics=diagnostics,
                                 dense_layout=dense_layout, launch_version=f"{route_name}_native_v1")
    run.__name__ = f"_run_{route_name}_route"
    return run


_ALL_OPS = tuple(SPMM_OP_NAMES.values())
_ROUTE_DTYPES = (torch.float32, torch.float64, torch.complex64, torch.complex128)

# Same ids, display names, ops and dtypes as spmm_csr.py:2452-2544.  The plain
# routes accumulate in the working precision; the accuracy routes use Dot2.
SPMM_CSR_ALGORITHMS = {
    "csr_base": SpmmCsrAlgorithm("csr_base", "Base", _ALL_OPS, SUPPORTED_SPMM_VALUE_DTYPES,
                                 _route_runner("csr_base", "Base", False)),
    "csr_base_accuracy": SpmmCsrAlgorithm("csr_base_accuracy", "BaseAccuracy", _ALL_OPS, _ROUTE_DTYPES,
                                          _route_runner("csr_base_accuracy", "BaseAccuracy", True)),
    "alpha_alg1_tle_opt": SpmmCsrAlgorithm("alpha_alg1_tle_opt", "TLEOpt", _ALL_OPS, _ROUTE_DTYPES,
                                           _route_runner("alpha_alg1_tle_opt", "TLEOpt", False)),
    "alpha_alg1_tle_opt2": SpmmCsrAlgorithm("alpha_alg1_tle_opt2", "TLEOpt2", _ALL_OPS, _ROUTE_DTYPES,
                                            _route_runner("alpha_alg1_tle_opt2", "TLEOpt2", False)),
    "spmm_csr_alg1": SpmmCsrAlgorithm("spmm_csr_alg1", "Alg1", _ALL_OPS, _ROUTE_DTYPES,
                                      _route_runner("spmm_csr_alg1", "Alg1", False)),
    "spmm_csr_alg2": SpmmCsrAlgorithm("spmm_csr_alg2", "Alg2", _ALL_OPS, _ROUTE_DTYPES,
                                      _route_runner("spmm_csr_alg2", "Alg2", False)),
    "spmm_csr_alg2_accuracy": SpmmCsrAlgorithm("spmm_csr_alg2_accuracy", "Alg2Accuracy", _ALL_OPS, _ROUTE_DTYPES,
                                               _route_runner("spmm_csr_alg2_accuracy", "Alg2Accuracy", True)),
    "spmm_csr_alg2_accuracy_hp": SpmmCsrAlgorithm(
        "spmm_csr_alg2_accuracy_hp", "Alg2AccuracyHP", _ALL_OPS, _ROUTE_DTYPES,
        _route_runner("spmm_csr_alg2_accuracy_hp", "Alg2AccuracyHP", True)),
}


def resolve_spmm_csr_algorithm(alg, op, dtype):
    token = _normalize_spmm_csr_alg(alg)
    if token == "auto":
        token = "csr_base"
    if token not in SPMM_CSR_ALGORITHMS:
        supported = ", ".join(sorted(SPMM_CSR_ALGORITHMS))
        raise ValueError(f"unsupported CSR SpMM algorithm {alg!r}; supported: auto, {supported}")
    algorithm = SPMM_CSR_ALGORITHMS[token]
    op_name = _spmm_op_to_name(op)
    if op_name not in algorithm.supported_ops:
        raise ValueError(f"algorithm {token!r} does not support op {op_name!r}")
    if dtype not in algorithm.supported_dtypes:
        raise TypeError(f"algorithm {token!r} does not support dtype {dtype}")
    return algorithm


def list_spmm_csr_algorithms(op=None, dtype=None):
    op_name = None if op is None else _spmm_op_to_name(op)
    names = []
    for name, algorithm in SPMM_CSR_ALGORITHMS.items():
        if op_name is not None and op_name not in algorithm.supported_ops:
            continue
        if dtype is not None and dtype not in algorithm.supported_dtypes:
            continue
        names.append(name)
    return tuple(names)


def prepare_spmm_csr_route(data, indices, indptr, shape, *, op="non", alg="auto"):
    """Prepare matrix-level CSR SpMM metadata for the route-based run API."""
    op_name = _spmm_op_to_name(_normalize_spmm_op(op))
    data, kernel_indices, kernel_indptr, n_rows, n_cols, row_lengths, max_row_nnz = _prepare_spmm_csr_matrix(
        data, indices, indptr, shape
    )
    resolved = _normalize_spmm_csr_alg(alg)
    if resolved != "auto":
        resolve_spmm_csr_algorithm(resolved, op_name, data.dtype)
    return PreparedCsrSpmmRoute(
        data=data, kernel_indices=kernel_indices, kernel_indptr=kernel_indptr, shape=shape, n_rows=n_rows,
        n_cols=n_cols, row_lengths=row_lengths, max_row_nnz=max_row_nnz, op=op_name, alg=resolved,
    )


def flagsparse_spmm_csr_run(prepared, B, *, alg=None, op=None, dense_layout="auto", return_time=False,
                            return_meta=False, timing=False, diagnostics=False):
    """Run a registered CSR SpMM route (spmm_csr.py:2607-2717 contract)."""
    if not isinstance(prepared, PreparedCsrSpmmRoute):
        raise TypeError("prepared must be a PreparedCsrSpmmRoute instance")
    op_name = prepared.op if op is None else _spmm_op_to_name(op)
    alg_name = prepared.alg if alg is None else _normalize_spmm_csr_alg(alg)
    algorithm = resolve_spmm_csr_algorithm(alg_name, op_name, prepared.data.dtype)
    dense_layout = _normalize_dense_layout(dense_layout)
    if B is None or not torch.is_tensor(B):
        raise TypeError("B must be a torch.Tensor")
    if B.ndim != 2:
        raise ValueError("B must be a 2D dense tensor")
    if not B.is_cuda:
        raise ValueError("B must be a CUDA tensor")
    if B.device != prepared.data.device:
        raise ValueError("B must be on the same CUDA device as sparse matrix data")
    if B.dtype != prepared.data.dtype:
        raise TypeError("B dtype must match sparse matrix dtype")

    start = torch.cuda.Event(enable_timing=True) if (return_time or return_meta) else None
    end = torch.cuda.Event(enable_timing=True) if (return_time or return_meta) else None
    if start is not None:
        torch.cuda.synchronize()
        start.record()
    route, plan, op_ms = _route_native(prepared, op_name, timing=bool(timing))
    C, route_meta = algorithm.run(route, plan, B, timing=bool(timing), diagnostics=bool(diagnostics),
                                  dense_layout=dense_layout)
    gpu_ms = None
    if end is not None:
        end.record()
        torch.cuda.synchronize()
        gpu_ms = start.elapsed_time(end)
    process_cpu_ms = float(route_meta.get("process_cpu_ms", 0.0) or 0.0)
    operator_ms = (process_cpu_ms + float(gpu_ms)) if gpu_ms is not None else None
    meta = None
    if return_meta:
        meta = {
            "alg": algorithm.name,
            "display_name": algorithm.display_name,
            "op": op_name,
            "operator_ms": operator_ms,
            "gpu_ms": gpu_ms,
            "process_cpu_ms": process_cpu_ms,
            "dense_layout": route_meta.get("dense_layout", dense_layout),
            "b_stride": route_meta.get("b_stride"),
            "c_stride": route_meta.get("c_stride"),
            "output_layout": route_meta.get("output_layout"),
        }
        if timing:
            meta["process_gpu_ms"] = float(op_ms or 0.0) + float(route_meta.get("process_gpu_ms") or 0.0)
            meta["compute_ms"] = route_meta.get("compute_ms")
        if diagnostics and "diagnostics" in route_meta:
            meta["diagnostics"] = route_meta["diagnostics"]
    if return_time and return_meta:
        return C, operator_ms, meta
    if return_time:
        return C, operator_ms
    if return_meta:
        return C, meta
    return C


# ---------------------------------------------------------------- spmm_csr_opt / _opt_alg1

_SPMM_OPT_LONG_ROW_THRESHOLD = 2048
_SPMM_OPT_SPLIT_BLOCK_NNZ = 256
# Row-length classes of the reference's alg1 buckets (spmm_csr.py:2798-2814);
# the native kernel has no per-bucket launch, the classes feed meta only.
_SPMM_CSR_ALG1_BUCKET_SPECS = (
    {"max_row_nnz": 32, "kind": "batched", "batch_rows": 8, "block_nnz": 32},
    {"max_row_nnz": 128, "kind": "batched", "batch_rows": 4, "block_nnz": 64},
    {"max_row_nnz": 512, "kind": "vector", "batch_rows": 1, "block_nnz": 128},
    {"max_row_nnz": _SPMM_OPT_LONG_ROW_THRESHOLD, "kind": "vector", "batch_rows": 1, "block_nnz": 128},
    {"max_row_nnz": None, "kind": "split", "batch_rows": 1, "block_nnz": _SPMM_OPT_SPLIT_BLOCK_NNZ},
)


class PreparedCsrSpmmOpt:
    """Cached CSR metadata for repeated SpMM-opt calls (spmm_csr.py:2720-2773)."""

    __slots__ = (
        "data",
        "kernel_indices",
        "kernel_indptr",
        "shape",
        "n_rows",
        "n_cols",
        "row_lengths",
        "max_row_nnz",
        "row_buckets",
        "supports_opt",
        "long_part_rows",
        "long_part_starts",
        "long_part_ends",
        "long_row_ids",
        "long_row_part_ptr",
        "long_row_fallback_only",
        "_native",
    )

    def __init__(self, data, kernel_indices, kernel_indptr, shape, n_rows, n_cols, row_lengths, max_row_nnz,
                 row_buckets, long_part_rows, long_part_starts, long_part_ends, long_row_ids, long_row_part_ptr,
                 long_row_fallback_only):
        self.data = data
        self.kernel_indices = kernel_indices
        self.kernel_indptr = kernel_indptr
        self.shape = (int(shape[0]), int(shape[1]))
        self.n_rows = int(n_rows)
        self.n_cols = int(n_cols)
        self.row_lengths = row_lengths
        self.max_row_nnz = int(max_row_nnz)
        self.row_buckets = row_buckets
        self.supports_opt = data.dtype in (torch.float32, torch.float64)
        self.long_part_rows = long_part_rows
        self.long_part_starts = long_part_starts
        self.long_part_ends = long_part_ends
        self.long_row_ids = long_row_ids
        self.long_row_part_ptr = long_row_part_ptr
        self.long_row_fallback_only = bool(long_row_fallback_only)
        self._native = None

    def native_plan(self):
        if self._native is None:
            self._native = _spmm_plan(self.kernel_indptr, self.n_rows, self.data.dtype)
        return self._native


def prepare_spmm_csr_opt_alg1(data, indices, indptr, shape):
    data, kernel_indices, kernel_indptr, n_rows, n_cols, row_lengths, max_row_nnz = _prepare_spmm_csr_matrix(
        data, indices, indptr, shape
    )
    row_index_dtype = torch.int32 if n_rows <= _INDEX_LIMIT_INT32 else torch.int64
    dev = data.device
    return PreparedCsrSpmmOpt(
        data=data, kernel_indices=kernel_indices, kernel_indptr=kernel_indptr, shape=shape, n_rows=n_rows,
        n_cols=n_cols, row_lengths=row_lengths, max_row_nnz=max_row_nnz, row_buckets=[],
        long_part_rows=torch.empty((0,), dtype=row_index_dtype, device=dev),
        long_part_starts=torch.empty((0,), dtype=torch.int64, device=dev),
        long_part_ends=torch.empty((0,), dtype=torch.int64, device=dev),
        long_row_ids=torch.empty((0,), dtype=row_index_dtype, device=dev),
        long_row_part_ptr=torch.zeros(1, dtype=torch.int64, device=dev),
        long_row_fallback_only=False,
    )


def prepare_spmm_csr_opt(data, indices, indptr, shape):
    return prepare_spmm_csr_opt_alg1(data, indices, indptr, shape)


def prepare_spmm_csr_opt_alg1_preprocess(data, indices, indptr, shape):
    return prepare_spmm_csr_opt_alg1(data, indices, indptr, shape)


def _build_spmm_csr_opt_runtime_symbolic(prepared):
    """Row classes and long-row split metadata (spmm_csr.py:3202-3246), built
    natively once and cached on ``prepared``; the launch itself needs only the
    unit plan."""
    if prepared.row_buckets:
        return prepared
    specs = _SPMM_CSR_ALG1_BUCKET_SPECS
    lists = _csr.bucketize_rows(prepared.kernel_indptr, prepared.n_rows, [s["max_row_nnz"] for s in specs])
    row_dtype = prepared.long_row_ids.dtype
    buckets = []
    lo = 0
    for spec, rows in zip(specs, lists):
        if rows.numel() > 0:
            buckets.append({"label": spec["kind"], "kind": spec["kind"], "rows": rows.to(row_dtype),
                            "min_row_nnz": lo, "max_row_nnz": spec["max_row_nnz"],
                            "batch_rows": spec["batch_rows"], "block_nnz": spec["block_nnz"]})
        lo = (spec["max_row_nnz"] or 0) + 1
    prepared.row_buckets = buckets
    long_rows = lists[-1].to(row_dtype)
    if long_rows.numel() > 0:
        ptr = prepared.kernel_indptr
        lr = long_rows.to(torch.int64)
        starts, ends = ptr[lr], ptr[lr + 1]
        parts = (ends - starts + _SPMM_OPT_SPLIT_BLOCK_NNZ - 1) // _SPMM_OPT_SPLIT_BLOCK_NNZ
        part_ptr = torch.zeros(lr.numel() + 1, dtype=torch.int64, device=ptr.device)
        part_ptr[1:] = torch.cumsum(parts, 0)
        owner = torch.repeat_interleave(torch.arange(lr.numel(), device=ptr.device), parts)
        k = torch.arange(owner.numel(), device=ptr.device) - part_ptr[owner]
        prepared.long_part_rows = long_rows[owner]
        prepared.long_part_starts = starts[owner] + k * _SPMM_OPT_SPLIT_BLOCK_NNZ
        prepared.long_part_ends = torch.minimum(prepared.long_part_starts + _SPMM_OPT_SPLIT_BLOCK_NNZ, ends[owner])
        prepared.long_row_ids = long_rows
        prepared.long_row_part_ptr = part_ptr
    return prepared


def _native_spmm_csr_impl_opt_prepared(prepared, B):
    C = torch.empty((prepared.n_rows, int(B.shape[1])), dtype=prepared.data.dtype, device=prepared.data.device)
    _native_spmm_into(prepared.data, prepared.kernel_indices, prepared.kernel_indptr, prepared.n_rows,
                      prepared.n_cols, B, prepared.native_plan(), C)
    return C, False


def _flagsparse_spmm_csr_opt_alg1_impl(data=None, indices=None, indptr=None, B=None, shape=None, prepared=None,
                                       out=None, return_time=False, return_meta=False,
                                       api_name="flagsparse_spmm_csr_opt_alg1"):
    if prepared is not None and not isinstance(prepared, PreparedCsrSpmmOpt):
        raise TypeError("prepared must be a PreparedCsrSpmmOpt instance")
    if prepared is None:
        if any(arg is None for arg in (data, indices, indptr, shape)):
            raise ValueError("data, indices, indptr, and shape are required when prepared is not provided")
        prepared = prepare_spmm_csr_opt_alg1(data, indices, indptr, shape)
    elif shape is not None:
        resolved = (int(shape[0]), int(shape[1]))
        if resolved != prepared.shape:
            raise ValueError(f"shape {resolved} does not match prepared.shape {prepared.shape}")
    if B is None:
        raise ValueError("B is required")
    if not prepared.supports_opt:
        raise TypeError(f"{api_name} only supports float32 and float64")
    if not B.is_cuda:
        raise ValueError("B must be a CUDA tensor")
    if B.device != prepared.data.device:
        raise ValueError("B must be on the same CUDA device as sparse matrix data")
    if B.ndim != 2:
        raise ValueError("B must be a 2D dense tensor")
    if B.dtype != prepared.data.dtype:
        raise TypeError("B dtype must match sparse matrix dtype")
    if B.shape[0] != prepared.n_cols:
        raise ValueError(f"B.shape[0] must be n_cols={prepared.n_cols}, got {B.shape[0]}")
    if out is not None:
        if not out.is_cuda:
            raise ValueError("out must be a CUDA tensor")
        if out.device != prepared.data.device:
            raise ValueError("out must be on the same CUDA device as sparse matrix data")
        if out.shape != (prepared.n_rows, int(B.shape[1])) or out.dtype != prepared.data.dtype:
            raise ValueError("out shape/dtype must match result")
    B = B.contiguous()
    do_timing = bool(return_time or return_meta)
    symbolic_ms = compute_ms = op_total_ms = None
    if do_timing:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
    runtime = _build_spmm_csr_opt_runtime_symbolic(prepared)
    if do_timing:
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        symbolic_ms = (t1 - t0) * 1000.0
    if out is not None and out.is_contiguous():
        C = _native_spmm_into(runtime.data, runtime.kernel_indices, runtime.kernel_indptr, runtime.n_rows,
                              runtime.n_cols, B, runtime.native_plan(), out)
    else:
        C, _fallback = _native_spmm_csr_impl_opt_prepared(runtime, B)
        if out is not None:
            out.copy_(C)
            C = out
    if do_timing:
        torch.cuda.synchronize()
        compute_ms = (time.perf_counter() - t1) * 1000.0
        op_total_ms = symbolic_ms + compute_ms
    if return_meta:
        meta = {
            "symbolic_ms": symbolic_ms,
            "compute_ms": compute_ms,
            "op_total_ms": op_total_ms,
            "long_part_count": int(runtime.long_part_rows.numel()),
            "long_row_count": int(runtime.long_row_ids.numel()),
            "bucket_count": int(len(runtime.row_buckets)),
        }
        if return_time:
            return C, op_total_ms, meta
        return C, meta
    if return_time:
        return C, op_total_ms
    return C


def flagsparse_spmm_csr_opt_alg1(data=None, indices=None, indptr=None, B=None, shape=None, prepared=None, out=None,
                                 return_time=False, return_meta=False):
    """CSR SpMM-opt alg1 (float32 / float64) on the native kernel."""
    return _flagsparse_spmm_csr_opt_alg1_impl(data, indices, indptr, B, shape, prepared, out, return_time,
                                              return_meta, api_name="flagsparse_spmm_csr_opt_alg1")


def flagsparse_spmm_csr_opt_alg1_preprocess(data=None, indices=None, indptr=None, B=None, shape=None, prepared=None,
                                            out=None, return_time=False, return_meta=False):
    """Compatibility alias of CSR SpMM-opt alg1."""
    return _flagsparse_spmm_csr_opt_alg1_impl(data, indices, indptr, B, shape, prepared, out, return_time,
                                              return_meta, api_name="flagsparse_spmm_csr_opt_alg1_preprocess")


def flagsparse_spmm_csr_opt(data=None, indices=None, indptr=None, B=None, shape=None, prepared=None, out=None,
                            return_time=False, return_meta=False):
    """Compatibility alias of CSR SpMM-opt alg1."""
    return flagsparse_spmm_csr_opt_alg1(data=data, indices=indices, indptr=indptr, B=B, shape=shape,
                                        prepared=prepared, out=out, return_time=return_time,
                                        return_meta=return_meta)
