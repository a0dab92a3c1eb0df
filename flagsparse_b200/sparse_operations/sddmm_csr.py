"""CSR SDDMM host code over the sm_100a native kernel.

Drop-in mirror of FlagSparse ``sparse_operations/sddmm_csr.py``: the same
``SDDMMPrepared`` slots (``:23-47``), launch-config table (``:50-57``),
pattern validation messages (``:60-92``), ``prepare_sddmm_csr`` (``:107-118``),
dense-input checks (``:219-243``), output checks (``:246-257``), diagnostic
variants (``:260-288``), ``_run_sddmm_prepared`` meta (``:291-384``),
and ``flagsparse_sddmm_csr`` (``:387-468``).  The compute is
``fsb_sddmm_csr``; ``allow_fallback`` is accepted for signature
compatibility but there is no fallback path (FlagSparse's torch fallback,
``_sddmm_reference`` at ``:471-483``, is not provided): a native failure
raises.
"""

import time

import torch

from .. import _native as nat

SUPPORTED_SDDMM_VALUE_DTYPES = (torch.float32, torch.float64)
SUPPORTED_SDDMM_DIAGNOSTIC_VARIANTS = ("baseline", "acc64", "acc64_out64", "altreduce")


class SDDMMPrepared:
    """Prepared CSR pattern metadata for SDDMM."""

    __slots__ = (
        "indices",
        "indptr",
        "shape",
        "n_rows",
        "n_cols",
        "nnz",
        "row_ids",
        "block_k",
        "num_warps",
    )

    def __init__(self, indices, indptr, shape, row_ids, block_k, num_warps):
        self.indices = indices
        self.indptr = indptr
        self.shape = (int(shape[0]), int(shape[1]))
        self.n_rows = self.shape[0]
        self.n_cols = self.shape[1]
        self.nnz = int(indices.numel())
        self.row_ids = row_ids
        self.block_k = int(block_k)
        self.num_warps = int(num_warps)


def _resolve_sddmm_launch_config(k):
    """(block_k, num_warps) the reference picks for dimension k; reported in meta."""
    if k <= 32:
        return 32, 2
    if k <= 64:
        return 64, 4
    if k <= 128:
        return 64, 4
    return 128, 8


def _prepare_sddmm_csr_pattern(indices, indptr, shape):
    if len(shape) != 2:
        raise ValueError("shape must be a 2-tuple")
    if indices.ndim != 1 or indptr.ndim != 1:
        raise ValueError("indices and indptr must be 1D tensors")
    n_rows, n_cols = int(shape[0]), int(shape[1])
    if n_rows < 0 or n_cols < 0:
        raise ValueError("shape dimensions must be non-negative")
    if indptr.numel() != n_rows + 1:
        raise ValueError(f"indptr length must be n_rows+1={n_rows + 1}, got {indptr.numel()}")
    if not indices.is_cuda or not indptr.is_cuda:
        raise ValueError("indices and indptr must be CUDA tensors")
    if indices.dtype != torch.int32:
        raise TypeError("indices dtype must be torch.int32")
    if indptr.dtype not in (torch.int32, torch.int64):
        raise TypeError("indptr dtype must be torch.int32 or torch.int64")
    from . import _csr

    indptr64 = indptr.to(torch.int64).contiguous()
    indices = indices.contiguous()
    nnz = int(indices.numel())
    facts = _csr.inspect_csr(indices, indptr64, n_rows, nnz)
    if facts["first"] != 0:
        raise ValueError("indptr[0] must be 0")
    if facts["last"] != nnz:
        raise ValueError(f"indptr[-1] must equal nnz={nnz}")
    if facts["decreasing"]:
        raise ValueError("indptr must be nondecreasing")
    if nnz > 0 and (facts["min_col"] < 0 or facts["max_col"] >= n_cols):
        raise IndexError("indices out of range for shape[1]")
    return indices, indptr64, (n_rows, n_cols)


def _build_row_ids(indptr):
    """int32 row of every nonzero (the reference's repeat_interleave), built natively."""
    n_rows = int(indptr.numel()) - 1
    if n_rows <= 0:
        return torch.empty(0, dtype=torch.int32, device=indptr.device)
    indptr = indptr.contiguous()
    nnz = int(indptr[-1].item())
    rows = torch.empty(nnz, dtype=torch.int32, device=indptr.device)
    nat.check(
        nat.lib().fsb_csr_row_ids(nat.ptr(indptr), nat.is64(indptr), n_rows, nnz, nat.ptr(rows),
                                  nat.stream_of(indptr.device)),
        "fsb_csr_row_ids",
    )
    return rows


def prepare_sddmm_csr(indices, indptr, shape, k_hint=64):
    indices, indptr, shape = _prepare_sddmm_csr_pattern(indices, indptr, shape)
    row_ids = _build_row_ids(indptr)
    block_k, num_warps = _resolve_sddmm_launch_config(int(k_hint))
    return SDDMMPrepared(indices=indices, indptr=indptr, shape=shape, row_ids=row_ids, block_k=block_k,
                         num_warps=num_warps)


def _validate_sddmm_dense_inputs(data, prepared, x, y):
    if x.ndim != 2 or y.ndim != 2:
        raise ValueError("x and y must be 2D dense tensors")
    if not x.is_cuda or not y.is_cuda:
        raise ValueError("x and y must be CUDA tensors")
    if x.device != y.device or x.device != prepared.indices.device:
        raise ValueError("x, y, and sparse pattern must be on the same CUDA device")
    if x.dtype not in SUPPORTED_SDDMM_VALUE_DTYPES:
        raise TypeError("x dtype must be torch.float32 or torch.float64")
    if y.dtype != x.dtype:
        raise TypeError("y dtype must match x dtype")
    if data is not None and data.dtype != x.dtype:
        raise TypeError("data dtype must match x/y dtype")
    if x.shape[0] != prepared.n_rows:
        raise ValueError(f"x.shape[0] must be n_rows={prepared.n_rows}, got {x.shape[0]}")
    if y.shape[0] != prepared.n_cols:
        raise ValueError(f"y.shape[0] must be n_cols={prepared.n_cols}, got {y.shape[0]}")
    if x.shape[1] != y.shape[1]:
        raise ValueError("x and y must have the same K dimension")
    if data is not None and data.numel() != prepared.nnz:
        raise ValueError("data length must equal nnz of sparse pattern")
    return int(x.shape[1])


def _prepare_validated_sddmm_out(prepared, x, out, out_dtype=None):
    nnz = prepared.nnz
    target = x.dtype if out_dtype is None else out_dtype
    if out is None:
        return torch.empty(nnz, dtype=target, device=x.device)
    if out.ndim != 1 or out.numel() != nnz:
        raise ValueError("out must be a 1D tensor with length nnz")
    if not out.is_cuda or out.device != x.device:
        raise ValueError("out must be a CUDA tensor on the same device as x")
    if out.dtype != target:
        raise TypeError("out dtype must match the requested output dtype")
    return out


def _normalize_sddmm_diagnostic_variant(variant):
    if variant is None:
        return "baseline"
    variant = str(variant).strip().lower()
    if variant not in SUPPORTED_SDDMM_DIAGNOSTIC_VARIANTS:
        supported = ", ".join(SUPPORTED_SDDMM_DIAGNOSTIC_VARIANTS)
        raise ValueError(f"Unsupported SDDMM diagnostic variant {variant!r}; expected one of: {supported}")
    return variant


def _sddmm_variant_flags(variant, value_dtype):
    """Native flags and accumulation name of a diagnostic variant (sddmm_csr.py:271-281)."""
    variant = _normalize_sddmm_diagnostic_variant(variant)
    if variant == "acc64":
        return nat.FSB_SDDMM_ACC64, "float64"
    if variant == "acc64_out64":
        return nat.FSB_SDDMM_ACC64 | nat.FSB_SDDMM_OUT64, "float64"
    return 0, ("float64" if value_dtype == torch.float64 else "float32")


def _resolve_sddmm_diagnostic_out_dtype(variant, value_dtype):
    if _normalize_sddmm_diagnostic_variant(variant) == "acc64_out64":
        return torch.float64
    return value_dtype


def _native_sddmm(row_ids, indices, x, y, data, alpha, beta, out, flags=0):
    """out = alpha * <x[row], y[col]> + beta * data on the native kernel (any of f16/bf16/f32/f64)."""
    nnz = int(indices.numel())
    if nnz == 0:
        return out
    k = int(x.shape[1])
    nat.check(
        nat.lib().fsb_sddmm_csr(
            nat.dtype_code(x.dtype), nat.ptr(row_ids), nat.ptr(indices), nnz,
            nat.ptr(x), int(x.stride(0)) if x.shape[0] > 1 else max(k, 1),
            nat.ptr(y), int(y.stride(0)) if y.shape[0] > 1 else max(k, 1), k,
            nat.ptr(data) if data is not None else None, float(alpha), float(beta), nat.ptr(out), int(flags),
            nat.stream_of(out.device),
        ),
        "fsb_sddmm_csr",
    )
    return out


def _run_sddmm_prepared(prepared, x, y, data, alpha, beta, out, allow_fallback=False, variant="baseline",
                        out_dtype=None):
    variant = _normalize_sddmm_diagnostic_variant(variant)
    target = _resolve_sddmm_diagnostic_out_dtype(variant, x.dtype) if out_dtype is None else out_dtype
    out = _prepare_validated_sddmm_out(prepared, x, out, out_dtype=target)
    flags, acc = _sddmm_variant_flags(variant, x.dtype)
    if target == torch.float64 and x.dtype != torch.float64:
        flags |= nat.FSB_SDDMM_ACC64 | nat.FSB_SDDMM_OUT64
        acc = "float64"
    if prepared.nnz == 0:
        return out, {"block_k": prepared.block_k, "num_warps": prepared.num_warps, "fallback_used": False,
                     "variant": variant, "acc_dtype": "float64" if target == torch.float64 else "float32",
                     "out_dtype": str(target).replace("torch.", "")}
    block_k, num_warps = _resolve_sddmm_launch_config(int(x.shape[1]))
    _native_sddmm(prepared.row_ids, prepared.indices, x.contiguous(), y.contiguous(),
                  data.contiguous() if data is not None else None, alpha, beta, out, flags)
    return out, {"block_k": block_k, "num_warps": num_warps, "fallback_used": False, "variant": variant,
                 "acc_dtype": acc, "out_dtype": str(out.dtype).replace("torch.", "")}


def flagsparse_sddmm_csr(data=None, indices=None, indptr=None, x=None, y=None, shape=None, alpha=1.0, beta=0.0,
                         prepared=None, out=None, return_time=False, return_meta=False, allow_fallback=False):
    """CSR SDDMM: out[p] = alpha * dot(x[row(p)], y[col(p)]) + beta * data[p]."""
    prepare_ms = 0.0
    if prepared is None:
        if any(v is None for v in (indices, indptr, shape)):
            raise ValueError("indices, indptr, and shape are required when prepared is not provided")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        k_hint = int(x.shape[1]) if (x is not None and x.ndim == 2) else 64
        prepared = prepare_sddmm_csr(indices, indptr, shape, k_hint=k_hint)
        torch.cuda.synchronize()
        prepare_ms = (time.perf_counter() - t0) * 1000.0
    elif not isinstance(prepared, SDDMMPrepared):
        raise TypeError("prepared must be a SDDMMPrepared instance")
    if x is None or y is None:
        raise ValueError("x and y are required")
    if data is None and float(beta) != 0.0:
        raise ValueError("data is required when beta is non-zero")
    k_dim = _validate_sddmm_dense_inputs(data, prepared, x, y)
    if k_dim == 0:
        out = _prepare_validated_sddmm_out(prepared, x, out)
        if beta == 0.0 or data is None:
            out.zero_()
        else:
            _native_sddmm(prepared.row_ids, prepared.indices, x, y, data, 0.0, beta, out)
        meta = {"prepare_ms": prepare_ms, "block_k": prepared.block_k, "num_warps": prepared.num_warps,
                "fallback_used": False}
        if return_time and return_meta:
            return out, 0.0, meta
        if return_time:
            return out, 0.0
        if return_meta:
            return out, meta
        return out
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out_tensor, launch_meta = _run_sddmm_prepared(prepared, x.contiguous(), y.contiguous(),
                                                  data.contiguous() if data is not None else None, alpha, beta, out,
                                                  allow_fallback=allow_fallback)
    torch.cuda.synchronize()
    elapsed_ms = (time.perf_counter() - t0) * 1000.0
    if return_time and return_meta:
        return out_tensor, elapsed_ms, {"prepare_ms": prepare_ms, **launch_meta}
    if return_time:
        return out_tensor, elapsed_ms
    if return_meta:
        return out_tensor, {"prepare_ms": prepare_ms, **launch_meta}
    return out_tensor

