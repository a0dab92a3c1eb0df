"""CSR SpMM opt-alg2 host code over the sm_100a native kernel.

Mirror of FlagSparse ``sparse_operations/spmm_csr_opt_alg2.py``: the same
``PreparedCsrSpmmOptAlg2`` slots (``:39-76``), prepare functions
(``:916-941``), runtime validation messages (``:943-975``), entry points
(``:1136-1241``) and meta keys (``:1073-1134``).  The reference launches one
Triton kernel per row-length bucket; here one ``fsb_spmm_csr`` launch covers
every row, and the buckets are reported as row-length classes in meta.
"""

import time

import torch

from . import _csr
from .spmm_csr import _native_spmm_into, _prepare_spmm_csr_matrix, _spmm_plan

SUPPORTED_SPMM_OPT_ALG2_DTYPES = (torch.float32, torch.float64, torch.complex64, torch.complex128)

# Labels, kinds and row-length bounds of the reference's alg2 buckets
# (spmm_csr_opt_alg2.py:79-178).
_SPMM_OPT_ALG2_CLASSES = (
    ("short_16", "batched2d", 16),
    ("short_64", "batched2d", 64),
    ("row_256", "row2d", 256),
    ("seg_1024", "row2d_segmented", 1024),
    ("seg_long", "row2d_segmented", None),
)


class PreparedCsrSpmmOptAlg2:
    """Cached CSR metadata for repeated alg2 CSR SpMM calls on the same sparse matrix."""

    __slots__ = (
        "data",
        "kernel_indices",
        "kernel_indptr",
        "shape",
        "n_rows",
        "n_cols",
        "row_lengths",
        "max_row_nnz",
        "opt_buckets",
        "supports_opt",
        "_native",
    )

    def __init__(self, data, kernel_indices, kernel_indptr, shape, n_rows, n_cols, row_lengths, max_row_nnz,
                 opt_buckets):
        self.data = data
        self.kernel_indices = kernel_indices
        self.kernel_indptr = kernel_indptr
        self.shape = (int(shape[0]), int(shape[1]))
        self.n_rows = int(n_rows)
        self.n_cols = int(n_cols)
        self.row_lengths = row_lengths
        self.max_row_nnz = int(max_row_nnz)
        self.opt_buckets = opt_buckets
        self.supports_opt = data.dtype in SUPPORTED_SPMM_OPT_ALG2_DTYPES
        self._native = None

    def native_plan(self):
        if self._native is None:
            self._native = _spmm_plan(self.kernel_indptr, self.n_rows, self.data.dtype)
        return self._native


def prepare_spmm_csr_opt_alg2(data, indices, indptr, shape):
    data, kernel_indices, kernel_indptr, n_rows, n_cols, row_lengths, max_row_nnz = _prepare_spmm_csr_matrix(
        data, indices, indptr, shape
    )
    return PreparedCsrSpmmOptAlg2(data=data, kernel_indices=kernel_indices, kernel_indptr=kernel_indptr, shape=shape,
                                  n_rows=n_rows, n_cols=n_cols, row_lengths=row_lengths, max_row_nnz=max_row_nnz,
                                  opt_buckets=[])


def prepare_spmm_csr_opt_alg2_preprocess(data, indices, indptr, shape):
    return prepare_spmm_csr_opt_alg2(data, indices, indptr, shape)


def _validate_spmm_opt_alg2_runtime_inputs(prepared, B, out):
    if not prepared.supports_opt:
        raise TypeError("flagsparse_spmm_csr_opt_alg2 only supports float32, float64, complex64, and complex128")
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
    if out is not None:
        if not out.is_cuda:
            raise ValueError("out must be a CUDA tensor")
        if out.device != prepared.data.device:
            raise ValueError("out must be on the same CUDA device as sparse matrix data")
        if out.shape != (prepared.n_rows, int(B.shape[1])) or out.dtype != prepared.data.dtype:
            raise ValueError("out shape/dtype must match result")


def _build_spmm_opt_alg2_row_classes(prepared):
    """Stable row lists per alg2 row-length class, built natively, cached."""
    if prepared.opt_buckets:
        return prepared.opt_buckets
    lists = _csr.bucketize_rows(prepared.kernel_indptr, prepared.n_rows, [c[2] for c in _SPMM_OPT_ALG2_CLASSES])
    buckets = []
    lo = 0
    for (label, kind, hi), rows in zip(_SPMM_OPT_ALG2_CLASSES, lists):
        if rows.numel() > 0:
            buckets.append({"label": label, "kind": kind, "rows": rows, "min_row_nnz": lo, "max_row_nnz": hi})
        lo = (hi or 0) + 1
    prepared.opt_buckets = buckets
    return buckets


def _device_summary(device):
    props = torch.cuda.get_device_properties(device)
    return {"device_name": str(props.name), "sm_count": int(props.multi_processor_count),
            "warp_size": int(getattr(props, "warp_size", 32) or 32)}


def _native_spmm_csr_impl_opt_alg2_prepared(prepared, B, out=None, opt_buckets=None, return_meta=False):
    n = int(B.shape[1])
    C = out if (out is not None and out.is_contiguous()) else torch.empty(
        (prepared.n_rows, n), dtype=prepared.data.dtype, device=prepared.data.device)
    plan = prepared.native_plan()
    _native_spmm_into(prepared.data, prepared.kernel_indices, prepared.kernel_indptr, prepared.n_rows,
                      prepared.n_cols, B, plan, C)
    if out is not None and C is not out:
        out.copy_(C)
        C = out
    meta = None
    if return_meta:
        buckets = prepared.opt_buckets if opt_buckets is None else opt_buckets
        hits = [{"bucket_label": b["label"], "kind": b["kind"], "row_count": int(b["rows"].numel())} for b in buckets]
        meta = {
            **_device_summary(prepared.data.device),
            "bucket_hits": hits,
            "launch_configs": [{"kernel": "fsb_spmm_csr", "units": int(plan.n_units),
                                "long_row_slots": int(plan.n_slots), "warps_per_block": 8}],
            "max_row_nnz": prepared.max_row_nnz,
            "n_dense_cols": n,
        }
    return C, meta


def flagsparse_spmm_csr_opt_alg2(data=None, indices=None, indptr=None, B=None, shape=None, prepared=None, out=None,
                                 return_time=False, return_meta=False):
    """CSR SpMM opt-alg2 on the native kernel (float32 / float64 / complex)."""
    if prepared is not None and not isinstance(prepared, PreparedCsrSpmmOptAlg2):
        raise TypeError("prepared must be a PreparedCsrSpmmOptAlg2 instance")
    if prepared is None:
        if any(arg is None for arg in (data, indices, indptr, shape)):
            raise ValueError("data, indices, indptr, and shape are required when prepared is not provided")
        prepared = prepare_spmm_csr_opt_alg2(data, indices, indptr, shape)
    elif shape is not None:
        resolved = (int(shape[0]), int(shape[1]))
        if resolved != prepared.shape:
            raise ValueError(f"shape {resolved} does not match prepared.shape {prepared.shape}")
    _validate_spmm_opt_alg2_runtime_inputs(prepared, B, out)
    B = B.contiguous()
    do_timing = bool(return_time or return_meta)
    symbolic_ms = compute_ms = op_total_ms = None
    if do_timing:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
    buckets = _build_spmm_opt_alg2_row_classes(prepared)
    if do_timing:
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        symbolic_ms = (t1 - t0) * 1000.0
    C, meta = _native_spmm_csr_impl_opt_alg2_prepared(prepared, B, out=out, opt_buckets=buckets,
                                                       return_meta=return_meta)
    if do_timing:
        torch.cuda.synchronize()
        compute_ms = (time.perf_counter() - t1) * 1000.0
        op_total_ms = symbolic_ms + compute_ms
    if return_meta:
        meta = dict(meta or {})
        meta.update({"symbolic_ms": symbolic_ms, "compute_ms": compute_ms, "op_total_ms": op_total_ms})
    if return_time and return_meta:
        return C, op_total_ms, meta
    if return_time:
        return C, op_total_ms
    if return_meta:
        return C, meta
    return C


def flagsparse_spmm_csr_opt_alg2_preprocess(data=None, indices=None, indptr=None, B=None, shape=None,
                                            prepared=None, out=None, return_time=False, return_meta=False):
    """Compatibility alias of CSR SpMM opt-alg2."""
    return flagsparse_spmm_csr_opt_alg2(data=data, indices=indices, indptr=indptr, B=B, shape=shape,
                                        prepared=prepared, out=out, return_time=return_time,
                                        return_meta=return_meta)
