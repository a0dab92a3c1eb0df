"""Shared dtypes, tolerances and helpers for the CSR operators.

Mirrors the public helpers of FlagSparse ``sparse_operations/_common.py``
(dtype tables ``:36-46``, ``_tolerance_for_dtype`` ``:113-122``, random CSR
builders ``:186-218``, timing helpers ``:340-405``).  Only torch is needed:
the compute path is the sm_100a native library, not Triton.
"""

import statistics
import time

import torch

SUPPORTED_VALUE_DTYPES = (
    torch.float16,
    torch.bfloat16,
    torch.float32,
    torch.float64,
    torch.complex64,
    torch.complex128,
)
SUPPORTED_INDEX_DTYPES = (torch.int32, torch.int64)
_INDEX_LIMIT_INT32 = 2**31 - 1

__all__ = (
    "SUPPORTED_VALUE_DTYPES",
    "SUPPORTED_INDEX_DTYPES",
    "_INDEX_LIMIT_INT32",
    "_is_complex_dtype",
    "_component_dtype_for_complex",
    "_tolerance_for_dtype",
    "_build_random_dense",
    "_build_random_csr",
    "_benchmark_cuda_op",
    "_benchmark_cuda_graph_op",
    "time",
    "torch",
)


def _is_complex_dtype(value_dtype):
    return value_dtype in (torch.complex64, torch.complex128)


def _component_dtype_for_complex(value_dtype):
    if value_dtype == torch.complex64:
        return torch.float32
    if value_dtype == torch.complex128:
        return torch.float64
    raise TypeError(f"Unsupported complex dtype: {value_dtype}")


def _tolerance_for_dtype(value_dtype):
    """(atol, rtol) per dtype, the same table FlagSparse applies to itself."""
    table = {
        torch.float16: (2e-3, 2e-3),
        torch.bfloat16: (1e-1, 1e-1),
        torch.float32: (1e-6, 1e-5),
        torch.complex64: (1e-6, 1e-5),
        torch.float64: (1e-10, 1e-8),
        torch.complex128: (1e-10, 1e-8),
    }
    return table.get(value_dtype, (1e-6, 1e-5))


def _build_random_dense(dense_size, value_dtype, device):
    if _is_complex_dtype(value_dtype):
        comp = _component_dtype_for_complex(value_dtype)
        return torch.complex(
            torch.randn(dense_size, dtype=comp, device=device),
            torch.randn(dense_size, dtype=comp, device=device),
        )
    if value_dtype in SUPPORTED_VALUE_DTYPES:
        return torch.randn(dense_size, dtype=value_dtype, device=device)
    raise TypeError(f"Unsupported value dtype: {value_dtype}")


def _build_random_csr(n_rows, n_cols, nnz, value_dtype, index_dtype, device):
    """Random CSR with uniformly placed nonzeros (duplicates allowed)."""
    if nnz <= 0 or n_rows <= 0 or n_cols <= 0:
        return (
            torch.empty(0, dtype=value_dtype, device=device),
            torch.empty(0, dtype=index_dtype, device=device),
            torch.zeros(n_rows + 1, dtype=torch.int64, device=device),
        )
    rows = torch.sort(torch.randint(0, n_rows, (nnz,), device=device)).values
    indptr = torch.zeros(n_rows + 1, dtype=torch.int64, device=device)
    indptr[1:] = torch.cumsum(torch.bincount(rows, minlength=n_rows), dim=0)
    indices = torch.randint(0, n_cols, (nnz,), dtype=index_dtype, device=device)
    return _build_random_dense(nnz, value_dtype, device), indices, indptr


def _benchmark_cuda_op(op, warmup, iters):
    """Mean wall time of ``op`` over ``iters`` calls after ``warmup`` calls (ms)."""
    output = None
    for _ in range(max(0, int(warmup))):
        output = op()
    iters = max(1, int(iters))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(iters):
        output = op()
    torch.cuda.synchronize()
    return output, (time.perf_counter() - t0) * 1000.0 / iters


def _benchmark_cuda_graph_op(op, *, graph_batch=100, warmup=20, repeats=10, capture_setup=None):
    """Median per-call time (ms) of ``op`` replayed from a CUDA graph of ``graph_batch`` calls."""
    graph_batch = max(1, int(graph_batch))
    torch.cuda.synchronize()
    stream = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(stream):
        if capture_setup is not None:
            capture_setup()
        op()
    stream.synchronize()
    with torch.cuda.graph(graph, stream=stream):
        for _ in range(graph_batch):
            op()
    stream.synchronize()
    with torch.cuda.stream(stream):
        for _ in range(max(0, int(warmup))):
            graph.replay()
    stream.synchronize()
    samples = []
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    for _ in range(max(1, int(repeats))):
        with torch.cuda.stream(stream):
            start.record()
            graph.replay()
            end.record()
        end.synchronize()
        samples.append(float(start.elapsed_time(end)) / graph_batch)
    return statistics.median(samples)
