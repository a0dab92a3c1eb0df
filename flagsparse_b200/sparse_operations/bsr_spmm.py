"""BSR SpMM with 16 x 16 blocks on the sm_100a tensor cores (``fsb_bsr16_spmm``).

FlagSparse has no BSR SpMM (its BSR support is SpMV, ``spmv_bsr.py``); this
operator serves matrices whose nonzeros come in dense 16 x 16 blocks, where a
block times a 16-row slab of B is a real dense contraction.  Values and B are
bfloat16 or float16; products accumulate in fp32 in tensor memory and C is
written in the value type.  Dense widths are multiples of 64 (one tcgen05.mma
covers a 128-column tile; a last tile of 64 columns loads and stores half).
"""

import torch

from .. import _native as nat
from . import _csr

SUPPORTED_BSR16_DTYPES = (torch.bfloat16, torch.float16)


class PreparedBsr16:
    """Validated BSR-16 pattern and values (int32 block columns, int64 block row pointers)."""

    __slots__ = ("blocks", "packed", "indices", "indptr", "shape", "n_brows", "n_bcols", "nnzb", "_err")

    # _err: one int32 in pinned host memory, which the kernel writes (a plain
    # store through the mapped address) when a bounded wait inside it expires.
    # The host reads it without synchronising: every call checks the word left
    # by earlier calls before it launches, and status() reports it on demand.

    def __init__(self, blocks, indices, indptr, shape):
        self.blocks = blocks
        # the blocks in the tensor cores' shared-memory layout, built once
        self.packed = torch.empty_like(blocks)
        nat.check(nat.lib().fsb_bsr16_pack(nat.dtype_code(blocks.dtype), nat.ptr(blocks), int(blocks.shape[0]),
                                           nat.ptr(self.packed), nat.stream_of(blocks.device)), "fsb_bsr16_pack")
        self.indices = indices
        self.indptr = indptr
        self.shape = (int(shape[0]), int(shape[1]))
        self.n_brows = self.shape[0] // 16
        self.n_bcols = self.shape[1] // 16
        self.nnzb = int(indices.numel())
        self._err = torch.zeros(1, dtype=torch.int32).pin_memory()

    def status(self, synchronize=False):
        """0, or 1 once a launch on this matrix gave up a bounded wait (its C is invalid).

        ``synchronize`` first waits for the work queued on the current stream."""
        if synchronize:
            torch.cuda.current_stream(self.blocks.device).synchronize()
        return int(self._err[0])

    def _raise_if_failed(self, when):
        if int(self._err[0]) != 0:
            self._err.zero_()
            raise RuntimeError(f"fsb_bsr16_spmm: a bounded wait inside the kernel expired ({when}); "
                               "the output of that call is invalid")


def prepare_spmm_bsr16(blocks, indices, indptr, shape):
    """Validate a BSR matrix of 16 x 16 blocks: ``blocks[nnzb, 16, 16]``, block columns
    ``indices[nnzb]``, block row pointers ``indptr[M/16 + 1]``, ``shape = (M, K)``."""
    if len(shape) != 2:
        raise ValueError("shape must be a 2-tuple: (n_rows, n_cols)")
    m, k = int(shape[0]), int(shape[1])
    if m < 0 or k < 0 or m % 16 or k % 16:
        raise ValueError("shape dimensions must be non-negative multiples of 16")
    if blocks.ndim != 3 or tuple(blocks.shape[1:]) != (16, 16):
        raise ValueError("blocks must have shape [nnzb, 16, 16]")
    if indices.ndim != 1 or indptr.ndim != 1:
        raise ValueError("indices and indptr must be 1D tensors")
    if blocks.shape[0] != indices.numel():
        raise ValueError("blocks and indices must have the same length (nnzb)")
    if indptr.numel() != m // 16 + 1:
        raise ValueError(f"indptr length must be n_rows/16+1={m // 16 + 1}, got {indptr.numel()}")
    if not all(t.is_cuda for t in (blocks, indices, indptr)):
        raise ValueError("blocks, indices, and indptr must be CUDA tensors")
    if blocks.dtype not in SUPPORTED_BSR16_DTYPES:
        raise TypeError("blocks dtype must be torch.bfloat16 or torch.float16")
    if indices.dtype not in (torch.int32, torch.int64) or indptr.dtype not in (torch.int32, torch.int64):
        raise TypeError("indices and indptr dtype must be torch.int32 or torch.int64")
    blocks = blocks.contiguous()
    indices = indices.contiguous()
    indptr = indptr.contiguous()
    facts = _csr.inspect_csr(indices, indptr, m // 16, indices.numel())
    if facts["first"] != 0:
        raise ValueError("indptr[0] must be 0")
    if facts["last"] != indices.numel():
        raise ValueError("indptr[-1] must equal nnzb")
    if facts["decreasing"]:
        raise ValueError("indptr must be nondecreasing")
    if indices.numel() and (facts["min_col"] < 0 or facts["max_col"] >= k // 16):
        raise IndexError("block indices out of range for n_cols/16")
    return PreparedBsr16(blocks, indices.to(torch.int32), indptr.to(torch.int64), (m, k))


def flagsparse_spmm_bsr16(blocks=None, indices=None, indptr=None, B=None, shape=None, prepared=None, out=None,
                          check_status=False):
    """C = A @ B for a BSR-16 matrix A on the tensor cores; returns C [M, N] in A's dtype.

    A failed launch (a bounded wait inside the kernel gave up) is reported
    without a synchronisation by the next call on the same prepared matrix,
    which raises before launching.  ``check_status`` waits for this call's
    kernel instead (one stream synchronisation) and raises at once.
    """
    if prepared is None:
        if any(v is None for v in (blocks, indices, indptr, shape)):
            raise ValueError("blocks, indices, indptr, and shape are required when prepared is not provided")
        prepared = prepare_spmm_bsr16(blocks, indices, indptr, shape)
    elif not isinstance(prepared, PreparedBsr16):
        raise TypeError("prepared must be a PreparedBsr16 instance")
    if B is None or B.ndim != 2:
        raise ValueError("B must be a 2D dense tensor")
    if B.shape[0] != prepared.shape[1]:
        raise ValueError(f"B.shape[0] must be n_cols={prepared.shape[1]}, got {B.shape[0]}")
    if B.dtype != prepared.blocks.dtype:
        raise TypeError("B dtype must match blocks dtype")
    if not B.is_cuda or B.device != prepared.blocks.device:
        raise ValueError("B must be a CUDA tensor on the same device as the sparse matrix")
    n = int(B.shape[1])
    if n % 64:
        raise ValueError("B.shape[1] must be a multiple of 64 for the tensor-core BSR path")
    prepared._raise_if_failed("an earlier call")
    B = B.contiguous()
    M = prepared.shape[0]
    if out is not None:
        if out.shape != (M, n) or out.dtype != B.dtype or not out.is_contiguous() or out.device != B.device:
            raise ValueError("out shape/dtype must match result")
        C = out
    else:
        C = torch.empty((M, n), dtype=B.dtype, device=B.device)
    nat.check(
        nat.lib().fsb_bsr16_spmm(
            nat.dtype_code(B.dtype), nat.ptr(prepared.packed), nat.ptr(prepared.indices), nat.ptr(prepared.indptr),
            prepared.n_brows, prepared.n_bcols, nat.ptr(B), n, n, nat.ptr(C), n, nat.ptr(prepared._err),
            nat.stream_of(B.device),
        ),
        "fsb_bsr16_spmm",
    )
    if check_status:
        torch.cuda.current_stream(B.device).synchronize()
        prepared._raise_if_failed("this call")
    return C
