"""Row-sharded CSR SpMV / SpMM across ranks (one process per GPU).

The CSR products shard by rows with no exchange on the data path: each rank
owns a contiguous block of rows, chosen so every rank holds about the same
number of nonzeros (one binary search of the nonzero prefix ``indptr`` per
boundary), keeps the global column indices, and multiplies its block by the
full x (or B), which every rank holds.  y (or C) comes out row-sharded; an
optional all-gather assembles it on every rank.

NCCL (``torch.distributed``, backend "nccl") carries the optional all-gather;
the sharding itself and the assembly logic also run on "gloo" for CPU tests.
"""

import numpy as np
import torch
import torch.distributed as dist

from .sparse_operations import _csr
from .sparse_operations.spmm_csr import _prepare_spmm_csr_matrix
from .sparse_operations.spmv_csr import flagsparse_spmv_csr, prepare_spmv_csr


def row_shards(indptr, world_size):
    """Contiguous row blocks ``[(r0, r1), ...]`` with nearly equal nonzero counts.

    Boundary k is the first row whose nonzero prefix reaches k * nnz / world_size
    (a binary search of indptr); empty blocks are allowed when there are fewer
    rows than ranks.
    """
    ptr = np.asarray(indptr.cpu() if torch.is_tensor(indptr) else indptr, dtype=np.int64)
    n_rows = ptr.size - 1
    nnz = int(ptr[-1])
    world_size = int(world_size)
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    bounds = [0]
    for k in range(1, world_size):
        target = (nnz * k + world_size - 1) // world_size
        r = int(np.searchsorted(ptr, target, side="left"))
        bounds.append(min(max(r, bounds[-1]), n_rows))
    bounds.append(n_rows)
    return [(bounds[k], bounds[k + 1]) for k in range(world_size)]


def gather_rows(local, shards, group=None):
    """All-gather row blocks of different lengths (dim 0) into the full result on every rank."""
    world = dist.get_world_size(group)
    rows = [r1 - r0 for r0, r1 in shards]
    if len(rows) != world:
        raise ValueError("one shard per rank is required")
    cap = max(rows) if rows else 0
    pad_shape = (cap,) + tuple(local.shape[1:])
    padded = torch.zeros(pad_shape, dtype=local.dtype, device=local.device)
    padded[: local.shape[0]].copy_(local)
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    return torch.cat([p[:n] for p, n in zip(parts, rows)], dim=0)


class ShardedCsr:
    """This rank's row block of a CSR matrix, for row-sharded SpMV and SpMM.

    ``data``, ``indices``, ``indptr`` describe the whole matrix (any device);
    only this rank's block is kept, on ``device``.  Products return the local
    rows, or the whole result with ``gather=True``.
    """

    def __init__(self, data, indices, indptr, shape, rank=None, world_size=None, device=None, group=None):
        self.group = group
        self.rank = dist.get_rank(group) if rank is None else int(rank)
        self.world_size = dist.get_world_size(group) if world_size is None else int(world_size)
        self.shape = (int(shape[0]), int(shape[1]))
        self.shards = row_shards(indptr, self.world_size)
        r0, r1 = self.shards[self.rank]
        self.row_begin, self.row_end = r0, r1
        device = device or data.device
        ptr = indptr.to(torch.int64)
        a, b = int(ptr[r0]), int(ptr[r1])
        self.indptr = (ptr[r0:r1 + 1] - a).to(device)
        self.indices = indices[a:b].to(device)
        self.data = data[a:b].to(device)
        self.local_shape = (r1 - r0, self.shape[1])
        self.prepared = prepare_spmv_csr(self.data, self.indices, self.indptr, self.local_shape)
        self._spmm = None  # (data, int32 indices, int64 indptr, SpmmPlan), built on the first spmm

    def _spmm_operands(self):
        if self._spmm is None:
            data, ind, ptr, n_rows, n_cols, _rl, _mx = _prepare_spmm_csr_matrix(
                self.data, self.indices, self.indptr, self.local_shape)
            self._spmm = (data, ind, ptr, _csr.SpmmPlan(ptr, n_rows, data.dtype))
        return self._spmm

    def spmv(self, x, gather=False, out=None):
        """y rows [row_begin, row_end) of A x (every row of A x with ``gather``)."""
        y = flagsparse_spmv_csr(x=x, prepared=self.prepared, out=out)
        return gather_rows(y, self.shards, self.group) if gather else y

    def spmm(self, B, gather=False):
        """C rows [row_begin, row_end) of A B (every row with ``gather``).

        The shard is validated and its SpMM plan built once, on the first call.
        """
        data, ind, ptr, plan = self._spmm_operands()
        if B.ndim != 2 or B.shape[0] != self.shape[1]:
            raise ValueError(f"B must be 2D with B.shape[0] == n_cols={self.shape[1]}")
        if B.dtype != data.dtype or B.device != data.device:
            raise TypeError("B must match the matrix dtype and device")
        B = B.contiguous()
        C = torch.empty((self.local_shape[0], int(B.shape[1])), dtype=data.dtype, device=data.device)
        _csr.spmm(data, ind, ptr, self.local_shape[0], self.shape[1], B, plan, C)
        return gather_rows(C, self.shards, self.group) if gather else C
