"""Sharded CSR SpMV / SpMM / SDDMM and batched steps across ranks (one process per GPU).

Every split has no exchange on the data path:
  * SpMV / SpMM shard by rows: each rank owns a contiguous block of rows,
    chosen so every rank holds about the same number of nonzeros (one binary
    search of the nonzero prefix ``indptr`` per boundary), keeps the global
    column indices, and multiplies its block by the full x (or B), which
    every rank holds.  y (or C) comes out row-sharded.
  * SDDMM shards by nonzero range: rank k computes the outputs of nonzeros
    [k nnz / world, (k+1) nnz / world) from the full x and y.
  * A batch of independent matrices shards by matrix: each rank takes a
    contiguous run of matrices holding about the same number of nonzeros
    and runs its own batched step over them.
An optional all-gather assembles the sharded result on every rank.

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


def nnz_shards(nnz, world_size):
    """Contiguous nonzero ranges ``[(p0, p1), ...]``, one per rank, sizes differing by at most one."""
    nnz, world_size = int(nnz), int(world_size)
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    bounds = [nnz * k // world_size for k in range(world_size + 1)]
    return [(bounds[k], bounds[k + 1]) for k in range(world_size)]


def matrix_shards(nnz_per_matrix, world_size):
    """Contiguous runs of matrices ``[(m0, m1), ...]`` with nearly equal nonzero counts.

    The same rule as row_shards, over the prefix of the matrices' nonzero
    counts: a rank's run ends at the first matrix whose prefix reaches
    k * total / world_size.
    """
    counts = np.asarray(nnz_per_matrix, dtype=np.int64)
    prefix = np.zeros(counts.size + 1, dtype=np.int64)
    np.cumsum(counts, out=prefix[1:])
    return row_shards(prefix, world_size)


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


class ShardedSddmm:
    """This rank's nonzero range of an SDDMM pattern:
    out[p] = alpha <x[row(p)], y[col(p)]> + beta data[p] for p in [p0, p1).

    ``indices``, ``indptr`` describe the whole pattern; this rank keeps the
    column and row index of each of its nonzeros on ``device``.  x and y are
    the whole dense operands on every rank.
    """

    def __init__(self, indices, indptr, shape, rank=None, world_size=None, device=None, group=None):
        from .sparse_operations.sddmm_csr import _build_row_ids

        self.group = group
        self.rank = dist.get_rank(group) if rank is None else int(rank)
        self.world_size = dist.get_world_size(group) if world_size is None else int(world_size)
        self.shape = (int(shape[0]), int(shape[1]))
        device = device or indices.device
        nnz = int(indices.numel())
        self.shards = nnz_shards(nnz, self.world_size)
        p0, p1 = self.shards[self.rank]
        self.nnz_begin, self.nnz_end = p0, p1
        row_ids = _build_row_ids(indptr.to(device=device, dtype=torch.int64))
        self.row_ids = row_ids[p0:p1].contiguous()
        self.indices = indices[p0:p1].to(device=device, dtype=torch.int32).contiguous()

    def sddmm(self, x, y, data=None, alpha=1.0, beta=0.0, gather=False):
        """out[p0:p1] of the SDDMM (every nonzero's output with ``gather``); ``data``, when
        given, is the whole value array (its [p0, p1) slice is read)."""
        from .sparse_operations.sddmm_csr import _native_sddmm

        if x.ndim != 2 or y.ndim != 2 or x.shape[0] != self.shape[0] or y.shape[0] != self.shape[1] \
                or x.shape[1] != y.shape[1]:
            raise ValueError("x must be n_rows x K and y n_cols x K")
        if x.dtype != y.dtype or x.device != y.device:
            raise TypeError("x and y must share dtype and device")
        local = data[self.nnz_begin:self.nnz_end].contiguous() if data is not None else None
        out = torch.empty(self.nnz_end - self.nnz_begin, dtype=x.dtype, device=x.device)
        _native_sddmm(self.row_ids, self.indices, x.contiguous(), y.contiguous(), local, alpha, beta, out)
        return gather_rows(out, self.shards, self.group) if gather else out


class ShardedBatch:
    """This rank's run of a batch of independent CSR matrices, as one BatchedCsr.

    ``matrices``: the whole batch as ``(data, indices, indptr, shape)``; only
    the rank's run ``[m0, m1)`` (balanced by nonzeros, matrix_shards) is kept
    and combined.  ``batch`` is the rank's BatchedCsr (its x / B / y / C views
    are indexed by the matrix id minus m0).
    """

    def __init__(self, matrices, n_dense=16, rank=None, world_size=None, device=None, group=None):
        from .sparse_operations.batched import BatchedCsr

        self.group = group
        self.rank = dist.get_rank(group) if rank is None else int(rank)
        self.world_size = dist.get_world_size(group) if world_size is None else int(world_size)
        self.count = len(matrices)
        self.shards = matrix_shards([int(m[1].numel()) for m in matrices], self.world_size)
        self.m0, self.m1 = self.shards[self.rank]
        mine = [(d.to(device) if device else d, i.to(device) if device else i, p.to(device) if device else p, sh)
                for d, i, p, sh in matrices[self.m0:self.m1]]
        self.batch = BatchedCsr(mine, n_dense=n_dense) if mine else None

    def owns(self, i):
        return self.m0 <= i < self.m1

    def run(self):
        """One step over the rank's matrices (y = A x and C = A B for each); returns (y, C)."""
        if self.batch is None:
            return None, None
        return self.batch.run()
