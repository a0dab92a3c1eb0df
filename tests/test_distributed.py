"""Row-sharded SpMV / SpMM: the shard plan and the row all-gather on 2 gloo ranks (CPU),
and the sharded products on one GPU (each shard run in turn, no collective)."""

import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from flagsparse_b200 import distributed as fsd
from flagsparse_b200 import workloads
from oracle import oracle
from tests.helpers import assert_spmv_close, assert_within, host, plain_error_bound


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_row_shards_balance_nonzeros(world):
    c = workloads.zipf_csr(n=20_000, seed=5)
    ptr = c["indptr"]
    shards = fsd.row_shards(ptr, world)
    assert shards[0][0] == 0 and shards[-1][1] == ptr.size - 1
    assert all(a <= b for a, b in shards) and all(shards[k][1] == shards[k + 1][0] for k in range(world - 1))
    nnz = int(ptr[-1])
    longest = int(np.diff(ptr).max())
    for r0, r1 in shards:
        assert int(ptr[r1] - ptr[r0]) <= -(-nnz // world) + longest


def test_row_shards_more_ranks_than_rows():
    ptr = np.array([0, 3, 3, 5], dtype=np.int64)
    shards = fsd.row_shards(ptr, 5)
    assert len(shards) == 5 and shards[-1][1] == 3
    assert sum(b - a for a, b in shards) == 3


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gloo_worker(rank, world, port, q):
    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
        c = workloads.poisson_csr(n=3000, seed=9)
        ptr, idx = c["indptr"], c["indices"]
        d = c["data"].astype(np.float64)
        x = c["x"].astype(np.float64)
        shards = fsd.row_shards(ptr, world)
        r0, r1 = shards[rank]
        # this rank's rows of A x, computed by the oracle on its row block
        lp = ptr[r0:r1 + 1] - ptr[r0]
        y_local = oracle.spmv(lp, idx[ptr[r0]:ptr[r1]], d[ptr[r0]:ptr[r1]], x)
        y = fsd.gather_rows(torch.from_numpy(y_local), shards)
        B = np.random.default_rng(1).standard_normal((3000, 5))
        C_local = oracle.spmm(lp, idx[ptr[r0]:ptr[r1]], d[ptr[r0]:ptr[r1]], B)
        C = fsd.gather_rows(torch.from_numpy(C_local), shards)
        ok = (np.array_equal(y.numpy(), oracle.spmv(ptr, idx, d, x))
              and np.array_equal(C.numpy(), oracle.spmm(ptr, idx, d, B)))
        q.put((rank, ok))
        dist.destroy_process_group()
    except Exception as exc:  # reported to the parent, which fails the test
        q.put((rank, repr(exc)))


def test_gather_rows_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert results == {0: True, 1: True}, results


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 3])
def test_sharded_products_on_one_gpu(world):
    c = workloads.zipf_csr(n=50_000, seed=6)
    data = torch.from_numpy(c["data"]).cuda()
    indices = torch.from_numpy(c["indices"]).cuda()
    indptr = torch.from_numpy(c["indptr"]).cuda()
    x = torch.from_numpy(c["x"]).cuda()
    B = torch.randn(c["shape"][1], 8, device="cuda")
    ys, Cs = [], []
    for rank in range(world):
        sh = fsd.ShardedCsr(data, indices, indptr, c["shape"], rank=rank, world_size=world)
        ys.append(sh.spmv(x))
        first = sh.spmm(B)
        Cs.append(sh.spmm(B))  # the second call reuses the shard's SpMM plan and scratch
        assert torch.equal(first, Cs[-1])
    y = host(torch.cat(ys)).astype(np.float64)
    C = host(torch.cat(Cs)).astype(np.float64)
    d = c["data"].astype(np.float64)
    x64 = c["x"].astype(np.float64)
    ref = oracle.spmv(c["indptr"], c["indices"], d, x64)
    scale = oracle.spmv_abs(c["indptr"], c["indices"], np.abs(d), np.abs(x64))
    assert_spmv_close(y, ref, scale, np.diff(c["indptr"]), "float32", f"sharded spmv x{world}")
    B64 = host(B).astype(np.float64)
    C_ref = oracle.spmm(c["indptr"], c["indices"], d, B64)
    C_scale = oracle.spmm(c["indptr"], c["indices"], np.abs(d), np.abs(B64))
    lens = np.broadcast_to(np.diff(c["indptr"])[:, None], C_ref.shape)
    assert_within(C, C_ref, plain_error_bound("float32", C_ref, C_scale, lens), f"sharded spmm x{world}")
