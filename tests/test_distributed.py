"""Sharded SpMV / SpMM (rows), SDDMM (nonzero ranges) and batches (matrices): the shard
plans and the all-gathers on 2 gloo ranks (CPU), and the sharded products on one GPU
(each shard run in turn, no collective)."""

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


@pytest.mark.parametrize("nnz,world", [(0, 2), (7, 3), (1_000_003, 8), (5, 8)])
def test_nnz_shards_cover_every_nonzero_once(nnz, world):
    shards = fsd.nnz_shards(nnz, world)
    assert len(shards) == world and shards[0][0] == 0 and shards[-1][1] == nnz
    assert all(shards[k][1] == shards[k + 1][0] for k in range(world - 1))
    sizes = [b - a for a, b in shards]
    assert max(sizes) - min(sizes) <= 1


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_matrix_shards_balance_nonzeros(world):
    counts = np.random.default_rng(3).integers(0, 5000, 256)
    shards = fsd.matrix_shards(counts, world)
    assert shards[0][0] == 0 and shards[-1][1] == counts.size
    assert all(shards[k][1] == shards[k + 1][0] for k in range(world - 1))
    total = int(counts.sum())
    for m0, m1 in shards:
        assert int(counts[m0:m1].sum()) <= -(-total // world) + int(counts.max())


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


def _gloo_worker_sddmm_batch(rank, world, port, q):
    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
        # SDDMM by nonzero range: each rank's outputs from the oracle, gathered
        c = workloads.poisson_csr(n=2000, seed=4)
        ptr, idx = c["indptr"], c["indices"]
        rng = np.random.default_rng(2)
        x, y = rng.standard_normal((2000, 6)), rng.standard_normal((2000, 6))
        full = oracle.sddmm(ptr, idx, x, y)
        shards = fsd.nnz_shards(idx.size, world)
        p0, p1 = shards[rank]
        local = full[p0:p1]  # what the rank's kernel computes
        got = fsd.gather_rows(torch.from_numpy(local.copy()), shards)
        ok = np.array_equal(got.numpy(), full)
        # batch by matrix: each rank's y blocks, gathered in matrix order
        mats = [workloads.poisson_csr(n=100 + 37 * i, seed=10 + i) for i in range(7)]
        ms = fsd.matrix_shards([m["indices"].size for m in mats], world)
        m0, m1 = ms[rank]
        ys = [oracle.spmv(m["indptr"], m["indices"], m["data"].astype(np.float64), m["x"].astype(np.float64))
              for m in mats]
        local = np.concatenate(ys[m0:m1]) if m1 > m0 else np.zeros(0)
        row_blocks = []
        r = 0
        for a, b in ms:
            n_rows = sum(mats[i]["shape"][0] for i in range(a, b))
            row_blocks.append((r, r + n_rows))
            r += n_rows
        got = fsd.gather_rows(torch.from_numpy(local), row_blocks)
        ok = ok and np.array_equal(got.numpy(), np.concatenate(ys))
        q.put((rank, ok))
        dist.destroy_process_group()
    except Exception as exc:  # reported to the parent, which fails the test
        q.put((rank, repr(exc)))


def test_sddmm_and_batch_shards_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_worker_sddmm_batch, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert results == {0: True, 1: True}, results


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


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 3])
def test_sharded_sddmm_on_one_gpu(world):
    g = workloads.chung_lu_graph(n=20_000, seed=7)
    indices = torch.from_numpy(g["indices"]).cuda()
    indptr = torch.from_numpy(g["indptr"]).cuda()
    gen = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn(g["shape"][0], 32, device="cuda", generator=gen)
    y = torch.randn(g["shape"][1], 32, device="cuda", generator=gen)
    data = torch.from_numpy(g["data"]).cuda()
    outs = [fsd.ShardedSddmm(indices, indptr, g["shape"], rank=r, world_size=world).sddmm(x, y, data, 1.25, 0.5)
            for r in range(world)]
    got = host(torch.cat(outs)).astype(np.float64)
    x64, y64 = host(x).astype(np.float64), host(y).astype(np.float64)
    d64 = g["data"].astype(np.float64)
    ref = oracle.sddmm(g["indptr"], g["indices"], x64, y64, d64, alpha=1.25, beta=0.5)
    scale = oracle.sddmm(g["indptr"], g["indices"], np.abs(x64), np.abs(y64), np.abs(d64), alpha=1.25, beta=0.5)
    assert_within(got, ref, plain_error_bound("float32", ref, scale, 34), f"sharded sddmm x{world}")


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 3])
def test_sharded_batch_on_one_gpu(world):
    mats = workloads.batched_mix(count=12, lo=1_000, hi=20_000, seed=8)
    dev_mats = [(torch.from_numpy(m["data"]).cuda(), torch.from_numpy(m["indices"]).cuda(),
                 torch.from_numpy(m["indptr"]).cuda(), m["shape"]) for m in mats]
    seen = set()
    for rank in range(world):
        sh = fsd.ShardedBatch(dev_mats, n_dense=16, rank=rank, world_size=world)
        if sh.batch is None:
            continue
        for i in range(sh.m0, sh.m1):
            sh.batch.x_view(i - sh.m0).copy_(torch.from_numpy(mats[i]["x"]))
            sh.batch.B_view(i - sh.m0).copy_(torch.from_numpy(mats[i]["B"]))
        sh.run()
        torch.cuda.synchronize()
        for i in range(sh.m0, sh.m1):
            seen.add(i)
            m = mats[i]
            d = m["data"].astype(np.float64)
            ref = oracle.spmv(m["indptr"], m["indices"], d, m["x"].astype(np.float64))
            scale = oracle.spmv_abs(m["indptr"], m["indices"], np.abs(d), np.abs(m["x"].astype(np.float64)))
            got = host(sh.batch.y_view(i - sh.m0)).astype(np.float64)
            assert_spmv_close(got, ref, scale, np.diff(m["indptr"]), "float32", f"batch shard matrix {i}")
    assert seen == set(range(len(mats)))
