"""Batched uneven CSR matrices: one graph launch for every SpMV and SpMM, checked per matrix."""

import numpy as np
import pytest
import torch

import flagsparse_b200 as fs
from flagsparse_b200 import workloads
from flagsparse_b200.sparse_operations import batched as bm
from oracle import oracle
from tests.helpers import assert_spmv_close, assert_within, host, plain_error_bound

pytestmark = pytest.mark.gpu


def _batch(count=24, lo=50, hi=20_000, seed=11):
    mats = workloads.batched_mix(count=count, lo=lo, hi=hi, seed=seed)
    dev = [(torch.from_numpy(m["data"]).cuda(), torch.from_numpy(m["indices"]).cuda(),
            torch.from_numpy(m["indptr"]).cuda(), m["shape"]) for m in mats]
    return mats, dev


def _check_all(b, mats, what):
    for i, m in enumerate(mats):
        x = host(b.x_view(i)).astype(np.float64)
        B = host(b.B_view(i)).astype(np.float64)
        d = m["data"].astype(np.float64)
        y_ref = oracle.spmv(m["indptr"], m["indices"], d, x)
        scale = oracle.spmv_abs(m["indptr"], m["indices"], d, x)
        assert_spmv_close(host(b.y_view(i)).astype(np.float64), y_ref, scale, np.diff(m["indptr"]), "float32",
                          f"{what} spmv {i}")
        C_ref = oracle.spmm(m["indptr"], m["indices"], d, B)
        C_scale = oracle.spmm(m["indptr"], m["indices"], np.abs(d), np.abs(B))
        lens = np.broadcast_to(np.diff(m["indptr"])[:, None], C_ref.shape)
        assert_within(host(b.C_view(i)).astype(np.float64), C_ref, plain_error_bound("float32", C_ref, C_scale, lens),
                      f"{what} spmm {i}")


def test_batched_graph_matches_oracle_per_matrix():
    mats, dev = _batch()
    b = fs.BatchedCsr(dev, n_dense=16)
    assert b.count == 24 and b.n_rows == sum(m["shape"][0] for m in mats)
    for i, m in enumerate(mats):
        b.x_view(i).copy_(torch.from_numpy(m["x"]))
        b.B_view(i).copy_(torch.from_numpy(m["B"]))
    b.run()
    torch.cuda.synchronize()
    _check_all(b, mats, "first replay")
    # new inputs in the same static buffers: the replay sees them
    g = torch.Generator(device="cuda").manual_seed(4)
    b.x.copy_(torch.rand(b.x.shape, device="cuda", generator=g) - 0.5)
    b.B.copy_(torch.rand(b.B.shape, device="cuda", generator=g) - 0.5)
    y0, C0 = (t.clone() for t in b.run())
    torch.cuda.synchronize()
    _check_all(b, mats, "second replay")
    y1, C1 = b.run()
    assert torch.equal(y0, y1) and torch.equal(C0, C1)


def test_batched_autotuner_picks_and_caches(tmp_path):
    mats, dev = _batch(count=10, seed=12)
    b = fs.BatchedCsr(dev, n_dense=16)
    for i, m in enumerate(mats):
        b.x_view(i).copy_(torch.from_numpy(m["x"]))
        b.B_view(i).copy_(torch.from_numpy(m["B"]))
    path = str(tmp_path / "tune.json")
    bm._TUNE_CACHE.clear()
    rep = b.tune(cache_path=path)
    assert rep["source"] == "measured"
    # every SpMM shape on one work item per warp, plus the best one on the persistent grid
    assert len(rep["spmv_trials"]) == len(bm.SPMV_CANDIDATES)
    assert len(rep["spmm_trials"]) == len(bm.SPMM_CANDIDATES) + 1
    assert [t["persistent"] for t in rep["spmm_trials"]].count(True) == 1
    # fp32 with a 16-column B: the one-kernel step applies and is timed too
    assert len(rep["fused_trials"]) == len(bm.SPMM_CANDIDATES) + 1
    fastest_v = min(rep["spmv_trials"], key=lambda t: t["ms"])
    fastest_m = min(rep["spmm_trials"], key=lambda t: t["ms"])
    fastest_f = min(rep["fused_trials"], key=lambda t: t["ms"])
    assert rep["fused"] == (fastest_f["ms"] < fastest_v["ms"] + fastest_m["ms"]) == b.fused
    best = fastest_f if b.fused else fastest_m
    assert b.spmv_cfg == {"cap": fastest_v["cap"], "chunk": fastest_v["chunk"]}
    assert b.spmm_cfg == {"cap": best["cap"], "chunk": best["chunk"], "persistent": best["persistent"]}
    b.run()
    torch.cuda.synchronize()
    _check_all(b, mats, "tuned")
    # a second batch with the same signature reuses the file cache
    bm._TUNE_CACHE.clear()
    b2 = fs.BatchedCsr(dev, n_dense=16)
    assert b2.tune(cache_path=path)["source"] == "cache"
    assert (b2.spmv_cfg, b2.spmm_cfg) == (b.spmv_cfg, b.spmm_cfg)


@pytest.mark.parametrize("cap", [32, 64, 128])
def test_spmv_smaller_windows_match(cap):
    """The SpMV kernel accepts any row-block window up to 128; every window meets the oracle bound."""
    c = workloads.zipf_csr(n=40_000, seed=13)
    A = (torch.from_numpy(c["data"]).cuda(), torch.from_numpy(c["indices"]).cuda(), torch.from_numpy(c["indptr"]).cuda())
    b = fs.BatchedCsr([(A[0], A[1], A[2], c["shape"])], n_dense=16)
    b.spmv_cfg = {"cap": cap, "chunk": 512}
    b.x.copy_(torch.from_numpy(c["x"]))
    b.step()
    torch.cuda.synchronize()
    d = c["data"].astype(np.float64)
    ref = oracle.spmv(c["indptr"], c["indices"], d, c["x"].astype(np.float64))
    scale = oracle.spmv_abs(c["indptr"], c["indices"], d, c["x"].astype(np.float64))
    assert_spmv_close(host(b.y).astype(np.float64), ref, scale, np.diff(c["indptr"]), "float32", f"cap {cap}")


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64, torch.complex64])
@pytest.mark.parametrize("fused", [False, True])
def test_batched_fused_and_unfused_steps_match_oracle(dtype, fused):
    """Both step forms, graph-captured: the one-kernel step for real values (complex values
    fall back to the SpMV and SpMM launches) and the two-launch step."""
    mats, _ = _batch(count=6, seed=15)
    dev_m = [(torch.from_numpy(m["data"]).cuda().to(dtype), torch.from_numpy(m["indices"]).cuda(),
              torch.from_numpy(m["indptr"]).cuda(), m["shape"]) for m in mats]
    b = fs.BatchedCsr(dev_m, n_dense=16)
    b.fused = fused
    g = torch.Generator(device="cuda").manual_seed(6)
    b.x.copy_(torch.rand(b.x.shape, device="cuda", generator=g).to(dtype))
    b.B.copy_(torch.rand(b.B.shape, device="cuda", generator=g).to(dtype))
    b.run()
    torch.cuda.synchronize()
    assert b.fused is (fused and not dtype.is_complex)
    dname = {torch.float32: "float32", torch.float64: "float64", torch.complex64: "complex64"}[dtype]
    for i, m in enumerate(mats):
        d = m["data"].astype(np.complex128 if dtype.is_complex else np.float64)
        x = host(b.x_view(i)).astype(d.dtype)
        B = host(b.B_view(i)).astype(d.dtype)
        ref = oracle.spmv(m["indptr"], m["indices"], d, x)
        scale = oracle.spmv_abs(m["indptr"], m["indices"], np.abs(d), np.abs(x))
        assert_spmv_close(host(b.y_view(i)), ref, scale, np.diff(m["indptr"]), dname, f"y {i}")
        C_ref = oracle.spmm(m["indptr"], m["indices"], d, B)
        C_scale = oracle.spmm(m["indptr"], m["indices"], np.abs(d), np.abs(B))
        lens = np.broadcast_to(np.diff(m["indptr"])[:, None], C_ref.shape)
        assert_within(host(b.C_view(i)), C_ref, plain_error_bound(dname, C_ref, C_scale, lens), f"C {i}")


def test_batched_validation():
    with pytest.raises(ValueError, match="non-empty"):
        fs.BatchedCsr([])
    bad = (torch.ones(2, device="cuda"), torch.tensor([0, 5], dtype=torch.int32, device="cuda"),
           torch.tensor([0, 1, 2], device="cuda"), (2, 3))
    with pytest.raises(IndexError, match="out of range"):
        fs.BatchedCsr([bad])
