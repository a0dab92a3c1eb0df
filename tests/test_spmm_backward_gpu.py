"""One-launch backward of Y = A X (fsb_spmm_csr_backward): dX = A^T dY and
dvals[p] = <dY[row(p)], X[col(p)]>, against the fp64 oracle with elementwise
error bounds, on patterns whose transposed rows are empty, short, longer than
the SpMM window and longer than one chunk (partials and tickets)."""

import numpy as np
import pytest
import torch

import flagsparse_b200 as fs
from flagsparse_b200.sparse_operations import _csr
from oracle import oracle
from tests.helpers import assert_within, dev, host, op_csr, plain_error_bound

pytestmark = pytest.mark.gpu

TORCH = {"float16": torch.float16, "bfloat16": torch.bfloat16, "float32": torch.float32, "float64": torch.float64}


def _pattern(n_rows, n_cols, seed):
    """Random sparse rows plus a few heavy columns: column 3 in every row (A^T row of
    n_rows nonzeros, several chunks), column 5 in 150 rows (one chunk, > window),
    columns n_cols-4.. never used (empty A^T rows), and every 97th row empty."""
    rng = np.random.default_rng(seed)
    rows = []
    for r in range(n_rows):
        if r % 97 == 0:
            rows.append(np.empty(0, dtype=np.int64))
            continue
        k = int(rng.integers(1, 12))
        cols = set(rng.integers(0, n_cols - 4, size=k).tolist())
        cols.add(3)
        if r % 7 == 0 and len(rows) < 1050:
            cols.add(5)
        rows.append(np.array(sorted(cols), dtype=np.int64))
    indptr = np.zeros(n_rows + 1, dtype=np.int64)
    indptr[1:] = np.cumsum([len(c) for c in rows])
    indices = np.concatenate(rows).astype(np.int32)
    data = rng.uniform(-1.0, 1.0, size=indices.size)
    return indptr, indices, data


def _run(dname, n, with_dvals=True, n_rows=2500, n_cols=700, seed=0):
    dt = TORCH[dname]
    indptr, indices, data = _pattern(n_rows, n_cols, seed)
    shape = (n_rows, n_cols)
    vals = dev(data, dt)
    p = fs.prepare_spmm_csr_autograd(vals, dev(indices), dev(indptr), shape)
    gen = torch.Generator(device="cuda").manual_seed(seed + 1)
    X = torch.randn(n_cols, n, device="cuda", generator=gen).to(dt)
    dY = torch.randn(n_rows, n, device="cuda", generator=gen).to(dt)
    dX = torch.full((n_cols, n), float("nan"), device="cuda").to(dt)
    dvals = torch.full_like(vals, float("nan")) if with_dvals else None
    ok = _csr.spmm_backward(vals, p.perm32, p.t_indices, p.t_indptr, n_rows, n_cols, dY,
                            X if with_dvals else None, dX, dvals, p.t_plan)
    return ok, (indptr, indices, host(vals).astype(np.float64), shape), host(X).astype(np.float64), \
        host(dY).astype(np.float64), dX, dvals, p


def _check(dname, mat, X, dY, dX, dvals, n):
    indptr, indices, v, shape = mat
    t_ptr, t_idx, t_v, _ = op_csr(indptr, indices, v, shape, "trans")
    ref = oracle.spmm(t_ptr, t_idx, t_v, dY)
    scale = oracle.spmm(t_ptr, t_idx, np.abs(t_v), np.abs(dY))
    lens = np.broadcast_to(np.diff(t_ptr)[:, None], ref.shape)
    assert_within(host(dX).astype(np.float64), ref, plain_error_bound(dname, ref, scale, lens), f"dX {dname} n={n}")
    if dvals is not None:
        dref = oracle.sddmm(indptr, indices, dY, X)
        dscale = oracle.sddmm(indptr, indices, np.abs(dY), np.abs(X))
        assert_within(host(dvals).astype(np.float64), dref, plain_error_bound(dname, dref, dscale, n),
                      f"dvals {dname} n={n}")


# every team width 1..32 appears: n * sizeof(value) / 16 lanes
CASES = [("float32", 4), ("float32", 8), ("float32", 36), ("float32", 64), ("float32", 128),
         ("float64", 2), ("float64", 6), ("float64", 64),
         ("bfloat16", 8), ("bfloat16", 24), ("bfloat16", 128), ("bfloat16", 256),
         ("float16", 8), ("float16", 64), ("float16", 256)]


@pytest.mark.parametrize("dname,n", CASES)
def test_backward_one_launch_against_oracle(dname, n):
    ok, mat, X, dY, dX, dvals, p = _run(dname, n)
    assert ok
    _check(dname, mat, X, dY, dX, dvals, n)
    assert p.t_plan.counters_clear()


@pytest.mark.parametrize("dname,n", [("float32", 64), ("bfloat16", 128), ("float64", 6)])
def test_backward_dx_only(dname, n):
    ok, mat, X, dY, dX, dvals, p = _run(dname, n, with_dvals=False, seed=2)
    assert ok and dvals is None
    _check(dname, mat, X, dY, dX, None, n)


def test_backward_repeat_bitwise():
    dt = torch.float32
    indptr, indices, data = _pattern(1500, 400, 7)
    vals = dev(data, dt)
    p = fs.prepare_spmm_csr_autograd(vals, dev(indices), dev(indptr), (1500, 400))
    X = torch.randn(400, 32, device="cuda")
    dY = torch.randn(1500, 32, device="cuda")
    outs = []
    for _ in range(3):
        dX = torch.empty(400, 32, device="cuda")
        dv = torch.empty_like(vals)
        assert _csr.spmm_backward(vals, p.perm32, p.t_indices, p.t_indptr, 1500, 400, dY, X, dX, dv, p.t_plan)
        outs.append((dX, dv))
    for dX, dv in outs[1:]:
        assert torch.equal(dX, outs[0][0]) and torch.equal(dv, outs[0][1])
    assert p.t_plan.counters_clear()


def test_backward_wide_rows_not_taken():
    """Rows wider than 512 bytes leave the kernel unlaunched; autograd then uses the separate kernels."""
    ok, *_ = _run("float32", 256, n_rows=300, n_cols=100)
    assert not ok
    indptr, indices, data = _pattern(300, 100, 3)
    vals = dev(data).requires_grad_(True)
    X = torch.randn(100, 256, dtype=torch.float64, device="cuda", requires_grad=True)
    p = fs.prepare_spmm_csr_autograd(vals.detach(), dev(indices), dev(indptr), (300, 100))
    G = torch.randn(300, 256, dtype=torch.float64, device="cuda")
    fs.flagsparse_spmm_csr_autograd(vals, X, prepared=p).backward(G)
    _check("float64", (indptr, indices, data, (300, 100)), host(X), host(G), X.grad, vals.grad, 256)


def test_autograd_takes_one_launch_path(monkeypatch):
    """The differentiable layer's backward goes through fsb_spmm_csr_backward when it applies."""
    calls = []
    real = _csr.spmm_backward

    def spy(*a, **k):
        r = real(*a, **k)
        calls.append(r)
        return r

    monkeypatch.setattr(_csr, "spmm_backward", spy)
    indptr, indices, data = _pattern(800, 300, 4)
    vals = dev(data, torch.float32).requires_grad_(True)
    X = torch.randn(300, 16, device="cuda", requires_grad=True)
    p = fs.prepare_spmm_csr_autograd(vals.detach(), dev(indices), dev(indptr), (800, 300))
    G = torch.randn(800, 16, device="cuda")
    fs.flagsparse_spmm_csr_autograd(vals, X, prepared=p).backward(G)
    assert calls == [True]
    _check("float32", (indptr, indices, host(vals).astype(np.float64), (800, 300)), host(X).astype(np.float64),
           host(G).astype(np.float64), X.grad, vals.grad, 16)
