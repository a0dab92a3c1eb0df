"""Differentiable CSR SpMM: gradients against finite differences, the oracle and torch's
sparse autograd."""

import numpy as np
import pytest
import torch

import flagsparse_b200 as fs
from flagsparse_b200 import workloads
from oracle import oracle
from tests.helpers import dev, host, op_csr, spmv_error_bound

pytestmark = pytest.mark.gpu


def _graph(n, seed=3):
    g = workloads.chung_lu_graph(n=n, mean_degree=25.0, seed=seed)
    return g["indptr"], g["indices"], g["data"].astype(np.float64), g["shape"]


def test_gradcheck_float64_small():
    mat = workloads.mask_csr(12, 9, seed=1, dtype=np.float64, long_rows=(4,))
    p = fs.prepare_spmm_csr_autograd(dev(mat["data"]), dev(mat["indices"]), dev(mat["indptr"]), mat["shape"])
    vals = dev(mat["data"]).requires_grad_(True)
    X = torch.randn(9, 3, dtype=torch.float64, device="cuda", requires_grad=True)
    assert torch.autograd.gradcheck(lambda v, x: fs.flagsparse_spmm_csr_autograd(v, x, prepared=p), (vals, X),
                                    eps=1e-6, atol=1e-9, rtol=1e-7)


def test_directional_finite_differences_chung_lu_1000():
    """Central differences of L = <G, A(v) X> along 8 random directions, float64."""
    indptr, indices, data, shape = _graph(1000)
    p = fs.prepare_spmm_csr_autograd(dev(data), dev(indices), dev(indptr), shape)
    gen = torch.Generator(device="cuda").manual_seed(0)
    vals = dev(data).requires_grad_(True)
    X = torch.randn(1000, 16, dtype=torch.float64, device="cuda", generator=gen, requires_grad=True)
    G = torch.randn(1000, 16, dtype=torch.float64, device="cuda", generator=gen)
    loss = (fs.flagsparse_spmm_csr_autograd(vals, X, prepared=p) * G).sum()
    gv, gx = torch.autograd.grad(loss, (vals, X))

    def L(v, x):
        return float((fs.flagsparse_spmm_csr_autograd(v, x, prepared=p) * G).sum())

    h = 1e-5
    for _ in range(8):
        dv = torch.randn(vals.shape, dtype=torch.float64, device="cuda", generator=gen)
        dx = torch.randn(X.shape, dtype=torch.float64, device="cuda", generator=gen)
        with torch.no_grad():
            fd = (L(vals + h * dv, X + h * dx) - L(vals - h * dv, X - h * dx)) / (2 * h)
        an = float((gv * dv).sum() + (gx * dx).sum())
        assert abs(fd - an) <= 1e-7 * max(1.0, abs(an)), (fd, an)


def _oracle_grads(indptr, indices, vals, X, G, shape):
    t_ptr, t_idx, t_vals, _ = op_csr(indptr, indices, vals, shape, "trans")
    dX = oracle.spmm(t_ptr, t_idx, t_vals, G)
    dv = oracle.sddmm(indptr, indices, G, X)
    Y = oracle.spmm(indptr, indices, vals, X)
    return Y, dX, dv


def _rel(got, ref):
    return float(np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-300))


@pytest.mark.parametrize("dname,thresh", [("float64", 1e-12), ("float32", 1e-6), ("bfloat16", 1e-2),
                                          ("float16", 5e-3)])
def test_forward_backward_against_oracle(dname, thresh):
    """Max relative error (FlagSparse's _spmm_relative_threshold metric) of Y, dX and dvals
    against the fp64 oracle on the same rounded inputs."""
    indptr, indices, data, shape = _graph(20_000, seed=4)
    dt = getattr(torch, dname)
    gen = torch.Generator(device="cuda").manual_seed(1)
    vals = dev(data, dt).requires_grad_(True)
    X = torch.randn(shape[1], 64, device="cuda", generator=gen).to(dt).requires_grad_(True)
    G = torch.randn(shape[0], 64, device="cuda", generator=gen).to(dt)
    p = fs.prepare_spmm_csr_autograd(vals.detach(), dev(indices), dev(indptr), shape)
    Y = fs.flagsparse_spmm_csr_autograd(vals, X, prepared=p)
    Y.backward(G)
    Yo, dXo, dvo = _oracle_grads(indptr, indices, host(vals).astype(np.float64), host(X).astype(np.float64),
                                 host(G).astype(np.float64), shape)
    assert _rel(host(Y).astype(np.float64), Yo) <= thresh
    assert _rel(host(X.grad).astype(np.float64), dXo) <= thresh
    assert _rel(host(vals.grad).astype(np.float64), dvo) <= thresh


@pytest.mark.parametrize("dname,thresh", [("float64", 1e-12), ("float32", 1e-6), ("bfloat16", 1e-2),
                                          ("float16", 5e-3)])
def test_gradients_match_torch_sparse_autograd(dname, thresh):
    """Y, dX and dvals against torch's own sparse autograd: torch.sparse.mm on a CPU
    sparse_csr_tensor that is a leaf, float64, on the same rounded inputs
    (20,000-node Chung-Lu graph, 64 features).  Half types are compared within
    FlagSparse's thresholds; CPU sparse CSR matmul has no half kernels, so the
    reference runs in float64 as the reference's own tests upcast."""
    indptr, indices, data, shape = _graph(20_000, seed=4)
    dt = getattr(torch, dname)
    gen = torch.Generator(device="cuda").manual_seed(5)
    vals = dev(data, dt).requires_grad_(True)
    X = torch.randn(shape[1], 64, device="cuda", generator=gen).to(dt).requires_grad_(True)
    G = torch.randn(shape[0], 64, device="cuda", generator=gen).to(dt)
    p = fs.prepare_spmm_csr_autograd(vals.detach(), dev(indices), dev(indptr), shape)
    Y = fs.flagsparse_spmm_csr_autograd(vals, X, prepared=p)
    Y.backward(G)

    X64 = torch.from_numpy(host(X).astype(np.float64)).requires_grad_(True)
    crow, colx = torch.from_numpy(indptr), torch.from_numpy(indices.astype(np.int64))
    A = torch.sparse_csr_tensor(crow, colx, torch.from_numpy(host(vals).astype(np.float64)), size=shape,
                                requires_grad=True)
    Yt = torch.sparse.mm(A, X64)
    Yt.backward(torch.from_numpy(host(G).astype(np.float64)))
    # torch's gradient of A lives on A's pattern: its values line up with vals
    assert torch.equal(A.grad.crow_indices(), crow) and torch.equal(A.grad.col_indices(), colx)
    assert _rel(host(Y).astype(np.float64), Yt.detach().numpy()) <= thresh
    assert _rel(host(X.grad).astype(np.float64), X64.grad.numpy()) <= thresh
    assert _rel(host(vals.grad).astype(np.float64), A.grad.values().numpy()) <= thresh


def test_values_change_between_steps():
    """The cached transpose regathers values every backward."""
    indptr, indices, data, shape = _graph(2000, seed=5)
    p = fs.prepare_spmm_csr_autograd(dev(data), dev(indices), dev(indptr), shape)
    X = torch.randn(shape[1], 8, dtype=torch.float64, device="cuda", requires_grad=True)
    for scale in (1.0, -3.0):
        v = dev(data * scale)
        G = torch.ones(shape[0], 8, dtype=torch.float64, device="cuda")
        X.grad = None
        fs.flagsparse_spmm_csr_autograd(v, X, prepared=p).backward(G)
        _, dXo, _ = _oracle_grads(indptr, indices, data * scale, host(X), host(G), shape)
        np.testing.assert_allclose(host(X.grad), dXo, rtol=1e-12, atol=1e-12)


def test_autograd_full_size_bf16_sampled():
    """500,000-node Chung-Lu graph, 128 features, bfloat16: forward + backward run, sampled rows of dX
    within FlagSparse's bfloat16 threshold of the fp64 result."""
    indptr, indices, data, shape = _graph(500_000)
    gen = torch.Generator(device="cuda").manual_seed(2)
    vals = dev(data, torch.bfloat16).requires_grad_(True)
    X = torch.randn(shape[1], 128, device="cuda", generator=gen).bfloat16().requires_grad_(True)
    p = fs.prepare_spmm_csr_autograd(vals.detach(), dev(indices), dev(indptr), shape)
    Y = fs.flagsparse_spmm_csr_autograd(vals, X, prepared=p)
    G = torch.randn(Y.shape, device="cuda", generator=gen).bfloat16()
    Y.backward(G)
    rows = np.sort(np.random.Generator(np.random.PCG64(6)).choice(shape[0], 500, replace=False))
    lens = np.diff(indptr)[rows]
    sub_ptr = np.zeros(rows.size + 1, dtype=np.int64)
    np.cumsum(lens, out=sub_ptr[1:])
    take = np.concatenate([np.arange(indptr[r], indptr[r + 1]) for r in rows])
    v64 = host(vals).astype(np.float64)
    # the graph is symmetric with symmetric values, so A^T rows equal A rows
    dX_ref = oracle.spmm(sub_ptr, indices[take], v64[take], host(G).astype(np.float64))
    got = host(X.grad[torch.from_numpy(rows).cuda()]).astype(np.float64)
    assert _rel(got, dX_ref) <= 1e-2
    assert torch.isfinite(vals.grad.float()).all()


@pytest.mark.parametrize("dname", ["bfloat16", "float32"])
@pytest.mark.parametrize("N", [16, 128])
def test_backward_long_column_sums_compensated(dname, N):
    """dX = A^T dY sums A's columns: column 0 holds 50,000 ones, and dY's rows 0 and
    49,999 are +big and -big with `unit` rows between (unit at or below half an fp32 ulp of
    big).  A plain fp32 sum absorbs every unit term and ends at 0; the backward sums rows
    over 1,024 nonzeros in fp64 (exact products), so dX[0] = 49,998 unit within the bound
    of a compensated (Dot2) sum, which the fp64 sum meets with room to spare.  dvals and
    the other columns stay within FlagSparse's thresholds of the fp64 oracle."""
    dt = getattr(torch, dname)
    n_long, k = 50_000, 8
    rng = np.random.Generator(np.random.PCG64(N))
    # row r < n_long: (r, 0) and one entry in columns 1..k-1; rows beyond: short random rows
    rows = [np.array([0, 1 + r % (k - 1)]) for r in range(n_long)] + [np.sort(rng.choice(k, 3, replace=False))
                                                                       for _ in range(32)]
    indptr = np.zeros(len(rows) + 1, dtype=np.int64)
    np.cumsum([len(r) for r in rows], out=indptr[1:])
    indices = np.concatenate(rows).astype(np.int32)
    data = np.ones(indices.size)
    shape = (len(rows), k)
    big, unit = 2.0**24, 1.0
    G = np.full((shape[0], N), unit)
    G[0], G[n_long - 1] = big, -big
    G[n_long:] = rng.standard_normal((32, N))
    X = rng.standard_normal((k, N))
    vals = dev(data, dt).requires_grad_(True)
    Xd = dev(X, dt).requires_grad_(True)
    p = fs.prepare_spmm_csr_autograd(vals.detach(), dev(indices), dev(indptr), shape)
    fs.flagsparse_spmm_csr_autograd(vals, Xd, prepared=p).backward(dev(G, dt))
    exact = np.full(N, (n_long - 2) * unit)
    S = np.full(N, 2 * big + (n_long - 2) * unit)
    got = host(Xd.grad[0]).astype(np.float64)
    bound = spmv_error_bound(dname, exact, S, n_long)
    assert np.all(np.abs(got - exact) <= bound), (got[:4], bound[:4])
    _, dXo, dvo = _oracle_grads(indptr, indices, data, host(Xd).astype(np.float64), host(dev(G, dt)).astype(np.float64),
                                shape)
    assert _rel(host(Xd.grad).astype(np.float64)[1:], dXo[1:]) <= (1e-2 if dname == "bfloat16" else 1e-6)
    assert _rel(host(vals.grad).astype(np.float64), dvo) <= (1e-2 if dname == "bfloat16" else 1e-6)
