"""CSR SDDMM on the native kernel against the oracle and FlagSparse's golden outputs."""

import numpy as np
import pytest
import torch

import flagsparse_b200 as fs
from flagsparse_b200 import workloads
from flagsparse_b200.sparse_operations import sddmm_csr as dm
from oracle import oracle
from tests.helpers import TORCH_DT, assert_within, dev, host, plain_error_bound, rounded

pytestmark = pytest.mark.gpu


def _pattern(m, n, seed, long_rows=()):
    mat = workloads.mask_csr(m, n, seed=seed, dtype=np.float64, long_rows=long_rows)
    return mat["indptr"], mat["indices"], mat["data"]


def _oracle(indptr, indices, x_r, y_r, d_r, alpha, beta):
    ref = oracle.sddmm(indptr, indices, x_r, y_r, d_r, alpha=alpha, beta=beta)
    scale = np.abs(alpha) * oracle.sddmm(indptr, indices, np.abs(x_r), np.abs(y_r), None, 1.0, 0.0)
    if d_r is not None:
        scale = scale + np.abs(beta) * np.abs(d_r)
    return ref, scale


@pytest.mark.parametrize("shape", ["8x10x8", "64x96x16", "50x40x37"])
@pytest.mark.parametrize("dname", ["float32", "float64"])
def test_sddmm_golden_cases(golden, shape, dname):
    g = golden("golden_sddmm.npz")
    tag = f"sddmm_{shape}"
    M, N, K = (int(v) for v in shape.split("x"))
    dt = TORCH_DT[dname]
    x, y, d = g[f"{tag}_{dname}_x"], g[f"{tag}_{dname}_y"], g[f"{tag}_{dname}_data"]
    out = fs.flagsparse_sddmm_csr(dev(d, dt), dev(g[tag + "_indices"]), dev(g[tag + "_indptr"]), dev(x, dt),
                                  dev(y, dt), (M, N), alpha=1.25, beta=0.5)
    ref, scale = _oracle(g[tag + "_indptr"], g[tag + "_indices"], x.astype(np.float64), y.astype(np.float64),
                         d.astype(np.float64), 1.25, 0.5)
    bound = plain_error_bound(dname, ref, scale, K)
    assert_within(host(out).astype(np.float64), ref, bound, f"{tag} vs oracle")
    assert_within(host(out).astype(np.float64), g[f"{tag}_{dname}_out"].astype(np.float64), 2 * bound,
                  f"{tag} vs reference")


@pytest.mark.parametrize("dname", ["float16", "bfloat16", "float32", "float64"])
@pytest.mark.parametrize("K", [1, 7, 32, 64, 128, 130, 200, 256, 300])
def test_sddmm_native_dtypes_and_widths(dname, K):
    """All value types the native kernel takes (the public API admits fp32 / fp64)."""
    indptr, indices, data = _pattern(40, 60, seed=K, long_rows=(2,))
    rng = np.random.Generator(np.random.PCG64(K))
    x_np, y_np = rng.standard_normal((40, K)), rng.standard_normal((60, K))
    dt = TORCH_DT[dname]
    x_r, y_r, d_r = rounded(x_np, dname), rounded(y_np, dname), rounded(data, dname)
    row_ids = dm._build_row_ids(dev(indptr))
    out = torch.empty(indices.size, dtype=dt, device="cuda")
    dm._native_sddmm(row_ids, dev(indices), dev(x_np, dt), dev(y_np, dt), dev(data, dt), 0.75, -1.5, out)
    ref, scale = _oracle(indptr, indices, x_r, y_r, d_r, 0.75, -1.5)
    assert_within(host(out).astype(np.float64), ref, plain_error_bound(dname, ref, scale, K), f"{dname} K={K}")


def test_sddmm_row_ids_match_reference_rule():
    c = workloads.zipf_csr(n=30_000, seed=21)
    for ptr_dt in (torch.int64, torch.int32):
        rows = dm._build_row_ids(dev(c["indptr"], ptr_dt))
        exp = np.repeat(np.arange(30_000, dtype=np.int32), np.diff(c["indptr"]))
        np.testing.assert_array_equal(host(rows), exp)


@pytest.mark.parametrize("variant", ["baseline", "altreduce", "acc64", "acc64_out64"])
def test_sddmm_diagnostic_variants(variant):
    indptr, indices, data = _pattern(64, 80, seed=3)
    rng = np.random.Generator(np.random.PCG64(5))
    K = 96
    x_np, y_np = rng.standard_normal((64, K)), rng.standard_normal((80, K))
    p = fs.prepare_sddmm_csr(dev(indices), dev(indptr), (64, 80), k_hint=K)
    x, y, d = dev(x_np, torch.float32), dev(y_np, torch.float32), dev(data, torch.float32)
    out, meta = dm._run_sddmm_prepared(p, x, y, d, 1.0, 0.25, None, variant=variant)
    ref, scale = _oracle(indptr, indices, rounded(x_np, "float32"), rounded(y_np, "float32"),
                         rounded(data, "float32"), 1.0, 0.25)
    if variant == "acc64_out64":
        assert out.dtype == torch.float64 and meta["acc_dtype"] == "float64"
        bound = plain_error_bound("float64", ref, scale, K)
    elif variant == "acc64":
        assert out.dtype == torch.float32 and meta["acc_dtype"] == "float64"
        bound = 2.0**-24 * np.abs(ref) + plain_error_bound("float64", ref, scale, K)
    else:
        bound = plain_error_bound("float32", ref, scale, K)
    assert_within(host(out).astype(np.float64), ref, bound, variant)
    assert meta["variant"] == variant and meta["fallback_used"] is False


def test_sddmm_beta_data_none_and_k_zero():
    indptr, indices, data = _pattern(10, 12, seed=6)
    p = fs.prepare_sddmm_csr(dev(indices), dev(indptr), (10, 12))
    x, y = torch.randn(10, 5, device="cuda"), torch.randn(12, 5, device="cuda")
    out = fs.flagsparse_sddmm_csr(x=x, y=y, prepared=p)
    ref, scale = _oracle(indptr, indices, host(x).astype(np.float64), host(y).astype(np.float64), None, 1.0, 0.0)
    assert_within(host(out).astype(np.float64), ref, plain_error_bound("float32", ref, scale, 5), "data None")
    d = dev(data, torch.float32)
    out0 = fs.flagsparse_sddmm_csr(d, x=torch.zeros(10, 0, device="cuda"), y=torch.zeros(12, 0, device="cuda"),
                                   prepared=p, beta=2.0)
    torch.testing.assert_close(out0, d * 2.0)
    with pytest.raises(ValueError, match="data is required when beta is non-zero"):
        fs.flagsparse_sddmm_csr(x=x, y=y, prepared=p, beta=1.0)


def test_sddmm_validation_messages_and_meta():
    indptr, indices, data = _pattern(10, 12, seed=7)
    with pytest.raises(TypeError, match="indices dtype must be torch.int32"):
        fs.prepare_sddmm_csr(dev(indices).long(), dev(indptr), (10, 12))
    p = fs.prepare_sddmm_csr(dev(indices), dev(indptr), (10, 12), k_hint=16)
    with pytest.raises(TypeError, match="x dtype must be torch.float32 or torch.float64"):
        fs.flagsparse_sddmm_csr(x=torch.randn(10, 4, device="cuda").half(), y=torch.randn(12, 4, device="cuda").half(),
                                prepared=p)
    with pytest.raises(ValueError, match=r"y.shape\[0\] must be n_cols=12"):
        fs.flagsparse_sddmm_csr(x=torch.randn(10, 4, device="cuda"), y=torch.randn(11, 4, device="cuda"), prepared=p)
    out, ms, meta = fs.flagsparse_sddmm_csr(x=torch.randn(10, 4, device="cuda"), y=torch.randn(12, 4, device="cuda"),
                                            prepared=p, return_time=True, return_meta=True)
    assert {"prepare_ms", "block_k", "num_warps", "fallback_used", "variant", "acc_dtype", "out_dtype"} <= set(meta)
    assert (meta["block_k"], meta["num_warps"]) == (32, 2)


def test_sddmm_full_size_backward_shape_sampled():
    """Chung-Lu graph, 500,000 rows, K = 128, bfloat16 (the SpMM backward's dvals): 20,000 sampled nonzeros."""
    g = workloads.chung_lu_graph()
    n = g["shape"][0]
    gen = torch.Generator(device="cuda").manual_seed(1)
    dY = torch.randn(n, 128, device="cuda", generator=gen).bfloat16()
    X = torch.randn(n, 128, device="cuda", generator=gen).bfloat16()
    indptr, indices = dev(g["indptr"]), dev(g["indices"])
    rows = dm._build_row_ids(indptr)
    out = torch.empty(indices.numel(), dtype=torch.bfloat16, device="cuda")
    dm._native_sddmm(rows, indices, dY, X, None, 1.0, 0.0, out)
    pick = torch.from_numpy(np.random.Generator(np.random.PCG64(8)).choice(indices.numel(), 20_000,
                                                                            replace=False)).cuda()
    r, c = rows[pick].long(), indices[pick].long()
    exact = (dY[r].double() * X[c].double()).sum(1)
    scale = (dY[r].double().abs() * X[c].double().abs()).sum(1)
    err = (out[pick].double() - exact).abs()
    assert bool((err <= 2.0**-8 * exact.abs() + 140 * 2.0**-24 * scale + 1e-30).all())
