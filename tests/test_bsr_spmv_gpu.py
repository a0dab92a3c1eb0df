"""BSR SpMV on the GPU against FlagSparse's own outputs (goldens) and the oracle.

Mirrors FlagSparse's BSR SpMV tests: op non / trans / conj, logical and padded
x lengths, the blockrow_reduce algorithm and its restrictions, meta keys.
"""

import numpy as np
import pytest
import torch

import flagsparse_b200 as fs
from oracle import oracle
from tests.helpers import TORCH_DT, assert_spmv_close, dev, host, rounded

pytestmark = pytest.mark.gpu

DTYPES = ("float32", "float64", "complex64", "complex128")


def _expected(blocks, indices, indptr, bd, n_bcols, x, op):
    ptr, idx, vals = oracle.bsr_to_csr(blocks, indices, indptr, bd)
    if op != "non":
        ptr, idx, perm = oracle.transpose(ptr, idx, n_bcols * bd)
        vals = vals[perm]
        if op == "conj":
            vals = np.conj(vals)
    ref = oracle.spmv(ptr, idx, vals, x)
    scale = oracle.spmv_abs(ptr, idx, np.abs(vals), np.abs(x))
    return ref, scale, np.diff(ptr)


@pytest.mark.parametrize("bd", [2, 3, 4, 16])
@pytest.mark.parametrize("dname", DTYPES)
@pytest.mark.parametrize("op", ["non", "trans", "conj"])
def test_bsr_spmv_golden(golden, bd, dname, op):
    g = golden("golden_bsr.npz")
    key = f"bsr{bd}_{dname}_{op}"
    if key + "_y" not in g:
        pytest.skip("conj equals trans for real dtypes")
    dt = TORCH_DT[dname]
    blocks, indices, indptr = g[f"bsr{bd}_{dname}_blocks"], g[f"bsr{bd}_indices"], g[f"bsr{bd}_indptr"]
    shape = tuple(int(v) for v in g[f"bsr{bd}_shape"])
    x = g[key + "_x"]
    y = fs.flagsparse_spmv_bsr(dev(blocks, dt), dev(indices), dev(indptr), dev(x, dt), shape=shape, block_dim=bd,
                               op=op)
    n_bcols = (shape[1] + bd - 1) // bd
    ref, scale, lens = _expected(blocks, indices, indptr, bd, n_bcols, x, op)
    assert y.shape == ref.shape
    assert_spmv_close(host(y), ref, scale, lens, dname, key)
    # FlagSparse's own result, within its summation error plus ours
    u = 2.0**-24 if dname in ("float32", "complex64") else 2.0**-53
    err = np.abs(host(y) - g[key + "_y"])
    assert np.all(err <= 4.0 * (lens + 2) * u * scale + 1e-300), key


def _random_bsr(rng, nbr, nbc, per_row, bd, dname):
    counts = rng.integers(0, 2 * per_row + 1, size=nbr)
    counts[rng.integers(0, nbr)] = 0
    counts = np.minimum(counts, nbc)
    ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    cols = np.concatenate([np.sort(rng.choice(nbc, size=c, replace=False)) for c in counts]).astype(np.int64)
    nnzb = int(ptr[-1])
    if dname.startswith("complex"):
        blocks = rng.standard_normal((nnzb, bd, bd)) + 1j * rng.standard_normal((nnzb, bd, bd))
    else:
        blocks = rng.standard_normal((nnzb, bd, bd))
    return ptr, cols, rounded(blocks, dname)


def _rand_x(rng, n, dname):
    if dname.startswith("complex"):
        return rounded(rng.standard_normal(n) + 1j * rng.standard_normal(n), dname)
    return rounded(rng.standard_normal(n), dname)


@pytest.mark.parametrize("bd", [2, 3, 4, 5, 8, 16, 32, 64])
@pytest.mark.parametrize("dname", DTYPES)
@pytest.mark.parametrize("op", ["non", "trans", "conj"])
@pytest.mark.parametrize("idx_dt", [torch.int32, torch.int64])
def test_bsr_spmv_random_matches_oracle(bd, dname, op, idx_dt):
    if op == "conj" and not dname.startswith("complex"):
        pytest.skip("conj equals trans for real dtypes")
    rng = np.random.default_rng(bd * 131 + len(dname) * 7 + len(op))
    nbr, nbc = max(3, 600 // bd), max(3, 500 // bd)
    ptr, cols, blocks = _random_bsr(rng, nbr, nbc, 6, bd, dname)
    dt = TORCH_DT[dname]
    shape = (nbr * bd - 1, nbc * bd)
    n_in = shape[0] if op != "non" else shape[1]   # logical length: padded by the operator
    x = _rand_x(rng, n_in, dname)
    x_pad = np.zeros((nbr if op != "non" else nbc) * bd, dtype=x.dtype)
    x_pad[:n_in] = x
    y = fs.flagsparse_spmv_bsr(dev(blocks, dt), dev(cols, idx_dt), dev(ptr, idx_dt), dev(x, dt), shape=shape,
                               block_dim=bd, op=op)
    ref, scale, lens = _expected(blocks, cols, ptr, bd, nbc, x_pad, op)
    assert y.shape == ref.shape and y.dtype == dt
    assert_spmv_close(host(y), ref, scale, lens, dname, f"bsr bd={bd} {dname} {op}")


def test_bsr_spmv_large_blocks_deterministic_and_prepared():
    rng = np.random.default_rng(3)
    bd, nbr, nbc = 16, 4096, 4096
    ptr, cols, blocks = _random_bsr(rng, nbr, nbc, 8, bd, "float32")
    dt = torch.float32
    x = _rand_x(rng, nbc * bd, "float32")
    p = fs.prepare_spmv_bsr(dev(blocks, dt), dev(cols), dev(ptr), (nbr * bd, nbc * bd), bd)
    xd = dev(x, dt)
    y1 = fs.flagsparse_spmv_bsr(x=xd, prepared=p)
    y2 = fs.flagsparse_spmv_bsr(x=xd, prepared=p)
    assert torch.equal(y1, y2)
    out = torch.empty(nbr * bd, dtype=dt, device="cuda")
    y3 = fs.flagsparse_spmv_bsr(x=xd, prepared=p, out=out)
    assert y3 is out and torch.equal(y3, y1)
    ref, scale, lens = _expected(blocks, cols, ptr, bd, nbc, x, "non")
    assert_spmv_close(host(y1), ref, scale, lens, "float32", "bsr16 large")


def test_bsr_spmv_blockrow_reduce_meta_and_limits():
    rng = np.random.default_rng(4)
    bd = 4
    ptr, cols, blocks = _random_bsr(rng, 300, 200, 20, bd, "float64")
    dt = torch.float64
    args = (dev(blocks, dt), dev(cols), dev(ptr))
    shape = (300 * bd, 200 * bd)
    x = dev(_rand_x(rng, 200 * bd, "float64"), dt)
    y, meta = fs.flagsparse_spmv_bsr(*args, x, shape=shape, block_dim=bd, use_opt=True, return_meta=True)
    assert meta["algorithm"] == "blockrow_reduce" and meta["op"] == "non"
    assert meta["padded_shape"] == shape and meta["nnzb"] == int(ptr[-1])
    lens = np.diff(ptr)
    want = []
    for label, lo, hi in (("le1", 0, 1), ("le4", 2, 4), ("le16", 5, 16), ("le64", 17, 64), ("gt64", 65, None)):
        n = int(np.count_nonzero((lens >= lo) & (lens <= (hi if hi is not None else 1 << 62))))
        if n:
            want.append({"bucket": label, "rows": n})
    assert meta["bucket_counts"] == want
    y_base = fs.flagsparse_spmv_bsr(*args, x, shape=shape, block_dim=bd)
    assert torch.equal(y, y_base)
    with pytest.raises(ValueError, match="only supports op='non'"):
        fs.flagsparse_spmv_bsr(*args, x, shape=shape, block_dim=bd, use_opt=True, op="trans")
    with pytest.raises(ValueError, match="block_dim values 2, 4, 8, and 16"):
        fs.prepare_spmv_bsr(dev(np.zeros((0, 3, 3)), dt), dev(np.zeros(0, np.int64)), dev(np.zeros(2, np.int64)),
                            (3, 3), 3, use_opt=True)


def test_bsr_spmv_validation_and_empty():
    dt = torch.float32
    blocks = torch.zeros(0, 4, 4, dtype=dt, device="cuda")
    idx = torch.zeros(0, dtype=torch.int64, device="cuda")
    ptr = torch.zeros(3, dtype=torch.int64, device="cuda")
    y = fs.flagsparse_spmv_bsr(blocks, idx, ptr, torch.ones(6, dtype=dt, device="cuda"), shape=(7, 6), block_dim=4)
    assert y.shape == (8,) and torch.equal(y, torch.zeros(8, dtype=dt, device="cuda"))
    with pytest.raises(TypeError, match="BSR SpMV supports float32"):
        fs.flagsparse_spmv_bsr(blocks.half(), idx, ptr, torch.ones(6, device="cuda").half(), shape=(7, 6),
                               block_dim=4)
    with pytest.raises(ValueError, match="block_dim must be greater than 1"):
        fs.prepare_spmv_bsr(torch.zeros(0, 1, 1, device="cuda"), idx, torch.zeros(8, dtype=torch.int64,
                                                                                 device="cuda"), (7, 6), 1)
    with pytest.raises(ValueError, match="indptr length must be n_block_rows"):
        fs.prepare_spmv_bsr(blocks, idx, torch.zeros(5, dtype=torch.int64, device="cuda"), (7, 6), 4)
    with pytest.raises(ValueError, match="x length must be 6 or padded length 8"):
        fs.flagsparse_spmv_bsr(blocks, idx, ptr, torch.ones(5, dtype=dt, device="cuda"), shape=(7, 6), block_dim=4)
    with pytest.raises(ValueError, match="transpose conflicts with op"):
        fs.flagsparse_spmv_bsr(blocks, idx, ptr, torch.ones(6, dtype=dt, device="cuda"), shape=(7, 6), block_dim=4,
                               op="non", transpose=True)
    p = fs.prepare_spmv_bsr(blocks, idx, ptr, (7, 6), 4)
    with pytest.raises(ValueError, match="does not match prepared.op"):
        fs.flagsparse_spmv_bsr(x=torch.ones(7, dtype=dt, device="cuda"), prepared=p, op="trans")
    with pytest.raises(ValueError, match="out shape/dtype must match result"):
        fs.flagsparse_spmv_bsr(x=torch.ones(6, dtype=dt, device="cuda"), prepared=p,
                               out=torch.empty(7, dtype=dt, device="cuda"))
    bad = torch.tensor([0, 5], dtype=torch.int64, device="cuda")
    with pytest.raises(IndexError, match="out of range for n_block_cols"):
        fs.prepare_spmv_bsr(torch.zeros(2, 4, 4, dtype=dt, device="cuda"), bad,
                            torch.tensor([0, 1, 2], dtype=torch.int64, device="cuda"), (7, 6), 4)
