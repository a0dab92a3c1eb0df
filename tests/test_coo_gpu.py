"""COO -> CSR on the GPU: the native conversion against the oracle (bit-exact
pattern and permutation), against FlagSparse's own conversion (goldens), and
the COO SpMV entry points against the oracle SpMV.

Mirrors FlagSparse's tests/pytest/test_spmv_coo_accuracy.py:230-263
(test_spmv_coo_tocsr_matches_torch, ..._prepared_path_matches_torch).
"""

import zlib

import numpy as np
import pytest
import torch

import flagsparse_b200 as fs
from flagsparse_b200.sparse_operations import _csr
from flagsparse_b200.sparse_operations import spmv_csr as spmv_mod
from oracle import oracle
from tests.helpers import TORCH_DT, assert_spmv_close, dev, host, rounded

pytestmark = pytest.mark.gpu


def _coo(rng, nr, nc, nnz, dup_frac=0.0, shuffle=True):
    """Random COO pattern; dup_frac of the entries repeat an earlier (row, col)."""
    n_new = nnz - int(nnz * dup_frac)
    if nr * nc <= 5_000_000:
        keys = rng.choice(nr * nc, size=n_new, replace=nr * nc < n_new)
    else:  # large pattern: draws with replacement (repeats are rare and allowed)
        keys = rng.integers(0, nr * nc, size=n_new)
    if nnz > n_new:
        keys = np.concatenate([keys, rng.choice(keys, size=nnz - n_new)])
    keys = rng.permutation(keys) if shuffle else np.sort(keys, kind="stable")
    return (keys // nc).astype(np.int64), (keys % nc).astype(np.int64)


@pytest.mark.parametrize("case", ["shuffled", "sorted", "dups", "empty_rows", "one_row", "one_col", "big"])
@pytest.mark.parametrize("idx_dt", [torch.int32, torch.int64])
def test_native_coo_to_csr_matches_oracle(case, idx_dt):
    rng = np.random.default_rng(zlib.crc32(f"{case}{idx_dt}".encode()))
    nr, nc, nnz, dup, shuffle = {
        "shuffled": (300, 200, 5000, 0.0, True),
        "sorted": (300, 200, 5000, 0.0, False),
        "dups": (50, 40, 3000, 0.3, True),
        "empty_rows": (20000, 64, 700, 0.0, True),
        "one_row": (1, 5000, 1200, 0.0, True),
        "one_col": (5000, 1, 1200, 0.0, True),
        "big": (200_000, 300_000, 2_000_000, 0.01, True),
    }[case]
    row, col = _coo(rng, nr, nc, nnz, dup, shuffle)
    r, c = dev(row, idx_dt), dev(col, idx_dt)
    unsorted, bad_r, bad_c = _csr.coo_inspect(r, c, nr, nc)
    assert (bad_r, bad_c) == (0, 0)
    keys = row * nc + col
    assert unsorted == int(np.count_nonzero(keys[1:] < keys[:-1]))
    indices, indptr, perm = _csr.coo_to_csr(r, c, nr, nc, ordered=(unsorted == 0))
    ptr_ref, idx_ref, perm_ref = oracle.coo_to_csr(row, col, nr, nc)
    np.testing.assert_array_equal(host(indptr), ptr_ref)
    np.testing.assert_array_equal(host(indices), idx_ref)
    if unsorted:
        np.testing.assert_array_equal(host(perm), perm_ref)
    else:
        assert perm is None
        np.testing.assert_array_equal(perm_ref, np.arange(nnz))


def test_native_coo_inspect_counts_out_of_range():
    row = dev(np.array([0, 3, 1, -1, 2], dtype=np.int64))
    col = dev(np.array([0, 1, 7, 2, 5], dtype=np.int64))
    assert _csr.coo_inspect(row, col, 3, 6) == (2, 2, 1)


@pytest.mark.parametrize("tag", ["shuf", "sorted", "i32", "emptyrows"])
def test_coo_to_csr_for_spmv_matches_flagsparse_golden(golden, tag):
    g = golden("golden_coo.npz")
    nr, nc = (int(v) for v in g[f"coo_{tag}_shape"])
    row, col = g[f"coo_{tag}_row"], g[f"coo_{tag}_col"]
    data = dev(g[f"coo_{tag}_data"])
    d_s, idx, ptr = spmv_mod.coo_to_csr_for_spmv(data, dev(row), dev(col), (nr, nc))
    assert idx.dtype == torch.int32 and ptr.dtype == torch.int64
    np.testing.assert_array_equal(host(ptr), g[f"coo_{tag}_indptr"])
    np.testing.assert_array_equal(host(idx), g[f"coo_{tag}_indices"])
    np.testing.assert_array_equal(host(d_s), g[f"coo_{tag}_data_s"])


def _coo_spmv_case(rng, nr, nc, nnz, dname, dup=0.0):
    row, col = _coo(rng, nr, nc, nnz, dup, True)
    if dname.startswith("complex"):
        data = rng.standard_normal(nnz) + 1j * rng.standard_normal(nnz)
        x = rng.standard_normal(nc) + 1j * rng.standard_normal(nc)
    else:
        data = rng.standard_normal(nnz)
        x = rng.standard_normal(nc)
    return row, col, rounded(data, dname), rounded(x, dname)


def _oracle_coo_spmv(row, col, data, x, nr, nc):
    ptr, idx, perm = oracle.coo_to_csr(row, col, nr, nc)
    d = np.asarray(data)[perm]
    return ptr, idx, oracle.spmv(ptr, idx, d, x), oracle.spmv_abs(ptr, idx, np.abs(d), np.abs(x))


@pytest.mark.parametrize("dname", ["float16", "bfloat16", "float32", "float64", "complex64", "complex128"])
@pytest.mark.parametrize("shape", [(1, 1), (8, 10), (513, 257), (4096, 2048)])
def test_spmv_coo_tocsr_matches_oracle(dname, shape):
    nr, nc = shape
    rng = np.random.default_rng(nr * 7 + nc)
    nnz = max(1, min(nr * nc, nr * 12))
    row, col, data, x = _coo_spmv_case(rng, nr, nc, nnz, dname, dup=0.05)
    dt = TORCH_DT[dname]
    y = fs.flagsparse_spmv_coo_tocsr(dev(data, dt), dev(row), dev(col), dev(x, dt), shape=shape)
    ptr, _, ref, scale = _oracle_coo_spmv(row, col, data, x, nr, nc)
    assert y.shape == (nr,) and y.dtype == dt
    assert_spmv_close(host(y), ref, scale, np.diff(ptr), dname, f"coo {dname} {shape}")


def test_spmv_coo_tocsr_prepared_path_and_out():
    rng = np.random.default_rng(5)
    nr, nc = 2000, 1500
    row, col, data, x = _coo_spmv_case(rng, nr, nc, 30000, "float32")
    dt = torch.float32
    prepared = fs.prepare_spmv_coo_tocsr(dev(data, dt), dev(row, torch.int32), dev(col, torch.int32), (nr, nc))
    assert prepared.shape == (nr, nc)
    out = torch.empty(nr, dtype=dt, device="cuda")
    y = fs.flagsparse_spmv_coo_tocsr(x=dev(x, dt), prepared=prepared, out=out)
    assert y is out
    y2, ms = fs.flagsparse_spmv_coo_tocsr(x=dev(x, dt), prepared=prepared, return_time=True)
    assert ms >= 0.0 and torch.equal(y, y2)
    ptr, _, ref, scale = _oracle_coo_spmv(row, col, data, x, nr, nc)
    assert_spmv_close(host(y), ref, scale, np.diff(ptr), "float32", "prepared coo")


def test_spmv_coo_tocsr_sorted_input_keeps_values():
    rng = np.random.default_rng(9)
    nr, nc = 700, 900
    row, col = _coo(rng, nr, nc, 9000, 0.0, shuffle=False)
    data = dev(rng.standard_normal(9000), torch.float64)
    d_s, idx, ptr = spmv_mod.coo_to_csr_for_spmv(data, dev(row), dev(col), (nr, nc), assume_sorted=True)
    assert d_s is data
    # unordered input is sorted even when assume_sorted is passed
    perm = rng.permutation(9000)
    d2, idx2, ptr2 = spmv_mod.coo_to_csr_for_spmv(data[dev(perm)], dev(row[perm]), dev(col[perm]), (nr, nc),
                                                  assume_sorted=True)
    assert torch.equal(ptr2, ptr) and torch.equal(idx2, idx) and torch.equal(d2, data)


def test_spmv_coo_tocsr_empty_and_validation():
    dt = torch.float32
    e64 = torch.empty(0, dtype=torch.int64, device="cuda")
    y = fs.flagsparse_spmv_coo_tocsr(torch.empty(0, dtype=dt, device="cuda"), e64, e64,
                                     torch.ones(4, dtype=dt, device="cuda"), shape=(3, 4))
    assert torch.equal(y, torch.zeros(3, dtype=dt, device="cuda"))
    d = torch.ones(3, dtype=dt, device="cuda")
    r = torch.tensor([0, 1, 2], device="cuda")
    c = torch.tensor([0, 1, 2], device="cuda")
    x = torch.ones(3, dtype=dt, device="cuda")
    with pytest.raises(TypeError, match="x dtype must match data dtype"):
        fs.flagsparse_spmv_coo_tocsr(d, r, c, x.double(), shape=(3, 3))
    with pytest.raises(ValueError, match="CUDA tensors"):
        fs.flagsparse_spmv_coo_tocsr(d, r.cpu(), c, x, shape=(3, 3))
    with pytest.raises(ValueError, match="same length"):
        fs.prepare_spmv_coo_tocsr(d, r[:2], c, (3, 3))
    with pytest.raises(IndexError, match="out of range for n_cols"):
        fs.flagsparse_spmv_coo_tocsr(d, r, c, x[:2], shape=(3, 2))
    with pytest.raises(RuntimeError, match="out of range for n_rows"):
        fs.flagsparse_spmv_coo_tocsr(d, r, c, x, shape=(2, 3))
    p = fs.prepare_spmv_coo_tocsr(d, r, c, (3, 3))
    with pytest.raises(ValueError, match="does not match prepared.shape"):
        fs.flagsparse_spmv_coo_tocsr(x=x, shape=(3, 4), prepared=p)
    with pytest.raises(TypeError, match="x is required"):
        fs.flagsparse_spmv_coo_tocsr(prepared=p)
