"""The MatrixMarket reader against FlagSparse's own test loader (goldens), CPU only."""

import os

import numpy as np
import pytest
import torch

from flagsparse_b200 import mtx

MTX_DIR = os.path.join(os.path.dirname(__file__), "golden", "mtx")
CASES = sorted(f[:-4] for f in os.listdir(MTX_DIR) if f.endswith(".mtx"))


@pytest.mark.parametrize("tag", CASES)
def test_mtx_reader_matches_flagsparse_loader(golden, tag):
    g = golden("golden_mtx.npz")
    data, indices, indptr, shape = mtx.load_mtx_to_csr_torch(os.path.join(MTX_DIR, tag + ".mtx"),
                                                             dtype=torch.float64, device=torch.device("cpu"))
    assert shape == tuple(int(v) for v in g[f"mtx_{tag}_shape"])
    assert indices.dtype == torch.int64 and indptr.dtype == torch.int64
    np.testing.assert_array_equal(indptr.numpy(), g[f"mtx_{tag}_indptr"])
    np.testing.assert_array_equal(indices.numpy(), g[f"mtx_{tag}_indices"])
    np.testing.assert_array_equal(data.numpy(), g[f"mtx_{tag}_data"])


def test_mtx_reader_large_file_roundtrip(tmp_path):
    rng = np.random.default_rng(0)
    n, nnz = 3000, 40000
    r = rng.integers(0, n, nnz)
    c = rng.integers(0, n, nnz)
    v = rng.standard_normal(nnz)
    path = tmp_path / "big.mtx"
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n%\n")
        f.write(f"{n} {n} {nnz}\n")
        for a, b, x in zip(r, c, v):
            f.write(f"{a + 1} {b + 1} {float(x)!r}\n")
    data, indices, indptr, shape = mtx.mtx_to_csr_arrays(str(path))
    dense = np.zeros((n, n))
    np.add.at(dense, (r, c), v)
    got = np.zeros((n, n))
    rows = np.repeat(np.arange(n), np.diff(indptr))
    got[rows, indices] = data
    np.testing.assert_allclose(got, dense, rtol=0, atol=1e-12)
    assert np.all(np.diff(indices)[np.diff(rows) == 0] > 0)


@pytest.mark.gpu
@pytest.mark.parametrize("tag", [t for t in CASES if t != "empty"])
def test_mtx_matrix_spmv_on_gpu(tag):
    """A MatrixMarket matrix read to the device runs through the native SpMV."""
    import flagsparse_b200 as fs
    from oracle import oracle

    data, indices, indptr, shape = mtx.load_mtx_to_csr_torch(os.path.join(MTX_DIR, tag + ".mtx"),
                                                             dtype=torch.float64, device=torch.device("cuda"))
    x = np.random.default_rng(7).standard_normal(shape[1])
    y = fs.flagsparse_spmv_csr(data, indices, indptr, torch.from_numpy(x).cuda(), shape=shape)
    ref = oracle.spmv(indptr.cpu().numpy(), indices.cpu().numpy().astype(np.int32), data.cpu().numpy(), x)
    np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=1e-12, atol=1e-14)
