"""Seeded synthetic CSR matrices with the shapes of the benchmark configurations.

All generators run on the host with numpy's PCG64 so a seed gives the same
matrix on every machine.  Returned arrays are numpy: ``indptr`` int64,
``indices`` int32 (sorted and distinct within each row), values as asked.

Configurations (sizes as in the hot-path benchmark table):
  1. ``poisson_csr``   4096 x 4096, row length max(1, Poisson(16)), seed 0.
  2. ``zipf_csr``      2,000,000 x 2,000,000, row length min(50000, ceil(2.887 Z)),
                       Z ~ Zipf(2) truncated at 50,000 (mean ~20), seed 1.
  3. ``zipf_csr``      1,000,000 x 1,000,000 with scale 32/6.93 (mean ~32), seed 2,
                       plus a dense B; ``bsr16`` gives the 16x16-block variant.
  4. ``chung_lu_graph`` symmetric power-law graph, values 1/sqrt(d_i d_j), seed 3.
  5. ``batched_mix``   256 matrices: 5-point stencils and Poisson(24) random rows, seed 4.
"""

import math

import numpy as np

ZIPF_EXPONENT = 2.0
ZIPF_CAP = 50_000
# E[Z] of Zipf(2) truncated at 50,000 is H(50000)/zeta_trunc(2) = 6.93; the
# scale 2.887 puts the mean row length near 20.
ZIPF_SCALE_MEAN20 = 2.887
ZIPF_MEAN_UNSCALED = 6.93


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def zipf_lengths(rng, n_rows, scale, exponent=ZIPF_EXPONENT, cap=ZIPF_CAP):
    """min(cap, ceil(scale * Z)) with Z ~ Zipf(exponent) truncated at cap (rejection)."""
    z = rng.zipf(exponent, n_rows)
    bad = z > cap
    while bad.any():
        z[bad] = rng.zipf(exponent, int(bad.sum()))
        bad = z > cap
    return np.minimum(cap, np.ceil(scale * z)).astype(np.int64)


def distinct_sorted_columns(rng, lengths, n_cols):
    """Per row, `len` distinct columns drawn uniformly, sorted ascending.

    Draws with replacement, sorts the (row, col) keys, redraws duplicates and
    repeats until every row's columns are distinct: the result is a uniform
    draw without replacement per row.
    """
    lengths = np.asarray(lengths, dtype=np.int64)
    if np.any(lengths > n_cols):
        raise ValueError("row length exceeds n_cols")
    n_rows = lengths.size
    indptr = np.zeros(n_rows + 1, dtype=np.int64)
    np.cumsum(lengths, out=indptr[1:])
    # Rows holding more than a quarter of the columns would make the redraw
    # loop a coupon-collector run; they are drawn without replacement after
    # the others (no such row exists in the full-size workloads, so their
    # draws are unaffected).
    dense = lengths > n_cols // 4
    sparse_len = np.where(dense, 0, lengths)
    nnz = int(sparse_len.sum())
    row_of = np.repeat(np.arange(n_rows, dtype=np.int64), sparse_len)
    key = row_of * n_cols + rng.integers(0, n_cols, nnz, dtype=np.int64)
    key.sort()
    while True:
        dup = np.nonzero(key[1:] == key[:-1])[0] + 1
        if dup.size == 0:
            break
        key[dup] = row_of[dup] * n_cols + rng.integers(0, n_cols, dup.size, dtype=np.int64)
        key.sort()
    sparse_cols = (key - row_of * n_cols).astype(np.int32)
    if not dense.any():
        return indptr, sparse_cols
    cols = np.empty(int(indptr[-1]), dtype=np.int32)
    is_sparse_pos = np.repeat(~dense, lengths)
    cols[is_sparse_pos] = sparse_cols
    for r in np.nonzero(dense)[0]:
        cols[indptr[r]:indptr[r + 1]] = np.sort(rng.choice(n_cols, int(lengths[r]), replace=False))
    return indptr, cols


def poisson_csr(n=4096, mean=16.0, seed=0, dtype=np.float32):
    """Configuration 1: square n x n, row length max(1, Poisson(mean)), U[-1,1] values and x."""
    rng = _rng(seed)
    lengths = np.maximum(1, rng.poisson(mean, n)).astype(np.int64)
    indptr, indices = distinct_sorted_columns(rng, lengths, n)
    data = rng.uniform(-1.0, 1.0, indices.size).astype(dtype)
    x = rng.uniform(-1.0, 1.0, n).astype(dtype)
    return {"indptr": indptr, "indices": indices, "data": data, "x": x, "shape": (n, n)}


def zipf_csr(n=2_000_000, scale=ZIPF_SCALE_MEAN20, seed=1, dtype=np.float32, values="uniform"):
    """Configurations 2 and 3: square power-law CSR with sorted distinct columns."""
    rng = _rng(seed)
    lengths = zipf_lengths(rng, n, scale, cap=min(ZIPF_CAP, n))
    indptr, indices = distinct_sorted_columns(rng, lengths, n)
    if values == "uniform":
        data = rng.uniform(-1.0, 1.0, indices.size).astype(dtype)
        x = rng.uniform(-1.0, 1.0, n).astype(dtype)
    else:
        data = rng.standard_normal(indices.size).astype(dtype)
        x = rng.standard_normal(n).astype(dtype)
    return {"indptr": indptr, "indices": indices, "data": data, "x": x, "shape": (n, n)}


def dense_normal(rows, cols, seed, dtype=np.float32):
    return _rng(seed).standard_normal((rows, cols), dtype=np.float32).astype(dtype)


def bsr16(n_block_rows=65_536, blocks_per_row=8, seed=2):
    """16x16-block BSR pattern: `blocks_per_row` distinct random block columns per block row.

    Returns block indptr/indices and N(0,1) fp32 block values [nnzb, 16, 16].
    """
    rng = _rng(seed)
    lengths = np.full(n_block_rows, blocks_per_row, dtype=np.int64)
    indptr, indices = distinct_sorted_columns(rng, lengths, n_block_rows)
    vals = rng.standard_normal((indices.size, 16, 16), dtype=np.float32)
    return {"indptr": indptr, "indices": indices, "blocks": vals, "block_shape": (n_block_rows, n_block_rows)}


def chung_lu_graph(n=500_000, mean_degree=25.0, exponent=2.5, seed=3):
    """Configuration 4: symmetric Chung-Lu graph, no self loops, values 1/sqrt(d_i d_j).

    Weights w_i follow a power law with the requested mean; about n*mean/2
    candidate edges (i, j) are drawn with probability proportional to w_i w_j,
    self loops dropped, duplicates merged, then both directions stored.
    """
    rng = _rng(seed)
    w = (np.arange(1, n + 1, dtype=np.float64)) ** (-1.0 / (exponent - 1.0))
    w *= mean_degree * n / w.sum()
    p = w / w.sum()
    m = int(round(n * mean_degree / 2.0))
    src = rng.choice(n, size=m, p=p)
    dst = rng.choice(n, size=m, p=p)
    keep = src != dst
    src, dst = src[keep], dst[keep]
    a = np.minimum(src, dst).astype(np.int64)
    b = np.maximum(src, dst).astype(np.int64)
    key = np.unique(a * n + b)
    a, b = key // n, key % n
    rows = np.concatenate([a, b])
    cols = np.concatenate([b, a])
    key = np.sort(rows * n + cols)
    rows, cols = key // n, key % n
    deg = np.bincount(rows, minlength=n).astype(np.int64)
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(deg, out=indptr[1:])
    vals = 1.0 / np.sqrt(deg[rows].astype(np.float64) * deg[cols].astype(np.float64))
    return {"indptr": indptr, "indices": cols.astype(np.int32), "data": vals.astype(np.float32), "shape": (n, n)}


def stencil5(side):
    """2-D 5-point Laplacian stencil on a side x side grid (values 4 / -1)."""
    n = side * side
    r = np.arange(n, dtype=np.int64)
    i, j = r // side, r % side
    cols, vals, rows = [], [], []
    for di, dj, v in ((-1, 0, -1.0), (0, -1, -1.0), (0, 0, 4.0), (0, 1, -1.0), (1, 0, -1.0)):
        ok = (i + di >= 0) & (i + di < side) & (j + dj >= 0) & (j + dj < side)
        rows.append(r[ok])
        cols.append((i[ok] + di) * side + (j[ok] + dj))
        vals.append(np.full(int(ok.sum()), v))
    rows, cols, vals = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=indptr[1:])
    return indptr, cols.astype(np.int32), vals.astype(np.float32)


def batched_mix(count=256, lo=1_000, hi=200_000, mean_len=24.0, n_dense=16, seed=4):
    """Configuration 5: `count` matrices with log-uniform row counts in [lo, hi].

    Even ids: 5-point stencil on a round(sqrt(rows))^2 grid; odd ids: random
    square CSR with Poisson(mean_len) row lengths (>= 1).  Each matrix comes
    with an x vector and an `n_dense`-column B, fp32.
    """
    rng = _rng(seed)
    mats = []
    for k in range(count):
        rows = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))
        if k % 2 == 0:
            side = max(2, int(round(math.sqrt(rows))))
            indptr, indices, data = stencil5(side)
            n = side * side
        else:
            n = rows
            lengths = np.minimum(n, np.maximum(1, rng.poisson(mean_len, n))).astype(np.int64)
            indptr, indices = distinct_sorted_columns(rng, lengths, n)
            data = rng.uniform(-1.0, 1.0, indices.size).astype(np.float32)
        x = rng.uniform(-1.0, 1.0, n).astype(np.float32)
        b = rng.uniform(-1.0, 1.0, (n, n_dense)).astype(np.float32)
        mats.append({"indptr": indptr, "indices": indices, "data": data, "x": x, "B": b, "shape": (n, n)})
    return mats


def mask_csr(m, n, seed, dtype=np.float64, density=None, long_rows=()):
    """Small mask-based random CSR like FlagSparse's accuracy tests
    (tests/pytest/test_spmv_csr_accuracy.py:66-82): density
    min(0.25, max(0.06, 32/(m n))), plus optional dense `long_rows`."""
    rng = _rng(seed)
    p = density if density is not None else min(0.25, max(0.06, 32.0 / max(m * n, 1)))
    mask = rng.random((m, n)) < p
    for r in long_rows:
        mask[r, :] = True
    if not mask.any():
        mask[0, 0] = True
    rows, cols = np.nonzero(mask)
    indptr = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=m), out=indptr[1:])
    nnz = rows.size
    if np.issubdtype(np.dtype(dtype), np.complexfloating):
        data = (rng.standard_normal(nnz) + 1j * rng.standard_normal(nnz)).astype(dtype)
    else:
        data = rng.standard_normal(nnz).astype(dtype)
    return {"indptr": indptr, "indices": cols.astype(np.int32), "data": data, "shape": (m, n)}
