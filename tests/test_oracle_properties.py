"""Size-independent properties of the oracle on random patterns (CPU only).

The golden fixtures pin the oracle to FlagSparse's own outputs on chosen
cases; these properties check the same functions on many random ones:
transposes compose to the identity, COO -> CSR and the transpose agree with
stable numpy sorts, the products are linear and consistent with each other,
and the unit plan covers every nonzero once within its window and chunk
limits.
"""

import numpy as np
from hypothesis import given, settings, strategies as st

from oracle import oracle


@st.composite
def patterns(draw, max_rows=120, max_cols=90):
    n_rows = draw(st.integers(0, max_rows))
    n_cols = draw(st.integers(1, max_cols))
    seed = draw(st.integers(0, 2**31 - 1))
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, min(n_cols, 12) + 1, size=n_rows)
    rows = [np.sort(rng.choice(n_cols, size=int(k), replace=False)) for k in lens]
    indptr = np.zeros(n_rows + 1, dtype=np.int64)
    indptr[1:] = np.cumsum(lens)
    indices = (np.concatenate(rows) if rows else np.empty(0)).astype(np.int32)
    data = rng.uniform(-1.0, 1.0, size=indices.size)
    return indptr, indices, data, n_rows, n_cols, rng


def _dense(indptr, indices, data, n_rows, n_cols):
    a = np.zeros((n_rows, n_cols))
    for r in range(n_rows):
        for p in range(indptr[r], indptr[r + 1]):
            a[r, indices[p]] += data[p]
    return a


@settings(max_examples=60, deadline=None, derandomize=True)
@given(patterns())
def test_transpose_twice_is_identity(pat):
    indptr, indices, data, n_rows, n_cols, _ = pat
    t_ptr, t_idx, perm = oracle.transpose(indptr, indices, n_cols)
    b_ptr, b_idx, perm2 = oracle.transpose(t_ptr, t_idx, n_rows)
    assert np.array_equal(b_ptr, indptr) and np.array_equal(b_idx, indices)
    assert np.array_equal(perm[perm2], np.arange(indices.size))
    assert np.allclose(_dense(t_ptr, t_idx, data[perm], n_cols, n_rows), _dense(indptr, indices, data, n_rows, n_cols).T)


@settings(max_examples=60, deadline=None, derandomize=True)
@given(patterns())
def test_transpose_matches_stable_argsort(pat):
    indptr, indices, _, n_rows, n_cols, _ = pat
    t_ptr, t_idx, perm = oracle.transpose(indptr, indices, n_cols)
    rows = np.repeat(np.arange(n_rows), np.diff(indptr))
    order = np.argsort(indices, kind="stable")
    assert np.array_equal(perm, order)
    assert np.array_equal(t_idx, rows[order])
    assert np.array_equal(t_ptr, np.concatenate([[0], np.cumsum(np.bincount(indices, minlength=n_cols))]))


@settings(max_examples=60, deadline=None, derandomize=True)
@given(patterns())
def test_coo_to_csr_matches_stable_lexsort(pat):
    indptr, indices, _, n_rows, n_cols, rng = pat
    rows = np.repeat(np.arange(n_rows), np.diff(indptr))
    shuf = rng.permutation(indices.size)
    r, c = rows[shuf], indices[shuf].astype(np.int64)
    ptr, idx, perm = oracle.coo_to_csr(r, c, n_rows, n_cols)
    order = np.lexsort((c, r))  # stable: by row, then column, then input position
    assert np.array_equal(perm, order)
    assert np.array_equal(idx, c[order])
    assert np.array_equal(ptr, indptr)


@settings(max_examples=40, deadline=None, derandomize=True)
@given(patterns(), st.floats(-3, 3), st.floats(-3, 3))
def test_spmv_linear_and_spmm_columnwise(pat, a, b):
    indptr, indices, data, n_rows, n_cols, rng = pat
    x, y = rng.standard_normal(n_cols), rng.standard_normal(n_cols)
    lhs = oracle.spmv(indptr, indices, data, a * x + b * y)
    rhs = a * oracle.spmv(indptr, indices, data, x) + b * oracle.spmv(indptr, indices, data, y)
    scale = oracle.spmv_abs(indptr, indices, np.abs(data), np.abs(x) * abs(a) + np.abs(y) * abs(b))
    assert np.all(np.abs(lhs - rhs) <= 1e-13 * (scale + 1e-300) + 1e-300)
    B = np.stack([x, y, a * x], axis=1)
    C = oracle.spmm(indptr, indices, data, B)
    for j in range(B.shape[1]):
        ref = oracle.spmv(indptr, indices, data, B[:, j])
        s = oracle.spmv_abs(indptr, indices, np.abs(data), np.abs(B[:, j]))
        assert np.all(np.abs(C[:, j] - ref) <= 1e-13 * (s + 1e-300) + 1e-300)


@settings(max_examples=40, deadline=None, derandomize=True)
@given(patterns())
def test_sddmm_matches_dense_dots(pat):
    indptr, indices, data, n_rows, n_cols, rng = pat
    k = int(rng.integers(1, 9))
    X, Y = rng.standard_normal((n_rows, k)), rng.standard_normal((n_cols, k))
    out = oracle.sddmm(indptr, indices, X, Y, data, alpha=1.5, beta=-0.25)
    rows = np.repeat(np.arange(n_rows), np.diff(indptr))
    ref = 1.5 * np.einsum("ij,ij->i", X[rows], Y[indices]) - 0.25 * data
    assert np.allclose(out, ref, rtol=1e-12, atol=1e-12)


@st.composite
def row_lengths(draw):
    n = draw(st.integers(1, 400))
    seed = draw(st.integers(0, 2**31 - 1))
    rng = np.random.default_rng(seed)
    lens = rng.integers(0, 9, size=n)
    heavy = rng.random(n) < 0.03
    lens[heavy] = rng.integers(100, 3000, size=int(heavy.sum()))
    return np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)


@settings(max_examples=60, deadline=None, derandomize=True)
@given(row_lengths(), st.sampled_from([4, 16, 64, 128, 224]), st.sampled_from([256, 512, 1024]))
def test_unit_plan_covers_every_nonzero_once(indptr, cap, chunk):
    _, _, units = oracle.spmv_plan(indptr, cap, chunk)
    lens = np.diff(indptr)
    nnz = int(indptr[-1])
    tags = units[:, 3]
    blocks = units[tags >= 0]
    chunks = units[tags < 0]
    assert np.all(np.diff((tags < 0).astype(int)) >= 0)  # row blocks first, then chunks
    covered = np.zeros(nnz, dtype=np.int32)
    row_seen = np.zeros(lens.size, dtype=np.int32)
    for b0, b1, r0, r1, nch, slot in blocks:
        assert r0 < r1 and r1 - r0 <= cap and nch == 1 and slot == -1
        assert np.all(lens[r0:r1] <= cap)
        assert b0 == indptr[r0] and b1 == indptr[r1] and b1 - b0 < 2 * cap
        covered[b0:b1] += 1
        row_seen[r0:r1] += 1
    slots = {}
    for b0, b1, r, tag, nch, slot in chunks:
        c = -(tag + 1)
        n = lens[r]
        assert n > cap and nch == -(-n // chunk) and 0 <= c < nch
        assert b0 == indptr[r] + c * chunk and b1 == min(indptr[r + 1], b0 + chunk)
        assert (slot == -1) == (nch == 1)
        if nch > 1:
            slots.setdefault(int(r), []).append((int(c), int(slot)))
        covered[b0:b1] += 1
        if c == 0:
            row_seen[r] += 1
    assert np.all(covered == 1)
    assert np.all(row_seen == 1)
    for r, cs in slots.items():  # a row's slots are consecutive, in chunk order
        cs.sort()
        assert [s - cs[0][1] for _, s in cs] == list(range(len(cs)))
