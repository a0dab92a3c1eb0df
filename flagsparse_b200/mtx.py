"""MatrixMarket (.mtx) coordinate files to CSR, for real-matrix validation.

Same reading as FlagSparse's test loader ``load_mtx_to_csr_torch``
(tests/test_spmv.py:116-190):

- the ``%%MatrixMarket`` banner gives the field and the symmetry; other
  ``%`` lines are comments; the first non-comment line is
  ``n_rows n_cols nnz``; the next ``nnz`` non-empty lines are entries;
- indices are 1-based; entries outside the matrix are dropped;
- ``pattern`` entries are 1.0; otherwise the third token is the value (the
  real part for complex fields);
- ``symmetric`` / ``hermitian`` mirror every off-diagonal entry,
  ``skew-symmetric`` mirrors it negated;
- repeated (row, col) entries are summed in file order, each entry followed
  by its mirror; the CSR has ascending columns per row.

Returns ``(data, indices, indptr, shape)`` with int64 indices and row
pointers.  The parsing is vectorised with numpy, so SuiteSparse-sized files
load in seconds.
"""

import numpy as np
import torch


def _read(file_path):
    field, symmetry = "real", "general"
    header = None
    entries = []
    with open(file_path, "r", encoding="utf-8") as f:
        for line in f:
            s = line.strip()
            if s.startswith("%%MatrixMarket"):
                tokens = s.split()
                if len(tokens) >= 5:
                    field, symmetry = tokens[3].lower(), tokens[4].lower()
                continue
            if s.startswith("%") or not s:
                continue
            if header is None:
                parts = s.split()
                header = (int(parts[0]), int(parts[1]), int(parts[2]) if len(parts) > 2 else 0)
                continue
            entries.append(s)
            if len(entries) >= header[2]:
                break
    if header is None:
        raise ValueError(f"Cannot parse .mtx header: {file_path}")
    return field, symmetry, header, entries


def mtx_to_csr_arrays(file_path):
    """numpy CSR of a .mtx file: (data float64, indices int64, indptr int64, shape)."""
    field, symmetry, (n_rows, n_cols, nnz), entries = _read(file_path)
    if nnz == 0 or not entries:
        return np.zeros(0), np.zeros(0, np.int64), np.zeros(n_rows + 1, np.int64), (n_rows, n_cols)
    pattern = field == "pattern"
    ncol = 2 if pattern else 3
    tok = np.array([e.split()[:ncol] for e in entries], dtype=object)
    r = tok[:, 0].astype(np.int64) - 1
    c = tok[:, 1].astype(np.int64) - 1
    v = np.ones(r.size) if pattern else tok[:, 2].astype(np.float64)
    keep = (r >= 0) & (r < n_rows) & (c >= 0) & (c < n_cols)
    r, c, v = r[keep], c[keep], v[keep]
    sym = symmetry in ("symmetric", "hermitian")
    skew = symmetry == "skew-symmetric"
    if sym or skew:
        # each entry, then its mirror (off-diagonal, inside the matrix), in file order
        mirror = (r != c) & (c < n_rows) & (r < n_cols)
        mr, mc, mv = c[mirror], r[mirror], (-v[mirror] if skew else v[mirror])
        order = np.concatenate([np.arange(r.size) * 2, np.nonzero(mirror)[0] * 2 + 1])
        rr = np.concatenate([r, mr])
        cc = np.concatenate([c, mc])
        vv = np.concatenate([v, mv])
        seq = np.argsort(order, kind="stable")
        r, c, v = rr[seq], cc[seq], vv[seq]
    key = r * max(n_cols, 1) + c
    perm = np.argsort(key, kind="stable")
    key_s, v_s = key[perm], v[perm]
    starts = np.concatenate([[0], np.nonzero(key_s[1:] != key_s[:-1])[0] + 1])
    ends = np.append(starts[1:], key_s.size)
    data = v_s[starts].copy()
    for j in np.nonzero(ends - starts > 1)[0]:
        acc = 0.0  # repeated entries: summed one by one in file order
        for t in v_s[starts[j]:ends[j]]:
            acc += float(t)
        data[j] = acc
    uk = key_s[starts]
    rows = uk // max(n_cols, 1)
    cols = uk % max(n_cols, 1)
    indptr = np.zeros(n_rows + 1, dtype=np.int64)
    np.add.at(indptr, rows + 1, 1)
    return data, cols.astype(np.int64), np.cumsum(indptr), (n_rows, n_cols)


def load_mtx_to_csr_torch(file_path, dtype=torch.float32, device=None):
    """Load a SuiteSparse / MatrixMarket .mtx file into CSR torch tensors on ``device``."""
    if device is None:
        device = torch.device("cuda" if torch.cuda.is_available() else "cpu")
    data, indices, indptr, shape = mtx_to_csr_arrays(file_path)
    return (torch.tensor(data, dtype=dtype, device=device), torch.from_numpy(indices).to(device),
            torch.from_numpy(indptr).to(device), shape)
