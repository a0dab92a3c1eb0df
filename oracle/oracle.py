"""numpy/ctypes front end of the C oracle (``csr_oracle.c``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, by ``__graft_entry__.smoke``
and by the CPU-baseline leg of ``bench.py``, always as the checker.  The
product package never imports it.

Inputs are numpy arrays (or anything ``np.asarray`` accepts).  Index arrays are
normalised to the oracle's layout (int64 indptr, int32 column indices).  See
``csr_oracle.c`` for the FlagSparse source lines each routine follows.
"""

import ctypes
import os
import subprocess

import numpy as np

_DIR = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_DIR, "liboracle.so")
_lib = None

_p = ctypes.c_void_p
_i64 = ctypes.c_int64
_int = ctypes.c_int
_dbl = ctypes.c_double

_SIGS = {
    "oracle_max_threads": (_int, []),
    "oracle_spmv_f32_acc64": (None, [_i64, _p, _p, _p, _p, _p, _int]),
    "oracle_spmv_dot2": (None, [_i64, _p, _p, _p, _p, _p, _int]),
    "oracle_spmv_dot2_c": (None, [_i64, _p, _p, _p, _p, _p, _int]),
    "oracle_spmm_dot2": (None, [_i64, _i64, _p, _p, _p, _p, _p, _int]),
    "oracle_spmm_f32_acc64": (None, [_i64, _i64, _p, _p, _p, _p, _p, _int]),
    "oracle_sddmm_dot2": (None, [_i64, _i64, _p, _p, _p, _p, _p, _dbl, _dbl, _p, _int]),
    "oracle_transpose": (None, [_i64, _i64, _p, _p, _p, _p, _p]),
    "oracle_coo_to_csr": (None, [_i64, _i64, _i64, _p, _p, _p, _p, _p]),
    "oracle_bucketize": (None, [_i64, _p, _p, _int, _p, _p]),
    "oracle_spmv_plan": (None, [_i64, _p, _i64, _i64, _p, _p, _p, _p]),
}


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _DIR], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        h = ctypes.CDLL(_LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib


def _a(x, dtype):
    return np.ascontiguousarray(np.asarray(x), dtype=dtype)


def _ptr(a):
    return a.ctypes.data if a.size else None


def max_threads():
    return int(lib().oracle_max_threads())


def csr_arrays(indptr, indices):
    return _a(indptr, np.int64), _a(indices, np.int32)


def spmv_f32_acc64(indptr, indices, data, x, nthreads=0):
    """fp32 SpMV with fp64 row sums, rounded to fp32 (FlagSparse's fp32 semantics)."""
    ptr, idx = csr_arrays(indptr, indices)
    data, x = _a(data, np.float32), _a(x, np.float32)
    m = ptr.size - 1
    y = np.empty(m, dtype=np.float32)
    lib().oracle_spmv_f32_acc64(m, _ptr(ptr), _ptr(idx), _ptr(data), _ptr(x), _ptr(y), int(nthreads))
    return y


def spmv(indptr, indices, data, x, nthreads=0):
    """Accurate SpMV (Dot2), returns float64 (or complex128 for complex input)."""
    ptr, idx = csr_arrays(indptr, indices)
    m = ptr.size - 1
    if np.iscomplexobj(data) or np.iscomplexobj(x):
        d = _a(data, np.complex128).view(np.float64)
        xv = _a(x, np.complex128).view(np.float64)
        y = np.empty(2 * m, dtype=np.float64)
        lib().oracle_spmv_dot2_c(m, _ptr(ptr), _ptr(idx), _ptr(d), _ptr(xv), _ptr(y), int(nthreads))
        return y.view(np.complex128)
    d, xv = _a(data, np.float64), _a(x, np.float64)
    y = np.empty(m, dtype=np.float64)
    lib().oracle_spmv_dot2(m, _ptr(ptr), _ptr(idx), _ptr(d), _ptr(xv), _ptr(y), int(nthreads))
    return y


def spmv_abs(indptr, indices, data, x, nthreads=0):
    """sum_k |a_k| |x_k| per row: the scale of the rounding-error bound of row r."""
    return spmv(indptr, indices, np.abs(np.asarray(data)).astype(np.float64),
                np.abs(np.asarray(x)).astype(np.float64), nthreads)


def _spmm_real(ptr, idx, data, b, nthreads):
    m = ptr.size - 1
    n = b.shape[1]
    d, bb = _a(data, np.float64), _a(b, np.float64)
    c = np.empty((m, n), dtype=np.float64)
    lib().oracle_spmm_dot2(m, n, _ptr(ptr), _ptr(idx), _ptr(d), _ptr(bb), _ptr(c), int(nthreads))
    return c


def spmm(indptr, indices, data, b, nthreads=0):
    """Accurate C = A B (Dot2 per entry); complex handled as four real products."""
    ptr, idx = csr_arrays(indptr, indices)
    b = np.asarray(b)
    if np.iscomplexobj(data) or np.iscomplexobj(b):
        d = np.asarray(data).astype(np.complex128)
        bc = b.astype(np.complex128)
        rr = _spmm_real(ptr, idx, d.real, bc.real, nthreads)
        ii = _spmm_real(ptr, idx, d.imag, bc.imag, nthreads)
        ri = _spmm_real(ptr, idx, d.real, bc.imag, nthreads)
        ir = _spmm_real(ptr, idx, d.imag, bc.real, nthreads)
        return (rr - ii) + 1j * (ri + ir)
    return _spmm_real(ptr, idx, data, b, nthreads)


def spmm_f32_acc64(indptr, indices, data, b, nthreads=0):
    ptr, idx = csr_arrays(indptr, indices)
    d, bb = _a(data, np.float32), _a(b, np.float32)
    m, n = ptr.size - 1, bb.shape[1]
    c = np.empty((m, n), dtype=np.float32)
    lib().oracle_spmm_f32_acc64(m, n, _ptr(ptr), _ptr(idx), _ptr(d), _ptr(bb), _ptr(c), int(nthreads))
    return c


def sddmm(indptr, indices, x, y, data=None, alpha=1.0, beta=0.0, nthreads=0):
    """out[p] = alpha <x[row(p)], y[col(p)]> + beta data[p] (Dot2), float64."""
    ptr, idx = csr_arrays(indptr, indices)
    xx, yy = _a(x, np.float64), _a(y, np.float64)
    m, k = ptr.size - 1, xx.shape[1]
    nnz = idx.size
    d = _a(data, np.float64) if data is not None else None
    out = np.empty(nnz, dtype=np.float64)
    lib().oracle_sddmm_dot2(m, k, _ptr(ptr), _ptr(idx), _ptr(xx), _ptr(yy),
                            _ptr(d) if d is not None else None, float(alpha), float(beta), _ptr(out), int(nthreads))
    return out


def transpose(indptr, indices, n_cols):
    """Stable CSR transpose: (t_indptr int64, t_indices int32, perm int64)."""
    ptr, idx = csr_arrays(indptr, indices)
    m = ptr.size - 1
    nnz = idx.size
    t_ptr = np.empty(int(n_cols) + 1, dtype=np.int64)
    t_idx = np.empty(nnz, dtype=np.int32)
    perm = np.empty(nnz, dtype=np.int64)
    lib().oracle_transpose(m, int(n_cols), _ptr(ptr), _ptr(idx), _ptr(t_ptr), _ptr(t_idx), _ptr(perm))
    return t_ptr, t_idx, perm


def coo_to_csr(row, col, n_rows, n_cols):
    """COO pattern -> CSR: (indptr int64, indices int32, perm int64), stable in (row, col) order."""
    r = _a(row, np.int64)
    c = _a(col, np.int64)
    nnz = r.size
    ptr = np.empty(int(n_rows) + 1, dtype=np.int64)
    idx = np.empty(nnz, dtype=np.int32)
    perm = np.empty(nnz, dtype=np.int64)
    lib().oracle_coo_to_csr(int(n_rows), int(n_cols), nnz, _ptr(r), _ptr(c), _ptr(ptr), _ptr(idx), _ptr(perm))
    return ptr, idx, perm


def bsr_to_csr(blocks, indices, indptr, block_dim):
    """Expand a BSR matrix (blocks [nnzb, bd, bd] row-major) to CSR over the padded
    shape: (indptr int64, indices int32, values), every stored block value kept.

    Restates the index arithmetic of FlagSparse's BSR SpMV kernels
    (sparse_operations/spmv_bsr.py:183-223: row = brow * bd + inner_row,
    col = bcol * bd + inner_col); the SpMV itself then runs on the CSR oracle.
    """
    bd = int(block_dim)
    bptr = _a(indptr, np.int64)
    bcol = _a(indices, np.int64)
    vals = np.asarray(blocks)
    nbr = bptr.size - 1
    lens = np.diff(bptr) * bd
    ptr = np.zeros(nbr * bd + 1, dtype=np.int64)
    ptr[1:] = np.cumsum(np.repeat(lens, bd))
    idx = np.empty(int(ptr[-1]), dtype=np.int32)
    out = np.empty(int(ptr[-1]), dtype=vals.dtype)
    for br in range(nbr):
        ks = np.arange(bptr[br], bptr[br + 1])
        for r in range(bd):
            row = br * bd + r
            a, b = ptr[row], ptr[row + 1]
            idx[a:b] = (bcol[ks][:, None] * bd + np.arange(bd)[None, :]).reshape(-1)
            out[a:b] = vals[ks, r, :].reshape(-1)
    return ptr, idx, out


def bucketize(indptr, upper_bounds):
    """Row lists per length bucket (ascending rows); None = unbounded."""
    ptr = _a(indptr, np.int64)
    m = ptr.size - 1
    ub = np.array([-1 if u is None else int(u) for u in upper_bounds], dtype=np.int64)
    rows = np.empty(max(m, 1), dtype=np.int32)
    counts = np.empty(ub.size, dtype=np.int64)
    lib().oracle_bucketize(m, _ptr(ptr), _ptr(ub), int(ub.size), _ptr(rows), _ptr(counts))
    out, off = [], 0
    for c in counts:
        out.append(rows[off:off + int(c)].copy())
        off += int(c)
    return out


def spmv_plan(indptr, cap, chunk):
    """(seg_row0, seg_unit0, units) of the native SpMV unit plan.

    ``units`` is int64 [n_units, 6]: nnz_begin, nnz_end, row, tag, n_chunks, slot.
    """
    ptr = _a(indptr, np.int64)
    m = ptr.size - 1
    totals = np.zeros(4, dtype=np.int64)
    lib().oracle_spmv_plan(m, _ptr(ptr), int(cap), int(chunk), _ptr(totals), None, None, None)
    s, u = int(totals[0]), int(totals[1])
    seg_row0 = np.empty(s + 1, dtype=np.int32)
    seg_unit0 = np.empty(s + 1, dtype=np.int32)
    units = np.empty((max(u, 1), 6), dtype=np.int64)
    lib().oracle_spmv_plan(m, _ptr(ptr), int(cap), int(chunk), _ptr(totals), _ptr(seg_row0), _ptr(seg_unit0),
                           _ptr(units))
    return seg_row0, seg_unit0, units[:u]
