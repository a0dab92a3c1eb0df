"""Native CSR plumbing shared by the SpMV / SpMM / SDDMM host code.

Thin wrappers over the C ABI: inspection (one synchronising read instead of
a chain of ``.item()`` calls), the stable transpose, stable row-length
bucketing and the SpMV unit plan.  Device memory comes from torch; every
computation runs in the native library.
"""

import ctypes

import torch

from .. import _native as nat


def inspect_csr(indices, indptr, n_rows, nnz):
    """Return a dict with indptr[0], indptr[-1], #decreasing steps, min/max column, max row length.

    One kernel, one device-to-host read.
    """
    out = torch.empty(6, dtype=torch.int64, device=indptr.device)
    if n_rows + 1 == 0:
        raise ValueError("indptr must have at least one entry")
    lib = nat.lib()
    idx = indices if (indices is not None and nnz > 0) else None
    nat.check(
        lib.fsb_csr_inspect(
            nat.ptr(idx), nat.is64(indices) if indices is not None else 0,
            nat.ptr(indptr), nat.is64(indptr), int(n_rows), int(nnz),
            nat.ptr(out), nat.stream_of(indptr.device),
        ),
        "fsb_csr_inspect",
    )
    v = out.tolist()
    return {
        "first": v[0],
        "last": v[1],
        "decreasing": v[2],
        "min_col": v[3] if nnz > 0 else None,
        "max_col": v[4] if nnz > 0 else None,
        "max_row_nnz": v[5] if n_rows > 0 else 0,
    }


def transpose_pattern(indices, indptr, shape, out_index_dtype, out_indptr_dtype):
    """Stable CSR transpose of the pattern.

    Returns ``(t_indices, t_indptr, perm)`` where ``perm[k]`` is the source
    position of transposed entry ``k``.  Identical to a stable argsort by
    column followed by bincount/cumsum.
    """
    n_rows, n_cols = int(shape[0]), int(shape[1])
    nnz = int(indices.numel())
    device = indices.device
    t_indices = torch.empty(nnz, dtype=out_index_dtype, device=device)
    t_indptr = torch.empty(n_cols + 1, dtype=out_indptr_dtype, device=device)
    perm = torch.empty(nnz, dtype=torch.int64, device=device)
    lib = nat.lib()
    ws_bytes = int(lib.fsb_csr_transpose_workspace_bytes(nnz, n_rows, n_cols)) if nnz > 0 else 0
    if ws_bytes < 0:
        raise RuntimeError("CSR transpose: nnz must be < 2^31")
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=device)
    nat.check(
        lib.fsb_csr_transpose(
            nat.ptr(indices), nat.is64(indices), nat.ptr(indptr), nat.is64(indptr),
            n_rows, n_cols, nnz, nat.ptr(ws), ws_bytes,
            nat.ptr(t_indices), 1 if out_index_dtype == torch.int64 else 0,
            nat.ptr(t_indptr), 1 if out_indptr_dtype == torch.int64 else 0,
            nat.ptr(perm), nat.stream_of(device),
        ),
        "fsb_csr_transpose",
    )
    return t_indices, t_indptr, perm


def coo_inspect(row, col, n_rows, n_cols):
    """(pairs out of (row, col) order, rows outside [0, n_rows), columns outside [0, n_cols)).

    One kernel, one device-to-host read.
    """
    out = torch.empty(3, dtype=torch.int64, device=row.device)
    nnz = int(row.numel())
    nat.check(
        nat.lib().fsb_coo_inspect(
            nat.ptr(row) if nnz else None, nat.is64(row), nat.ptr(col) if nnz else None, nat.is64(col), nnz,
            int(n_rows), int(n_cols), nat.ptr(out), nat.stream_of(row.device),
        ),
        "fsb_coo_inspect",
    )
    unsorted, bad_rows, bad_cols = out.tolist()
    return unsorted, bad_rows, bad_cols


def coo_to_csr(row, col, n_rows, n_cols, ordered):
    """CSR pattern of a COO pattern: ``(indices int32, indptr int64, perm)``.

    ``ordered``: the pairs are already in (row, col) order; then ``perm`` is
    None (identity).  Otherwise ``perm`` (int64) holds the source position of
    every CSR entry, from a stable sort (repeated pairs keep their order).
    """
    nnz = int(row.numel())
    device = row.device
    indices = torch.empty(nnz, dtype=torch.int32, device=device)
    indptr = torch.empty(int(n_rows) + 1, dtype=torch.int64, device=device)
    lib = nat.lib()
    perm = ws = None
    ws_bytes = 0
    if not ordered and nnz > 0:
        ws_bytes = int(lib.fsb_coo_to_csr_workspace_bytes(nnz, int(n_rows), int(n_cols)))
        if ws_bytes < 0:
            raise RuntimeError("COO to CSR: nnz must be < 2^31")
        ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=device)
        perm = torch.empty(nnz, dtype=torch.int64, device=device)
    nat.check(
        lib.fsb_coo_to_csr(
            nat.ptr(row) if nnz else None, nat.is64(row), nat.ptr(col) if nnz else None, nat.is64(col), nnz,
            int(n_rows), int(n_cols), 1 if ordered else 0, nat.ptr(ws), ws_bytes, nat.ptr(indices) if nnz else None,
            nat.ptr(indptr), nat.ptr(perm), nat.stream_of(device),
        ),
        "fsb_coo_to_csr",
    )
    return indices, indptr, perm


def gather_values(values, perm, conj=False):
    """values[perm] (conjugated for complex when ``conj``), computed natively."""
    out = torch.empty(perm.numel(), dtype=values.dtype, device=values.device)
    nat.check(
        nat.lib().fsb_gather_values(
            nat.dtype_code(values.dtype), nat.ptr(values), nat.ptr(perm), int(perm.numel()),
            1 if conj else 0, nat.ptr(out), nat.stream_of(values.device),
        ),
        "fsb_gather_values",
    )
    return out


def bucketize_rows(indptr, n_rows, upper_bounds):
    """Stable row lists per row-length bucket.

    ``upper_bounds[b]`` is the inclusive upper length of bucket ``b`` (``None``
    = unbounded); bucket 0 includes empty rows.  Returns a list of int32
    tensors (views into one buffer), one per bucket.
    """
    nb = len(upper_bounds)
    device = indptr.device
    rows = torch.empty(max(int(n_rows), 1), dtype=torch.int32, device=device)
    counts = torch.zeros(nb, dtype=torch.int64, device=device)
    ub = (ctypes.c_int64 * nb)(*[-1 if u is None else int(u) for u in upper_bounds])
    lib = nat.lib()
    ws_bytes = int(lib.fsb_csr_bucketize_workspace_bytes(int(n_rows), nb))
    ws = torch.empty(max(ws_bytes, 8), dtype=torch.uint8, device=device)
    nat.check(
        lib.fsb_csr_bucketize(
            nat.ptr(indptr), nat.is64(indptr), int(n_rows), ub, nb,
            nat.ptr(ws), ws_bytes, nat.ptr(rows), nat.ptr(counts), nat.stream_of(device),
        ),
        "fsb_csr_bucketize",
    )
    out = []
    off = 0
    for c in counts.tolist():
        out.append(rows[off:off + c])
        off += c
    return out


class NativeSpmvPlan:
    """Device arrays of the SpMV unit plan plus its scratch (see fsb_spmv_plan)."""

    __slots__ = ("seg_row0", "seg_unit0", "units", "partials", "counters", "cap", "chunk_nnz",
                 "n_segs", "n_units", "n_slots", "n_block_units", "dtype", "flags", "_struct")

    def __init__(self, indptr, n_rows, dtype, cap=None, chunk_nnz=None, fast_short_rows=False, scratch=True):
        lib = nat.lib()
        code = nat.dtype_code(dtype)
        device = indptr.device
        self.dtype = dtype
        self.cap = int(cap) if cap is not None else int(lib.fsb_spmv_default_cap(code))
        self.chunk_nnz = int(chunk_nnz) if chunk_nnz is not None else int(lib.fsb_spmv_default_chunk(code))
        n_rows = int(n_rows)
        st = nat.stream_of(device)
        ws_bytes = int(lib.fsb_spmv_plan_workspace_bytes(n_rows))
        ws = torch.empty(max(ws_bytes, 8), dtype=torch.uint8, device=device)
        totals = torch.zeros(4, dtype=torch.int64, device=device)
        if n_rows > 0:
            nat.check(
                lib.fsb_spmv_plan_analyze(nat.ptr(indptr), nat.is64(indptr), n_rows, self.cap,
                                          self.chunk_nnz, nat.ptr(ws), ws_bytes, nat.ptr(totals), st),
                "fsb_spmv_plan_analyze",
            )
        self.n_segs, self.n_units, self.n_slots, self.n_block_units = (int(v) for v in totals.tolist())
        self.seg_row0 = torch.empty(self.n_segs + 1, dtype=torch.int32, device=device)
        self.seg_unit0 = torch.empty(self.n_segs + 1, dtype=torch.int32, device=device)
        # fsb_spmv_unit: int64 nnz_begin, nnz_end; int32 row, tag, n_chunks, slot (32 bytes)
        self.units = torch.empty((max(self.n_units, 1), 4), dtype=torch.int64, device=device)
        if n_rows > 0:
            nat.check(
                lib.fsb_spmv_plan_build(nat.ptr(indptr), nat.is64(indptr), n_rows, self.cap,
                                        self.chunk_nnz, nat.ptr(ws), ws_bytes, nat.ptr(self.seg_row0),
                                        nat.ptr(self.seg_unit0), nat.ptr(self.units), st),
                "fsb_spmv_plan_build",
            )
        if scratch:
            pbytes = int(lib.fsb_spmv_partial_bytes(code))
            self.partials = torch.empty(max(self.n_slots * pbytes, 16), dtype=torch.uint8, device=device)
            self.counters = torch.zeros(max(self.n_slots, 1), dtype=torch.int32, device=device)
        else:  # the caller attaches scratch (see SpmmPlan)
            self.partials = None
            self.counters = None
        self.flags = nat.FSB_SPMV_FAST_SHORT_ROWS if fast_short_rows else 0
        self._struct = nat.SpmvPlan(
            nat.ptr(self.seg_row0), nat.ptr(self.seg_unit0), nat.ptr(self.units),
            self.n_segs, self.n_units, self.n_slots, self.n_block_units, self.cap, self.chunk_nnz,
            nat.ptr(self.partials), nat.ptr(self.counters), self.flags, 0,
        )

    def set_fast_short_rows(self, on):
        self.flags = nat.FSB_SPMV_FAST_SHORT_ROWS if on else 0
        self._struct.flags = self.flags

    def struct_ref(self):
        return ctypes.byref(self._struct)

    def unit_table(self):
        """Host copy of the unit descriptors as columns (begin, end, row, tag, n_chunks, slot)."""
        u = self.units[: self.n_units].cpu()
        packed = u[:, 2]
        row = (packed & 0xFFFFFFFF).to(torch.int64)
        row = torch.where(row >= 2**31, row - 2**32, row)
        tag = packed >> 32
        nch = (u[:, 3] & 0xFFFFFFFF).to(torch.int64)
        slot = u[:, 3] >> 32
        return u[:, 0].numpy(), u[:, 1].numpy(), row.numpy(), tag.numpy(), nch.numpy(), slot.numpy()


class SpmmPlan:
    """The SpMM launch plan: a unit plan built with the SpMM window and chunk,
    plus long-row scratch sized per dense width N (allocated once per N and
    reused; fsb_spmm_csr leaves the tickets zero after every call)."""

    def __init__(self, indptr, n_rows, dtype, cap=None, chunk_nnz=None):
        lib = nat.lib()
        code = nat.dtype_code(dtype)
        self.dtype = dtype
        cap = int(lib.fsb_spmm_default_cap(code)) if cap is None else int(cap)
        chunk_nnz = int(lib.fsb_spmm_default_chunk(code)) if chunk_nnz is None else int(chunk_nnz)
        self.plan = NativeSpmvPlan(indptr, n_rows, dtype, cap=cap, chunk_nnz=chunk_nnz, scratch=False)
        self._scratch = {}  # n -> (partials, counters, SpmvPlan struct)

    @property
    def n_units(self):
        return self.plan.n_units

    @property
    def n_slots(self):
        return self.plan.n_slots

    def struct_for(self, n, compensated=False, tile_bytes=0, persistent=False):
        """ctypes reference to an fsb_spmv_plan with scratch for dense width ``n``.

        ``tile_bytes``: column tile of the team kernel (0 = the library's choice);
        ``persistent``: the team kernel's persistent grid (FSB_SPMM_PERSISTENT)."""
        key = int(n)
        entry = self._scratch.get(key)
        if entry is None:
            pb, tk = ctypes.c_int64(0), ctypes.c_int64(0)
            nat.check(nat.lib().fsb_spmm_scratch_layout(nat.dtype_code(self.dtype), key, ctypes.byref(pb),
                                                        ctypes.byref(tk)), "fsb_spmm_scratch_layout")
            device = self.plan.units.device
            slots = self.plan.n_slots
            partials = torch.empty(max(slots * pb.value, 16), dtype=torch.uint8, device=device)
            counters = torch.zeros(max(slots * tk.value, 1), dtype=torch.int32, device=device)
            st = nat.SpmvPlan.from_buffer_copy(self.plan._struct)
            st.partials = nat.ptr(partials)
            st.counters = nat.ptr(counters)
            entry = (partials, counters, st)
            self._scratch[key] = entry
        st = entry[2]
        st.flags = (nat.FSB_SPMM_COMPENSATED if compensated else 0) | (nat.FSB_SPMM_PERSISTENT if persistent else 0)
        st.tile_bytes = int(tile_bytes)
        return ctypes.byref(st)

    def counters_clear(self):
        """True when every ticket is zero (the state each call must leave)."""
        return all(int(c.abs().sum().item()) == 0 for _, c, _ in self._scratch.values())


def spmm_spmv(data, indices, indptr, n_rows, n_cols, B, plan, out, x, y, compensated=False, persistent=False):
    """out = A @ B and y = A @ x in one launch through fsb_spmm_spmv_csr.

    Returns False (nothing launched) when the fused kernel does not apply
    (complex values, wide or misaligned dense rows, N a multiple of 256).
    """
    n = int(B.shape[1])
    rc = nat.lib().fsb_spmm_spmv_csr(
        nat.dtype_code(data.dtype), nat.ptr(data), nat.ptr(indices), nat.ptr(indptr), int(n_rows), int(n_cols),
        nat.ptr(B), int(B.stride(0)) if B.shape[0] > 1 else max(n, 1), n, nat.ptr(out),
        int(out.stride(0)) if out.shape[0] > 1 else max(n, 1), nat.ptr(x), nat.ptr(y),
        plan.struct_for(n, compensated, persistent=persistent), nat.stream_of(out.device),
    )
    if rc == nat.FSB_ERR_UNSUPPORTED:
        return False
    nat.check(rc, "fsb_spmm_spmv_csr")
    return True


def _ld(t, n):
    return int(t.stride(0)) if t.shape[0] > 1 else max(n, 1)


def spmm_backward(vals, perm32, t_indices, t_indptr, n_rows, n_cols, dY, X, dX, dvals, t_plan):
    """dX = A^T dY and, when ``dvals`` is given, dvals = <dY[row(p)], X[col(p)]> in one
    launch through fsb_spmm_csr_backward.

    ``vals`` are A's values (A order), ``perm32`` int32 with A's position of each
    nonzero of A^T, ``t_plan`` A^T's SpmmPlan.  Returns False (nothing launched)
    when the kernel does not apply (complex values, rows wider than 512 bytes,
    unaligned rows); the caller then runs the separate kernels.
    """
    n = int(dY.shape[1])
    rc = nat.lib().fsb_spmm_csr_backward(
        nat.dtype_code(vals.dtype), nat.ptr(vals), nat.ptr(perm32), nat.ptr(t_indices), nat.ptr(t_indptr),
        int(n_rows), int(n_cols), nat.ptr(dY), _ld(dY, n), nat.ptr(X), _ld(X, n) if X is not None else 0, n,
        nat.ptr(dX), _ld(dX, n), nat.ptr(dvals), t_plan.struct_for(n), nat.stream_of(dX.device),
    )
    if rc == nat.FSB_ERR_UNSUPPORTED:
        return False
    nat.check(rc, "fsb_spmm_csr_backward")
    return True


def spmm(data, indices, indptr, n_rows, n_cols, B, plan, out, compensated=False, tile_bytes=0, persistent=False):
    """out[:n_rows, :N] = A @ B through fsb_spmm_csr.

    ``indices`` int32, ``indptr`` int64, ``B`` and ``out`` row-major 2-D with
    unit column stride; ``plan`` a SpmmPlan of this matrix; ``tile_bytes`` the
    column tile of the team kernel (0 = the library's choice); ``persistent``
    its persistent grid.
    """
    n = int(B.shape[1])
    nat.check(
        nat.lib().fsb_spmm_csr(
            nat.dtype_code(data.dtype), nat.ptr(data), nat.ptr(indices), nat.ptr(indptr), int(n_rows), int(n_cols),
            nat.ptr(B), int(B.stride(0)) if B.shape[0] > 1 else max(n, 1), n, nat.ptr(out),
            int(out.stride(0)) if out.shape[0] > 1 else max(n, 1),
            plan.struct_for(n, compensated, tile_bytes, persistent),
            nat.stream_of(out.device),
        ),
        "fsb_spmm_csr",
    )
    return out
