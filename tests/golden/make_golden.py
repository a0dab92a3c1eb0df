"""Generate golden vectors by running FlagSparse's own code on seeded inputs: small
cases whole, and sampled rows of the full-size configurations 2-4.

Runs only where the FlagSparse source tree is available (pass its ``src``
directory as argv[1]); the committed ``*.npz`` files are what the tests read.
The Triton kernels run on the CPU under ``TRITON_INTERPRET=1``.  FlagSparse's
public entry points insist on CUDA tensors, so this script calls the same
internal functions they call (prepare logic restated line by line where it
only validates), e.g. ``_transpose_csr_for_spmv``, ``_build_spmv_opt_buckets``,
``_triton_spmv_csr_impl_prepared``, ``_triton_spmm_csr_impl`` and
``_run_sddmm_prepared``.

Usage:  python tests/golden/make_golden.py <FlagSparse>/src
"""

import os
import sys

os.environ["TRITON_INTERPRET"] = "1"

import numpy as np  # noqa: E402
import torch  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from flagsparse_b200 import workloads  # noqa: E402

TORCH_DT = {
    "float16": torch.float16,
    "bfloat16": torch.bfloat16,
    "float32": torch.float32,
    "float64": torch.float64,
    "complex64": torch.complex64,
    "complex128": torch.complex128,
}


def np_of(t):
    t = t.detach().cpu()
    if t.dtype in (torch.float16, torch.bfloat16):
        return t.to(torch.float32).numpy()
    return t.numpy()


def rand_vec(rng, n, dtype):
    if dtype.is_complex:
        v = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        return torch.from_numpy(v).to(dtype)
    return torch.from_numpy(rng.standard_normal(n)).to(dtype)


def ref_prepared_spmv(m, data, indices, indptr, shape, op):
    """FlagSparse prepare_spmv_csr (spmv_csr.py:614-687) minus the CUDA checks."""
    op_code = m._normalize_spmv_op(op)
    if m._spmv_op_transposes(op_code):
        if op_code == m.SPMV_OP_CONJ_TRANS and data.dtype.is_complex:
            data = data.conj().resolve_conj()
        data, indices, indptr, shape = m._transpose_csr_for_spmv(data, indices, indptr, shape)
    n_rows, n_cols = int(shape[0]), int(shape[1])
    row_lengths = indptr[1:] - indptr[:-1]
    max_row_nnz = int(row_lengths.max().item()) if n_rows > 0 else 0
    block_nnz = 256
    max_segments = max((max_row_nnz + block_nnz - 1) // block_nnz, 1)
    while max_segments > 2048 and block_nnz < 65536:
        block_nnz *= 2
        max_segments = max((max_row_nnz + block_nnz - 1) // block_nnz, 1)
    return m.PreparedCsrSpmv(
        data=data.contiguous(), kernel_indices=indices.contiguous(), kernel_indptr=indptr.contiguous(),
        shape=shape, n_rows=n_rows, n_cols=n_cols, block_nnz=block_nnz, max_segments=max_segments,
        opt_max_segments=None, row_lengths=row_lengths, max_row_nnz=max_row_nnz, op=op_code,
    )


def spmv_cases(m, out):
    rng = np.random.Generator(np.random.PCG64(101))
    mats = {
        "small": workloads.mask_csr(40, 56, seed=11, dtype=np.float64),
        "wide": workloads.mask_csr(24, 5000, seed=12, dtype=np.float64, density=0.002, long_rows=(5,)),
    }
    for mname, mat in mats.items():
        out[f"spmv_{mname}_indptr"] = mat["indptr"]
        out[f"spmv_{mname}_indices"] = mat["indices"]
        out[f"spmv_{mname}_shape"] = np.array(mat["shape"])
        base = mat["data"]
        base_c = base + 1j * rng.standard_normal(base.size)
        out[f"spmv_{mname}_data_real"] = base
        out[f"spmv_{mname}_data_cplx"] = base_c
        for dname, dt in TORCH_DT.items():
            for op in ("non", "trans", "conj"):
                if op == "conj" and not dt.is_complex:
                    continue
                src = base_c if dt.is_complex else base
                data = torch.from_numpy(src).to(dt)
                indices = torch.from_numpy(mat["indices"]).to(torch.int32)
                indptr = torch.from_numpy(mat["indptr"]).to(torch.int64)
                p = ref_prepared_spmv(m, data, indices, indptr, mat["shape"], op)
                x = rand_vec(rng, p.n_cols, dt)
                y = m._triton_spmv_csr_impl_prepared(p, x)
                key = f"spmv_{mname}_{dname}_{op}"
                out[key + "_x"] = np_of(x)
                out[key + "_y"] = np_of(y)
                if dt in (torch.float32, torch.float64) and op == "non":
                    buckets = m._build_spmv_opt_buckets(
                        p.row_lengths, p.max_row_nnz, torch.int32, fp64=dt == torch.float64
                    )
                    yo = m._triton_spmv_csr_impl_opt_prepared(p, x, opt_buckets=buckets)
                    out[key + "_yopt"] = np_of(yo)
                    out[key + "_nbuckets"] = np.array(len(buckets))
                    for b, bucket in enumerate(buckets):
                        out[key + f"_bucket{b}_rows"] = bucket["rows"].numpy()
                        out[key + f"_bucket{b}_max_segs"] = np.array(bucket["max_segs"])


def config1_case(m, out):
    c = workloads.poisson_csr()
    data = torch.from_numpy(c["data"])
    p = ref_prepared_spmv(m, data, torch.from_numpy(c["indices"]), torch.from_numpy(c["indptr"]), c["shape"], "non")
    y = m._triton_spmv_csr_impl_prepared(p, torch.from_numpy(c["x"]))
    out["config1_f32_y"] = np_of(y)
    out["config1_nnz"] = np.array(c["indices"].size)


def transpose_cases(m, out):
    rng = np.random.Generator(np.random.PCG64(7))
    # unsorted columns with duplicates and empty rows: stability matters
    n_rows, n_cols, nnz = 30, 17, 140
    rows = np.sort(rng.integers(0, n_rows, nnz))
    rows[rows == 4] = 5  # row 4 empty
    indptr = np.zeros(n_rows + 1, dtype=np.int64)
    np.cumsum(np.bincount(rows, minlength=n_rows), out=indptr[1:])
    cols = rng.integers(0, n_cols - 2, nnz).astype(np.int32)  # last two columns empty
    data = rng.standard_normal(nnz)
    for idx_dt, ptr_dt, tag in ((torch.int32, torch.int64, "i32p64"), (torch.int64, torch.int32, "i64p32")):
        td, ti, tp, shape = m._transpose_csr_for_spmv(
            torch.from_numpy(data), torch.from_numpy(cols).to(idx_dt), torch.from_numpy(indptr).to(ptr_dt),
            (n_rows, n_cols),
        )
        out[f"transpose_{tag}_data"] = td.numpy()
        out[f"transpose_{tag}_indices"] = ti.numpy()
        out[f"transpose_{tag}_indptr"] = tp.numpy()
        out[f"transpose_{tag}_indices_dtype"] = np.array(str(ti.dtype))
        out[f"transpose_{tag}_indptr_dtype"] = np.array(str(tp.dtype))
    out["transpose_src_indptr"] = indptr
    out["transpose_src_indices"] = cols
    out["transpose_src_data"] = data
    out["transpose_shape"] = np.array((n_rows, n_cols))


def spmm_cases(sm, out):
    rng = np.random.Generator(np.random.PCG64(202))
    for (M, K, N, seed) in ((64, 96, 16, 21), (40, 30, 5, 22), (33, 3000, 64, 23)):
        mat = workloads.mask_csr(M, K, seed=seed, dtype=np.float64,
                                 density=0.004 if K > 1000 else None, long_rows=(2,) if K > 1000 else ())
        tag = f"spmm_{M}x{K}x{N}"
        out[tag + "_indptr"] = mat["indptr"]
        out[tag + "_indices"] = mat["indices"]
        base = mat["data"]
        base_c = base + 1j * rng.standard_normal(base.size)
        out[tag + "_data_real"] = base
        out[tag + "_data_cplx"] = base_c
        for dname in ("float32", "float64", "complex64"):
            dt = TORCH_DT[dname]
            data = torch.from_numpy(base_c if dt.is_complex else base).to(dt)
            if dt.is_complex:
                B = torch.from_numpy(rng.standard_normal((K, N)) + 1j * rng.standard_normal((K, N))).to(dt)
            else:
                B = torch.from_numpy(rng.standard_normal((K, N))).to(dt)
            indices = torch.from_numpy(mat["indices"]).to(torch.int32)
            indptr = torch.from_numpy(mat["indptr"]).to(torch.int64)
            max_row = int((indptr[1:] - indptr[:-1]).max().item())
            launch = sm._resolve_spmm_base_triton_launch(dt, N, max_row)
            C = sm._triton_spmm_csr_impl(
                data, indices, indptr, B, M, N, block_n=launch["block_n"], block_nnz=launch["block_nnz"],
                num_warps=launch["num_warps"], num_stages=launch["num_stages"],
            )
            out[f"{tag}_{dname}_B"] = np_of(B)
            out[f"{tag}_{dname}_C"] = np_of(C)


def sddmm_cases(dm, out):
    rng = np.random.Generator(np.random.PCG64(303))
    for (M, N, K, seed) in ((8, 10, 8, 31), (64, 96, 16, 32), (50, 40, 37, 33)):
        mat = workloads.mask_csr(M, N, seed=seed, dtype=np.float64)
        tag = f"sddmm_{M}x{N}x{K}"
        out[tag + "_indptr"] = mat["indptr"]
        out[tag + "_indices"] = mat["indices"]
        for dname in ("float32", "float64"):
            dt = TORCH_DT[dname]
            x = torch.from_numpy(rng.standard_normal((M, K)) * 0.125).to(dt)
            y = torch.from_numpy(rng.standard_normal((N, K)) * 0.125).to(dt)
            data = torch.from_numpy(mat["data"]).to(dt)
            indices = torch.from_numpy(mat["indices"]).to(torch.int32)
            indptr = torch.from_numpy(mat["indptr"]).to(torch.int64)
            row_ids = dm._build_row_ids(indptr)
            bk, nw = dm._resolve_sddmm_launch_config(K)
            p = dm.SDDMMPrepared(indices=indices, indptr=indptr, shape=(M, N), row_ids=row_ids, block_k=bk,
                                 num_warps=nw)
            res, _meta = dm._run_sddmm_prepared(p, x, y, data, 1.25, 0.5, None)
            out[f"{tag}_{dname}_x"] = x.numpy()
            out[f"{tag}_{dname}_y"] = y.numpy()
            out[f"{tag}_{dname}_data"] = data.numpy()
            out[f"{tag}_{dname}_out"] = res.numpy()


def coo_cases(m, out):
    """coo_to_csr_for_spmv (spmv_csr.py:957-984) on distinct (row, col) pairs in
    shuffled, sorted and empty-row layouts; int32 and int64 index inputs."""
    rng = np.random.default_rng(21)
    cases = [("shuf", 40, 33, 300, True, torch.int64), ("sorted", 25, 50, 200, False, torch.int64),
             ("i32", 64, 17, 400, True, torch.int32), ("emptyrows", 500, 40, 120, True, torch.int64)]
    for tag, nr, nc, nnz, shuffle, idt in cases:
        keys = np.sort(rng.choice(nr * nc, size=nnz, replace=False))
        if shuffle:
            keys = rng.permutation(keys)
        row = torch.from_numpy(keys // nc).to(idt)
        col = torch.from_numpy(keys % nc).to(idt)
        data = torch.from_numpy(rng.standard_normal(nnz)).to(torch.float32)
        d_s, idx, ptr = m.coo_to_csr_for_spmv(data, row, col, (nr, nc))
        out[f"coo_{tag}_shape"] = np.array([nr, nc], dtype=np.int64)
        out[f"coo_{tag}_row"] = row.numpy()
        out[f"coo_{tag}_col"] = col.numpy()
        out[f"coo_{tag}_data"] = data.numpy()
        out[f"coo_{tag}_data_s"] = np_of(d_s)
        out[f"coo_{tag}_indices"] = idx.numpy()
        out[f"coo_{tag}_indptr"] = ptr.numpy()


def bsr_cases(bm, out):
    """_triton_spmv_bsr_kernel (spmv_bsr.py:603-671) for op non / trans / conj on small
    BSR matrices with ragged logical shapes (padded rows and columns)."""
    rng = np.random.default_rng(31)
    for bd in (2, 3, 4, 16):
        nbr, nbc = 9, 7
        counts = rng.integers(0, 4, size=nbr)
        counts[2] = 0
        ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        cols = np.concatenate([np.sort(rng.choice(nbc, size=c, replace=False)) for c in counts]).astype(np.int64)
        nnzb = int(ptr[-1])
        shape = (nbr * bd - 1, nbc * bd - 1)
        out[f"bsr{bd}_indptr"] = ptr
        out[f"bsr{bd}_indices"] = cols
        out[f"bsr{bd}_shape"] = np.array(shape, dtype=np.int64)
        for dname in ("float32", "float64", "complex64", "complex128"):
            dt = TORCH_DT[dname]
            blocks = rand_vec(rng, nnzb * bd * bd, dt).reshape(nnzb, bd, bd)
            out[f"bsr{bd}_{dname}_blocks"] = np_of(blocks)
            for op_name, op_code in (("non", 0), ("trans", 1), ("conj", 2)):
                if op_name == "conj" and not dt.is_complex:
                    continue
                n_in = nbr * bd if op_code else nbc * bd
                x = rand_vec(rng, n_in, dt)
                p = bm.PreparedBsrSpmv(blocks, torch.from_numpy(cols), torch.from_numpy(ptr), shape, bd, nbr, nbc,
                                       128, 1, int(counts.max()), op=op_code)
                y = bm._triton_spmv_bsr_kernel(p, x, op_code)
                out[f"bsr{bd}_{dname}_{op_name}_x"] = np_of(x)
                out[f"bsr{bd}_{dname}_{op_name}_y"] = np_of(y)


def mtx_cases(tests_dir, out):
    """FlagSparse's test loader load_mtx_to_csr_torch (tests/test_spmv.py:116-190)
    on the .mtx fixtures in tests/golden/mtx, read on the CPU."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("fs_test_spmv", os.path.join(tests_dir, "test_spmv.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mdir = os.path.join(HERE, "mtx")
    for name in sorted(os.listdir(mdir)):
        data, indices, indptr, shape = mod.load_mtx_to_csr_torch(os.path.join(mdir, name), dtype=torch.float64,
                                                                 device=torch.device("cpu"))
        tag = name[:-4]
        out[f"mtx_{tag}_data"] = data.numpy()
        out[f"mtx_{tag}_indices"] = indices.numpy()
        out[f"mtx_{tag}_indptr"] = indptr.numpy()
        out[f"mtx_{tag}_shape"] = np.array(shape, dtype=np.int64)


def sample_rows(indptr, n_long, n_random, seed):
    """The n_long longest rows plus n_random other rows (sorted, distinct)."""
    lens = np.diff(indptr)
    longest = np.argsort(-lens, kind="stable")[:n_long]
    rest = np.setdiff1d(np.arange(lens.size), longest)
    rnd = np.random.Generator(np.random.PCG64(seed)).choice(rest, n_random, replace=False)
    return np.sort(np.concatenate([longest, rnd]))


def sub_csr(c, rows):
    """Rows `rows` of CSR c with all of its columns: (indptr, indices, positions taken)."""
    lens = np.diff(c["indptr"])[rows]
    ptr = np.zeros(rows.size + 1, dtype=np.int64)
    np.cumsum(lens, out=ptr[1:])
    take = np.concatenate([np.arange(c["indptr"][r], c["indptr"][r + 1]) for r in rows])
    return ptr, c["indices"][take], take


def config_cases(m, sm, dm, out):
    """FlagSparse's own kernels on sampled rows of the full-size configurations.

    Each of its kernels computes a row (SpMV, SpMM) or a nonzero (SDDMM) from
    that row's entries and the dense operands alone, so its output on a
    row subset equals those rows of its output on the whole matrix.  The tests
    regenerate the same seeded inputs and compare the native result on the
    whole matrix at these rows.
    """
    # configuration 2: 2,000,000 x 2,000,000 Zipf(2), fp32 and the fp64 drop-in
    c = workloads.zipf_csr()
    rows = sample_rows(c["indptr"], 6, 250, seed=41)
    ptr, idx, take = sub_csr(c, rows)
    out["config2_rows"] = rows
    for dname in ("float32", "float64"):
        dt = TORCH_DT[dname]
        data = torch.from_numpy(c["data"][take]).to(dt)
        x = torch.from_numpy(c["x"]).to(dt)
        p = ref_prepared_spmv(m, data, torch.from_numpy(idx), torch.from_numpy(ptr), (rows.size, c["shape"][1]),
                              "non")
        out[f"config2_{dname}_y"] = np_of(m._triton_spmv_csr_impl_prepared(p, x))
        buckets = m._build_spmv_opt_buckets(p.row_lengths, p.max_row_nnz, torch.int32, fp64=dt == torch.float64)
        out[f"config2_{dname}_yopt"] = np_of(m._triton_spmv_csr_impl_opt_prepared(p, x, opt_buckets=buckets))
    del c
    # configuration 3: 1,000,000 x 1,000,000 power law (mean ~30), fp32, B = dense_normal(K, 64, seed 2)
    c = workloads.zipf_csr(n=1_000_000, scale=32.0 / workloads.ZIPF_MEAN_UNSCALED, seed=2, dtype=np.float32,
                           values="normal")
    rows = sample_rows(c["indptr"], 4, 150, seed=42)
    ptr, idx, take = sub_csr(c, rows)
    B = torch.from_numpy(workloads.dense_normal(c["shape"][1], 64, seed=2))
    indptr_t = torch.from_numpy(ptr)
    max_row = int(np.diff(ptr).max())
    launch = sm._resolve_spmm_base_triton_launch(torch.float32, 64, max_row)
    C = sm._triton_spmm_csr_impl(
        torch.from_numpy(c["data"][take]), torch.from_numpy(idx).to(torch.int32), indptr_t, B, rows.size, 64,
        block_n=launch["block_n"], block_nnz=launch["block_nnz"], num_warps=launch["num_warps"],
        num_stages=launch["num_stages"],
    )
    out["config3_rows"] = rows
    out["config3_float32_N64_C"] = np_of(C)
    del c, B
    # configuration 4: SDDMM of dY and X (500,000 x 128 each, dense_normal seeds 3 and 4) on the
    # Chung-Lu graph's pattern, fp32 (out[p] = <dY[row(p)], X[col(p)]>)
    g = workloads.chung_lu_graph()
    rows = sample_rows(g["indptr"], 4, 150, seed=43)
    ptr, idx, take = sub_csr(g, rows)
    dY = torch.from_numpy(workloads.dense_normal(g["shape"][0], 128, seed=3))[torch.from_numpy(rows)]
    X = torch.from_numpy(workloads.dense_normal(g["shape"][1], 128, seed=4))
    indptr_t = torch.from_numpy(ptr)
    row_ids = dm._build_row_ids(indptr_t)
    bk, nw = dm._resolve_sddmm_launch_config(128)
    prep = dm.SDDMMPrepared(indices=torch.from_numpy(idx).to(torch.int32), indptr=indptr_t,
                            shape=(rows.size, g["shape"][1]), row_ids=row_ids, block_k=bk, num_warps=nw)
    res, _meta = dm._run_sddmm_prepared(prep, dY, X, None, 1.0, 0.0, None)
    out["config4_rows"] = rows
    out["config4_float32_K128_sddmm"] = np_of(res)


def main():
    src = sys.argv[1] if len(sys.argv) > 1 else None
    if not src or not os.path.isdir(src):
        raise SystemExit("usage: make_golden.py <FlagSparse>/src")
    sys.path.insert(0, src)
    from flagsparse.sparse_operations import sddmm_csr as dm
    from flagsparse.sparse_operations import spmv_bsr as bm
    from flagsparse.sparse_operations import spmm_csr as sm
    from flagsparse.sparse_operations import spmv_csr as m

    torch.manual_seed(0)
    groups = {
        "golden_spmv.npz": lambda o: (spmv_cases(m, o), transpose_cases(m, o)),
        "golden_config1.npz": lambda o: config1_case(m, o),
        "golden_spmm.npz": lambda o: spmm_cases(sm, o),
        "golden_sddmm.npz": lambda o: sddmm_cases(dm, o),
        "golden_coo.npz": lambda o: coo_cases(m, o),
        "golden_bsr.npz": lambda o: bsr_cases(bm, o),
        "golden_mtx.npz": lambda o: mtx_cases(os.path.join(os.path.dirname(src), "tests"), o),
        "golden_configs.npz": lambda o: config_cases(m, sm, dm, o),
    }
    only = set(sys.argv[2:])
    for fname, fn in groups.items():
        if only and fname not in only:
            continue
        out = {}
        fn(out)
        np.savez_compressed(os.path.join(HERE, fname), **out)
        print(fname, len(out), "arrays")


if __name__ == "__main__":
    main()
