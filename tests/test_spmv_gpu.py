"""GPU parity of the native CSR SpMV against the oracle and FlagSparse's outputs.

Every call goes through the public mirror (flagsparse_b200.flagsparse_spmv_csr),
which reaches the kernel through the C ABI.  Expected values come from the
CPU oracle (pinned to FlagSparse's goldens in test_oracle_golden.py) and,
where a golden exists, from FlagSparse's own Triton output directly.
"""

import numpy as np
import pytest
import torch

import flagsparse_b200 as fs
from flagsparse_b200 import workloads
from flagsparse_b200.sparse_operations import _csr
from flagsparse_b200.sparse_operations import spmv_csr as spmv_mod
from oracle import oracle
from tests.helpers import TORCH_DT, assert_spmv_close, dev, host, op_csr, rounded

pytestmark = pytest.mark.gpu

DTYPES = ("float16", "bfloat16", "float32", "float64", "complex64", "complex128")
# north-star parity tolerance against FlagSparse's own output (rtol), plus the
# reference's own summation error for the dtypes it evaluates in place
REF_RTOL = {"float16": 2.0**-10, "bfloat16": 2.0**-7, "float32": 1e-5, "complex64": 1e-5,
            "float64": 1e-12, "complex128": 1e-12}
REF_ATOL = {"float16": 1e-5, "bfloat16": 1e-5, "float32": 1e-9, "complex64": 2e-5,
            "float64": 1e-14, "complex128": 1e-14}


def _run_spmv(indptr, indices, data, x, shape, dname, op="non", idx_dt=torch.int32, ptr_dt=torch.int64, **kw):
    dt = TORCH_DT[dname]
    return fs.flagsparse_spmv_csr(
        dev(data, dt), dev(indices, idx_dt), dev(indptr, ptr_dt), dev(x, dt), shape=shape, op=op, **kw
    )


def _check_against_oracle(y, indptr, indices, data64, x64, shape, op, dname, what):
    p, i, d, _ = op_csr(indptr, indices, data64, shape, op)
    ref = oracle.spmv(p, i, d, x64)
    scale = oracle.spmv_abs(p, i, np.abs(d), np.abs(x64))
    assert_spmv_close(host(y), ref, scale, np.diff(p), dname, what)


@pytest.mark.parametrize("mname", ["small", "wide"])
@pytest.mark.parametrize("dname", DTYPES)
@pytest.mark.parametrize("op", ["non", "trans", "conj"])
@pytest.mark.parametrize("idx", ["i32p64", "i64p64", "i32p32", "i64p32"])
def test_spmv_golden_cases(golden, mname, dname, op, idx):
    if op == "conj" and not dname.startswith("complex"):
        pytest.skip("conj equals trans for real dtypes")
    g = golden("golden_spmv.npz")
    key = f"spmv_{mname}_{dname}_{op}"
    indptr, indices = g[f"spmv_{mname}_indptr"], g[f"spmv_{mname}_indices"]
    shape = tuple(int(v) for v in g[f"spmv_{mname}_shape"])
    base = g[f"spmv_{mname}_data_cplx"] if dname.startswith("complex") else g[f"spmv_{mname}_data_real"]
    idx_dt = torch.int64 if idx.startswith("i64") else torch.int32
    ptr_dt = torch.int64 if idx.endswith("p64") else torch.int32
    x = g[key + "_x"]
    y = _run_spmv(indptr, indices, base, x, shape, dname, op=op, idx_dt=idx_dt, ptr_dt=ptr_dt)
    assert y.dtype == TORCH_DT[dname]
    data64, x64 = rounded(base, dname), rounded(x, dname)
    _check_against_oracle(y, indptr, indices, data64, x64, shape, op, dname, key)
    # FlagSparse's own output on the same inputs
    ref = g[key + "_y"]
    got = host(y)
    p, i, d, _ = op_csr(indptr, indices, data64, shape, op)
    scale = oracle.spmv_abs(p, i, np.abs(d), np.abs(x64))
    err = np.abs(got - ref)
    assert np.all(err <= REF_RTOL[dname] * np.abs(ref) + REF_ATOL[dname] * scale + 1e-30), key


@pytest.mark.parametrize("mname", ["small", "wide"])
@pytest.mark.parametrize("dname", ["float32", "float64"])
def test_spmv_opt_buckets_bit_exact(golden, mname, dname):
    """use_opt builds FlagSparse's bucket row lists; they match its own bit for bit."""
    g = golden("golden_spmv.npz")
    key = f"spmv_{mname}_{dname}_non"
    shape = tuple(int(v) for v in g[f"spmv_{mname}_shape"])
    dt = TORCH_DT[dname]
    p = fs.prepare_spmv_csr(dev(g[f"spmv_{mname}_data_real"], dt), dev(g[f"spmv_{mname}_indices"], torch.int32),
                            dev(g[f"spmv_{mname}_indptr"]), shape)
    y, meta = fs.flagsparse_spmv_csr(x=dev(g[key + "_x"], dt), prepared=p, use_opt=True, return_meta=True)
    assert meta["bucket_count"] == int(g[key + "_nbuckets"])
    buckets = spmv_mod._build_spmv_opt_runtime_buckets(p)
    for b, bucket in enumerate(buckets):
        np.testing.assert_array_equal(host(bucket["rows"]), g[key + f"_bucket{b}_rows"])
        assert bucket["max_segs"] == int(g[key + f"_bucket{b}_max_segs"])
    np.testing.assert_allclose(host(y), g[key + "_yopt"], rtol=REF_RTOL[dname], atol=REF_RTOL[dname])


@pytest.mark.parametrize("tag,idx_dt,ptr_dt", [("i32p64", torch.int32, torch.int64), ("i64p32", torch.int64, torch.int32)])
def test_transpose_bit_exact(golden, tag, idx_dt, ptr_dt):
    g = golden("golden_spmv.npz")
    shape = tuple(int(v) for v in g["transpose_shape"])
    td, ti, tp, tshape = spmv_mod._transpose_csr_for_spmv(
        dev(g["transpose_src_data"]), dev(g["transpose_src_indices"], idx_dt), dev(g["transpose_src_indptr"], ptr_dt),
        shape,
    )
    assert tshape == (shape[1], shape[0])
    assert str(ti.dtype) == str(g[f"transpose_{tag}_indices_dtype"])
    assert str(tp.dtype) == str(g[f"transpose_{tag}_indptr_dtype"])
    np.testing.assert_array_equal(host(ti), g[f"transpose_{tag}_indices"])
    np.testing.assert_array_equal(host(tp), g[f"transpose_{tag}_indptr"])
    np.testing.assert_array_equal(host(td), g[f"transpose_{tag}_data"])


def test_transpose_bit_exact_large():
    c = workloads.zipf_csr(n=300_000, seed=9)
    n = c["shape"][1]
    t_ptr, t_idx, perm = oracle.transpose(c["indptr"], c["indices"], n)
    ti, tp, dperm = _csr.transpose_pattern(dev(c["indices"]), dev(c["indptr"]), c["shape"], torch.int32, torch.int64)
    np.testing.assert_array_equal(host(tp), t_ptr)
    np.testing.assert_array_equal(host(ti), t_idx)
    np.testing.assert_array_equal(host(dperm), perm)


@pytest.mark.parametrize("n,seed", [(50_000, 3), (400_000, 4)])
def test_plan_and_buckets_bit_exact(n, seed):
    c = workloads.zipf_csr(n=n, seed=seed)
    indptr = dev(c["indptr"])
    for dname in ("float32", "float64", "complex128"):
        plan = _csr.NativeSpmvPlan(indptr, n, TORCH_DT[dname])
        seg_row0, seg_unit0, units = oracle.spmv_plan(c["indptr"], plan.cap, plan.chunk_nnz)
        np.testing.assert_array_equal(host(plan.seg_row0), seg_row0)
        np.testing.assert_array_equal(host(plan.seg_unit0), seg_unit0)
        for got, exp in zip(plan.unit_table(), units.T):
            np.testing.assert_array_equal(got, exp)
        assert plan.n_slots == int(np.count_nonzero(units[:, 5] >= 0))
        assert plan.n_block_units == int(np.count_nonzero(units[:, 3] >= 0))
    bounds = [64, 512, 4096, None]
    got = _csr.bucketize_rows(indptr, n, bounds)
    exp = oracle.bucketize(c["indptr"], bounds)
    for a, b in zip(got, exp):
        np.testing.assert_array_equal(host(a), b)


def _edge_matrix(kind):
    rng = np.random.Generator(np.random.PCG64(77))
    if kind == "empty_rows":        # nnz == 0, every row empty
        return np.zeros(9, dtype=np.int64), np.zeros(0, dtype=np.int32), (8, 5)
    if kind == "single_long_row":   # one 50,000-nonzero row among empty rows
        lens = np.zeros(7, dtype=np.int64)
        lens[3] = 50_000
        ptr, idx = workloads.distinct_sorted_columns(rng, lens, 60_000)
        return ptr, idx, (7, 60_000)
    if kind == "one_column":        # n_cols == 1
        lens = rng.integers(0, 2, 100)
        ptr, idx = workloads.distinct_sorted_columns(rng, lens, 1)
        return ptr, idx, (100, 1)
    if kind == "boundaries":        # rows right at the window / chunk edges
        lens = np.array([1023, 1024, 1025, 0, 4095, 4096, 4097, 8192, 8193, 2047, 2048, 2049, 1, 0, 513])
        ptr, idx = workloads.distinct_sorted_columns(rng, lens, 9000)
        return ptr, idx, (lens.size, 9000)
    if kind == "many_empty":        # long runs of empty rows between dense ones
        lens = np.zeros(20_000, dtype=np.int64)
        lens[::997] = 1500
        ptr, idx = workloads.distinct_sorted_columns(rng, lens, 3000)
        return ptr, idx, (lens.size, 3000)
    raise ValueError(kind)


@pytest.mark.parametrize("kind", ["empty_rows", "single_long_row", "one_column", "boundaries", "many_empty"])
@pytest.mark.parametrize("dname", ["float32", "float64", "complex64", "bfloat16"])
@pytest.mark.parametrize("op", ["non", "trans"])
def test_spmv_edge_cases(kind, dname, op):
    ptr, idx, shape = _edge_matrix(kind)
    rng = np.random.Generator(np.random.PCG64(5))
    nnz = idx.size
    if dname.startswith("complex"):
        data = rng.uniform(-1, 1, nnz) + 1j * rng.uniform(-1, 1, nnz)
        xlen = shape[1] if op == "non" else shape[0]
        x = rng.uniform(-1, 1, xlen) + 1j * rng.uniform(-1, 1, xlen)
    else:
        data = rng.uniform(-1, 1, nnz)
        x = rng.uniform(-1, 1, shape[1] if op == "non" else shape[0])
    y = _run_spmv(ptr, idx, data, x, shape, dname, op=op)
    assert y.shape == ((shape[0],) if op == "non" else (shape[1],))
    _check_against_oracle(y, ptr, idx, rounded(data, dname), rounded(x, dname), shape, op, dname, kind)


def test_spmv_zero_rows():
    y = fs.flagsparse_spmv_csr(torch.zeros(0, device="cuda"), torch.zeros(0, dtype=torch.int32, device="cuda"),
                               torch.zeros(1, dtype=torch.int64, device="cuda"), torch.randn(4, device="cuda"),
                               shape=(0, 4))
    assert y.shape == (0,)


def test_spmv_repeat_calls_are_bitwise_deterministic():
    c = workloads.zipf_csr(n=200_000, seed=6)
    p = fs.prepare_spmv_csr(dev(c["data"]), dev(c["indices"]), dev(c["indptr"]), c["shape"])
    x = dev(c["x"])
    y0 = fs.flagsparse_spmv_csr(x=x, prepared=p)
    for _ in range(3):
        y1 = fs.flagsparse_spmv_csr(x=x, prepared=p)
        assert torch.equal(y0, y1)
    assert int(p.native_plan().counters.abs().sum().item()) == 0


@pytest.mark.parametrize("dname", ["float32", "float64"])
def test_spmv_config2_full_size_against_oracle(dname):
    """2,000,000 x 2,000,000 Zipf(2) matrix (~39M nonzeros): every row within the Dot2 bound."""
    dt = np.float32 if dname == "float32" else np.float64
    c = workloads.zipf_csr(n=2_000_000, seed=1, dtype=dt)
    y = _run_spmv(c["indptr"], c["indices"], c["data"], c["x"], c["shape"], dname)
    ref = oracle.spmv(c["indptr"], c["indices"], c["data"], c["x"])
    scale = oracle.spmv_abs(c["indptr"], c["indices"], np.abs(c["data"]), np.abs(c["x"]))
    assert_spmv_close(host(y), ref, scale, np.diff(c["indptr"]), dname, "config2")
    if dname == "float32":
        # the reference's fp32 semantics (fp64 row sums rounded to fp32)
        ref32 = oracle.spmv_f32_acc64(c["indptr"], c["indices"], c["data"], c["x"])
        rel = np.abs(host(y) - ref32) / np.maximum(np.abs(ref32), 1e-30)
        assert np.mean(host(y) == ref32) > 0.99
        assert np.all(np.abs(host(y) - ref32) <= 1e-5 * np.abs(ref32) + 1e-6 * scale), rel.max()


def test_spmv_linearity_at_scale():
    """A(a x + b z) == a A x + b A z within the rounding bound (size-independent property)."""
    c = workloads.zipf_csr(n=2_000_000, seed=1, dtype=np.float64)
    p = fs.prepare_spmv_csr(dev(c["data"]), dev(c["indices"]), dev(c["indptr"]), c["shape"])
    x = dev(c["x"])
    z = torch.flip(x, [0])
    lhs = fs.flagsparse_spmv_csr(x=0.5 * x + 0.25 * z, prepared=p)
    rhs = 0.5 * fs.flagsparse_spmv_csr(x=x, prepared=p) + 0.25 * fs.flagsparse_spmv_csr(x=z, prepared=p)
    scale = fs.flagsparse_spmv_csr(x=torch.ones_like(x), prepared=fs.prepare_spmv_csr(
        dev(np.abs(c["data"])), dev(c["indices"]), dev(c["indptr"]), c["shape"]))
    assert bool(torch.all((lhs - rhs).abs() <= 1e-14 * scale + 1e-300))


# ---- host policy, mirroring tests/pytest/test_spmv_csr_accuracy.py:141-247 ----

def _small_f32(index_dtype=torch.int32):
    m = workloads.mask_csr(12, 9, seed=3)
    return (dev(m["data"], torch.float32), dev(m["indices"], index_dtype), dev(m["indptr"], index_dtype), m)


def test_prepared_transpose_mismatch_rejected():
    data, indices, indptr, _ = _small_f32()
    p = fs.prepare_spmv_csr(data, indices, indptr, (12, 9), transpose=True)
    with pytest.raises(ValueError, match="does not match prepared.transpose"):
        fs.flagsparse_spmv_csr(x=torch.randn(12, device="cuda"), prepared=p, transpose=False)


def test_prepared_op_mismatch_rejected():
    data, indices, indptr, _ = _small_f32()
    p = fs.prepare_spmv_csr(data.to(torch.complex64), indices, indptr, (12, 9), op="conj")
    with pytest.raises(ValueError, match="does not match prepared.op"):
        fs.flagsparse_spmv_csr(x=torch.randn(12, device="cuda").to(torch.complex64), prepared=p, op="trans")


def test_int64_auto_fallback_to_int32(monkeypatch):
    data, indices, indptr, m = _small_f32(torch.int64)
    x = torch.randn(9, device="cuda")
    state = {"forced": False}
    original = spmv_mod._native_spmv_csr_impl_prepared

    def fail_int64_once(prepared, x_in, **kw):
        if prepared.kernel_indices.dtype == torch.int64 and not state["forced"]:
            state["forced"] = True
            raise RuntimeError("forced int64 launch failure")
        return original(prepared, x_in, **kw)

    monkeypatch.setattr(spmv_mod, "_native_spmv_csr_impl_prepared", fail_int64_once)
    y = fs.flagsparse_spmv_csr(data, indices, indptr, x, shape=(12, 9), index_fallback_policy="auto")
    assert state["forced"]
    ref = oracle.spmv(m["indptr"], m["indices"], host(data), host(x))
    np.testing.assert_allclose(host(y), ref, rtol=1.3e-6, atol=1.3e-6)


def test_int64_strict_no_fallback(monkeypatch):
    data, indices, indptr, _ = _small_f32(torch.int64)

    def fail_int64(prepared, x_in, **kw):
        raise RuntimeError("forced int64 launch failure")

    monkeypatch.setattr(spmv_mod, "_native_spmv_csr_impl_prepared", fail_int64)
    with pytest.raises(RuntimeError, match="forced int64 launch failure"):
        fs.flagsparse_spmv_csr(data, indices, indptr, torch.randn(9, device="cuda"), shape=(12, 9),
                               index_fallback_policy="strict")


def test_int64_auto_refuses_unsafe_fallback(monkeypatch):
    limit = spmv_mod._INDEX_LIMIT_INT32
    p = spmv_mod.PreparedCsrSpmv(
        data=torch.ones(1, device="cuda"),
        kernel_indices=torch.tensor([limit + 1], dtype=torch.int64, device="cuda"),
        kernel_indptr=torch.tensor([0, 1], dtype=torch.int64, device="cuda"),
        shape=(1, limit + 2), n_rows=1, n_cols=limit + 2, block_nnz=256, max_segments=1, max_row_nnz=1,
        opt_buckets=[], transpose=False, index_fallback_policy="auto",
    )

    def fail_launch(_p, _x, use_opt=False, **kw):
        raise RuntimeError("forced native int64 failure")

    monkeypatch.setattr(spmv_mod, "_run_spmv_prepared", fail_launch)
    with pytest.raises(RuntimeError, match="int32 fallback is unsafe"):
        spmv_mod._run_spmv_prepared_with_fallback(p, torch.empty(0, device="cuda"), use_opt=False)


def test_validation_messages():
    data, indices, indptr, _ = _small_f32()
    x = torch.randn(9, device="cuda")
    with pytest.raises(ValueError, match="op must be one of"):
        fs.flagsparse_spmv_csr(data, indices, indptr, x, shape=(12, 9), op="bad")
    with pytest.raises(ValueError, match="transpose conflicts with op"):
        fs.flagsparse_spmv_csr(data, indices, indptr, x, shape=(12, 9), op="non", transpose=True)
    with pytest.raises(ValueError, match="x length must be n_cols=9"):
        fs.flagsparse_spmv_csr(data, indices, indptr, torch.randn(12, device="cuda"), shape=(12, 9))
    with pytest.raises(ValueError, match="out shape/dtype must match result"):
        fs.flagsparse_spmv_csr(data, indices, indptr, x, shape=(12, 9), out=torch.empty(9, device="cuda"))
    with pytest.raises(IndexError, match="indices out of range"):
        fs.flagsparse_spmv_csr(data, indices, indptr, torch.randn(3, device="cuda"), shape=(12, 3))
    bad_ptr = indptr.clone()
    bad_ptr[3] = bad_ptr[4] + 1
    with pytest.raises(ValueError, match="non-decreasing"):
        fs.flagsparse_spmv_csr(data, indices, bad_ptr, x, shape=(12, 9))


def test_out_and_meta_contract():
    data, indices, indptr, m = _small_f32()
    x = torch.randn(9, device="cuda")
    out = torch.empty(12, device="cuda")
    y, ms, meta = fs.flagsparse_spmv_csr(data, indices, indptr, x, shape=(12, 9), out=out, return_time=True,
                                         return_meta=True)
    assert y is out
    assert ms == pytest.approx(meta["op_total_ms"])
    assert set(meta) == {"symbolic_ms", "compute_ms", "op_total_ms", "bucket_count"}
    assert meta["bucket_count"] == 0


def test_spmv_fast_short_rows_mode_within_plain_bound():
    """Opt-in plain sums for rows of <= cap nonzeros: each such row within gamma_n * S."""
    c = workloads.zipf_csr(n=400_000, seed=8, dtype=np.float32)
    p = fs.prepare_spmv_csr(dev(c["data"]), dev(c["indices"]), dev(c["indptr"]), c["shape"])
    plan = p.native_plan()
    plan.set_fast_short_rows(True)
    y = host(fs.flagsparse_spmv_csr(x=dev(c["x"]), prepared=p))
    ref = oracle.spmv(c["indptr"], c["indices"], c["data"], c["x"])
    scale = oracle.spmv_abs(c["indptr"], c["indices"], np.abs(c["data"]), np.abs(c["x"]))
    lens = np.diff(c["indptr"])
    u = 2.0**-24
    n = lens.astype(np.float64) + 2
    plain = u * np.abs(ref) + n * u / (1 - n * u) * scale
    short = lens <= plan.cap
    assert np.all(np.abs(y[short] - ref[short]) <= plain[short] + 1e-30)
    assert_spmv_close(y[~short], ref[~short], scale[~short], lens[~short], "float32", "long rows")
    plan.set_fast_short_rows(False)
