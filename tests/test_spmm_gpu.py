"""CSR SpMM on the native kernel against the oracle and FlagSparse's golden outputs.

Every comparison is against the exact product (the oracle's Dot2 SpMM on the
same rounded inputs) within the rounding-error bound of the route's
accumulation: a working-precision sum for the plain routes, the Dot2 bound
for the accuracy routes.  The golden cases also hold the reference's own
outputs on the same inputs.
"""

import numpy as np
import pytest
import torch

import flagsparse_b200 as fs
from flagsparse_b200 import workloads
from flagsparse_b200.sparse_operations import _csr
from flagsparse_b200.sparse_operations import spmm_csr as sm
from oracle import oracle
from tests.helpers import (TORCH_DT, assert_within, dev, host, op_csr, plain_error_bound, rounded,
                           spmv_error_bound)

pytestmark = pytest.mark.gpu

DTYPES = ("float16", "bfloat16", "float32", "float64", "complex64", "complex128")


def _dense(rng, rows, cols, dname):
    if dname.startswith("complex"):
        return rng.standard_normal((rows, cols)) + 1j * rng.standard_normal((rows, cols))
    return rng.standard_normal((rows, cols))


def _oracle_spmm(indptr, indices, data_r, shape, B_r, op):
    p, i, d, _ = op_csr(indptr, indices, data_r, shape, op)
    ref = oracle.spmm(p, i, d, B_r)
    scale = np.real(oracle.spmm(p, i, np.abs(d), np.abs(B_r)))
    lens = np.diff(p)[:, None]
    return ref, scale, lens


def _check(C, ref, scale, lens, dname, what, compensated=False):
    got = host(C).astype(ref.dtype)
    if compensated:
        bound = spmv_error_bound(dname, np.abs(ref), scale, np.broadcast_to(lens, ref.shape))
    else:
        bound = plain_error_bound(dname, ref, scale, np.broadcast_to(lens, ref.shape))
    assert_within(got, ref, bound, what)


def _run_case(mat, N, dname, op="non", seed=0, idx_dt=torch.int32, ptr_dt=torch.int64, route=None):
    rng = np.random.Generator(np.random.PCG64(seed))
    dt = TORCH_DT[dname]
    m, k = mat["shape"]
    data = mat["data"]
    if dname.startswith("complex") and not np.iscomplexobj(data):
        data = data + 1j * rng.standard_normal(data.size)
    k_eff = m if op != "non" else k
    B_np = _dense(rng, k_eff, N, dname)
    d_r, B_r = rounded(data, dname), rounded(B_np, dname)
    A = (dev(data, dt), dev(mat["indices"], idx_dt), dev(mat["indptr"], ptr_dt))
    B = dev(B_np, dt)
    if route is None:
        C = fs.flagsparse_spmm_csr(*A, B, mat["shape"], op=op)
    else:
        p = fs.prepare_spmm_csr_route(*A, mat["shape"], op=op, alg=route)
        C = fs.flagsparse_spmm_csr_run(p, B)
    ref, scale, lens = _oracle_spmm(mat["indptr"], mat["indices"], d_r, mat["shape"], B_r, op)
    return C, ref, scale, lens


# ---------------------------------------------------------------- golden (reference outputs)

@pytest.mark.parametrize("shape", ["64x96x16", "40x30x5", "33x3000x64"])
@pytest.mark.parametrize("dname", ["float32", "float64", "complex64"])
def test_spmm_golden_cases(golden, shape, dname):
    g = golden("golden_spmm.npz")
    tag = f"spmm_{shape}"
    M, K, N = (int(v) for v in shape.split("x"))
    base = g[tag + ("_data_cplx" if dname.startswith("complex") else "_data_real")]
    dt = TORCH_DT[dname]
    B_np = g[f"{tag}_{dname}_B"]
    C = fs.flagsparse_spmm_csr(dev(base, dt), dev(g[tag + "_indices"]), dev(g[tag + "_indptr"]), dev(B_np, dt),
                               (M, K))
    d_r = rounded(base, dname)
    ref, scale, lens = _oracle_spmm(g[tag + "_indptr"], g[tag + "_indices"], d_r, (M, K), B_np.astype(
        np.complex128 if dname.startswith("complex") else np.float64), "non")
    _check(C, ref, scale, lens, dname, f"{tag} {dname} vs oracle")
    # and against the reference's own output: both within their bounds of the exact result
    golden_c = g[f"{tag}_{dname}_C"]
    bound = 2 * plain_error_bound(dname, ref, scale, np.broadcast_to(lens, ref.shape))
    assert_within(host(C).astype(ref.dtype), golden_c.astype(ref.dtype), bound, f"{tag} {dname} vs reference")


# ---------------------------------------------------------------- dtypes x ops x widths

@pytest.mark.parametrize("dname", DTYPES)
@pytest.mark.parametrize("op", ["non", "trans", "conj"])
@pytest.mark.parametrize("N", [1, 5, 16, 64, 130])
def test_spmm_dtypes_ops_widths(dname, op, N):
    if op == "conj" and not dname.startswith("complex"):
        pytest.skip("conj equals trans for real dtypes")
    mat = workloads.mask_csr(48, 70, seed=40 + N, dtype=np.float64, long_rows=(3,))
    C, ref, scale, lens = _run_case(mat, N, dname, op=op, seed=N)
    _check(C, ref, scale, lens, dname, f"{dname} {op} N={N}")


@pytest.mark.parametrize("idx_dt,ptr_dt", [(torch.int64, torch.int64), (torch.int32, torch.int32),
                                           (torch.int64, torch.int32)])
def test_spmm_index_dtypes(idx_dt, ptr_dt):
    mat = workloads.mask_csr(60, 50, seed=7, dtype=np.float64)
    C, ref, scale, lens = _run_case(mat, 32, "float32", idx_dt=idx_dt, ptr_dt=ptr_dt)
    _check(C, ref, scale, lens, "float32", f"{idx_dt} {ptr_dt}")


@pytest.mark.parametrize("dname", ["float32", "bfloat16", "float64", "complex128"])
@pytest.mark.parametrize("N", [64, 300])
def test_spmm_long_rows_multi_chunk(dname, N):
    """Power-law rows up to thousands of nonzeros: multi-chunk rows reduce through scratch."""
    c = workloads.zipf_csr(n=20_000, seed=11, dtype=np.float64)
    mat = {"indptr": c["indptr"], "indices": c["indices"], "data": c["data"], "shape": c["shape"]}
    assert int(np.diff(c["indptr"]).max()) > 4 * 256
    C, ref, scale, lens = _run_case(mat, N, dname, seed=3)
    _check(C, ref, scale, lens, dname, f"zipf {dname} N={N}")


def _long_row_matrix(n_long, n_short):
    """Row 0: n_long nonzeros (value 1) in columns 0 .. n_long-1; row 1: a random row of
    n_short nonzeros (plain sums); row 2 empty."""
    rng = np.random.Generator(np.random.PCG64(17))
    k = n_long + 64
    cols1 = np.sort(rng.choice(k, n_short, replace=False))
    indptr = np.array([0, n_long, n_long + n_short, n_long + n_short], dtype=np.int64)
    indices = np.concatenate([np.arange(n_long), cols1]).astype(np.int32)
    data = np.concatenate([np.ones(n_long), rng.standard_normal(n_short)])
    return indptr, indices, data, k


def _compensated_bound(dname, ref, scale):
    """Rows over 1,024 nonzeros: each step's 4 products per team sum plainly, then fold
    into a compensated (Dot2) accumulator, and the partials combine compensated:
    |C - exact| <= (u_out + 2 u_acc) |exact| + gamma_6 sum|a||b|, whatever the length."""
    u, ua = {"bfloat16": 2.0**-8, "float16": 2.0**-11, "float32": 2.0**-24}[dname], 2.0**-24
    return (u + 2 * ua) * np.abs(ref) + 6 * ua / (1 - 6 * ua) * scale + 1e-30


@pytest.mark.parametrize("dname", ["bfloat16", "float16", "float32"])
@pytest.mark.parametrize("N", [16, 64, 128])
def test_long_rows_sum_compensated(dname, N):
    """A 50,000-nonzero row in the fp32-accumulated types sums compensated.  Its first
    product is +big and its last -big with 49,998 products of `unit` between, unit at or
    below half an fp32 ulp of big: a plain fp32 sum absorbs every unit term into big and
    ends at 0, while the compensated sum keeps them (exact: 49,998 unit).  A random row of
    the same length meets the same bound against the oracle."""
    dt = TORCH_DT[dname]
    big, unit = (2.0**15, 2.0**-10) if dname == "float16" else (2.0**24, 1.0)
    indptr, indices, data, k = _long_row_matrix(50_000, 50)
    rng = np.random.Generator(np.random.PCG64(N))
    B = np.full((k, N), unit)
    B[0] = big
    B[49_999] = -big
    B[50_000:] = rng.standard_normal((64, N))
    C = fs.flagsparse_spmm_csr(dev(data, dt), dev(indices), dev(indptr), dev(B, dt), (3, k))
    exact = np.full(N, 49_998 * unit)
    got = host(C[0]).astype(np.float64)
    assert_within(got, exact, _compensated_bound(dname, exact, np.full(N, 2 * big + 49_998 * unit)),
                  f"{dname} N={N} cancelling long row")
    assert np.all(host(C[2]) == 0)
    d2 = rng.standard_normal(data.size)
    B2 = rng.standard_normal((k, N))
    C2 = fs.flagsparse_spmm_csr(dev(d2, dt), dev(indices), dev(indptr), dev(B2, dt), (3, k))
    d_r, B_r = rounded(d2, dname), rounded(B2, dname)
    ref = oracle.spmm(indptr, indices, d_r, B_r)
    scale = oracle.spmm(indptr, indices, np.abs(d_r), np.abs(B_r))
    got = host(C2).astype(np.float64)
    assert_within(got[0], ref[0], _compensated_bound(dname, ref[0], scale[0]), f"{dname} N={N} random long row")
    assert_within(got[1], ref[1], plain_error_bound(dname, ref[1], scale[1], 50), f"{dname} N={N} short row")


@pytest.mark.parametrize("route", sorted(sm.SPMM_CSR_ALGORITHMS))
@pytest.mark.parametrize("dname", ["float32", "float64", "complex64"])
def test_spmm_every_route(route, dname):
    mat = workloads.zipf_csr(n=3000, seed=12, dtype=np.float64)
    mat = {"indptr": mat["indptr"], "indices": mat["indices"], "data": mat["data"], "shape": mat["shape"]}
    C, ref, scale, lens = _run_case(mat, 24, dname, seed=5, route=route)
    compensated = "accuracy" in route
    _check(C, ref, scale, lens, dname, f"route {route} {dname}", compensated=compensated)


def test_accuracy_routes_are_compensated():
    """Ill-conditioned rows: the accuracy route stays within the Dot2 bound, the plain one may not."""
    rng = np.random.Generator(np.random.PCG64(9))
    m, k, n = 64, 4096, 8
    indptr = np.arange(m + 1, dtype=np.int64) * 2048
    indices = np.concatenate([np.sort(rng.choice(k, 2048, replace=False)) for _ in range(m)]).astype(np.int32)
    data = rng.standard_normal(indptr[-1]) * np.exp2(rng.integers(-20, 20, indptr[-1]))
    mat = {"indptr": indptr, "indices": indices, "data": data, "shape": (m, k)}
    C, ref, scale, lens = _run_case(mat, n, "float32", seed=2, route="csr_base_accuracy")
    _check(C, ref, scale, lens, "float32", "accuracy route", compensated=True)


# ---------------------------------------------------------------- layouts / strides / out

def test_spmm_misaligned_and_strided_operands():
    """B and out views whose rows are not 16-byte aligned take the narrow-vector path."""
    mat = workloads.mask_csr(40, 33, seed=8, dtype=np.float64)
    rng = np.random.Generator(np.random.PCG64(1))
    big = torch.from_numpy(rng.standard_normal((33, 71))).float().cuda()
    B = big[:, 1:66]  # row stride 71, base offset 4 bytes
    A = (dev(mat["data"], torch.float32), dev(mat["indices"]), dev(mat["indptr"]))
    plan = _csr.SpmmPlan(A[2], 40, torch.float32)
    out_big = torch.full((40, 70), float("nan"), device="cuda")
    out = out_big[:, 3:68]
    _csr.spmm(A[0], A[1], A[2], 40, 33, B, plan, out)
    ref, scale, lens = _oracle_spmm(mat["indptr"], mat["indices"], rounded(mat["data"], "float32"), (40, 33),
                                    host(B).astype(np.float64), "non")
    _check(out, ref, scale, lens, "float32", "strided")
    assert torch.isnan(out_big[:, :3]).all() and torch.isnan(out_big[:, 68:]).all()


def test_spmm_route_col_major_layout():
    mat = workloads.mask_csr(30, 20, seed=9, dtype=np.float64)
    rng = np.random.Generator(np.random.PCG64(2))
    B_np = rng.standard_normal((20, 12))
    B_col = torch.from_numpy(B_np).float().cuda().t().contiguous().t()
    p = fs.prepare_spmm_csr_route(dev(mat["data"], torch.float32), dev(mat["indices"]), dev(mat["indptr"]), (30, 20))
    C, meta = fs.flagsparse_spmm_csr_run(p, B_col, dense_layout="col", return_meta=True)
    assert meta["dense_layout"] == "col" and meta["output_layout"] == "col"
    assert C.stride(0) == 1
    ref, scale, lens = _oracle_spmm(mat["indptr"], mat["indices"], rounded(mat["data"], "float32"), (30, 20),
                                    rounded(B_np, "float32"), "non")
    _check(C, ref, scale, lens, "float32", "col layout")


def test_spmm_out_parameter_and_meta():
    mat = workloads.mask_csr(16, 24, seed=10, dtype=np.float64)
    A = (dev(mat["data"], torch.float32), dev(mat["indices"]), dev(mat["indptr"]))
    B = torch.randn(24, 8, device="cuda")
    out = torch.empty(16, 8, device="cuda")
    C, ms, meta = fs.flagsparse_spmm_csr(*A, B, (16, 24), out=out, return_time=True, return_meta=True)
    assert C is out and ms >= 0
    assert set(meta) == {"symbolic_ms", "compute_ms", "op_total_ms", "op"} and meta["op"] == "non"
    Ct, meta_t = fs.flagsparse_spmm_csr(*A, torch.randn(16, 8, device="cuda"), (16, 24), op="trans",
                                        return_meta=True)
    assert Ct.shape == (24, 8) and meta_t["op"] == "trans" and meta_t["symbolic_ms"] >= 0


# ---------------------------------------------------------------- edge cases / determinism

@pytest.mark.parametrize("kind", ["empty_rows", "all_empty", "one_column", "single_long_row", "zero_cols_B"])
def test_spmm_edge_cases(kind):
    rng = np.random.Generator(np.random.PCG64(4))
    if kind == "empty_rows":
        lens = np.array([0, 3, 0, 0, 5, 0, 1, 0] * 20)
    elif kind == "all_empty":
        lens = np.zeros(50, dtype=np.int64)
    elif kind == "one_column":
        lens = np.ones(40, dtype=np.int64)
    elif kind == "single_long_row":
        lens = np.array([0, 5000, 0])
    else:
        lens = np.array([2, 1, 3])
    m = lens.size
    k = 1 if kind == "one_column" else 6000
    indptr = np.zeros(m + 1, dtype=np.int64)
    np.cumsum(lens, out=indptr[1:])
    indices = np.concatenate([np.sort(rng.choice(k, int(n), replace=False)) for n in lens]).astype(np.int32) \
        if indptr[-1] else np.zeros(0, dtype=np.int32)
    data = rng.standard_normal(indices.size)
    N = 0 if kind == "zero_cols_B" else 17
    mat = {"indptr": indptr, "indices": indices, "data": data, "shape": (m, k)}
    C, ref, scale, lens2 = _run_case(mat, N, "float32", seed=6)
    assert C.shape == (m, N)
    if N:
        _check(C, ref, scale, lens2, "float32", kind)


def test_spmm_zero_rows():
    C = fs.flagsparse_spmm_csr(torch.zeros(0, device="cuda"), torch.zeros(0, dtype=torch.int32, device="cuda"),
                               torch.zeros(1, dtype=torch.int64, device="cuda"), torch.randn(4, 3, device="cuda"),
                               (0, 4))
    assert C.shape == (0, 3)


def test_spmm_repeat_calls_bitwise_and_tickets_reset():
    c = workloads.zipf_csr(n=50_000, seed=13)
    A = (dev(c["data"]), dev(c["indices"]), dev(c["indptr"]))
    p = fs.prepare_spmm_csr_route(*A, c["shape"])
    B = torch.randn(c["shape"][1], 64, device="cuda")
    C0 = fs.flagsparse_spmm_csr_run(p, B)
    for _ in range(3):
        assert torch.equal(fs.flagsparse_spmm_csr_run(p, B), C0)
    _route, plan, _ = sm._route_native(p, "non")
    assert plan.n_slots > 0 and plan.counters_clear()


@pytest.mark.parametrize("dname,N,tile", [("float32", 16, 0), ("float32", 128, 0), ("bfloat16", 64, 0),
                                         ("float64", 32, 0), ("float32", 128, 128), ("bfloat16", 256, 256)])
def test_spmm_persistent_grid_bitwise(dname, N, tile):
    """The persistent grid (FSB_SPMM_PERSISTENT) runs the same work items as one item per
    warp, so the products are bitwise equal -- with narrower column tiles too, and for the
    fused SpMV + SpMM launch."""
    c = workloads.zipf_csr(n=300_000, seed=21, dtype=np.float64)
    dt = TORCH_DT[dname]
    data, ind, ptr = dev(c["data"], dt), dev(c["indices"]), dev(c["indptr"])
    n = c["shape"][0]
    plan = _csr.SpmmPlan(ptr, n, dt)
    B = torch.randn(c["shape"][1], N, device="cuda", dtype=torch.float64).to(dt)
    C = [torch.empty(n, N, device="cuda", dtype=dt) for _ in range(2)]
    for C_i, persistent in zip(C, (False, True)):
        _csr.spmm(data, ind, ptr, n, c["shape"][1], B, plan, C_i, tile_bytes=tile, persistent=persistent)
    assert torch.equal(C[0], C[1])
    ref, scale, lens = _oracle_spmm(c["indptr"], c["indices"], rounded(c["data"], dname), c["shape"],
                                    rounded(host(B), dname), "non")
    _check(C[1], ref, scale, lens, dname, f"persistent {dname} N={N}")
    if dname != "float32" or N != 16:
        return
    x = torch.randn(c["shape"][1], device="cuda", dtype=dt)
    ys = [torch.empty(n, device="cuda", dtype=dt) for _ in range(2)]
    for C_i, y_i, persistent in zip(C, ys, (False, True)):
        assert _csr.spmm_spmv(data, ind, ptr, n, c["shape"][1], B, plan, C_i, x, y_i, persistent=persistent)
    assert torch.equal(C[0], C[1]) and torch.equal(ys[0], ys[1])


# ---------------------------------------------------------------- opt entry points / API contract

def test_spmm_opt_entry_points_agree():
    c = workloads.zipf_csr(n=8_000, seed=14, dtype=np.float64)
    A = (dev(c["data"]), dev(c["indices"]), dev(c["indptr"]))
    B = torch.randn(c["shape"][1], 32, dtype=torch.float64, device="cuda")
    base = fs.flagsparse_spmm_csr(*A, B, c["shape"])
    p1 = fs.prepare_spmm_csr_opt(*A, c["shape"])
    C1, meta1 = fs.flagsparse_spmm_csr_opt(B=B, prepared=p1, return_meta=True)
    C1b = fs.flagsparse_spmm_csr_opt_alg1_preprocess(*A, B=B, shape=c["shape"])
    p2 = fs.prepare_spmm_csr_opt_alg2(*A, c["shape"])
    C2, meta2 = fs.flagsparse_spmm_csr_opt_alg2(B=B, prepared=p2, return_meta=True)
    for C in (C1, C1b, C2):
        assert torch.equal(C, base)
    assert {"long_part_count", "long_row_count", "bucket_count"} <= set(meta1)
    lens = np.diff(c["indptr"])
    assert meta1["long_row_count"] == int((lens > 2048).sum())
    assert meta1["long_part_count"] == int(np.ceil(lens[lens > 2048] / 256).sum())
    assert sum(h["row_count"] for h in meta2["bucket_hits"]) == c["shape"][0]


def test_spmm_validation_messages():
    A = (torch.randn(3, device="cuda"), torch.tensor([0, 1, 2], dtype=torch.int32, device="cuda"),
         torch.tensor([0, 1, 2, 3], device="cuda"))
    with pytest.raises(ValueError, match=r"B.shape\[0\] must be n_cols=8"):
        fs.flagsparse_spmm_csr(*A, torch.randn(5, 2, device="cuda"), (3, 8))
    with pytest.raises(ValueError, match="out shape/dtype must match result"):
        fs.flagsparse_spmm_csr(*A, torch.randn(8, 2, device="cuda"), (3, 8), out=torch.empty(3, 3, device="cuda"))
    with pytest.raises(ValueError, match="transpose conflicts with op"):
        fs.flagsparse_spmm_csr(*A, torch.randn(3, 2, device="cuda"), (3, 8), op="non", transpose=True)
    with pytest.raises(ValueError, match="op must be one of"):
        fs.flagsparse_spmm_csr(*A, torch.randn(8, 2, device="cuda"), (3, 8), op="bad")
    with pytest.raises(TypeError, match="B dtype must match data dtype"):
        fs.flagsparse_spmm_csr(*A, torch.randn(8, 2, dtype=torch.float64, device="cuda"), (3, 8))
    with pytest.raises(IndexError, match="indices out of range"):
        fs.flagsparse_spmm_csr(*A, torch.randn(2, 2, device="cuda"), (3, 2))
    with pytest.raises(ValueError, match="unsupported CSR SpMM algorithm"):
        fs.resolve_spmm_csr_algorithm("nope", "non", torch.float32)
    with pytest.raises(TypeError, match="does not support dtype"):
        fs.resolve_spmm_csr_algorithm("csr_base_accuracy", "non", torch.bfloat16)
    with pytest.raises(TypeError, match="only supports float32 and float64"):
        fs.flagsparse_spmm_csr_opt(A[0].half(), A[1], A[2], torch.randn(8, 2, device="cuda").half(), (3, 8))


def test_route_meta_and_diagnostics():
    mat = workloads.mask_csr(20, 20, seed=15, dtype=np.float64)
    p = fs.prepare_spmm_csr_route(dev(mat["data"], torch.float32), dev(mat["indices"]), dev(mat["indptr"]),
                                  (20, 20), op="trans", alg="alg2")
    C, ms, meta = fs.flagsparse_spmm_csr_run(p, torch.randn(20, 4, device="cuda"), return_time=True,
                                             return_meta=True, timing=True, diagnostics=True)
    assert meta["alg"] == "spmm_csr_alg2" and meta["display_name"] == "Alg2" and meta["op"] == "trans"
    assert {"operator_ms", "gpu_ms", "process_cpu_ms", "process_gpu_ms", "compute_ms", "diagnostics"} <= set(meta)
    assert ms == meta["operator_ms"]
    assert fs.list_spmm_csr_algorithms(dtype=torch.bfloat16) == ("csr_base",)


# ---------------------------------------------------------------- full size: sampled rows + linearity

@pytest.mark.parametrize("dname,N", [("float32", 64), ("bfloat16", 128)])
def test_spmm_power_law_1m_sampled_rows(dname, N):
    """1,000,000-row power-law matrix (mean 32 per row): 2,000 sampled rows
    against the oracle, and linearity A(B1 + B2) = A B1 + A B2 on every row."""
    c = workloads.zipf_csr(n=1_000_000, scale=32.0 / workloads.ZIPF_MEAN_UNSCALED, seed=2, dtype=np.float32,
                           values="normal")
    dt = TORCH_DT[dname]
    A = (dev(c["data"], dt), dev(c["indices"]), dev(c["indptr"]))
    p = fs.prepare_spmm_csr_route(*A, c["shape"])
    g = torch.Generator(device="cuda").manual_seed(2)
    B1 = torch.randn(c["shape"][1], N, device="cuda", generator=g).to(dt)
    B2 = torch.randn(c["shape"][1], N, device="cuda", generator=g).to(dt)
    C1 = fs.flagsparse_spmm_csr_run(p, B1)
    rows = np.sort(np.random.Generator(np.random.PCG64(3)).choice(c["shape"][0], 2000, replace=False))
    rows = np.unique(np.concatenate([rows, np.argsort(np.diff(c["indptr"]))[-20:]]))  # include the longest rows
    lens = np.diff(c["indptr"])[rows]
    sub_ptr = np.zeros(rows.size + 1, dtype=np.int64)
    np.cumsum(lens, out=sub_ptr[1:])
    take = np.concatenate([np.arange(c["indptr"][r], c["indptr"][r + 1]) for r in rows])
    d_r = rounded(c["data"][take].astype(np.float64), dname)
    ref = oracle.spmm(sub_ptr, c["indices"][take], d_r, host(B1).astype(np.float64))
    scale = oracle.spmm(sub_ptr, c["indices"][take], np.abs(d_r), np.abs(host(B1).astype(np.float64)))
    bound = plain_error_bound(dname, ref, scale, np.broadcast_to(lens[:, None], ref.shape))
    assert_within(host(C1[torch.from_numpy(rows).cuda()]).astype(np.float64), ref, bound, "sampled rows")
    if dname == "float32":
        C2 = fs.flagsparse_spmm_csr_run(p, B2)
        C12 = fs.flagsparse_spmm_csr_run(p, B1 + B2)
        diff = (C12 - (C1 + C2)).abs()
        scale_all = fs.flagsparse_spmm_csr_run(fs.prepare_spmm_csr_route(A[0].abs(), A[1], A[2], c["shape"]),
                                               B1.abs() + B2.abs())
        lens_t = torch.from_numpy(np.diff(c["indptr"])).cuda().float()[:, None] + 3
        assert bool((diff <= 4 * lens_t * 2.0**-24 * scale_all + 1e-30).all())
