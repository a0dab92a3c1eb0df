"""BSR-16 SpMM on the tcgen05 tensor cores against the oracle.

The oracle multiplies the equivalent CSR matrix (every 16 x 16 block expanded
to 256 nonzeros) with Dot2 sums on the same bf16 / f16 inputs; the kernel
accumulates exact 16-bit products in fp32 and rounds once to the value type.
"""

import numpy as np
import pytest
import torch

import flagsparse_b200 as fs
from flagsparse_b200 import workloads
from oracle import oracle
from tests.helpers import assert_within, host, plain_error_bound

pytestmark = pytest.mark.gpu

NAME = {torch.bfloat16: "bfloat16", torch.float16: "float16"}


def _bsr_to_csr(indptr, indices, blocks):
    """Expanded CSR (int64 indptr, int32 indices, float64 values) of a BSR-16 matrix."""
    n_brows = indptr.size - 1
    per_row = np.diff(indptr)
    ptr = np.zeros(n_brows * 16 + 1, dtype=np.int64)
    ptr[1:] = np.repeat(per_row * 16, 16)
    np.cumsum(ptr, out=ptr)
    cols, vals = [], []
    for br in range(n_brows):
        b0, b1 = indptr[br], indptr[br + 1]
        if b0 == b1:
            continue
        bc = indices[b0:b1]
        c = (bc[:, None] * 16 + np.arange(16)[None, :]).reshape(-1)  # row-independent column list
        cols.append(np.tile(c, 16))
        vals.append(blocks[b0:b1].transpose(1, 0, 2).reshape(-1))  # [row i][block][col j]
    cols = np.concatenate(cols).astype(np.int32) if cols else np.zeros(0, np.int32)
    vals = np.concatenate(vals).astype(np.float64) if vals else np.zeros(0)
    return ptr, cols, vals


def _case(n_brows, n_bcols, per_row, seed, empty=()):
    rng = np.random.Generator(np.random.PCG64(seed))
    lens = np.array([0 if r in empty else min(per_row, n_bcols) for r in range(n_brows)], dtype=np.int64)
    indptr = np.zeros(n_brows + 1, dtype=np.int64)
    np.cumsum(lens, out=indptr[1:])
    indices = np.concatenate([np.sort(rng.choice(n_bcols, int(l), replace=False)) for l in lens]).astype(np.int32)
    blocks = rng.standard_normal((indices.size, 16, 16)).astype(np.float32)
    return indptr, indices, blocks


def _check(C, indptr, indices, blocks_r, B_r, dname, rows=None):
    ptr, cols, vals = _bsr_to_csr(indptr, indices, blocks_r)
    if rows is not None:
        lens = np.diff(ptr)[rows]
        sub = np.zeros(rows.size + 1, dtype=np.int64)
        np.cumsum(lens, out=sub[1:])
        take = np.concatenate([np.arange(ptr[r], ptr[r + 1]) for r in rows])
        ptr, cols, vals = sub, cols[take], vals[take]
    ref = oracle.spmm(ptr, cols, vals, B_r)
    scale = oracle.spmm(ptr, cols, np.abs(vals), np.abs(B_r))
    lens = np.diff(ptr)[:, None]
    got = host(C if rows is None else C[torch.from_numpy(rows).cuda()]).astype(np.float64)
    assert_within(got, ref, plain_error_bound(dname, ref, scale, np.broadcast_to(lens, ref.shape)), "bsr16")


@pytest.mark.parametrize("dt", [torch.bfloat16, torch.float16])
@pytest.mark.parametrize("n_brows,n_bcols,per_row,N,empty", [
    (1, 1, 1, 128, ()),
    (8, 8, 3, 128, ()),
    (64, 64, 8, 256, (3, 17)),
    (700, 900, 8, 384, (0, 699)),
    (8, 8, 3, 64, (2,)),
    (300, 200, 6, 192, (0, 299)),
])
def test_bsr16_against_oracle(dt, n_brows, n_bcols, per_row, N, empty):
    indptr, indices, blocks = _case(n_brows, n_bcols, per_row, seed=n_brows + N, empty=empty)
    rng = np.random.Generator(np.random.PCG64(N))
    blocks_t = torch.from_numpy(blocks).to(dt).cuda()
    B = torch.from_numpy(rng.standard_normal((n_bcols * 16, N)).astype(np.float32)).to(dt).cuda()
    C = fs.flagsparse_spmm_bsr16(blocks_t, torch.from_numpy(indices).cuda(), torch.from_numpy(indptr).cuda(), B,
                                 (n_brows * 16, n_bcols * 16), check_status=True)
    _check(C, indptr, indices, host(blocks_t), host(B).astype(np.float64), NAME[dt])
    for r in empty:
        assert bool((C[r * 16:(r + 1) * 16] == 0).all())


def test_bsr16_full_size_sampled_rows_and_determinism():
    """65,536 x 65,536 blocks (M = K = 1,048,576), 8 blocks per block row, N = 128, bf16:
    600 sampled rows against the oracle; repeated calls bitwise equal."""
    c = workloads.bsr16()
    n = c["block_shape"][0] * 16
    blocks = torch.from_numpy(c["blocks"]).to(torch.bfloat16).cuda()
    p = fs.prepare_spmm_bsr16(blocks, torch.from_numpy(c["indices"]).cuda(), torch.from_numpy(c["indptr"]).cuda(),
                              (n, n))
    g = torch.Generator(device="cuda").manual_seed(2)
    B = torch.randn(n, 128, device="cuda", generator=g).bfloat16()
    C = fs.flagsparse_spmm_bsr16(B=B, prepared=p, check_status=True)
    rows = np.sort(np.random.Generator(np.random.PCG64(5)).choice(n, 600, replace=False))
    # expand only the sampled rows' block rows
    brows = np.unique(rows // 16)
    sub_ptr = np.zeros(brows.size + 1, dtype=np.int64)
    np.cumsum(np.diff(c["indptr"])[brows], out=sub_ptr[1:])
    take = np.concatenate([np.arange(c["indptr"][b], c["indptr"][b + 1]) for b in brows])
    local = np.searchsorted(brows, rows // 16) * 16 + rows % 16
    ptr, cols, vals = _bsr_to_csr(sub_ptr, c["indices"][take], host(blocks)[take])
    lens = np.diff(ptr)[local]
    sp = np.zeros(local.size + 1, dtype=np.int64)
    np.cumsum(lens, out=sp[1:])
    tk = np.concatenate([np.arange(ptr[r], ptr[r + 1]) for r in local])
    B64 = host(B).astype(np.float64)
    ref = oracle.spmm(sp, cols[tk], vals[tk], B64)
    scale = oracle.spmm(sp, cols[tk], np.abs(vals[tk]), np.abs(B64))
    got = host(C[torch.from_numpy(rows).cuda()]).astype(np.float64)
    assert_within(got, ref, plain_error_bound("bfloat16", ref, scale, np.broadcast_to(lens[:, None], ref.shape)),
                  "bsr16 full size")
    assert torch.equal(fs.flagsparse_spmm_bsr16(B=B, prepared=p), C)


@pytest.mark.parametrize("N", [128, 192])
def test_bsr16_b_larger_than_l2(N):
    """A dense operand larger than L2 (40,000 block columns, K = 640,000 rows), N = 128 and
    192 (a last tile of 64 columns): every row against the oracle, the error word left clear."""
    indptr, indices, blocks = _case(300, 40_000, 8, seed=N, empty=(5,))
    blocks_t = torch.from_numpy(blocks).bfloat16().cuda()
    g = torch.Generator(device="cuda").manual_seed(N)
    B = torch.randn(40_000 * 16, N, device="cuda", generator=g).bfloat16()
    assert B.numel() * 2 > 126 * 2**20
    p = fs.prepare_spmm_bsr16(blocks_t, torch.from_numpy(indices).cuda(), torch.from_numpy(indptr).cuda(),
                              (300 * 16, 40_000 * 16))
    C = fs.flagsparse_spmm_bsr16(B=B, prepared=p)
    assert p.status(synchronize=True) == 0
    _check(C, indptr, indices, host(blocks_t), host(B).astype(np.float64), "bfloat16")
    assert bool((C[5 * 16:6 * 16] == 0).all())


def test_bsr16_agrees_with_csr_spmm_on_expanded_matrix():
    indptr, indices, blocks = _case(300, 400, 6, seed=9)
    blocks_t = torch.from_numpy(blocks).bfloat16().cuda()
    B = torch.randn(400 * 16, 128, device="cuda").bfloat16()
    C_bsr = fs.flagsparse_spmm_bsr16(blocks_t, torch.from_numpy(indices).cuda(), torch.from_numpy(indptr).cuda(), B,
                                     (300 * 16, 400 * 16))
    ptr, cols, vals = _bsr_to_csr(indptr, indices, host(blocks_t))
    C_csr = fs.flagsparse_spmm_csr(torch.from_numpy(vals).bfloat16().cuda(), torch.from_numpy(cols).cuda(),
                                   torch.from_numpy(ptr).cuda(), B, (300 * 16, 400 * 16))
    # both are fp32 sums of the same exact products, in different orders, rounded to
    # bfloat16: each within u_bf16 |c| + gamma_n S of the exact value (n = 96 terms)
    scale = fs.flagsparse_spmm_csr(torch.from_numpy(np.abs(vals)).float().cuda(), torch.from_numpy(cols).cuda(),
                                   torch.from_numpy(ptr).cuda(), B.float().abs(), (300 * 16, 400 * 16))
    diff = (C_bsr.float() - C_csr.float()).abs()
    bound = 2.0**-8 * (C_bsr.float().abs() + C_csr.float().abs()) + 2 * 100 * 2.0**-24 * scale + 1e-30
    assert bool((diff <= bound).all())


def test_bsr16_validation_and_out():
    indptr, indices, blocks = _case(4, 4, 2, seed=1)
    args = (torch.from_numpy(blocks).bfloat16().cuda(), torch.from_numpy(indices).cuda(),
            torch.from_numpy(indptr).cuda())
    with pytest.raises(ValueError, match="multiple of 64"):
        fs.flagsparse_spmm_bsr16(*args, torch.randn(64, 96, device="cuda").bfloat16(), (64, 64))
    with pytest.raises(TypeError, match="bfloat16 or torch.float16"):
        fs.prepare_spmm_bsr16(args[0].float(), args[1], args[2], (64, 64))
    with pytest.raises(ValueError, match="multiples of 16"):
        fs.prepare_spmm_bsr16(*args, (63, 64))
    out = torch.empty(64, 128, device="cuda").bfloat16()
    C = fs.flagsparse_spmm_bsr16(*args, torch.randn(64, 128, device="cuda").bfloat16(), (64, 64), out=out)
    assert C is out
