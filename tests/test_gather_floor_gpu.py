"""The two measurement kernels: the SpMV x-gather floor (fsb_spmv_gather_floor) and
the SpMM B-row gather floor through TMA (fsb_spmm_gather_floor_tma), against float64
sums of the same products computed with torch on the GPU."""

import numpy as np
import pytest
import torch

from flagsparse_b200 import _native as nat

pytestmark = pytest.mark.gpu


def _inputs(nnz, k, dt, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    cols = torch.randint(0, k, (nnz,), generator=g, device="cuda", dtype=torch.int32)
    vals = torch.randn(nnz, generator=g, device="cuda").to(dt)
    return vals, cols


@pytest.mark.parametrize("dt", [torch.float32, torch.float64, torch.bfloat16])
def test_spmv_gather_floor_sums_every_product(dt):
    nnz, k = 1_000_003, 70_000
    vals, cols = _inputs(nnz, k, dt, 1)
    x = torch.randn(k, device="cuda").to(dt)
    out = torch.zeros(148 * 8, dtype=torch.float64, device="cuda")
    nat.check(nat.lib().fsb_spmv_gather_floor(nat.dtype_code(dt), nat.ptr(vals), nat.ptr(cols), 0, nnz, nat.ptr(x),
                                              nat.ptr(out), out.numel(), nat.stream_of(out.device)),
              "fsb_spmv_gather_floor")
    ref = (vals.double() * x.double()[cols.long()]).sum()
    scale = (vals.double().abs() * x.double().abs()[cols.long()]).sum()
    assert abs(float(out.sum() - ref)) <= 1e-9 * float(scale)  # fp64 sums of 1e6 exact products


@pytest.mark.parametrize("dt,n", [(torch.float32, 128), (torch.float32, 64), (torch.bfloat16, 128),
                                  (torch.float16, 256)])
@pytest.mark.parametrize("nnz", [100_003, 8 * 1776])
def test_spmm_gather_floor_tma_per_warp_sums(dt, n, nnz):
    """Warp w sums nonzeros [w * per, (w + 1) * per) of value * B row: each warp's row of
    out against the float64 sum of its products, within the fp32 summation bound."""
    k = 5_000
    vals, cols = _inputs(nnz, k, dt, 2)
    B = torch.randn(k, n, device="cuda").to(dt)
    rows = 148 * 3 * 4
    out = torch.full((rows, n), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    nat.check(nat.lib().fsb_spmm_gather_floor_tma(nat.dtype_code(dt), nat.ptr(vals), nat.ptr(cols), nnz, nat.ptr(B), k,
                                                  n, n, nat.ptr(out), rows, nat.ptr(err), nat.stream_of(B.device)),
              "fsb_spmm_gather_floor_tma")
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    per = -(-nnz // rows)
    owner = torch.arange(nnz, device="cuda") // per
    terms = vals.double()[:, None] * B.double()[cols.long()]
    ref = torch.zeros(rows, n, dtype=torch.float64, device="cuda").index_add_(0, owner, terms)
    scale = torch.zeros(rows, n, dtype=torch.float64, device="cuda").index_add_(0, owner, terms.abs())
    gamma = (per + 1) * 2.0**-24
    bound = 2.0**-24 * ref.abs() + gamma * scale + 1e-30
    assert torch.all((out.double() - ref).abs() <= bound)


def test_spmm_gather_floor_tma_rejects():
    B = torch.zeros(16, 32, device="cuda")  # 128-byte rows: not a gather floor width
    v = torch.zeros(4, device="cuda")
    c = torch.zeros(4, dtype=torch.int32, device="cuda")
    out = torch.zeros(8, 32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    lib = nat.lib()
    st = nat.stream_of(B.device)
    assert lib.fsb_spmm_gather_floor_tma(nat.dtype_code(torch.float32), nat.ptr(v), nat.ptr(c), 4, nat.ptr(B), 16, 32,
                                         32, nat.ptr(out), 8, nat.ptr(err), st) == nat.FSB_ERR_UNSUPPORTED
    assert lib.fsb_spmm_gather_floor_tma(nat.dtype_code(torch.float32), nat.ptr(v), nat.ptr(c), 4, nat.ptr(B), 16, 32,
                                         32, nat.ptr(out), 6, nat.ptr(err), st) == nat.FSB_ERR_INVALID_ARG
    assert lib.fsb_spmm_gather_floor_tma(nat.dtype_code(torch.float64), nat.ptr(v), nat.ptr(c), 4, nat.ptr(B), 16, 16,
                                         16, nat.ptr(out), 8, nat.ptr(err), st) == nat.FSB_ERR_UNSUPPORTED
