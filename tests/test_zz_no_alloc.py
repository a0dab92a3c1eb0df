"""fsb_spmv_csr_static_scratch: SpMV that allocates nothing, through the C ABI.

The entry point takes its long-row scratch from a file-scope device array of
the library instead of the plan, so these tests hand it a plan whose
``partials`` / ``counters`` are NULL and compare every result bit for bit
with fsb_spmv_csr on the same plan (caller scratch), on two calls in a row.
The file name sorts last so it also runs after every other test module.
"""

import ctypes

import numpy as np
import pytest
import torch

from flagsparse_b200 import _native as nat
from flagsparse_b200 import workloads
from flagsparse_b200.sparse_operations import _csr

from tests.helpers import TORCH_DT, dev


def _no_scratch_copy(plan):
    s = plan._struct
    c = nat.SpmvPlan.from_buffer_copy(s)
    c.partials = None
    c.counters = None
    return c


def _call(fn, data, indices, indptr, n_rows, n_cols, x, y, plan_ref):
    return fn(
        nat.dtype_code(data.dtype), nat.ptr(data), nat.ptr(indices), nat.is64(indices),
        nat.ptr(indptr), nat.is64(indptr), int(n_rows), int(n_cols),
        nat.ptr(x), nat.ptr(y), plan_ref, nat.stream_of(x.device),
    )


def _bits(t):
    t = t.detach()
    if t.is_complex():
        t = torch.view_as_real(t)
    width = {2: torch.int16, 4: torch.int32, 8: torch.int64}[t.element_size()]
    return t.contiguous().view(width)


def test_oversized_plan_is_rejected_before_any_work():
    """A plan above the built-in slot count fails with FSB_ERR_TOO_LARGE; no device is touched."""
    lib = nat.lib()
    p = nat.SpmvPlan()
    p.n_units = 1
    p.n_slots = nat.FSB_SPMV_STATIC_MAX_SLOTS + 1
    p.cap, p.chunk_nnz = 128, 512
    rc = lib.fsb_spmv_csr_static_scratch(2, None, None, 0, None, 1, 10, 10, None, None, ctypes.byref(p), None)
    assert rc == nat.FSB_ERR_TOO_LARGE
    assert "scratch" in nat.status_text(rc)
    p.n_slots = -1
    assert lib.fsb_spmv_csr_static_scratch(2, None, None, 0, None, 1, 10, 10, None, None, ctypes.byref(p),
                                           None) == nat.FSB_ERR_INVALID_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("dname", ["bfloat16", "float32", "float64", "complex128"])
@pytest.mark.parametrize("idx_dt,ptr_dt", [(torch.int32, torch.int64), (torch.int64, torch.int32)])
def test_static_scratch_matches_caller_scratch(dname, idx_dt, ptr_dt):
    c = workloads.zipf_csr(n=300_000, seed=9, dtype=np.float64)
    n = c["shape"][0]
    dt = TORCH_DT[dname]
    data = dev(c["data"], dt)
    if dt.is_complex:
        data = data + 0.5j * dev(c["data"][::-1].copy(), dt)
    indices = dev(c["indices"], idx_dt)
    indptr = dev(c["indptr"], ptr_dt)
    x = dev(c["x"], dt)
    plan = _csr.NativeSpmvPlan(indptr, n, dt)
    assert 0 < plan.n_slots <= nat.FSB_SPMV_STATIC_MAX_SLOTS  # long rows use the scratch
    bare = _no_scratch_copy(plan)
    lib = nat.lib()
    for call in range(2):
        y_ref = torch.empty(n, dtype=dt, device="cuda")
        y_st = torch.full((n,), float("nan"), dtype=dt, device="cuda")
        nat.check(_call(lib.fsb_spmv_csr, data, indices, indptr, n, n, x, y_ref, plan.struct_ref()), "fsb_spmv_csr")
        nat.check(_call(lib.fsb_spmv_csr_static_scratch, data, indices, indptr, n, n, x, y_st, ctypes.byref(bare)),
                  "fsb_spmv_csr_static_scratch")
        torch.cuda.synchronize()
        assert torch.equal(_bits(y_st), _bits(y_ref)), f"call {call}"


@pytest.mark.gpu
def test_static_scratch_at_full_power_law_size():
    """2,000,000-row power-law matrix (38.9 M nonzeros): its plan fits the built-in scratch."""
    c = workloads.zipf_csr()
    n = c["shape"][0]
    data, indices, indptr, x = dev(c["data"]), dev(c["indices"]), dev(c["indptr"]), dev(c["x"])
    plan = _csr.NativeSpmvPlan(indptr, n, torch.float32)
    assert 0 < plan.n_slots <= nat.FSB_SPMV_STATIC_MAX_SLOTS
    bare = _no_scratch_copy(plan)
    lib = nat.lib()
    y_ref = torch.empty(n, dtype=torch.float32, device="cuda")
    nat.check(_call(lib.fsb_spmv_csr, data, indices, indptr, n, n, x, y_ref, plan.struct_ref()), "fsb_spmv_csr")
    for call in range(2):
        y_st = torch.full((n,), float("nan"), device="cuda")
        nat.check(_call(lib.fsb_spmv_csr_static_scratch, data, indices, indptr, n, n, x, y_st, ctypes.byref(bare)),
                  "fsb_spmv_csr_static_scratch")
        torch.cuda.synchronize()
        assert torch.equal(_bits(y_st), _bits(y_ref)), f"call {call}"


@pytest.mark.gpu
def test_static_scratch_plan_without_long_rows():
    """Plans with no multi-chunk rows never touch the scratch (n_slots == 0)."""
    c = workloads.poisson_csr()
    n = c["shape"][0]
    data, indices, indptr, x = dev(c["data"]), dev(c["indices"]), dev(c["indptr"]), dev(c["x"])
    plan = _csr.NativeSpmvPlan(indptr, n, torch.float32)
    assert plan.n_slots == 0
    bare = _no_scratch_copy(plan)
    lib = nat.lib()
    y_ref = torch.empty(n, device="cuda")
    y_st = torch.full((n,), float("nan"), device="cuda")
    nat.check(_call(lib.fsb_spmv_csr, data, indices, indptr, n, n, x, y_ref, plan.struct_ref()), "fsb_spmv_csr")
    nat.check(_call(lib.fsb_spmv_csr_static_scratch, data, indices, indptr, n, n, x, y_st, ctypes.byref(bare)),
              "fsb_spmv_csr_static_scratch")
    torch.cuda.synchronize()
    assert torch.equal(_bits(y_st), _bits(y_ref))
