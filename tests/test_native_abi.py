"""The C-ABI library loads on a CPU-only host and exports every declared symbol."""

import ctypes
import os
import re

from flagsparse_b200 import _native

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    include = os.path.join(REPO, "include")
    for fname in os.listdir(include):
        if fname.endswith(".h"):
            text = open(os.path.join(include, fname)).read()
            names |= set(re.findall(r"FSB_API\s+[A-Za-z_][A-Za-z0-9_ \*]*?\b(fsb_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_native.LIB_PATH)
    declared = _declared_symbols()
    assert declared, "no declarations found"
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    assert _declared_symbols() == set(_native.exported_symbols())


def test_status_strings_and_version():
    lib = _native.lib()
    assert lib.fsb_version() >= 100
    assert _native.status_text(0) == "ok"
    assert "wait" in _native.status_text(_native.FSB_ERR_TIMEOUT)
    assert _native.status_text(-99) == "unknown status"


def test_size_queries_need_no_gpu():
    lib = _native.lib()
    assert lib.fsb_spmv_partial_bytes(2) == 8
    assert lib.fsb_spmv_partial_bytes(5) == 32
    assert lib.fsb_spmv_partial_bytes(42) == -1
    assert lib.fsb_spmv_default_cap(2) == 224 and lib.fsb_spmv_default_cap(3) == 128
    assert lib.fsb_spmv_default_chunk(2) % 256 == 0
    assert lib.fsb_spmv_plan_workspace_bytes(10_000) > 0
    assert lib.fsb_csr_transpose_workspace_bytes(1 << 40, 10, 10) == -1


def test_invalid_arguments_are_rejected_without_touching_the_device():
    lib = _native.lib()
    # null indptr / negative sizes return FSB_ERR_INVALID_ARG before any launch
    assert lib.fsb_csr_inspect(None, 0, None, 0, 5, 0, None, None) == _native.FSB_ERR_INVALID_ARG
    assert lib.fsb_spmv_plan_analyze(None, 0, -1, 1024, 4096, None, 0, None, None) == _native.FSB_ERR_INVALID_ARG
    assert lib.fsb_gather_values(2, None, None, 3, 0, None, None) == _native.FSB_ERR_INVALID_ARG
    assert lib.fsb_spmv_csr(2, None, None, 0, None, 0, 4, 4, None, None, None, None) == _native.FSB_ERR_INVALID_ARG


def _declared_param_counts():
    counts = {}
    include = os.path.join(REPO, "include")
    for fname in os.listdir(include):
        if not fname.endswith(".h"):
            continue
        text = open(os.path.join(include, fname)).read()
        for m in re.finditer(r"FSB_API\s+[A-Za-z_][A-Za-z0-9_ \*]*?\b(fsb_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", text):
            params = " ".join(m.group(2).split())
            counts[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return counts


def test_binding_argument_counts_match_the_header():
    """Every ctypes signature has as many arguments as its C declaration."""
    counts = _declared_param_counts()
    assert set(counts) == set(_native.exported_symbols())
    wrong = {n: (c, len(_native._SIGNATURES[n][1])) for n, c in counts.items() if c != len(_native._SIGNATURES[n][1])}
    assert not wrong, wrong


def test_backward_entry_rejects_bad_arguments_without_a_launch():
    lib = _native.lib()
    # no plan, negative width, missing dX: rejected on the host
    assert lib.fsb_spmm_csr_backward(2, None, None, None, None, 4, 4, None, 8, None, 8, 8, None, 8, None, None,
                                     None) == _native.FSB_ERR_INVALID_ARG
    plan = _native.SpmvPlan()
    assert lib.fsb_spmm_csr_backward(2, None, None, None, None, 4, 4, None, 8, None, 8, -1, None, 8, None,
                                     ctypes.byref(plan), None) == _native.FSB_ERR_INVALID_ARG
    # n == 0 is left to the separate kernels
    assert lib.fsb_spmm_csr_backward(2, None, None, None, None, 4, 4, None, 8, None, 8, 0, ctypes.c_void_p(16), 8,
                                     None, ctypes.byref(plan), None) == _native.FSB_ERR_UNSUPPORTED
