"""The drop-in surface: registry, exported names, signatures, route table (CPU only)."""

import inspect
import os
import re

import pytest
import torch

import flagsparse_b200 as fs
from flagsparse_b200.sparse_operations import sddmm_csr as dm
from flagsparse_b200.sparse_operations import spmm_csr as sm
from flagsparse_b200.sparse_operations import spmv_csr as vm

REGISTRY = os.path.join(os.path.dirname(fs.__file__), "conf", "operators.yaml")
# FlagSparse label / kind values that its registry test skips (tests/ci/test_operator_registry.py:63-86)
IGNORED = {"flagsparse", "sparse", "triton", "public-api", "csr", "coo", "csc", "bsr", "sell", "optimized",
           "alpha-sparse", "descriptor", "format", "Sparse", "SparseLinearAlg", "SparseSolver", "SparseFormat",
           "Utility"}


def _text():
    with open(REGISTRY, encoding="utf-8") as f:
        return f.read()


def test_registry_shape_ids_and_interfaces():
    text = _text()
    body = "\n".join(line for line in text.splitlines() if not line.startswith("#")).lstrip("\n")
    assert body.startswith("ops:\n")
    for snippet in ("description: |", "for:", "labels:", "kind:", "stages:"):
        assert snippet in text
    ids = re.findall(r"^  - id: ([a-z0-9_]+)$", text, flags=re.MULTILINE)
    assert ids == ["spmv_csr", "spmm_csr", "spmm_csr_opt", "spmm_csr_opt_alg1", "spmm_csr_opt_alg2", "sddmm_csr",
                   "spmv_bsr", "spmv_coo_tocsr"]
    names = set(re.findall(r"^      - ([A-Za-z_][A-Za-z0-9_]*)$", text, flags=re.MULTILINE)) - IGNORED
    assert names and names <= set(fs.__all__)


def test_every_export_resolves():
    for name in fs.__all__:
        assert getattr(fs, name) is not None, name
    with pytest.raises(AttributeError):
        fs.flagsparse_not_a_function  # noqa: B018


def _params(fn):
    return [(p.name, p.default) for p in inspect.signature(fn).parameters.values()]


E = inspect.Parameter.empty

SIGNATURES = {
    # flagsparse spmv_csr.py:837-853 / :614-624
    "flagsparse_spmv_csr": [("data", None), ("indices", None), ("indptr", None), ("x", None), ("shape", None),
                            ("block_nnz", 256), ("max_segments", None), ("out", None), ("return_time", False),
                            ("return_meta", False), ("use_opt", False), ("prepared", None), ("transpose", None),
                            ("op", None), ("index_fallback_policy", "auto")],
    "prepare_spmv_csr": [("data", E), ("indices", E), ("indptr", E), ("shape", E), ("block_nnz", 256),
                         ("max_segments", None), ("transpose", False), ("op", None),
                         ("index_fallback_policy", "auto")],
    # spmm_csr.py:3981-3995, :2577, :2607-2618
    "flagsparse_spmm_csr": [("data", E), ("indices", E), ("indptr", E), ("B", E), ("shape", E), ("block_n", None),
                            ("block_nnz", None), ("max_segments", None), ("out", None), ("return_time", False),
                            ("transpose", None), ("op", None), ("return_meta", False)],
    "prepare_spmm_csr_route": [("data", E), ("indices", E), ("indptr", E), ("shape", E), ("op", "non"),
                               ("alg", "auto")],
    "flagsparse_spmm_csr_run": [("prepared", E), ("B", E), ("alg", None), ("op", None), ("dense_layout", "auto"),
                                ("return_time", False), ("return_meta", False), ("timing", False),
                                ("diagnostics", False)],
    # sddmm_csr.py:389-403, :107
    "flagsparse_sddmm_csr": [("data", None), ("indices", None), ("indptr", None), ("x", None), ("y", None),
                             ("shape", None), ("alpha", 1.0), ("beta", 0.0), ("prepared", None), ("out", None),
                             ("return_time", False), ("return_meta", False), ("allow_fallback", False)],
    "prepare_sddmm_csr": [("indices", E), ("indptr", E), ("shape", E), ("k_hint", 64)],
    # spmv_bsr.py:895-912, :510-522
    "flagsparse_spmv_bsr": [("data", None), ("indices", None), ("indptr", None), ("x", None), ("shape", None),
                            ("block_dim", None), ("block_nnz", 128), ("max_segments", None), ("out", None),
                            ("return_time", False), ("return_meta", False), ("prepared", None), ("transpose", None),
                            ("op", None), ("use_opt", False), ("index_fallback_policy", "auto")],
    "prepare_spmv_bsr": [("data", E), ("indices", E), ("indptr", E), ("shape", E), ("block_dim", E),
                         ("block_nnz", 128), ("max_segments", None), ("transpose", False), ("op", None),
                         ("use_opt", False), ("index_fallback_policy", "auto")],
    # spmv_csr.py:987-995, :1020-1033
    "prepare_spmv_coo_tocsr": [("data", E), ("row", E), ("col", E), ("shape", E), ("block_nnz", 256),
                               ("max_segments", None), ("assume_sorted", False)],
    "flagsparse_spmv_coo_tocsr": [("data", None), ("row", None), ("col", None), ("x", None), ("shape", None),
                                  ("block_nnz", 256), ("max_segments", None), ("out", None), ("return_time", False),
                                  ("use_opt", True), ("prepared", None), ("assume_sorted", False)],
}
OPT = [("data", None), ("indices", None), ("indptr", None), ("B", None), ("shape", None), ("prepared", None),
       ("out", None), ("return_time", False), ("return_meta", False)]
for _n in ("flagsparse_spmm_csr_opt", "flagsparse_spmm_csr_opt_alg1", "flagsparse_spmm_csr_opt_alg1_preprocess",
           "flagsparse_spmm_csr_opt_alg2", "flagsparse_spmm_csr_opt_alg2_preprocess"):
    SIGNATURES[_n] = OPT
for _n in ("prepare_spmm_csr_opt", "prepare_spmm_csr_opt_alg1", "prepare_spmm_csr_opt_alg1_preprocess",
           "prepare_spmm_csr_opt_alg2", "prepare_spmm_csr_opt_alg2_preprocess"):
    SIGNATURES[_n] = [("data", E), ("indices", E), ("indptr", E), ("shape", E)]


@pytest.mark.parametrize("name", sorted(SIGNATURES))
def test_public_signatures_match_reference(name):
    assert _params(getattr(fs, name)) == SIGNATURES[name]


def test_route_table_matches_reference():
    real_cplx = (torch.float32, torch.float64, torch.complex64, torch.complex128)
    expected = {
        "csr_base": "Base", "csr_base_accuracy": "BaseAccuracy", "alpha_alg1_tle_opt": "TLEOpt",
        "alpha_alg1_tle_opt2": "TLEOpt2", "spmm_csr_alg1": "Alg1", "spmm_csr_alg2": "Alg2",
        "spmm_csr_alg2_accuracy": "Alg2Accuracy", "spmm_csr_alg2_accuracy_hp": "Alg2AccuracyHP",
    }
    assert list(sm.SPMM_CSR_ALGORITHMS) == list(expected)
    for name, algo in sm.SPMM_CSR_ALGORITHMS.items():
        assert algo.name == name and algo.display_name == expected[name]
        assert algo.supported_ops == ("non", "trans", "conj")
        assert algo.supported_dtypes == (sm.SUPPORTED_SPMM_VALUE_DTYPES if name == "csr_base" else real_cplx)
    assert fs.list_spmm_csr_algorithms(dtype=torch.float16) == ("csr_base",)
    for alias, name in (("base", "csr_base"), ("alg1", "spmm_csr_alg1"), ("csr_alg2_accuracy_hp",
                                                                            "spmm_csr_alg2_accuracy_hp")):
        assert fs.resolve_spmm_csr_algorithm(alias, 0, torch.float32).name == name
    assert fs.resolve_spmm_csr_algorithm("auto", "trans", torch.float32).name == "csr_base"


@pytest.mark.parametrize("norm", [vm._normalize_spmv_op, sm._normalize_spmm_op])
def test_op_normalisation(norm):
    assert [norm(v) for v in (None, 0, 1, 2, "non", " TRANS ", "conj")] == [0, 0, 1, 2, 0, 1, 2]
    assert norm(None, transpose=True) == 1
    for bad in (3, "x", 1.5j, object()):
        with pytest.raises(ValueError, match="op must be one of: 0=non, 1=trans, 2=conj"):
            norm(bad)


def test_dense_layout_and_tolerance_helpers():
    assert sm._normalize_dense_layout("auto") == "row" and sm._normalize_dense_layout("F") == "col"
    with pytest.raises(ValueError, match="dense_layout must be one of"):
        sm._normalize_dense_layout("diag")
    assert sm._spmm_relative_threshold(torch.bfloat16) == 1e-2
    assert sm._spmm_relative_threshold(torch.complex128) == 1e-12
    a = torch.tensor([[1.0, 2.0], [3.0, 4.0]])
    m = sm._spmm_validation_metrics(a + 1e-3, a)
    assert m["max_abs_error"] == pytest.approx(1e-3, rel=1e-3) and m["matches_threshold"] is False
    assert sm._spmm_error_metrics(a[:0], a[:0])["max_relative_error"] == 0.0


def test_alg1_launch_configuration_rules():
    assert sm._select_spmm_alg1_warp_and_factor(128) == (32, 4)
    assert sm._select_spmm_alg1_warp_and_factor(7) == (8, 1)
    cfg = sm._resolve_spmm_alg1_launch_config(64, 1000)
    assert (cfg["block_n"], cfg["block_nnz"], cfg["required_segments"]) == (64, 32, 32)
    with pytest.raises(ValueError, match="requires more CSR segments"):
        sm._resolve_spmm_alg1_launch_config(64, 1000, max_segments=3)
    assert dm._resolve_sddmm_launch_config(128) == (64, 4) and dm._resolve_sddmm_launch_config(200) == (128, 8)


def test_sddmm_variant_names():
    assert dm._normalize_sddmm_diagnostic_variant(None) == "baseline"
    with pytest.raises(ValueError, match="Unsupported SDDMM diagnostic variant"):
        dm._normalize_sddmm_diagnostic_variant("fast")
