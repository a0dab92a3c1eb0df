"""flagsparse_b200: a B200 (sm_100a) drop-in for FlagSparse's CSR hot path.

Same public names and lazy export map as FlagSparse ``__init__.py``
(``__all__`` ``:19-154``, ``_OPS_EXPORTS`` ``:156-272``, ``__getattr__``
``:297-306``), restricted to the CSR SpMV / SpMM / SDDMM operators (with the COO-to-CSR
SpMV on-ramp and the BSR SpMV) this package implements.  ``import flagsparse_b200 as flagsparse`` is the switch.
"""

__version__ = "1.0.0"

_OPS_EXPORTS = {
    "PreparedCsrSpmv",
    "PreparedCsrSpmmOpt",
    "PreparedCsrSpmmOptAlg2",
    "PreparedCsrSpmmRoute",
    "SDDMMPrepared",
    "SpmmCsrAlgorithm",
    "SpmmCsrAlgorithmUnavailable",
    "prepare_spmv_csr",
    "prepare_spmv_coo_tocsr",
    "prepare_spmv_bsr",
    "prepare_spmm_csr_route",
    "prepare_spmm_csr_opt",
    "prepare_spmm_csr_opt_alg1",
    "prepare_spmm_csr_opt_alg1_preprocess",
    "prepare_spmm_csr_opt_alg2",
    "prepare_spmm_csr_opt_alg2_preprocess",
    "prepare_sddmm_csr",
    "flagsparse_spmv_csr",
    "flagsparse_spmv_coo_tocsr",
    "flagsparse_spmv_bsr",
    "flagsparse_spmm_csr",
    "flagsparse_spmm_csr_run",
    "flagsparse_spmm_csr_opt",
    "flagsparse_spmm_csr_opt_alg1",
    "flagsparse_spmm_csr_opt_alg1_preprocess",
    "flagsparse_spmm_csr_opt_alg2",
    "flagsparse_spmm_csr_opt_alg2_preprocess",
    "flagsparse_sddmm_csr",
    "list_spmm_csr_algorithms",
    "resolve_spmm_csr_algorithm",
    # batched uneven matrices in one graph launch (no FlagSparse counterpart)
    "BatchedCsr",
    # BSR-16 SpMM on the tensor cores (no FlagSparse counterpart)
    "PreparedBsr16",
    "prepare_spmm_bsr16",
    "flagsparse_spmm_bsr16",
    # differentiable SpMM (no FlagSparse counterpart)
    "CsrSpmmFunction",
    "PreparedCsrSpmmAutograd",
    "prepare_spmm_csr_autograd",
    "flagsparse_spmm_csr_autograd",
}

__all__ = sorted(_OPS_EXPORTS)


def __getattr__(name):
    if name in _OPS_EXPORTS:
        from . import sparse_operations as _ops

        return getattr(_ops, name)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")


def __dir__():
    return sorted(set(globals()) | _OPS_EXPORTS)
