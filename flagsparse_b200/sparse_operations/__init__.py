"""CSR SpMV / SpMM / SDDMM operators on the sm_100a native library.

Mirrors the CSR hot-path part of FlagSparse ``sparse_operations/__init__.py``
(``:18-137``, ``:149-268``): the same names, imported eagerly, plus the
differentiable SpMM of ``autograd`` and the tensor-core BSR-16 SpMM of
``bsr_spmm`` and the batched graph launch of ``batched`` (none has a
FlagSparse counterpart).
"""

from ._common import SUPPORTED_INDEX_DTYPES, SUPPORTED_VALUE_DTYPES
from .autograd import (
    CsrSpmmFunction,
    PreparedCsrSpmmAutograd,
    flagsparse_spmm_csr_autograd,
    prepare_spmm_csr_autograd,
)
from .batched import BatchedCsr
from .bsr_spmm import PreparedBsr16, flagsparse_spmm_bsr16, prepare_spmm_bsr16
from .sddmm_csr import SDDMMPrepared, flagsparse_sddmm_csr, prepare_sddmm_csr
from .spmm_csr import (
    SPMM_CSR_ALGORITHMS,
    PreparedCsrSpmmOpt,
    PreparedCsrSpmmRoute,
    SpmmCsrAlgorithm,
    SpmmCsrAlgorithmUnavailable,
    flagsparse_spmm_csr,
    flagsparse_spmm_csr_opt,
    flagsparse_spmm_csr_opt_alg1,
    flagsparse_spmm_csr_opt_alg1_preprocess,
    flagsparse_spmm_csr_run,
    list_spmm_csr_algorithms,
    prepare_spmm_csr_opt,
    prepare_spmm_csr_opt_alg1,
    prepare_spmm_csr_opt_alg1_preprocess,
    prepare_spmm_csr_route,
    resolve_spmm_csr_algorithm,
)
from .spmm_csr_opt_alg2 import (
    PreparedCsrSpmmOptAlg2,
    flagsparse_spmm_csr_opt_alg2,
    flagsparse_spmm_csr_opt_alg2_preprocess,
    prepare_spmm_csr_opt_alg2,
    prepare_spmm_csr_opt_alg2_preprocess,
)
from .spmv_bsr import PreparedBsrSpmv, flagsparse_spmv_bsr, prepare_spmv_bsr
from .spmv_csr import (
    PreparedCsrSpmv,
    flagsparse_spmv_coo_tocsr,
    flagsparse_spmv_csr,
    prepare_spmv_coo_tocsr,
    prepare_spmv_csr,
)

__all__ = [
    "SUPPORTED_INDEX_DTYPES",
    "SUPPORTED_VALUE_DTYPES",
    "SPMM_CSR_ALGORITHMS",
    "BatchedCsr",
    "CsrSpmmFunction",
    "PreparedBsr16",
    "PreparedCsrSpmmAutograd",
    "PreparedCsrSpmmOpt",
    "PreparedCsrSpmmOptAlg2",
    "PreparedCsrSpmmRoute",
    "PreparedBsrSpmv",
    "PreparedCsrSpmv",
    "SDDMMPrepared",
    "SpmmCsrAlgorithm",
    "SpmmCsrAlgorithmUnavailable",
    "flagsparse_sddmm_csr",
    "flagsparse_spmm_bsr16",
    "flagsparse_spmm_csr",
    "flagsparse_spmm_csr_autograd",
    "flagsparse_spmm_csr_opt",
    "flagsparse_spmm_csr_opt_alg1",
    "flagsparse_spmm_csr_opt_alg1_preprocess",
    "flagsparse_spmm_csr_opt_alg2",
    "flagsparse_spmm_csr_opt_alg2_preprocess",
    "flagsparse_spmm_csr_run",
    "flagsparse_spmv_bsr",
    "flagsparse_spmv_coo_tocsr",
    "flagsparse_spmv_csr",
    "list_spmm_csr_algorithms",
    "prepare_sddmm_csr",
    "prepare_spmm_bsr16",
    "prepare_spmm_csr_autograd",
    "prepare_spmm_csr_opt",
    "prepare_spmm_csr_opt_alg1",
    "prepare_spmm_csr_opt_alg1_preprocess",
    "prepare_spmm_csr_opt_alg2",
    "prepare_spmm_csr_opt_alg2_preprocess",
    "prepare_spmm_csr_route",
    "prepare_spmv_bsr",
    "prepare_spmv_coo_tocsr",
    "prepare_spmv_csr",
    "resolve_spmm_csr_algorithm",
]
