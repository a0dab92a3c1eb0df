"""CSR SpMV / SpMM / SDDMM operators on the sm_100a native library.

Mirrors the hot-path part of FlagSparse ``sparse_operations/__init__.py``
(``:18-137``, ``:149-268``): the same names, imported eagerly.
"""

from ._common import SUPPORTED_INDEX_DTYPES, SUPPORTED_VALUE_DTYPES
from .spmv_csr import (
    PreparedCsrSpmv,
    flagsparse_spmv_csr,
    prepare_spmv_csr,
)

__all__ = [
    "SUPPORTED_INDEX_DTYPES",
    "SUPPORTED_VALUE_DTYPES",
    "PreparedCsrSpmv",
    "flagsparse_spmv_csr",
    "prepare_spmv_csr",
]
