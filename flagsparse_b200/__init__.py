"""flagsparse_b200: a B200 (sm_100a) drop-in for FlagSparse's CSR hot path.

Same public names and lazy export map as FlagSparse ``__init__.py``
(``__all__`` ``:19-154``, ``_OPS_EXPORTS`` ``:156-272``, ``__getattr__``
``:297-306``), restricted to the CSR SpMV / SpMM / SDDMM operators this
package implements.  ``import flagsparse_b200 as flagsparse`` is the switch.
"""

__version__ = "1.0.0"

_OPS_EXPORTS = {
    "PreparedCsrSpmv",
    "prepare_spmv_csr",
    "flagsparse_spmv_csr",
}

__all__ = sorted(_OPS_EXPORTS)


def __getattr__(name):
    if name in _OPS_EXPORTS:
        from . import sparse_operations as _ops

        return getattr(_ops, name)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")


def __dir__():
    return sorted(set(globals()) | _OPS_EXPORTS)
