"""ctypes binding of the sm_100a C ABI (``include/flagsparse_b200.h``).

The host mirror of the FlagSparse operators calls the native library only
through this module.  There is no fallback: if the shared library is missing
or a call returns a non-zero status, a ``RuntimeError`` is raised.
"""

import ctypes
import os
import threading

import torch

_PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG_DIR, "_lib", "libflagsparse_b200.so")

FSB_OK = 0
FSB_ERR_INVALID_ARG = -1
FSB_ERR_UNSUPPORTED = -2
FSB_ERR_LAUNCH = -3
FSB_ERR_TIMEOUT = -4
FSB_ERR_CUDA = -5
FSB_ERR_WORKSPACE = -6
FSB_ERR_TOO_LARGE = -7

DTYPE_CODE = {
    torch.float16: 0,
    torch.bfloat16: 1,
    torch.float32: 2,
    torch.float64: 3,
    torch.complex64: 4,
    torch.complex128: 5,
}

_c_i32 = ctypes.c_int32
_c_i64 = ctypes.c_int64
_c_int = ctypes.c_int
_c_ptr = ctypes.c_void_p
_c_i64p = ctypes.POINTER(ctypes.c_int64)


class SpmvPlan(ctypes.Structure):
    """Mirror of ``fsb_spmv_plan``."""

    _fields_ = [
        ("seg_row0", _c_ptr),
        ("seg_unit0", _c_ptr),
        ("units", _c_ptr),
        ("n_segs", _c_i64),
        ("n_units", _c_i64),
        ("n_slots", _c_i64),
        ("n_block_units", _c_i64),
        ("cap", _c_i32),
        ("chunk_nnz", _c_i32),
        ("partials", _c_ptr),
        ("counters", _c_ptr),
        ("flags", _c_i32),
        ("tile_bytes", _c_i32),
    ]


FSB_SPMV_FAST_SHORT_ROWS = 1
FSB_SPMV_STATIC_MAX_SLOTS = 65536
FSB_SPMM_COMPENSATED = 2
FSB_SPMM_PERSISTENT = 4
FSB_SDDMM_ACC64 = 1
FSB_SDDMM_OUT64 = 2


# name -> (restype, argtypes)
_SIGNATURES = {
    "fsb_version": (_c_int, []),
    "fsb_status_string": (ctypes.c_char_p, [_c_int]),
    "fsb_csr_inspect": (_c_int, [_c_ptr, _c_int, _c_ptr, _c_int, _c_i64, _c_i64, _c_ptr, _c_ptr]),
    "fsb_csr_bucketize_workspace_bytes": (_c_i64, [_c_i64, _c_int]),
    "fsb_csr_bucketize": (
        _c_int,
        [_c_ptr, _c_int, _c_i64, _c_i64p, _c_int, _c_ptr, _c_i64, _c_ptr, _c_ptr, _c_ptr],
    ),
    "fsb_csr_transpose_workspace_bytes": (_c_i64, [_c_i64, _c_i64, _c_i64]),
    "fsb_csr_transpose": (
        _c_int,
        [_c_ptr, _c_int, _c_ptr, _c_int, _c_i64, _c_i64, _c_i64, _c_ptr, _c_i64,
         _c_ptr, _c_int, _c_ptr, _c_int, _c_ptr, _c_ptr],
    ),
    "fsb_gather_values": (_c_int, [_c_int, _c_ptr, _c_ptr, _c_i64, _c_int, _c_ptr, _c_ptr]),
    "fsb_bsr_spmv": (
        _c_int, [_c_int, _c_ptr, _c_ptr, _c_int, _c_ptr, _c_int, _c_i64, _c_i64, _c_int, _c_ptr, _c_ptr, _c_ptr]
    ),
    "fsb_bsr_transpose_values": (_c_int, [_c_int, _c_ptr, _c_ptr, _c_i64, _c_int, _c_int, _c_ptr, _c_ptr]),
    "fsb_coo_inspect": (_c_int, [_c_ptr, _c_int, _c_ptr, _c_int, _c_i64, _c_i64, _c_i64, _c_ptr, _c_ptr]),
    "fsb_coo_to_csr_workspace_bytes": (_c_i64, [_c_i64, _c_i64, _c_i64]),
    "fsb_coo_to_csr": (
        _c_int,
        [_c_ptr, _c_int, _c_ptr, _c_int, _c_i64, _c_i64, _c_i64, _c_int, _c_ptr, _c_i64, _c_ptr, _c_ptr, _c_ptr,
         _c_ptr],
    ),
    "fsb_spmv_default_cap": (_c_i32, [_c_int]),
    "fsb_spmv_default_chunk": (_c_i32, [_c_int]),
    "fsb_spmv_partial_bytes": (_c_i64, [_c_int]),
    "fsb_spmv_plan_workspace_bytes": (_c_i64, [_c_i64]),
    "fsb_spmv_plan_analyze": (
        _c_int, [_c_ptr, _c_int, _c_i64, _c_i32, _c_i32, _c_ptr, _c_i64, _c_ptr, _c_ptr]
    ),
    "fsb_spmv_plan_build": (
        _c_int,
        [_c_ptr, _c_int, _c_i64, _c_i32, _c_i32, _c_ptr, _c_i64, _c_ptr, _c_ptr, _c_ptr, _c_ptr],
    ),
    "fsb_spmv_csr": (
        _c_int,
        [_c_int, _c_ptr, _c_ptr, _c_int, _c_ptr, _c_int, _c_i64, _c_i64, _c_ptr, _c_ptr,
         ctypes.POINTER(SpmvPlan), _c_ptr],
    ),
    "fsb_spmm_default_cap": (_c_i32, [_c_int]),
    "fsb_spmm_default_chunk": (_c_i32, [_c_int]),
    "fsb_spmm_scratch_layout": (_c_int, [_c_int, _c_i64, _c_i64p, _c_i64p]),
    "fsb_spmm_csr": (
        _c_int,
        [_c_int, _c_ptr, _c_ptr, _c_ptr, _c_i64, _c_i64, _c_ptr, _c_i64, _c_i64, _c_ptr, _c_i64,
         ctypes.POINTER(SpmvPlan), _c_ptr],
    ),
    "fsb_spmm_spmv_csr": (
        _c_int,
        [_c_int, _c_ptr, _c_ptr, _c_ptr, _c_i64, _c_i64, _c_ptr, _c_i64, _c_i64, _c_ptr, _c_i64, _c_ptr, _c_ptr,
         ctypes.POINTER(SpmvPlan), _c_ptr],
    ),
    "fsb_spmm_csr_backward": (
        _c_int,
        [_c_int, _c_ptr, _c_ptr, _c_ptr, _c_ptr, _c_i64, _c_i64, _c_ptr, _c_i64, _c_ptr, _c_i64, _c_i64, _c_ptr,
         _c_i64, _c_ptr, ctypes.POINTER(SpmvPlan), _c_ptr],
    ),
    "fsb_csr_row_ids":(_c_int, [_c_ptr, _c_int, _c_i64, _c_i64, _c_ptr, _c_ptr]),
    "fsb_sddmm_csr": (
        _c_int,
        [_c_int, _c_ptr, _c_ptr, _c_i64, _c_ptr, _c_i64, _c_ptr, _c_i64, _c_i64, _c_ptr,
         ctypes.c_double, ctypes.c_double, _c_ptr, _c_int, _c_ptr],
    ),
    "fsb_bsr16_pack": (_c_int, [_c_int, _c_ptr, _c_i64, _c_ptr, _c_ptr]),
    "fsb_bsr16_spmm": (
        _c_int,
        [_c_int, _c_ptr, _c_ptr, _c_ptr, _c_i64, _c_i64, _c_ptr, _c_i64, _c_i64, _c_ptr, _c_i64, _c_ptr, _c_ptr],
    ),
    "fsb_spmv_gather_floor": (
        _c_int, [_c_int, _c_ptr, _c_ptr, _c_int, _c_i64, _c_ptr, _c_ptr, _c_i64, _c_ptr],
    ),
    "fsb_spmm_gather_floor_tma": (
        _c_int, [_c_int, _c_ptr, _c_ptr, _c_i64, _c_ptr, _c_i64, _c_i64, _c_i64, _c_ptr, _c_i64, _c_ptr, _c_ptr],
    ),
    "fsb_spmv_csr_static_scratch": (
        _c_int,
        [_c_int, _c_ptr, _c_ptr, _c_int, _c_ptr, _c_int, _c_i64, _c_i64, _c_ptr, _c_ptr,
         ctypes.POINTER(SpmvPlan), _c_ptr],
    ),
}

_lib = None
_lock = threading.Lock()


def exported_symbols():
    """Names this binding expects the library to export."""
    return sorted(_SIGNATURES)


def lib():
    """Load the native library once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"flagsparse_b200 native library not found at {LIB_PATH}; "
                    "build it with `python -m flagsparse_b200._build`"
                )
            handle = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in _SIGNATURES.items():
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            _lib = handle
    return _lib


def status_text(status):
    return lib().fsb_status_string(int(status)).decode()


def check(status, what):
    if status != FSB_OK:
        raise RuntimeError(f"{what} failed: {status_text(status)} (status {status})")


def ptr(t):
    """Device (or host) address of a tensor, or NULL for None / empty."""
    if t is None:
        return None
    return t.data_ptr() or None


def stream_of(device):
    return torch.cuda.current_stream(device).cuda_stream


def dtype_code(dtype):
    code = DTYPE_CODE.get(dtype)
    if code is None:
        raise TypeError(f"unsupported value dtype {dtype}")
    return code


def is64(t):
    return 1 if t.dtype == torch.int64 else 0
