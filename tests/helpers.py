"""Helpers shared by the GPU parity tests: device tensors from numpy, error bounds."""

import numpy as np
import torch

from oracle import oracle

TORCH_DT = {
    "float16": torch.float16,
    "bfloat16": torch.bfloat16,
    "float32": torch.float32,
    "float64": torch.float64,
    "complex64": torch.complex64,
    "complex128": torch.complex128,
}

# unit roundoff of the output dtype
UNIT = {
    "float16": 2.0**-11,
    "bfloat16": 2.0**-8,
    "float32": 2.0**-24,
    "complex64": 2.0**-24,
    "float64": 2.0**-53,
    "complex128": 2.0**-53,
}
# half the smallest subnormal of the output dtype: the absolute error that
# rounding a result into the subnormal range can add (Higham, sec. 2.1)
ETA = {
    "float16": 2.0**-25,
    "bfloat16": 2.0**-134,
    "float32": 2.0**-150,
    "complex64": 2.0**-150,
    "float64": 0.0,
    "complex128": 0.0,
}
# unit roundoff of the accumulation type
ACC_UNIT = {
    "float16": 2.0**-24,
    "bfloat16": 2.0**-24,
    "float32": 2.0**-24,
    "complex64": 2.0**-24,
    "float64": 2.0**-53,
    "complex128": 2.0**-53,
}


def dev(a, dtype=None, device="cuda"):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.to(device)


def host(t):
    t = t.detach().cpu()
    if t.dtype in (torch.float16, torch.bfloat16):
        t = t.to(torch.float32)
    return t.numpy()


def rounded(values, dname):
    """numpy float64/complex128 copy of `values` after rounding to dtype `dname`."""
    t = torch.from_numpy(np.ascontiguousarray(values)).to(TORCH_DT[dname])
    if t.dtype.is_complex:
        return t.to(torch.complex128).numpy()
    return t.to(torch.float64).numpy()


def spmv_error_bound(dname, ref, scale, row_len):
    """Bound for the native (compensated) SpMV against the exact result.

    A compensated dot product of n terms obeys
    |y - exact| <= u_acc |exact| + gamma_n^2 S, gamma_n = n u_acc / (1 - n u_acc),
    S = sum |a||x| (Ogita, Rump, Oishi 2005, Prop. 4.5).  Rounding to the
    output type adds u_out |exact|; complex products count four terms each.
    """
    u, ua = UNIT[dname], ACC_UNIT[dname]
    n = 4.0 * np.maximum(np.asarray(row_len, dtype=np.float64), 1.0) + 8.0
    gamma = n * ua / (1.0 - n * ua)
    return (u + 2.0 * ua) * np.abs(ref) + gamma * gamma * scale + ETA[dname] + 1e-300


def assert_spmv_close(y, ref, scale, row_len, dname, what=""):
    y = np.asarray(y)
    bound = spmv_error_bound(dname, ref, scale, row_len)
    if np.iscomplexobj(ref):
        err = np.maximum(np.abs(y.real - ref.real), np.abs(y.imag - ref.imag))
        bound = spmv_error_bound(dname, np.maximum(np.abs(ref.real), np.abs(ref.imag)), scale, row_len)
    else:
        err = np.abs(y - ref)
    bad = np.nonzero(err > bound)[0]
    assert bad.size == 0, f"{what}: {bad.size} rows out of bound, first {bad[:5]}, err {err[bad[:5]]}, bound {bound[bad[:5]]}"


def op_csr(indptr, indices, data, shape, op):
    if op == "non":
        return indptr, indices, data, shape
    t_ptr, t_idx, perm = oracle.transpose(indptr, indices, shape[1])
    d = np.asarray(data)[perm]
    if op == "conj":
        d = np.conj(d)
    return t_ptr, t_idx, d, (shape[1], shape[0])


def plain_error_bound(dname, ref, scale, n_terms):
    """Bound for a working-precision sum of n products against the exact result:
    |c - exact| <= u_out |exact| + gamma_n S, gamma_n = n u_acc / (1 - n u_acc),
    S = sum |a||b| (Higham, Accuracy and Stability, eq. 3.5); complex products
    count four terms."""
    u, ua = UNIT[dname], ACC_UNIT[dname]
    n = np.maximum(np.asarray(n_terms, dtype=np.float64), 1.0)
    if dname.startswith("complex"):
        n = 4.0 * n
    n = n + 2.0
    gamma = n * ua / (1.0 - n * ua)
    return 2.0 * u * np.abs(ref) + gamma * scale + ETA[dname] + 1e-300


def assert_within(got, ref, bound, what=""):
    got = np.asarray(got)
    if np.iscomplexobj(ref) or np.iscomplexobj(got):
        err = np.maximum(np.abs(np.real(got) - np.real(ref)), np.abs(np.imag(got) - np.imag(ref)))
    else:
        err = np.abs(got - ref)
    bad = np.argwhere(err > bound)
    assert bad.size == 0, (f"{what}: {len(bad)} entries out of bound, first {bad[:3].tolist()}, "
                           f"err {err[tuple(bad[:3].T)]}, bound {np.broadcast_to(bound, err.shape)[tuple(bad[:3].T)]}")
