"""Shared dtype tables, tolerances and helpers of the SpMV/SpMM operators.

Mirrors the parts of FlagSparse's ``sparse_operations/_common.py`` that the
CSR/COO SpMV and SpMM operators use (dtype tables ``_common.py:25-36``,
tolerances ``:123-134``, random CSR builder ``:223-238``, timing helper
``:353-371``).  The CuPy interop of the reference is not part of this path.
"""

import time

import torch

_TORCH_COMPLEX32_DTYPE = getattr(torch, "complex32", None)
if _TORCH_COMPLEX32_DTYPE is None:
    _TORCH_COMPLEX32_DTYPE = getattr(torch, "chalf", None)

_SUPPORTED_VALUE_DTYPES = [torch.float16, torch.bfloat16, torch.float32, torch.float64]
if _TORCH_COMPLEX32_DTYPE is not None:
    _SUPPORTED_VALUE_DTYPES.append(_TORCH_COMPLEX32_DTYPE)
_SUPPORTED_VALUE_DTYPES.extend([torch.complex64, torch.complex128])
SUPPORTED_VALUE_DTYPES = tuple(_SUPPORTED_VALUE_DTYPES)
SUPPORTED_INDEX_DTYPES = (torch.int32, torch.int64)
_INDEX_LIMIT_INT32 = 2**31 - 1

__all__ = (
    "SUPPORTED_VALUE_DTYPES",
    "SUPPORTED_INDEX_DTYPES",
    "_INDEX_LIMIT_INT32",
    "_torch_complex32_dtype",
    "_is_complex32_dtype",
    "_is_complex_dtype",
    "_component_dtype_for_complex",
    "_tolerance_for_dtype",
    "_build_random_dense",
    "_build_random_csr",
    "_benchmark_cuda_op",
    "time",
    "torch",
)


def _torch_complex32_dtype():
    return _TORCH_COMPLEX32_DTYPE


def _is_complex32_dtype(value_dtype):
    return _TORCH_COMPLEX32_DTYPE is not None and value_dtype == _TORCH_COMPLEX32_DTYPE


def _is_complex_dtype(value_dtype):
    return _is_complex32_dtype(value_dtype) or value_dtype in (torch.complex64, torch.complex128)


def _component_dtype_for_complex(value_dtype):
    if _is_complex32_dtype(value_dtype):
        return torch.float16
    if value_dtype == torch.complex64:
        return torch.float32
    if value_dtype == torch.complex128:
        return torch.float64
    raise TypeError(f"Unsupported complex dtype: {value_dtype}")


def _tolerance_for_dtype(value_dtype):
    """(atol, rtol) per value dtype, as FlagSparse ``_common.py:123-134``."""
    if value_dtype == torch.float16:
        return 2e-3, 2e-3
    if _is_complex32_dtype(value_dtype):
        return 5e-3, 5e-3
    if value_dtype == torch.bfloat16:
        return 1e-1, 1e-1
    if value_dtype in (torch.float32, torch.complex64):
        return 1e-6, 1e-5
    if value_dtype in (torch.float64, torch.complex128):
        return 1e-10, 1e-8
    return 1e-6, 1e-5


def _build_random_dense(dense_size, value_dtype, device):
    if value_dtype in (torch.float16, torch.bfloat16, torch.float32, torch.float64):
        return torch.randn(dense_size, dtype=value_dtype, device=device)
    if _is_complex_dtype(value_dtype):
        comp = _component_dtype_for_complex(value_dtype)
        return torch.complex(torch.randn(dense_size, dtype=comp, device=device),
                             torch.randn(dense_size, dtype=comp, device=device))
    raise TypeError(f"Unsupported value dtype: {value_dtype}")


def _build_random_csr(n_rows, n_cols, nnz, value_dtype, index_dtype, device):
    """Random CSR with uniformly drawn row ids and columns (``_common.py:223-238``)."""
    if nnz <= 0 or n_rows <= 0 or n_cols <= 0:
        indptr = torch.zeros(n_rows + 1, dtype=torch.int64, device=device)
        return (torch.empty(0, dtype=value_dtype, device=device),
                torch.empty(0, dtype=index_dtype, device=device), indptr)
    row_choices, _ = torch.sort(torch.randint(0, n_rows, (nnz,), device=device))
    nnz_per_row = torch.bincount(row_choices, minlength=n_rows)
    indptr = torch.zeros(n_rows + 1, dtype=torch.int64, device=device)
    indptr[1:] = torch.cumsum(nnz_per_row, dim=0)
    indices = torch.randint(0, n_cols, (nnz,), dtype=index_dtype, device=device)
    data = _build_random_dense(nnz, value_dtype, device)
    return data, indices, indptr


def _benchmark_cuda_op(op, warmup, iters):
    """Wall-clock mean of ``iters`` calls after ``warmup`` (``_common.py:353-371``)."""
    warmup = max(0, int(warmup))
    iters = max(1, int(iters))
    output = None
    for _ in range(warmup):
        output = op()
    torch.cuda.synchronize()
    start_time = time.perf_counter()
    for _ in range(iters):
        output = op()
    torch.cuda.synchronize()
    elapsed_ms = (time.perf_counter() - start_time) * 1000.0 / iters
    return output, elapsed_ms


