"""Matrix Market (.mtx) files to CSR tensors through the native parser.

``load_mtx_to_csr`` mirrors FlagSparse's ``load_mtx_to_csr_torch``
(tests/test_spmv.py:103-178): same arguments, same result
``(data, indices, indptr, shape)`` with int64 indices and row offsets, same
handling of pattern, symmetric, hermitian and skew-symmetric files,
duplicates and out-of-range entries.  The parse runs in C++ on the host's
threads (``fsb_mtx_open``); values are summed in float64 and rounded to
``dtype`` once, as FlagSparse's are.
"""

import ctypes
import os

import torch

from . import _native as nat


def load_mtx_to_csr(file_path, dtype=torch.float32, device=None, threads=0):
    """(data, indices, indptr, (n_rows, n_cols)) of a .mtx file on ``device``
    (default: CUDA when available)."""
    if device is None:
        device = torch.device("cuda" if torch.cuda.is_available() else "cpu")
    lib = nat.library()
    n_rows, n_cols, nnz = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
    handle = lib.fsb_mtx_open(os.fsencode(str(file_path)), ctypes.byref(n_rows), ctypes.byref(n_cols),
                              ctypes.byref(nnz), int(threads))
    if not handle:
        msg = lib.fsb_last_error().decode()
        raise ValueError(msg)
    try:
        indptr = torch.empty(n_rows.value + 1, dtype=torch.int64)
        indices = torch.empty(nnz.value, dtype=torch.int64)
        values = torch.empty(nnz.value, dtype=torch.float64)
        rc = lib.fsb_mtx_read(handle, indptr.data_ptr(), indices.data_ptr() if nnz.value else None,
                              values.data_ptr() if nnz.value else None)
        nat.check(rc, "fsb_mtx_read")
    finally:
        lib.fsb_mtx_close(handle)
    data = values.to(dtype)
    return data.to(device), indices.to(device), indptr.to(device), (n_rows.value, n_cols.value)
