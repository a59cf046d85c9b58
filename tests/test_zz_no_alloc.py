"""fsb_spmv_csr_noalloc: the allocation-free merge-path SpMV entry point.

Some callers cannot allocate device memory: a C program or plug-in that is
handed device pointers by a host framework which owns all device memory, or a
latency-critical loop in which cudaMalloc's implicit device-wide
synchronisation is unacceptable.  For them the library keeps the merge-path
scratch (tile coordinates and per-tile carries) in a fixed device array, so
the caller passes only the matrix, x and y.

The test calls the entry point through the C ABI twice in a row, with
different inputs, and compares each result with the existing merge-path
entry point (fsb_spmv_csr, scratch passed in by the caller), within the float32
bound used by the other parity tests.  It also checks that sizes beyond the
fixed scratch are rejected.  This file is collected last.
"""

import ctypes

import pytest
import torch

from flagsparse_public_b200 import _native as nat
from flagsparse_public_b200 import _plan
from tests.gpu_cases import EDGE_LENGTHS, csr_from_lengths, dense
from tests.numerics import scaled_error

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")
ITEMS = 512


def _reference_spmv(d_data, d_idx, d_ptr, n_rows, n_cols, d_x, acc):
    y = torch.empty(n_rows, dtype=d_data.dtype, device=DEV)
    _plan.run_spmv(d_data, d_idx, d_ptr, n_rows, n_cols, d_x, y, acc,
                   _plan.KernelPlan(nat.ALGO_MERGE, items_per_unit=ITEMS))
    return y


def _noalloc_spmv(d_data, d_idx, d_ptr, n_rows, n_cols, d_x, acc):
    y = torch.full((n_rows,), float("nan"), dtype=d_data.dtype, device=DEV)
    m = nat.make_csr(d_data, d_idx, d_ptr, n_rows, n_cols)
    rc = nat.library().fsb_spmv_csr_noalloc(m, nat.ptr(d_x), nat.ptr(y), nat.dtype_code(y.dtype), acc, ITEMS,
                                            nat.stream_handle(DEV))
    nat.check(rc, "fsb_spmv_csr_noalloc")
    return y


@pytest.mark.parametrize("acc", [nat.ACC_WIDE, nat.ACC_NATIVE], ids=["wide", "native"])
def test_noalloc_matches_merge_path_on_two_calls(acc):
    # first call: skewed rows with empty rows and long rows crossing tiles
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths(EDGE_LENGTHS["skewed"], 20000, seed=41)
    d = (data.to(DEV), indices.to(DEV), indptr.to(DEV))
    x = dense((n_cols,), 42, torch.float32).to(DEV)
    ref = _reference_spmv(*d, n_rows, n_cols, x, acc)
    got = _noalloc_spmv(*d, n_rows, n_cols, x, acc)
    mag = (torch.zeros(n_rows, dtype=torch.float64).index_add_(
        0, torch.repeat_interleave(torch.arange(n_rows), indptr[1:] - indptr[:-1]),
        (data.double() * x.cpu().double()[indices.long()]).abs()))
    assert scaled_error(got, ref.cpu().double(), mag) <= 1e-5

    # second call, different matrix and vector: no state may leak between calls
    data2, indices2, indptr2, (n_rows2, n_cols2) = csr_from_lengths(EDGE_LENGTHS["long_rows"] * 3, 13000, seed=43)
    d2 = (data2.to(DEV), indices2.to(DEV), indptr2.to(DEV))
    x2 = dense((n_cols2,), 44, torch.float32).to(DEV)
    ref2 = _reference_spmv(*d2, n_rows2, n_cols2, x2, acc)
    got2 = _noalloc_spmv(*d2, n_rows2, n_cols2, x2, acc)
    mag2 = (torch.zeros(n_rows2, dtype=torch.float64).index_add_(
        0, torch.repeat_interleave(torch.arange(n_rows2), indptr2[1:] - indptr2[:-1]),
        (data2.double() * x2.cpu().double()[indices2.long()]).abs()))
    assert scaled_error(got2, ref2.cpu().double(), mag2) <= 1e-5


def test_noalloc_rejects_sizes_beyond_fixed_scratch():
    lib = nat.library()
    m = nat.FsbCsr()
    m.value_dtype, m.index_dtype, m.ptr_dtype, m.row_map_dtype = nat.FSB_F32, nat.FSB_I32, nat.FSB_I64, nat.FSB_I32
    m.n_rows, m.n_cols, m.nnz = 1_000_000, 1_000_000, 16_000_000  # 16.5 M path items > 16384 tiles x 512
    m.values = m.col_idx = m.row_ptr = 1  # never dereferenced: rejected before any launch
    rc = lib.fsb_spmv_csr_noalloc(m, ctypes.c_void_p(1), ctypes.c_void_p(1), nat.FSB_F32, nat.ACC_NATIVE, ITEMS,
                                  nat.stream_handle(DEV))
    assert rc == nat.FSB_ERR_LIMIT
    assert b"exceed the fixed scratch" in lib.fsb_last_error()
