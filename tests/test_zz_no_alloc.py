"""fsb_spmv_csr_noalloc: the allocation-free merge-path SpMV entry point.

Some callers cannot allocate device memory: a C program or plug-in that is
handed device pointers by a host framework which owns all device memory, or a
latency-critical loop in which cudaMalloc's implicit device-wide
synchronisation is unacceptable.  For them the library keeps the merge-path
scratch (tile coordinates and per-tile carries) in a fixed device array, so
the caller passes only the matrix, x and y.

The tests call the entry point through the C ABI twice in a row, with
different inputs, and require each result to equal, bit for bit, the existing
merge-path entry point (fsb_spmv_csr, scratch passed in by the caller) with
the same tile size -- both run the same partition, tile and carry kernels --
and to lie within the float32 / float64 bounds of the other parity tests of
the FP64 oracle.  One case fills the fixed array to its last tile with the
widest (16-byte) accumulator; sizes one path item beyond the array are
rejected.  This file is collected last.
"""

import ctypes

import pytest
import torch

from flagsparse_public_b200 import _native as nat
from flagsparse_public_b200 import _plan
from oracle import oracle as orc
from tests.gpu_cases import EDGE_LENGTHS, csr_from_lengths, dense
from tests.numerics import scaled_error

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")
MAX_TILES = 16384  # the fixed array's tile capacity (fsb_spmv.cu)


def _reference_spmv(d_data, d_idx, d_ptr, n_rows, n_cols, d_x, acc, items):
    y = torch.empty(n_rows, dtype=d_data.dtype, device=DEV)
    _plan.run_spmv(d_data, d_idx, d_ptr, n_rows, n_cols, d_x, y, acc,
                   _plan.KernelPlan(nat.ALGO_MERGE, items_per_unit=items))
    return y


def _noalloc_spmv(d_data, d_idx, d_ptr, n_rows, n_cols, d_x, acc, items):
    y = torch.full((n_rows,), float("nan"), dtype=d_data.dtype, device=DEV)
    m = nat.make_csr(d_data, d_idx, d_ptr, n_rows, n_cols)
    rc = nat.library().fsb_spmv_csr_noalloc(m, nat.ptr(d_x), nat.ptr(y), nat.dtype_code(y.dtype), acc, items,
                                            nat.stream_handle(DEV))
    nat.check(rc, "fsb_spmv_csr_noalloc")
    return y


def _check_case(data, indices, indptr, n_rows, n_cols, x, acc, items, bound):
    """The allocation-free result equals fsb_spmv_csr's bit for bit and is
    within ``bound`` of the FP64 oracle (condition-scaled)."""
    d = (data.to(DEV), indices.to(DEV), indptr.to(DEV))
    dx = x.to(DEV)
    ref = _reference_spmv(*d, n_rows, n_cols, dx, acc, items)
    got = _noalloc_spmv(*d, n_rows, n_cols, dx, acc, items)
    torch.cuda.synchronize()
    assert torch.equal(got, ref)
    exact, mag = orc.spmv_csr_exact(data, indices, indptr, x)
    assert scaled_error(got.cpu(), exact, mag) <= bound


@pytest.mark.parametrize("acc", [nat.ACC_WIDE, nat.ACC_NATIVE], ids=["wide", "native"])
def test_noalloc_matches_merge_path_on_two_calls(acc):
    items = 512
    bound = 1e-5 if acc == nat.ACC_WIDE else 3e-5
    # first call: skewed rows with empty rows and long rows crossing tiles
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths(EDGE_LENGTHS["skewed"], 20000, seed=41)
    _check_case(data, indices, indptr, n_rows, n_cols, dense((n_cols,), 42, torch.float32), acc, items, bound)
    # second call, different matrix and vector: no state may leak between calls
    data2, indices2, indptr2, (n_rows2, n_cols2) = csr_from_lengths(EDGE_LENGTHS["long_rows"] * 3, 13000, seed=43)
    _check_case(data2, indices2, indptr2, n_rows2, n_cols2, dense((n_cols2,), 44, torch.float32), acc, items, bound)


def _csr_with_items(n_rows, total_items, n_cols, seed, dtype):
    """CSR whose rows + nonzeros add up to exactly ``total_items``: uniform
    columns, row lengths spread evenly (the remainder on the first rows)."""
    nnz = total_items - n_rows
    base, extra = divmod(nnz, n_rows)
    lengths = torch.full((n_rows,), base, dtype=torch.int64)
    lengths[:extra] += 1
    g = torch.Generator().manual_seed(seed)
    indptr = torch.zeros(n_rows + 1, dtype=torch.int64)
    indptr[1:] = torch.cumsum(lengths, 0)
    rows = torch.repeat_interleave(torch.arange(n_rows), lengths)
    cols = torch.randint(0, n_cols, (nnz,), generator=g)
    key, _ = torch.sort(rows * n_cols + cols)  # duplicates allowed: CSR does not forbid them
    indices = (key % n_cols).to(torch.int32)
    if dtype.is_complex:
        data = torch.complex(torch.rand(nnz, generator=g, dtype=torch.float64) * 2 - 1,
                             torch.rand(nnz, generator=g, dtype=torch.float64) * 2 - 1).to(dtype)
    else:
        data = (torch.rand(nnz, generator=g, dtype=torch.float64) * 2 - 1).to(dtype)
    return data, indices, indptr


def test_noalloc_fills_the_fixed_scratch_to_its_last_tile():
    # exactly MAX_TILES tiles of 128 items with complex128 values: the 16-byte
    # accumulators of the carries occupy the whole array
    items = 128
    n_rows, n_cols = 65536, 50000
    data, indices, indptr = _csr_with_items(n_rows, MAX_TILES * items, n_cols, 45, torch.complex128)
    assert -(-(n_rows + data.numel()) // items) == MAX_TILES
    x = dense((n_cols,), 46, torch.complex128)
    for _ in range(2):  # two calls in a row on the full array
        _check_case(data, indices, indptr, n_rows, n_cols, x, nat.ACC_NATIVE, items, 1e-12)


def _limit_status(n_rows, nnz, items):
    lib = nat.library()
    m = nat.FsbCsr()
    m.value_dtype, m.index_dtype, m.ptr_dtype, m.row_map_dtype = nat.FSB_F32, nat.FSB_I32, nat.FSB_I64, nat.FSB_I32
    m.n_rows, m.n_cols, m.nnz = n_rows, 1_000_000, nnz
    m.values = m.col_idx = m.row_ptr = 1  # never dereferenced: rejected before any launch
    return lib.fsb_spmv_csr_noalloc(m, ctypes.c_void_p(1), ctypes.c_void_p(1), nat.FSB_F32, nat.ACC_NATIVE, items,
                                    nat.stream_handle(DEV)), lib


@pytest.mark.parametrize("items", [128, 512, 1024])
def test_noalloc_rejects_one_item_beyond_fixed_scratch(items):
    # MAX_TILES * items + 1 path items need MAX_TILES + 1 tiles
    n_rows = 1000
    rc, lib = _limit_status(n_rows, MAX_TILES * items + 1 - n_rows, items)
    assert rc == nat.FSB_ERR_LIMIT
    assert b"exceed the fixed scratch" in lib.fsb_last_error()
    # far beyond the array: 1 M rows + 16 M nonzeros = 17 M path items
    rc, _ = _limit_status(1_000_000, 16_000_000, items)
    assert rc == nat.FSB_ERR_LIMIT
