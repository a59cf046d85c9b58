"""The C-ABI library loads on a machine without a GPU and exports every entry
point include/flagsparse_b200.h declares (no kernel is launched here)."""

import ctypes
import os
import re

from flagsparse_public_b200 import _native as nat
from tests.conftest import ROOT

HEADER = os.path.join(ROOT, "include", "flagsparse_b200.h")


def declared_in_header():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fsb_[a-z0-9_]+)\s*\(", text)))


def test_header_declarations_are_bound():
    declared = declared_in_header()
    assert declared, "no declarations parsed"
    assert declared == nat.declared_symbols()


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(nat.LIB_PATH)
    for name in declared_in_header():
        assert hasattr(lib, name), name


def test_abi_version_and_status_strings():
    lib = nat.library()
    assert lib.fsb_abi_version() == 2
    assert lib.fsb_status_string(0) == b"ok"
    assert b"workspace" in lib.fsb_status_string(nat.FSB_ERR_WORKSPACE)


def test_workspace_query_is_host_only():
    lib = nat.library()
    m = nat.FsbCsr()
    m.value_dtype, m.index_dtype, m.ptr_dtype = nat.FSB_F32, nat.FSB_I32, nat.FSB_I64
    m.n_rows, m.n_cols, m.nnz = 1000, 1000, 5000
    rows = nat.make_plan(nat.ALGO_ROWS, lanes=4)
    assert lib.fsb_workspace_bytes(0, m, 1, nat.ACC_NATIVE, nat.FSB_F32, rows) == 0
    merge = nat.make_plan(nat.ALGO_MERGE, items_per_unit=1024, n_units=6)
    # carry_row (int64) + carry and head partials per unit, 256-byte aligned
    assert lib.fsb_workspace_bytes(0, m, 1, nat.ACC_WIDE, nat.FSB_F32, merge) == 3 * 256
    assert lib.fsb_workspace_bytes(1, m, 64, nat.ACC_NATIVE, nat.FSB_F32, merge) == 256 + 2 * 1536


def test_invalid_arguments_rejected_without_launch():
    lib = nat.library()
    rc = lib.fsb_spmv_csr(None, None, None, nat.FSB_F32, 0, None, None, 0, None)
    assert rc == nat.FSB_ERR_INVALID
    assert b"null" in lib.fsb_last_error()
    rc = lib.fsb_merge_partition(None, nat.FSB_I64, 10, 10, 128, 0, None, 1, None)
    assert rc == nat.FSB_ERR_INVALID


def test_spmm_rejects_oversized_units_on_the_host():
    """The launchers check items_per_unit before touching the device."""
    import torch
    lib = nat.library()
    for algo in (nat.ALGO_MERGE, nat.ALGO_SEQ):
        csr = nat.FsbCsr()
        csr.value_dtype, csr.index_dtype, csr.ptr_dtype, csr.row_map_dtype = nat.FSB_F32, nat.FSB_I32, nat.FSB_I64, nat.FSB_I32
        csr.n_rows, csr.n_cols, csr.nnz = 4, 4, 4
        csr.values = csr.col_idx = csr.row_ptr = 16  # never dereferenced: rejected first
        plan = nat.make_plan(algo, items_per_unit=(1 << 24) + 1, n_units=1, coords=None)
        plan.unit_coords = 16
        rc = lib.fsb_spmm_csr(ctypes.byref(csr), 16, 8, 8, 16, 8, nat.FSB_F32, nat.ACC_NATIVE, ctypes.byref(plan), 16,
                              1 << 20, None)
        assert rc == nat.FSB_ERR_INVALID, (algo, rc)


def test_header_constants_match_the_binding():
    """Every #define the Python binding mirrors has the header's value."""
    text = open(HEADER).read()
    defines = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define\s+(FSB_[A-Z0-9_]+)\s+(-?\d+)", text)}
    mirrored = {
        "FSB_F16": nat.FSB_F16, "FSB_BF16": nat.FSB_BF16, "FSB_F32": nat.FSB_F32, "FSB_F64": nat.FSB_F64,
        "FSB_C64": nat.FSB_C64, "FSB_C128": nat.FSB_C128, "FSB_I32": nat.FSB_I32, "FSB_I64": nat.FSB_I64,
        "FSB_C32": nat.FSB_C32, "FSB_ACC_NATIVE": nat.ACC_NATIVE, "FSB_ACC_WIDE": nat.ACC_WIDE,
        "FSB_ACC_COMP": nat.ACC_COMP, "FSB_ALGO_ROWS": nat.ALGO_ROWS, "FSB_ALGO_MERGE": nat.ALGO_MERGE,
        "FSB_ALGO_FLAT": nat.ALGO_FLAT, "FSB_ALGO_GATHER": nat.ALGO_GATHER, "FSB_ALGO_SEQ": nat.ALGO_SEQ,
        "FSB_PLAN_TMA_GATHER": nat.PLAN_TMA_GATHER, "FSB_BSR_STAGE_TMA": nat.BSR_STAGE_TMA,
        "FSB_BSR_STAGE_THREADS": nat.BSR_STAGE_THREADS, "FSB_ERR_UNSUPPORTED": nat.FSB_ERR_UNSUPPORTED,
        "FSB_ERR_WORKSPACE": nat.FSB_ERR_WORKSPACE, "FSB_OK": nat.FSB_OK,
        "FSB_GATHER_FLOOR_VARIANTS": nat.GATHER_FLOOR_VARIANTS,
    }
    for name, value in mirrored.items():
        assert defines.get(name) == value, name
