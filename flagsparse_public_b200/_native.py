"""ctypes binding of ``libflagsparse_b200.so`` (the C ABI in include/flagsparse_b200.h).

Every compute entry point receives device pointers taken from torch tensors and
the handle of torch's current CUDA stream; torch only provides memory and the
stream.  There is no fallback: if the library is missing or a launch fails the
caller gets an exception.
"""

import ctypes
import os
import threading

import torch

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
# FSB_LIB_PATH selects another build of the same library (same ABI).
LIB_PATH = os.environ.get("FSB_LIB_PATH") or os.path.join(PKG_DIR, "libflagsparse_b200.so")

FSB_OK = 0
FSB_ERR_INVALID = -1
FSB_ERR_UNSUPPORTED = -2
FSB_ERR_LAUNCH = -3
FSB_ERR_WORKSPACE = -4
FSB_ERR_TIMEOUT = -5
FSB_ERR_LIMIT = -6

FSB_F16, FSB_BF16, FSB_F32, FSB_F64, FSB_C64, FSB_C128, FSB_I32, FSB_I64 = range(8)
ACC_NATIVE, ACC_WIDE, ACC_COMP = 0, 1, 2
ALGO_ROWS, ALGO_MERGE, ALGO_FLAT, ALGO_GATHER, ALGO_SEQ = 0, 1, 2, 3, 4
PLAN_TMA_GATHER = 1  # fsb_plan.flags: SEQ with B rows staged by TMA tile::gather4
PLAN_OVERLAP_LAUNCH = 2  # fsb_plan.flags: ROWS SpMV with programmatic dependent launch
GATHER_FLOOR_VARIANTS = 4  # fsb_gather_floor variants (gathers in flight x resident warps)
DIAG_NATIVE, DIAG_WIDE, DIAG_KAHAN, DIAG_KAHAN_WIDE = 0, 1, 2, 3  # fsb_spmm_csr_diag accumulations
BSR_STAGE_TMA, BSR_STAGE_THREADS = 0, 1

_DTYPE_CODES = {
    torch.float16: FSB_F16,
    torch.bfloat16: FSB_BF16,
    torch.float32: FSB_F32,
    torch.float64: FSB_F64,
    torch.complex64: FSB_C64,
    torch.complex128: FSB_C128,
    torch.int32: FSB_I32,
    torch.int64: FSB_I64,
}
FSB_C32 = 8
if getattr(torch, "complex32", None) is not None:
    _DTYPE_CODES[torch.complex32] = FSB_C32


class FsbCsr(ctypes.Structure):
    _fields_ = [
        ("values", ctypes.c_void_p),
        ("col_idx", ctypes.c_void_p),
        ("row_ptr", ctypes.c_void_p),
        ("row_map", ctypes.c_void_p),
        ("value_dtype", ctypes.c_int32),
        ("index_dtype", ctypes.c_int32),
        ("ptr_dtype", ctypes.c_int32),
        ("row_map_dtype", ctypes.c_int32),
        ("n_rows", ctypes.c_int64),
        ("n_cols", ctypes.c_int64),
        ("nnz", ctypes.c_int64),
    ]


class FsbPlan(ctypes.Structure):
    _fields_ = [
        ("algo", ctypes.c_int32),
        ("lanes", ctypes.c_int32),
        ("items_per_unit", ctypes.c_int32),
        ("n_tile", ctypes.c_int32),
        ("n_units", ctypes.c_int64),
        ("unit_coords", ctypes.c_void_p),
        ("row_cap", ctypes.c_int64),
        ("comp_threshold", ctypes.c_int64),
        ("grid_blocks", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("unit_runs", ctypes.c_void_p),
        ("tickets", ctypes.c_void_p),
        ("ticket_slots", ctypes.c_int64),
    ]


class FsbStruct(ctypes.Structure):
    _fields_ = [
        ("run_col", ctypes.c_void_p),
        ("run_off", ctypes.c_void_p),
        ("run_len", ctypes.c_void_p),
        ("tile_base", ctypes.c_void_p),
        ("tile_span", ctypes.c_void_p),
        ("max_span", ctypes.c_int32),
        ("chunk_nnz", ctypes.c_int32),
        ("n_long", ctypes.c_int64),
        ("long_rows", ctypes.c_void_p),
        ("n_chunks", ctypes.c_int64),
        ("chunk_row", ctypes.c_void_p),
        ("chunk_ptr", ctypes.c_void_p),
        ("xblock", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("n_xblocks", ctypes.c_int64),
        ("seg_ptr", ctypes.c_void_p),
        ("seg_val", ctypes.c_void_p),
        ("seg_off", ctypes.c_void_p),
        ("lt_groups", ctypes.c_int64),
        ("lt_col_blocks", ctypes.c_int64),
        ("lt_rec_cap", ctypes.c_int32),
        ("lt_rows", ctypes.c_int32),
        ("lt_cols", ctypes.c_int32),
        ("reserved3", ctypes.c_int32),
        ("lt_rec", ctypes.c_void_p),
        ("lt_seg_start", ctypes.c_void_p),
        ("lt_seg_len", ctypes.c_void_p),
        ("lt_row_start", ctypes.c_void_p),
    ]


# name -> (restype, argtypes)
_SIGNATURES = {
    "fsb_abi_version": (ctypes.c_int, []),
    "fsb_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "fsb_last_error": (ctypes.c_char_p, []),
    "fsb_device_error": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int), ctypes.c_int]),
    "fsb_selftest_wait_timeout": (ctypes.c_int, [ctypes.c_int64, ctypes.c_void_p]),
    "fsb_workspace_bytes": (
        ctypes.c_int64,
        [ctypes.c_int, ctypes.POINTER(FsbCsr), ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.POINTER(FsbPlan)],
    ),
    "fsb_merge_partition": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32, ctypes.c_int64,
         ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p],
    ),
    "fsb_csr_check_workspace_bytes": (ctypes.c_int64, [ctypes.c_int64, ctypes.c_int64]),
    "fsb_csr_check": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p],
    ),
    "fsb_merge_runs": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
         ctypes.c_void_p],
    ),
    "fsb_spmv_csr": (
        ctypes.c_int,
        [ctypes.POINTER(FsbCsr), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
         ctypes.POINTER(FsbPlan), ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p],
    ),
    "fsb_spmv_csr_checked_workspace_bytes": (ctypes.c_int64, [ctypes.POINTER(FsbCsr), ctypes.c_int, ctypes.c_int]),
    "fsb_spmv_csr_checked": (
        ctypes.c_int,
        [ctypes.POINTER(FsbCsr), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
         ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(FsbPlan), ctypes.c_void_p],
    ),
    "fsb_coo_coalesce": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
         ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "fsb_spmm_csr_diag": (
        ctypes.c_int,
        [ctypes.POINTER(FsbCsr), ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
         ctypes.c_int, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p],
    ),
    "fsb_spmv_csr_noalloc": (
        ctypes.c_int,
        [ctypes.POINTER(FsbCsr), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int32,
         ctypes.c_void_p],
    ),
    "fsb_spmm_csr": (
        ctypes.c_int,
        [ctypes.POINTER(FsbCsr), ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
         ctypes.c_int, ctypes.c_int, ctypes.POINTER(FsbPlan), ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p],
    ),
    "fsb_spmv_coo_atomic": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int64,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p],
    ),
    "fsb_spmm_coo_atomic": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int64,
         ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
         ctypes.c_void_p],
    ),
    "fsb_struct_rows": (
        ctypes.c_int,
        [ctypes.POINTER(FsbCsr), ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
         ctypes.c_void_p],
    ),
    "fsb_struct_tiles": (
        ctypes.c_int,
        [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
         ctypes.c_void_p],
    ),
    "fsb_struct_workspace_bytes": (ctypes.c_int64, [ctypes.c_int, ctypes.POINTER(FsbStruct), ctypes.c_int64]),
    "fsb_struct_spmv": (
        ctypes.c_int,
        [ctypes.POINTER(FsbCsr), ctypes.POINTER(FsbStruct), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
         ctypes.c_int64, ctypes.c_void_p],
    ),
    "fsb_struct_spmm": (
        ctypes.c_int,
        [ctypes.POINTER(FsbCsr), ctypes.POINTER(FsbStruct), ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
         ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p],
    ),
    "fsb_bsr_spmm_tc": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int64,
         ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
         ctypes.c_int64, ctypes.c_int, ctypes.c_void_p],
    ),
    "fsb_sorted_keys_to_offsets": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "fsb_sort_workspace_bytes": (ctypes.c_int64, [ctypes.c_int64, ctypes.c_int, ctypes.c_int]),
    "fsb_stable_sort": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p],
    ),
    "fsb_run_starts_workspace_bytes": (ctypes.c_int64, [ctypes.c_int64]),
    "fsb_run_starts": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p],
    ),
    "fsb_sddmm_csr": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
         ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_void_p],
    ),
    "fsb_mtx_open": (
        ctypes.c_void_p,
        [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
         ctypes.POINTER(ctypes.c_int64), ctypes.c_int],
    ),
    "fsb_mtx_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "fsb_mtx_close": (None, [ctypes.c_void_p]),
    "fsb_csr_features": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_int64,
         ctypes.c_void_p, ctypes.c_void_p],
    ),
    "fsb_mlp_param_count": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "fsb_mlp_forward": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p],
    ),
    "fsb_mlp_backward": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p,
         ctypes.c_void_p, ctypes.c_void_p],
    ),
    "fsb_adam_step": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_float,
         ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_float, ctypes.c_void_p],
    ),
    "fsb_gather_floor": (
        ctypes.c_int,
        [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p,
         ctypes.c_int64, ctypes.c_int, ctypes.c_void_p],
    ),
}

_lib = None
_lock = threading.Lock()


class NativeLibraryError(RuntimeError):
    """The CUDA library is missing or failed to load."""


def library():
    """Load (once) and return the ctypes handle of libflagsparse_b200.so."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise NativeLibraryError(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                "or `python flagsparse_public_b200/_build.py`; there is no non-CUDA fallback"
            )
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def device_error(reset=True):
    """Sticky device error word of the mbarrier-waiting kernels (synchronises)."""
    v = ctypes.c_int(0)
    check(library().fsb_device_error(ctypes.byref(v), int(bool(reset))), "fsb_device_error")
    return v.value


def declared_symbols():
    return sorted(_SIGNATURES)


def dtype_code(dtype):
    try:
        return _DTYPE_CODES[dtype]
    except KeyError:
        raise TypeError(f"dtype {dtype} has no kernel support") from None


def check(status, what):
    if status != FSB_OK:
        lib = library()
        msg = lib.fsb_last_error().decode(errors="replace")
        kind = lib.fsb_status_string(status).decode()
        raise RuntimeError(f"{what} failed ({kind}): {msg}")


def stream_handle(device):
    """torch's current stream on ``device`` as a cudaStream_t."""
    if isinstance(device, int):
        idx = device
    else:
        idx = torch.device(device).index
        if idx is None:
            idx = torch.cuda.current_device()
    return ctypes.c_void_p(torch._C._cuda_getCurrentRawStream(idx))


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() > 0 else ctypes.c_void_p(0)


_figures = threading.local()


def csr_check(row_ptr, col_idx, n_rows):
    """The eight structural figures of fsb_csr_check (row_ptr[0],
    row_ptr[n_rows], rows of negative length, negative column indices, largest
    column index, longest row, sum of squared row lengths, empty rows),
    written by its kernels into a pinned buffer of this thread and read after
    one stream synchronisation."""
    buf = getattr(_figures, "buf", None)
    if buf is None:
        buf = _figures.buf = torch.empty(8, dtype=torch.int64).pin_memory()
    n_rows, nnz = int(n_rows), int(col_idx.numel())
    lib = library()
    nbytes = int(lib.fsb_csr_check_workspace_bytes(n_rows, nnz))
    ws = torch.empty(nbytes, dtype=torch.uint8, device=row_ptr.device)
    rc = lib.fsb_csr_check(ptr(row_ptr), dtype_code(row_ptr.dtype), n_rows, ptr(col_idx), dtype_code(col_idx.dtype),
                           nnz, ctypes.c_void_p(buf.data_ptr()), ptr(ws), nbytes, stream_handle(row_ptr.device))
    check(rc, "fsb_csr_check")
    torch.cuda.current_stream(row_ptr.device).synchronize()
    return buf.tolist()


def make_csr(values, col_idx, row_ptr, n_rows, n_cols, row_map=None):
    m = FsbCsr()
    m.values = values.data_ptr() if values.numel() > 0 else 0
    m.col_idx = col_idx.data_ptr() if col_idx.numel() > 0 else 0
    m.row_ptr = row_ptr.data_ptr()
    m.row_map = row_map.data_ptr() if row_map is not None and row_map.numel() > 0 else 0
    m.value_dtype = dtype_code(values.dtype)
    m.index_dtype = dtype_code(col_idx.dtype)
    m.ptr_dtype = dtype_code(row_ptr.dtype)
    m.row_map_dtype = dtype_code(row_map.dtype) if row_map is not None else m.index_dtype
    m.n_rows = int(n_rows)
    m.n_cols = int(n_cols)
    m.nnz = int(values.numel())
    return m


def make_plan(algo, lanes=32, items_per_unit=0, n_tile=0, coords=None, n_units=0, row_cap=0, comp_threshold=0,
              grid_blocks=0, flags=0, runs=None, tickets=None):
    p = FsbPlan()
    p.algo = int(algo)
    p.lanes = int(lanes)
    p.items_per_unit = int(items_per_unit)
    p.n_tile = int(n_tile)
    p.n_units = int(n_units)
    p.unit_coords = coords.data_ptr() if coords is not None else 0
    p.row_cap = int(row_cap)
    p.comp_threshold = int(comp_threshold)
    p.grid_blocks = int(grid_blocks)
    p.flags = int(flags)
    p.unit_runs = runs.data_ptr() if runs is not None and runs.numel() > 0 else 0
    p.tickets = tickets.data_ptr() if tickets is not None and tickets.numel() > 0 else 0
    p.ticket_slots = int(tickets.numel()) if tickets is not None else 0
    return p
