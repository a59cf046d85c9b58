"""COO SpMM: FlagSparse's ``spmm_coo`` operator API on sm_100a kernels.

Follows FlagSparse ``sparse_operations/spmm_coo.py`` (validation
``_prepare_spmm_coo_inputs`` :312-371, routes :526-669,
``flagsparse_spmm_coo`` :671-694).  FlagSparse canonicalises on every call
(coalesce duplicates, lexicographic sort, float32 -> float64 copies of A and
B, ``:11-120``) and then runs one program per row run.  The product is linear
in the entries, so duplicates need no merging: here the nonzeros are ordered
by row with a stable sort, row offsets come from a histogram, and the CSR
kernels of ``libflagsparse_b200.so`` accumulate in the reference's compute
precision (float32 -> float64, complex64 -> complex128, half types -> float32)
in registers.  ``_coalesce_coo_entries``, ``_sort_coo_lex_inplace`` and
``_seg_starts_from_sorted_rows`` keep the reference's structural semantics.
"""

from ._common import *
from .. import _native as _nat
from .. import _plan
from .spmm_csr import (
    SUPPORTED_SPMM_VALUE_DTYPES,
    _select_spmm_alg1_warp_and_factor,
    _spmm_coo_reference_tolerance,
    _spmm_relative_threshold,
    _spmm_validation_metrics,
)


def _spmm_coo_compute_dtype(value_dtype):
    if _is_complex_dtype(value_dtype):
        return torch.complex128 if value_dtype == torch.complex64 else value_dtype
    if value_dtype in (torch.float16, torch.bfloat16):
        return torch.float32
    if value_dtype == torch.float32:
        return torch.float64
    return value_dtype


def _sort_coo_lex_inplace(data, row, col, n_cols, n_rows=None):
    """Lexicographic (row, col) order with int64 indices (FlagSparse ``spmm_coo.py:21-32``)."""
    row64 = row.to(torch.int64)
    col64 = col.to(torch.int64)
    if data.numel() == 0:
        return data.contiguous(), row64, col64
    key = row64 * max(1, int(n_cols)) + col64
    bound = None if n_rows is None else max(1, int(n_rows)) * max(1, int(n_cols))
    _, order = _plan.stable_sort(key, key_bound=bound)
    return data[order].contiguous(), row64[order].contiguous(), col64[order].contiguous()


def _coalesce_coo_device(data, row, col, shape):
    """Duplicate merge on the device without a host read: the (row, col) keys
    stably sorted (fsb_stable_sort), runs of equal keys (fsb_run_starts) and
    their values summed in sorted order (fsb_coo_coalesce).  Returns buffers
    of nnz entries (values, int64 rows, int64 cols) and the device count of
    distinct entries; safe to record in a CUDA graph."""
    n_rows, n_cols = int(shape[0]), int(shape[1])
    key = row.to(torch.int64) * max(1, n_cols) + col.to(torch.int64)
    sorted_key, order = _plan.stable_sort(key, key_bound=max(1, n_rows) * max(1, n_cols))
    ukeys, uvals, count = _plan.coalesce_sorted(sorted_key, order, data.contiguous())
    return uvals, ukeys // max(1, n_cols), ukeys % max(1, n_cols), count


def _coalesce_coo_entries(data, row, col, shape):
    """Merge duplicate (row, col) entries by summing values (FlagSparse ``spmm_coo.py:35-51``,
    which calls torch's coalesce): on CUDA tensors the device merge above,
    equal to torch's coalesce bit for bit, with one host read of the count;
    host tensors (the reference's own fixtures) go through torch."""
    n_rows, n_cols = int(shape[0]), int(shape[1])
    if data.numel() == 0:
        z = torch.empty(0, dtype=torch.int64, device=data.device)
        return data.contiguous(), z, z.clone()
    if data.is_cuda:
        vals, rows, cols, count = _coalesce_coo_device(data, row, col, shape)
        m = int(count.item())
        return vals[:m].contiguous(), rows[:m].contiguous(), cols[:m].contiguous()
    coo = torch.sparse_coo_tensor(torch.stack([row.to(torch.int64), col.to(torch.int64)]), data,
                                  size=(n_rows, n_cols), device=data.device, dtype=data.dtype).coalesce()
    idx = coo.indices()
    return coo.values().contiguous(), idx[0].contiguous(), idx[1].contiguous()


def _seg_starts_from_sorted_rows(row_i32, nnz, device):
    """int32 row-run offsets of sorted COO (FlagSparse ``spmm_coo.py:121-132``)."""
    if nnz == 0:
        return None
    return _plan.run_starts(row_i32, torch.int32)


def _prepare_spmm_coo_inputs(data, row, col, B, shape):
    if len(shape) != 2:
        raise ValueError("shape must be a 2-tuple: (n_rows, n_cols)")
    if data.ndim != 1 or row.ndim != 1 or col.ndim != 1:
        raise ValueError("data, row, and col must be 1D tensors")
    if B.ndim != 2:
        raise ValueError("B must be a 2D dense tensor")
    n_rows, n_cols = int(shape[0]), int(shape[1])
    if n_rows < 0 or n_cols < 0:
        raise ValueError("shape dimensions must be non-negative")
    if data.numel() != row.numel() or data.numel() != col.numel():
        raise ValueError("data, row, and col must have the same length (nnz)")
    if B.shape[0] != n_cols:
        raise ValueError(f"B.shape[0] must be n_cols={n_cols}, got {B.shape[0]}")
    if not all(t.is_cuda for t in (data, row, col, B)):
        raise ValueError("data, row, col, and B must be CUDA tensors")
    if not all(t.device == data.device for t in (row, col, B)):
        raise ValueError("data, row, col, and B must be on the same CUDA device")
    if data.dtype not in SUPPORTED_SPMM_VALUE_DTYPES:
        raise TypeError("data dtype must be one of: float16, bfloat16, float32, float64, complex64, complex128")
    if B.dtype != data.dtype:
        raise TypeError("B dtype must match data dtype")
    if row.dtype not in SUPPORTED_INDEX_DTYPES:
        raise TypeError("row dtype must be torch.int32 or torch.int64")
    if col.dtype not in SUPPORTED_INDEX_DTYPES:
        raise TypeError("col dtype must be torch.int32 or torch.int64")
    nnz = data.numel()
    if nnz > _INDEX_LIMIT_INT32:
        raise ValueError("nnz exceeds the int32 range supported by the Triton COO kernel")
    # the index checks read the device: skipped while a CUDA graph records
    # the call (the caller checks the indices before capturing)
    if nnz > 0 and not torch.cuda.is_current_stream_capturing():
        lim = torch.stack([row.min().to(torch.int64), row.max().to(torch.int64), col.min().to(torch.int64),
                           col.max().to(torch.int64)]).tolist()
        min_row, max_row, min_col, max_col = lim
        if min_row < 0 or max_row >= n_rows:
            raise IndexError("row indices out of range for n_rows")
        if min_col < 0 or max_col >= n_cols:
            raise IndexError("col indices out of range for n_cols")
        if max_row > _INDEX_LIMIT_INT32:
            raise ValueError("row indices exceed the int32 range supported by the Triton kernel")
        if max_col > _INDEX_LIMIT_INT32:
            raise ValueError("column indices exceed the int32 range supported by the Triton kernel")
    data = data.contiguous()
    row = row.contiguous()
    col = col.contiguous()
    B = B.contiguous()
    kernel_row = row.to(torch.int32) if row.dtype == torch.int64 else row
    kernel_col = col.to(torch.int32) if col.dtype == torch.int64 else col
    return data, kernel_row, kernel_col, B, n_rows, n_cols, int(B.shape[1])


def _resolve_spmm_coo_launch_config(n_dense_cols, nnz, block_n=None, block_nnz=256):
    warp_size, factor = _select_spmm_alg1_warp_and_factor(n_dense_cols)
    if block_n is None:
        block_n = warp_size * factor
    if block_nnz is None:
        block_nnz = 256
    if block_n <= 0 or block_nnz <= 0:
        raise ValueError("block_n and block_nnz must be positive when provided")
    return {
        "block_n": int(block_n),
        "block_nnz": int(block_nnz),
        "required_nnz_tiles": int(-(-nnz // block_nnz) if nnz > 0 else 0),
        "heuristic_warp_size": int(warp_size),
        "heuristic_factor": int(factor),
    }


def _normalize_spmm_coo_route(route):
    route = "rowrun" if route is None else str(route).lower()
    if route not in ("rowrun", "atomic"):
        raise ValueError("route must be 'rowrun' or 'atomic'")
    return route


def _acc_mode_for(value_dtype):
    return _nat.ACC_WIDE if value_dtype in (torch.float32, torch.complex64) else _nat.ACC_NATIVE


def _take(values, order):
    """values[order]; complex32 entries move as their 32-bit patterns."""
    if _is_complex32_dtype(values.dtype):
        return values.view(torch.int32)[order].view(values.dtype)
    return values[order]


def _coo_rows_to_csr(data, row, col, n_rows):
    """Order nonzeros by row (stable) and build int64 row offsets."""
    row64 = row.to(torch.int64)
    if data.numel() > 1:
        sorted_rows, order = _plan.stable_sort(row64, key_bound=n_rows)
        data, col, row64 = _take(data, order), col[order], sorted_rows
    indptr = _plan.sorted_keys_to_offsets(row64, n_rows)
    return data.contiguous(), col.contiguous(), indptr


def _triton_spmm_coo_impl(data, row, col, B, n_rows, n_dense_cols, block_n, block_nnz, route="rowrun",
                          output_dtype=None):
    """COO SpMM by route; ``block_n`` / ``block_nnz`` are the reference's Triton
    tile sizes and do not change the result."""
    del block_n, block_nnz
    route = _normalize_spmm_coo_route(route)
    out_dtype = output_dtype if output_dtype is not None else data.dtype
    device = data.device
    if n_rows == 0 or n_dense_cols == 0 or B.shape[0] == 0 or data.numel() == 0:
        return torch.zeros((n_rows, n_dense_cols), dtype=out_dtype, device=device)
    if route == "rowrun":
        d, c, indptr = _coo_rows_to_csr(data, row, col, n_rows)
        C = torch.empty((n_rows, n_dense_cols), dtype=data.dtype, device=device)
        # the merge-path plan needs only the sizes the host knows (rows +
        # nonzeros per unit): no statistics read from the device
        nnz = data.numel()
        stats = _plan.MatrixStats(n_rows, B.shape[0], nnz, nnz, nnz / max(n_rows, 1), 0.0, 0)
        plan = _plan.default_spmm_plan(stats, n_dense_cols, data.dtype)
        _plan.run_spmm(d, c, indptr, n_rows, B.shape[0], B, C, _acc_mode_for(data.dtype), plan)
        return C if C.dtype == out_dtype else C.to(out_dtype)
    acc_dtype = _spmm_coo_compute_dtype(data.dtype)
    if _is_complex32_dtype(data.dtype):
        acc_dtype = torch.complex64  # float32 pairs: no float16 atomics
    C_acc = torch.zeros((n_rows, n_dense_cols), dtype=acc_dtype, device=device)
    row_k = row if row.dtype == col.dtype else row.to(col.dtype)
    lib = _nat.library()
    rc = lib.fsb_spmm_coo_atomic(_nat.ptr(data), _nat.ptr(row_k), _nat.ptr(col), _nat.dtype_code(data.dtype),
                                 _nat.dtype_code(col.dtype), data.numel(), _nat.ptr(B), int(B.stride(0)),
                                 n_dense_cols, _nat.ptr(C_acc), int(C_acc.stride(0)), _nat.dtype_code(acc_dtype),
                                 _nat.stream_handle(device))
    _nat.check(rc, "fsb_spmm_coo_atomic")
    return C_acc.to(out_dtype)


def _run_spmm_coo_route(data, row, col, B, shape, block_n=None, block_nnz=256, out=None, return_time=False,
                        route="rowrun"):
    route = _normalize_spmm_coo_route(route)
    if block_n is not None and block_n <= 0:
        raise ValueError("block_n must be positive when provided")
    if block_nnz is not None and block_nnz <= 0:
        raise ValueError("block_nnz must be positive when provided")
    data, kernel_row, kernel_col, B, n_rows, _n_cols, n_dense_cols = _prepare_spmm_coo_inputs(
        data, row, col, B, shape)
    output_dtype = data.dtype
    launch = _resolve_spmm_coo_launch_config(n_dense_cols, data.numel(), block_n=block_n, block_nnz=block_nnz)
    if out is not None:
        if not out.is_cuda:
            raise ValueError("out must be a CUDA tensor")
        if out.device != data.device:
            raise ValueError("out must be on the same CUDA device as the inputs")
        if out.shape != (n_rows, n_dense_cols) or out.dtype != output_dtype:
            raise ValueError("out shape/dtype must match result")
    t0 = None
    if return_time:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
    C = _triton_spmm_coo_impl(data, kernel_row, kernel_col, B, n_rows, n_dense_cols, block_n=launch["block_n"],
                              block_nnz=launch["block_nnz"], route=route, output_dtype=output_dtype)
    elapsed_ms = None
    if return_time:
        torch.cuda.synchronize()
        elapsed_ms = (time.perf_counter() - t0) * 1000.0
    if out is not None:
        out.copy_(C)
        C = out
    if return_time:
        return C, elapsed_ms
    return C


def flagsparse_spmm_coo(data, row, col, B, shape, block_n=None, block_nnz=256, out=None, return_time=False):
    """COO SpMM: C = A @ B (row-run route)."""
    return _run_spmm_coo_route(data, row, col, B, shape, block_n=block_n, block_nnz=block_nnz, out=out,
                               return_time=return_time, route="rowrun")
