"""CSR SpMM opt-alg2: FlagSparse's device-aware SpMM API on sm_100a kernels.

Follows FlagSparse ``sparse_operations/spmm_csr_opt_alg2.py``
(``PreparedCsrSpmmOptAlg2`` :20-57, ``prepare_spmm_csr_opt_alg2`` :632-653,
``flagsparse_spmm_csr_opt_alg2`` :801-850 with ``return_time`` /
``return_meta``).  The reference picked Triton warps/stages per row-length
bucket from device properties; here the launch is the CUDA kernel plan of the
matrix, and ``meta`` reports that plan together with the device properties
and the reference's row-length bucket hits.
"""

from ._common import *
from .. import _native as _nat
from .. import _plan
from .spmm_csr import (
    _prepare_spmm_csr_matrix,
    _spmm_coo_reference_tolerance,
    _spmm_plan_for,
)

SUPPORTED_SPMM_OPT_ALG2_DTYPES = (torch.float32, torch.float64)

# Row-length buckets of FlagSparse alg2 (spmm_csr_opt_alg2.py:60-158), reported
# in meta["bucket_hits"]; (label, min_row_nnz, max_row_nnz).
_ALG2_BUCKETS = (
    ("short_16", 0, 16),
    ("short_64", 17, 64),
    ("row_256", 65, 256),
    ("seg_1024", 257, 1024),
    ("seg_long", 1025, None),
)


class PreparedCsrSpmmOptAlg2:
    """Cached CSR metadata for repeated alg2 CSR SpMM calls on the same sparse matrix."""

    __slots__ = (
        "data",
        "kernel_indices",
        "kernel_indptr",
        "shape",
        "n_rows",
        "n_cols",
        "row_lengths",
        "max_row_nnz",
        "opt_buckets",
        "supports_opt",
        "_stats",
        "_plans",
    )

    def __init__(self, data, kernel_indices, kernel_indptr, shape, n_rows, n_cols, row_lengths, max_row_nnz,
                 opt_buckets):
        self.data = data
        self.kernel_indices = kernel_indices
        self.kernel_indptr = kernel_indptr
        self.shape = (int(shape[0]), int(shape[1]))
        self.n_rows = int(n_rows)
        self.n_cols = int(n_cols)
        self.row_lengths = row_lengths
        self.max_row_nnz = int(max_row_nnz)
        self.opt_buckets = opt_buckets
        self.supports_opt = data.dtype in SUPPORTED_SPMM_OPT_ALG2_DTYPES
        self._stats = None
        self._plans = {}


def _normalize_spmm_opt_alg2_device_props(device):
    props = torch.cuda.get_device_properties(device)
    return {
        "device_name": str(getattr(props, "name", "cuda")),
        "warp_size": int(getattr(props, "warp_size", 32) or 32),
        "sm_count": int(getattr(props, "multi_processor_count", 0) or 0),
        "max_threads_per_mp": int(getattr(props, "max_threads_per_multi_processor", 2048) or 2048),
        "max_threads_per_block": int(getattr(props, "max_threads_per_block", 1024) or 1024),
        "shared_memory_per_block": int(getattr(props, "shared_memory_per_block", 0) or 0),
        "capability": (int(getattr(props, "major", 0) or 0), int(getattr(props, "minor", 0) or 0)),
    }


def _build_spmm_opt_alg2_buckets(row_lengths, dtype):
    """Row counts per FlagSparse alg2 row-length bucket (one device->host read)."""
    del dtype
    if row_lengths.numel() == 0:
        return []
    counts = []
    for _label, lo, hi in _ALG2_BUCKETS:
        if hi is None:
            counts.append((row_lengths >= lo).sum())
        elif lo <= 0:
            counts.append((row_lengths <= hi).sum())
        else:
            counts.append(((row_lengths >= lo) & (row_lengths <= hi)).sum())
    vals = torch.stack(counts).tolist()
    return [{"label": b[0], "row_count": int(c)} for b, c in zip(_ALG2_BUCKETS, vals) if c > 0]


def prepare_spmm_csr_opt_alg2(data, indices, indptr, shape):
    (data, kernel_indices, kernel_indptr, n_rows, n_cols, row_lengths, max_row_nnz) = _prepare_spmm_csr_matrix(
        data, indices, indptr, shape
    )
    opt_buckets = _build_spmm_opt_alg2_buckets(row_lengths, data.dtype)
    return PreparedCsrSpmmOptAlg2(
        data=data, kernel_indices=kernel_indices, kernel_indptr=kernel_indptr, shape=shape, n_rows=n_rows,
        n_cols=n_cols, row_lengths=row_lengths, max_row_nnz=max_row_nnz, opt_buckets=opt_buckets,
    )


def _validate_spmm_opt_alg2_runtime_inputs(prepared, B, out):
    if not prepared.supports_opt:
        raise TypeError("flagsparse_spmm_csr_opt_alg2 only supports float32 and float64")
    if B is None:
        raise ValueError("B is required")
    if B.ndim != 2:
        raise ValueError("B must be a 2D dense tensor")
    if not B.is_cuda:
        raise ValueError("B must be a CUDA tensor")
    if B.device != prepared.data.device:
        raise ValueError("B must be on the same CUDA device as sparse matrix data")
    if B.dtype != prepared.data.dtype:
        raise TypeError("B dtype must match sparse matrix dtype")
    if B.shape[0] != prepared.n_cols:
        raise ValueError(f"B.shape[0] must be n_cols={prepared.n_cols}, got {B.shape[0]}")
    if out is not None:
        if not out.is_cuda:
            raise ValueError("out must be a CUDA tensor")
        if out.device != prepared.data.device:
            raise ValueError("out must be on the same CUDA device as sparse matrix data")
        if out.shape != (prepared.n_rows, int(B.shape[1])) or out.dtype != prepared.data.dtype:
            raise ValueError("out shape/dtype must match result")


def _triton_spmm_csr_impl_opt_alg2_prepared(prepared, B, return_meta=False, out=None):
    n_dense = int(B.shape[1])
    C = out if out is not None else torch.empty((prepared.n_rows, n_dense), dtype=B.dtype, device=B.device)
    launch_configs = []
    if prepared.n_rows > 0 and n_dense > 0:
        plan = _spmm_plan_for(prepared, "alg2", n_dense, (B, C, _nat.ACC_NATIVE))
        _plan.run_spmm(prepared.data, prepared.kernel_indices, prepared.kernel_indptr, prepared.n_rows,
                       prepared.n_cols, B, C, _nat.ACC_NATIVE, plan)
        desc = plan.describe()
        desc.update({"bucket_label": "all_rows", "row_count": prepared.n_rows})
        launch_configs.append(desc)
    elif C.numel():
        C.zero_()
    meta = None
    if return_meta:
        props = _normalize_spmm_opt_alg2_device_props(prepared.data.device)
        bucket_hits = [{"bucket_label": b["label"], "kind": "single_launch", "row_count": b["row_count"]}
                       for b in prepared.opt_buckets]
        meta = {
            "device_name": props["device_name"],
            "sm_count": props["sm_count"],
            "warp_size": props["warp_size"],
            "bucket_hits": bucket_hits,
            "launch_configs": launch_configs,
            "max_row_nnz": prepared.max_row_nnz,
            "n_dense_cols": n_dense,
        }
    return C, meta


def flagsparse_spmm_csr_opt_alg2(data=None, indices=None, indptr=None, B=None, shape=None, prepared=None, out=None,
                                 return_time=False, return_meta=False):
    """CSR SpMM opt-alg2 (float32/float64, value-precision accumulation)."""
    if prepared is not None and not isinstance(prepared, PreparedCsrSpmmOptAlg2):
        raise TypeError("prepared must be a PreparedCsrSpmmOptAlg2 instance")
    if prepared is None:
        if any(arg is None for arg in (data, indices, indptr, shape)):
            raise ValueError("data, indices, indptr, and shape are required when prepared is not provided")
        prepared = prepare_spmm_csr_opt_alg2(data, indices, indptr, shape)
    elif shape is not None:
        resolved_shape = (int(shape[0]), int(shape[1]))
        if resolved_shape != prepared.shape:
            raise ValueError(f"shape {resolved_shape} does not match prepared.shape {prepared.shape}")
    _validate_spmm_opt_alg2_runtime_inputs(prepared, B, out)
    B = B.contiguous()
    direct = out is not None and out.is_contiguous()
    t0 = None
    if return_time:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
    C, meta = _triton_spmm_csr_impl_opt_alg2_prepared(prepared, B, return_meta=return_meta,
                                                      out=out if direct else None)
    elapsed_ms = None
    if return_time:
        torch.cuda.synchronize()
        elapsed_ms = (time.perf_counter() - t0) * 1000.0
    if out is not None:
        if C.data_ptr() != out.data_ptr():
            out.copy_(C)
        C = out
    if return_time and return_meta:
        return C, elapsed_ms, meta
    if return_time:
        return C, elapsed_ms
    if return_meta:
        return C, meta
    return C


def _spmm_opt_alg2_reference_error(candidate, reference, value_dtype):
    atol, rtol = _spmm_coo_reference_tolerance(value_dtype)
    if candidate.numel() == 0:
        return 0.0
    diff = torch.abs(candidate - reference)
    denom = atol + rtol * torch.abs(reference)
    return float(torch.max(diff / denom).item())
