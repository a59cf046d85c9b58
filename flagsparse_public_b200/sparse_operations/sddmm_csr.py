"""CSR SDDMM: out[p] = alpha * dot(x[row(p)], y[col(p)]) + beta * data[p].

Same API as FlagSparse's ``sddmm_csr.py``: ``SDDMMPrepared`` (same slots,
:9-33), ``prepare_sddmm_csr`` (:93-105, pattern validation :46-79 with the
same messages), ``flagsparse_sddmm_csr`` (:350-422: keywords, defaults,
``return_time`` / ``return_meta`` results, dense-input validation :205-226,
``out`` validation :229-240).  The product runs in ``fsb_sddmm_csr``
(sm_100a); ``allow_fallback`` is accepted for compatibility, but there is no
non-CUDA path to fall back to (``fallback_used`` is always False).
"""

from ._common import *
from .. import _native as _nat
from .. import _plan

SUPPORTED_SDDMM_VALUE_DTYPES = (torch.float32, torch.float64)


class SDDMMPrepared:
    """Prepared CSR pattern metadata for SDDMM."""

    __slots__ = ("indices", "indptr", "shape", "n_rows", "n_cols", "nnz", "row_ids", "block_k", "num_warps")

    def __init__(self, indices, indptr, shape, row_ids, block_k, num_warps):
        self.indices = indices
        self.indptr = indptr
        self.shape = (int(shape[0]), int(shape[1]))
        self.n_rows = self.shape[0]
        self.n_cols = self.shape[1]
        self.nnz = int(indices.numel())
        self.row_ids = row_ids
        self.block_k = int(block_k)
        self.num_warps = int(num_warps)


def _resolve_sddmm_launch_config(k):
    # reported in meta like FlagSparse's (sddmm_csr.py:36-43); the kernel
    # sizes its lane groups from k itself
    if k <= 32:
        return 32, 2
    if k <= 128:
        return 64, 4
    return 128, 8


def _prepare_sddmm_csr_pattern(indices, indptr, shape):
    if len(shape) != 2:
        raise ValueError("shape must be a 2-tuple")
    if indices.ndim != 1 or indptr.ndim != 1:
        raise ValueError("indices and indptr must be 1D tensors")
    n_rows, n_cols = int(shape[0]), int(shape[1])
    if n_rows < 0 or n_cols < 0:
        raise ValueError("shape dimensions must be non-negative")
    if indptr.numel() != n_rows + 1:
        raise ValueError(f"indptr length must be n_rows+1={n_rows + 1}, got {indptr.numel()}")
    if not indices.is_cuda or not indptr.is_cuda:
        raise ValueError("indices and indptr must be CUDA tensors")
    if indices.dtype != torch.int32:
        raise TypeError("indices dtype must be torch.int32")
    if indptr.dtype not in (torch.int32, torch.int64):
        raise TypeError("indptr dtype must be torch.int32 or torch.int64")
    indptr64 = indptr.to(torch.int64).contiguous()
    indices = indices.contiguous()
    nnz = int(indices.numel())
    if indptr64.numel() > 0 and int(indptr64[0].item()) != 0:
        raise ValueError("indptr[0] must be 0")
    if indptr64.numel() > 0 and int(indptr64[-1].item()) != nnz:
        raise ValueError(f"indptr[-1] must equal nnz={nnz}")
    if indptr64.numel() > 1 and bool(torch.any(indptr64[1:] < indptr64[:-1]).item()):
        raise ValueError("indptr must be nondecreasing")
    if nnz > 0:
        min_col = int(indices.min().item())
        max_col = int(indices.max().item())
        if min_col < 0 or max_col >= n_cols:
            raise IndexError("indices out of range for shape[1]")
    return indices, indptr64, (n_rows, n_cols)


def _build_row_ids(indptr):
    n_rows = int(indptr.numel()) - 1
    if n_rows <= 0:
        return torch.empty(0, dtype=torch.int32, device=indptr.device)
    counts = indptr[1:] - indptr[:-1]
    return torch.repeat_interleave(torch.arange(n_rows, dtype=torch.int32, device=indptr.device), counts)


def prepare_sddmm_csr(indices, indptr, shape, k_hint=64):
    indices, indptr, shape = _prepare_sddmm_csr_pattern(indices, indptr, shape)
    row_ids = _build_row_ids(indptr)
    block_k, num_warps = _resolve_sddmm_launch_config(int(k_hint))
    return SDDMMPrepared(indices=indices, indptr=indptr, shape=shape, row_ids=row_ids, block_k=block_k,
                         num_warps=num_warps)


def _validate_sddmm_dense_inputs(data, prepared, x, y):
    if x.ndim != 2 or y.ndim != 2:
        raise ValueError("x and y must be 2D dense tensors")
    if not x.is_cuda or not y.is_cuda:
        raise ValueError("x and y must be CUDA tensors")
    if x.device != y.device or x.device != prepared.indices.device:
        raise ValueError("x, y, and sparse pattern must be on the same CUDA device")
    if x.dtype not in SUPPORTED_SDDMM_VALUE_DTYPES:
        raise TypeError("x dtype must be torch.float32 or torch.float64")
    if y.dtype != x.dtype:
        raise TypeError("y dtype must match x dtype")
    if data is not None and data.dtype != x.dtype:
        raise TypeError("data dtype must match x/y dtype")
    if x.shape[0] != prepared.n_rows:
        raise ValueError(f"x.shape[0] must be n_rows={prepared.n_rows}, got {x.shape[0]}")
    if y.shape[0] != prepared.n_cols:
        raise ValueError(f"y.shape[0] must be n_cols={prepared.n_cols}, got {y.shape[0]}")
    if x.shape[1] != y.shape[1]:
        raise ValueError("x and y must have the same K dimension")
    if data is not None and data.numel() != prepared.nnz:
        raise ValueError("data length must equal nnz of sparse pattern")
    return int(x.shape[1])


def _prepare_validated_sddmm_out(prepared, x, out, out_dtype=None):
    nnz = prepared.nnz
    target_dtype = x.dtype if out_dtype is None else out_dtype
    if out is None:
        return torch.empty(nnz, dtype=target_dtype, device=x.device)
    if out.ndim != 1 or out.numel() != nnz:
        raise ValueError("out must be a 1D tensor with length nnz")
    if not out.is_cuda or out.device != x.device:
        raise ValueError("out must be a CUDA tensor on the same device as x")
    if out.dtype != target_dtype:
        raise TypeError("out dtype must match the requested output dtype")
    return out


def _run_sddmm_prepared(prepared, x, y, data, alpha, beta, out):
    out = _prepare_validated_sddmm_out(prepared, x, out)
    k = int(x.shape[1])
    block_k, num_warps = _resolve_sddmm_launch_config(k)
    meta = {"block_k": block_k, "num_warps": num_warps, "fallback_used": False, "variant": "baseline",
            "acc_dtype": "float64" if x.dtype == torch.float64 else "float32",
            "out_dtype": str(out.dtype).replace("torch.", "")}
    if prepared.nnz == 0:
        return out, meta
    x = x.contiguous()
    y = y.contiguous()
    if not out.is_contiguous():
        raise ValueError("out must be contiguous")
    d = data.contiguous() if data is not None else None
    lib = _nat.library()
    rc = lib.fsb_sddmm_csr(_nat.ptr(prepared.indices), _nat.dtype_code(prepared.indices.dtype),
                           _nat.ptr(prepared.row_ids), prepared.nnz, prepared.n_rows, prepared.n_cols, _nat.ptr(x),
                           int(x.stride(0)), _nat.ptr(y), int(y.stride(0)), k, _nat.ptr(d) if d is not None else None,
                           _nat.ptr(out), _nat.dtype_code(x.dtype), float(alpha),
                           float(beta) if d is not None else 0.0, _nat.stream_handle(x.device))
    _nat.check(rc, "fsb_sddmm_csr")
    _plan.LAUNCHES["count"] += 1
    return out, meta


def flagsparse_sddmm_csr(data=None, indices=None, indptr=None, x=None, y=None, shape=None, alpha=1.0, beta=0.0,
                         prepared=None, out=None, return_time=False, return_meta=False, allow_fallback=False):
    """CSR SDDMM: out[p] = alpha * dot(x[row(p)], y[col(p)]) + beta * data[p]."""
    prepare_ms = 0.0
    if prepared is None:
        if any(v is None for v in (indices, indptr, shape)):
            raise ValueError("indices, indptr, and shape are required when prepared is not provided")
        torch.cuda.synchronize()
        t_prepare0 = time.perf_counter()
        k_hint = int(x.shape[1]) if (x is not None and x.ndim == 2) else 64
        prepared = prepare_sddmm_csr(indices, indptr, shape, k_hint=k_hint)
        torch.cuda.synchronize()
        prepare_ms = (time.perf_counter() - t_prepare0) * 1000.0
    elif not isinstance(prepared, SDDMMPrepared):
        raise TypeError("prepared must be a SDDMMPrepared instance")
    if x is None or y is None:
        raise ValueError("x and y are required")
    if data is None and float(beta) != 0.0:
        raise ValueError("data is required when beta is non-zero")
    k_dim = _validate_sddmm_dense_inputs(data, prepared, x, y)
    if k_dim == 0:
        out = _prepare_validated_sddmm_out(prepared, x, out)
        if beta == 0.0 or data is None:
            out.zero_()
        else:
            out.copy_(data * beta)
        meta = {"prepare_ms": prepare_ms, "block_k": prepared.block_k, "num_warps": prepared.num_warps,
                "fallback_used": False}
        if return_time and return_meta:
            return out, 0.0, meta
        if return_time:
            return out, 0.0
        if return_meta:
            return out, meta
        return out
    t0 = None
    if return_time:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
    out_tensor, launch_meta = _run_sddmm_prepared(prepared, x, y, data, alpha, beta, out)
    elapsed_ms = 0.0
    if return_time:
        torch.cuda.synchronize()
        elapsed_ms = (time.perf_counter() - t0) * 1000.0
    if return_time and return_meta:
        return out_tensor, elapsed_ms, {"prepare_ms": prepare_ms, **launch_meta}
    if return_time:
        return out_tensor, elapsed_ms
    if return_meta:
        return out_tensor, {"prepare_ms": prepare_ms, **launch_meta}
    return out_tensor
