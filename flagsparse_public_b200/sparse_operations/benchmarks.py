"""FlagSparse's benchmark entry points for the SpMV / SpMM path.

Each function builds a random CSR matrix with FlagSparse's generator
(``_build_random_csr``), times this package's operator with FlagSparse's
timing helper (``_benchmark_cuda_op``: warm-up, then wall time over ``iters``
synchronised calls), checks it against a higher-precision PyTorch sparse
product, and returns FlagSparse's result dictionary.  The key names are
FlagSparse's, so scripts that read them keep working: ``triton_*`` keys hold
this package's sm_100a kernels.  The cuSPARSE leg runs through CuPy when it
is importable, as FlagSparse's does; otherwise it is reported unavailable with
FlagSparse's reason string.

Reference: ``benchmark_spmv_case`` (benchmarks.py:345-507),
``benchmark_spmm_case`` (spmm_csr.py:2351-2573), ``benchmark_spmm_opt_case``
(spmm_csr.py:2226-2348), ``benchmark_spmm_opt_alg2_case``
(spmm_csr_opt_alg2.py:862-972), ``benchmark_sddmm_case`` (sddmm_csr.py:472-568).
"""

import time

import torch

from ._common import _benchmark_cuda_op, _build_random_csr, _build_random_dense, _tolerance_for_dtype
from .spmm_csr import (
    _resolve_spmm_alg1_launch_config,
    _spmm_opt_reference_error,
    _spmm_relative_threshold,
    _spmm_validation_metrics,
    flagsparse_spmm_csr,
    flagsparse_spmm_csr_opt,
    prepare_spmm_csr_opt,
)
from .spmm_csr_opt_alg2 import (
    SUPPORTED_SPMM_OPT_ALG2_DTYPES,
    _spmm_opt_alg2_reference_error,
    flagsparse_spmm_csr_opt_alg2,
    prepare_spmm_csr_opt_alg2,
)
from .spmv_csr import (
    SPMV_OP_NON,
    _normalize_spmv_op,
    _spmv_op_to_name,
    _spmv_op_transposes,
    flagsparse_spmv_csr,
    prepare_spmv_csr,
)

try:  # optional, as in FlagSparse: the cuSPARSE leg needs CuPy
    import cupy as cp
    import cupyx.scipy.sparse as cpx_sparse
except Exception:  # pragma: no cover - CuPy is absent on the test machines
    cp = None
    cpx_sparse = None

_CUPY_DTYPES = (torch.float32, torch.float64, torch.complex64, torch.complex128)
_NO_CUPY = "CuPy/cuSPARSE is not available"


def _wide(dtype):
    """Reference precision: float32 -> float64, complex64 -> complex128, half
    types -> float32, others unchanged."""
    if dtype == torch.float32:
        return torch.float64
    if dtype == torch.complex64:
        return torch.complex128
    if dtype in (torch.float16, torch.bfloat16):
        return torch.float32
    return dtype


def _csr_reference(data, indices, indptr, shape, dtype):
    return torch.sparse_csr_tensor(indptr.to(torch.int64), indices.to(torch.int64), data.to(dtype), size=shape,
                                   device=data.device)


def _cupy_csr(data, indices, indptr, shape):
    return cpx_sparse.csr_matrix((cp.asarray(data), cp.asarray(indices.to(torch.int64)), cp.asarray(indptr)),
                                 shape=shape)


def _first_call_ms(fn):
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fn()
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) * 1000.0


def benchmark_spmv_case(n_rows=4096, n_cols=4096, nnz=65536, value_dtype=torch.float32, index_dtype=torch.int32,
                        warmup=20, iters=200, block_nnz=256, max_segments=None, run_cusparse=True, transpose=False,
                        op=None, index_fallback_policy="auto"):
    """CSR SpMV (``flagsparse_spmv_csr`` on a prepared matrix) against a
    PyTorch sparse reference and, with CuPy, cuSPARSE."""
    device = torch.device("cuda")
    data, indices, indptr = _build_random_csr(n_rows, n_cols, nnz, value_dtype, index_dtype, device)
    op_code = _normalize_spmv_op(op, transpose=transpose)
    if op is not None and bool(transpose) and op_code == SPMV_OP_NON:
        raise ValueError("transpose=True conflicts with op=non")
    transpose = _spmv_op_transposes(op_code)
    x_size, y_size = (n_rows, n_cols) if transpose else (n_cols, n_rows)
    x = _build_random_dense(x_size, value_dtype, device)
    shape = (n_rows, n_cols)
    prepared = prepare_spmv_csr(data, indices, indptr, shape, block_nnz=block_nnz, max_segments=max_segments,
                                op=op_code, index_fallback_policy=index_fallback_policy)
    ours_y, ours_ms = _benchmark_cuda_op(lambda: flagsparse_spmv_csr(x=x, prepared=prepared, return_time=False),
                                         warmup=warmup, iters=iters)
    # reference: the same operator as a COO product on a wider copy, rounded
    # to the value type
    ref_dtype = _wide(value_dtype)
    rows = torch.repeat_interleave(torch.arange(n_rows, device=device, dtype=torch.int64),
                                   (indptr[1:] - indptr[:-1]).to(torch.int64))
    cols = indices.to(torch.int64)
    vals = data.to(ref_dtype)
    if transpose:
        rows, cols = cols, rows
        if _spmv_op_to_name(op_code) == "conj":
            vals = vals.conj()
    A = torch.sparse_coo_tensor(torch.stack([rows, cols]), vals, (y_size, x_size), device=device).coalesce()
    expected = torch.sparse.mm(A, x.to(ref_dtype).unsqueeze(1)).squeeze(1).to(value_dtype)
    atol, rtol = _tolerance_for_dtype(value_dtype)
    match = bool(torch.allclose(ours_y, expected, atol=atol, rtol=rtol))
    max_err = float(torch.max(torch.abs(ours_y - expected)).item()) if y_size > 0 else 0.0
    cu_ms = cu_match = cu_err = None
    cu_reason = None
    if run_cusparse:
        if cp is None or cpx_sparse is None:
            cu_reason = _NO_CUPY
        elif value_dtype not in _CUPY_DTYPES:
            cu_reason = "float16/bfloat16 not supported by CuPy sparse; skipped"
        else:
            try:
                M = _cupy_csr(data, indices, indptr, shape)
                if op_code != SPMV_OP_NON:
                    M = M.T.conj() if _spmv_op_to_name(op_code) == "conj" else M.T
                cu_vals, cu_ms = _benchmark_cuda_op(lambda: torch.as_tensor(M @ cp.asarray(x), device=device),
                                                    warmup=warmup, iters=iters)
                cu_match = bool(torch.allclose(cu_vals, expected, atol=atol, rtol=rtol))
                cu_err = float(torch.max(torch.abs(cu_vals - expected)).item()) if y_size > 0 else 0.0
            except Exception as exc:  # noqa: BLE001 - reported like FlagSparse does
                cu_reason = str(exc)
    return {
        "parameters": {"n_rows": n_rows, "n_cols": n_cols, "nnz": nnz, "value_dtype": str(value_dtype),
                       "index_dtype": str(index_dtype), "op": _spmv_op_to_name(op_code), "transpose": transpose,
                       "index_fallback_policy": str(index_fallback_policy).lower(), "warmup": warmup,
                       "iters": iters},
        "performance": {"triton_ms": ours_ms, "cusparse_ms": cu_ms,
                        "triton_speedup_vs_cusparse": (cu_ms / ours_ms if cu_ms is not None and ours_ms > 0
                                                       else None)},
        "verification": {"triton_match_reference": match, "triton_max_error": max_err,
                         "cusparse_match_reference": cu_match, "cusparse_max_error": cu_err},
        "backend_status": {"cusparse_unavailable_reason": cu_reason},
        "samples": {"triton": ours_y, "reference": expected},
    }


def benchmark_spmm_case(n_rows=4096, n_cols=4096, nnz=65536, n_dense_cols=32, value_dtype=torch.float32,
                        index_dtype=torch.int32, warmup=20, iters=200, block_n=None, block_nnz=None,
                        max_segments=None, run_cusparse=True):
    """CSR SpMM, ALG1 (``flagsparse_spmm_csr``), against PyTorch
    ``sparse.mm`` and, with CuPy, cuSPARSE."""
    device = torch.device("cuda")
    data, indices, indptr = _build_random_csr(n_rows, n_cols, nnz, value_dtype, index_dtype, device)
    B = _build_random_dense((n_cols, n_dense_cols), value_dtype, device)
    shape = (n_rows, n_cols)
    max_row_nnz = int(torch.max(indptr[1:] - indptr[:-1]).item()) if n_rows > 0 else 0
    launch = _resolve_spmm_alg1_launch_config(n_dense_cols, max_row_nnz, block_n=block_n, block_nnz=block_nnz,
                                              max_segments=max_segments)
    kwargs = {"data": data, "indices": indices, "indptr": indptr, "B": B, "shape": shape,
              "block_n": launch["block_n"], "block_nnz": launch["block_nnz"],
              "max_segments": launch["max_segments"], "return_time": False}
    first_ms = _first_call_ms(lambda: flagsparse_spmm_csr(**kwargs))
    ours_C, ours_ms = _benchmark_cuda_op(lambda: flagsparse_spmm_csr(**kwargs), warmup=warmup, iters=iters)
    # PyTorch: the CSR product timed in the value type; the reference is the
    # same product on a wider copy, rounded to the value type (COO when CSR
    # is refused for this dtype)
    pt_reason, pt_format, pt_ms = None, "CSR", None
    try:
        pt_A = _csr_reference(data, indices, indptr, shape, value_dtype)
        ref_A = _csr_reference(data, indices, indptr, shape, _wide(value_dtype))
        expected = torch.sparse.mm(ref_A, B.to(_wide(value_dtype))).to(value_dtype)
    except Exception as exc:  # noqa: BLE001 - reported like FlagSparse does
        pt_format, pt_reason = "COO", f"CSR fallback: {exc}"
        rows = torch.repeat_interleave(torch.arange(n_rows, device=device, dtype=torch.int64),
                                       (indptr[1:] - indptr[:-1]).to(torch.int64))
        pt_A = torch.sparse_coo_tensor(torch.stack([rows, indices.to(torch.int64)]), data, shape,
                                       device=device).coalesce()
        expected = torch.sparse.mm(pt_A.to(_wide(value_dtype)), B.to(_wide(value_dtype))).to(value_dtype)
    pt_values = expected
    try:
        pt_values, pt_ms = _benchmark_cuda_op(lambda: torch.sparse.mm(pt_A, B), warmup=warmup, iters=iters)
    except Exception as exc:  # noqa: BLE001
        pt_reason = str(exc) if pt_reason is None else f"{pt_reason}; timing: {exc}"
    ours = _spmm_validation_metrics(ours_C, expected)
    cu_ms = cu_reason = cu_metrics = None
    if run_cusparse:
        if cp is None or cpx_sparse is None:
            cu_reason = _NO_CUPY
        elif value_dtype not in _CUPY_DTYPES:
            cu_reason = "float16/bfloat16 not supported by CuPy sparse; skipped"
        else:
            try:
                M = _cupy_csr(data, indices, indptr, shape)
                Bc = cp.asarray(B)
                cu_vals, cu_ms = _benchmark_cuda_op(lambda: M @ Bc, warmup=warmup, iters=iters)
                cu_metrics = _spmm_validation_metrics(torch.as_tensor(cu_vals, device=device), expected)
            except Exception as exc:  # noqa: BLE001
                cu_reason = str(exc)
    threshold = _spmm_relative_threshold(value_dtype)
    cu = (lambda k: cu_metrics[k] if cu_metrics is not None else None)
    return {
        "parameters": {"format": "csr", "n_rows": n_rows, "n_cols": n_cols, "nnz": nnz,
                       "n_dense_cols": n_dense_cols, "value_dtype": str(value_dtype),
                       "index_dtype": str(index_dtype), "warmup": warmup, "iters": iters,
                       "block_n": launch["block_n"], "block_nnz": launch["block_nnz"],
                       "max_segments": launch["max_segments"], "required_segments": launch["required_segments"],
                       "alg1_warp_size": launch["warp_size"], "alg1_factor": launch["factor"],
                       "auto_max_segments": launch["auto_max_segments"], "run_cusparse": run_cusparse},
        "performance": {"pytorch_ms": pt_ms, "triton_ms": ours_ms, "triton_first_call_ms": first_ms,
                        "cusparse_ms": cu_ms,
                        "triton_speedup_vs_pytorch": pt_ms / ours_ms if pt_ms is not None and ours_ms > 0 else None,
                        "triton_speedup_vs_cusparse": cu_ms / ours_ms if cu_ms is not None and ours_ms > 0 else None},
        "verification": {
            "triton_match_reference": ours["strict_allclose_match"],
            "triton_match_pytorch": ours["strict_allclose_match"],
            "triton_max_error": ours["max_abs_error"], "triton_max_abs_error": ours["max_abs_error"],
            "triton_max_relative_error": ours["max_relative_error"],
            "triton_sum_relative_error": ours["sum_relative_error"],
            "triton_relative_threshold": ours["relative_threshold"],
            "triton_strict_allclose_match": ours["strict_allclose_match"],
            "pytorch_match_reference": True, "pytorch_max_error": 0.0, "pytorch_max_abs_error": 0.0,
            "pytorch_max_relative_error": 0.0, "pytorch_sum_relative_error": 0.0,
            "pytorch_relative_threshold": threshold,
            "cusparse_match_reference": cu("strict_allclose_match"),
            "cusparse_match_pytorch": cu("strict_allclose_match"),
            "cusparse_max_error": cu("max_abs_error"), "cusparse_max_abs_error": cu("max_abs_error"),
            "cusparse_max_relative_error": cu("max_relative_error"),
            "cusparse_sum_relative_error": cu("sum_relative_error"),
            "cusparse_relative_threshold": cu("relative_threshold") if cu_metrics is not None else threshold,
            "cusparse_strict_allclose_match": cu("strict_allclose_match"),
        },
        "backend_status": {"pytorch_unavailable_reason": pt_reason, "pytorch_sparse_format": pt_format,
                           "cusparse_unavailable_reason": cu_reason, "flagsparse_internal_route": "csr-alg1"},
        "samples": {"pytorch": pt_values, "triton": ours_C},
    }


def benchmark_spmm_opt_case(n_rows=4096, n_cols=4096, nnz=65536, n_dense_cols=32, value_dtype=torch.float32,
                            index_dtype=torch.int32, warmup=20, iters=200, run_cusparse=True):
    """CSR SpMM, ALG1 against opt, both against a float64 PyTorch reference
    (error in units of FlagSparse's COO tolerance: at most 1 passes)."""
    if value_dtype not in (torch.float32, torch.float64):
        raise TypeError("benchmark_spmm_opt_case only supports float32 and float64")
    device = torch.device("cuda")
    data, indices, indptr = _build_random_csr(n_rows, n_cols, nnz, value_dtype, index_dtype, device)
    B = _build_random_dense((n_cols, n_dense_cols), value_dtype, device)
    shape = (n_rows, n_cols)
    prepared = prepare_spmm_csr_opt(data, indices, indptr, shape)
    base_first = _first_call_ms(lambda: flagsparse_spmm_csr(data, indices, indptr, B, shape))
    base_values, base_ms = _benchmark_cuda_op(lambda: flagsparse_spmm_csr(data, indices, indptr, B, shape),
                                              warmup=warmup, iters=iters)
    opt_first = _first_call_ms(lambda: flagsparse_spmm_csr_opt(B=B, prepared=prepared))
    opt_values, opt_ms = _benchmark_cuda_op(lambda: flagsparse_spmm_csr_opt(B=B, prepared=prepared),
                                            warmup=warmup, iters=iters)
    ref = torch.sparse.mm(_csr_reference(data, indices, indptr, shape, _wide(value_dtype)),
                          B.to(_wide(value_dtype))).to(value_dtype)
    pt_ms = None
    try:
        pt_A = _csr_reference(data, indices, indptr, shape, value_dtype)
        _, pt_ms = _benchmark_cuda_op(lambda: torch.sparse.mm(pt_A, B), warmup=warmup, iters=iters)
    except Exception:  # noqa: BLE001
        pt_ms = None
    cu_ms = None
    if run_cusparse and cp is not None and cpx_sparse is not None:
        try:
            M, Bc = _cupy_csr(data, indices, indptr, shape), cp.asarray(B)
            _, cu_ms = _benchmark_cuda_op(lambda: M @ Bc, warmup=warmup, iters=iters)
        except Exception:  # noqa: BLE001
            cu_ms = None
    err_base = _spmm_opt_reference_error(base_values, ref, value_dtype)
    err_opt = _spmm_opt_reference_error(opt_values, ref, value_dtype)
    return {
        "parameters": {"n_rows": n_rows, "n_cols": n_cols, "nnz": nnz, "n_dense_cols": n_dense_cols,
                       "value_dtype": str(value_dtype), "index_dtype": str(index_dtype)},
        "performance": {"base_ms": base_ms, "base_first_call_ms": base_first, "opt_ms": opt_ms,
                        "opt_first_call_ms": opt_first, "pt_ms": pt_ms, "cu_ms": cu_ms,
                        "opt_vs_base": base_ms / opt_ms if opt_ms and opt_ms > 0 else None,
                        "opt_vs_pt": pt_ms / opt_ms if pt_ms is not None and opt_ms > 0 else None,
                        "opt_vs_cu": cu_ms / opt_ms if cu_ms is not None and opt_ms > 0 else None},
        "verification": {"err_base": err_base, "err_opt": err_opt, "base_ok": err_base <= 1.0,
                         "opt_ok": err_opt <= 1.0, "status": "PASS" if err_opt <= 1.0 else "FAIL"},
        "backend_status": {"long_row_fallback_used": bool(prepared.long_row_fallback_only),
                           "flagsparse_internal_route": "csr-opt-bucketed"},
        "samples": {"base": base_values, "opt": opt_values, "reference": ref},
    }


def benchmark_spmm_opt_alg2_case(n_rows=4096, n_cols=4096, nnz=65536, n_dense_cols=32, value_dtype=torch.float32,
                                 index_dtype=torch.int32, warmup=20, iters=200, run_cusparse=True):
    """CSR SpMM: ALG1, opt and opt-alg2 against a float64 PyTorch reference
    and, with CuPy, cuSPARSE's result."""
    if value_dtype not in SUPPORTED_SPMM_OPT_ALG2_DTYPES:
        raise TypeError("benchmark_spmm_opt_alg2_case only supports float32 and float64")
    device = torch.device("cuda")
    data, indices, indptr = _build_random_csr(n_rows, n_cols, nnz, value_dtype, index_dtype, device)
    B = _build_random_dense((n_cols, n_dense_cols), value_dtype, device)
    shape = (n_rows, n_cols)
    prepared_opt = prepare_spmm_csr_opt(data, indices, indptr, shape)
    prepared_alg2 = prepare_spmm_csr_opt_alg2(data, indices, indptr, shape)
    base_values, base_ms = _benchmark_cuda_op(lambda: flagsparse_spmm_csr(data, indices, indptr, B, shape),
                                              warmup=warmup, iters=iters)
    opt_values, opt_ms = _benchmark_cuda_op(lambda: flagsparse_spmm_csr_opt(B=B, prepared=prepared_opt),
                                            warmup=warmup, iters=iters)
    alg2_values, alg2_ms = _benchmark_cuda_op(lambda: flagsparse_spmm_csr_opt_alg2(B=B, prepared=prepared_alg2),
                                              warmup=warmup, iters=iters)
    torch_ref = torch.sparse.mm(_csr_reference(data, indices, indptr, shape, _wide(value_dtype)),
                                B.to(_wide(value_dtype))).to(value_dtype)
    torch_ms = None
    try:
        pt_A = _csr_reference(data, indices, indptr, shape, value_dtype)
        _, torch_ms = _benchmark_cuda_op(lambda: torch.sparse.mm(pt_A, B), warmup=warmup, iters=iters)
    except Exception:  # noqa: BLE001
        torch_ms = None
    cu_ref = cu_ms = cu_reason = None
    if run_cusparse:
        if cp is None or cpx_sparse is None:
            cu_reason = _NO_CUPY
        else:
            try:
                M, Bc = _cupy_csr(data, indices, indptr, shape), cp.asarray(B)
                cu_vals, cu_ms = _benchmark_cuda_op(lambda: M @ Bc, warmup=warmup, iters=iters)
                cu_ref = torch.as_tensor(cu_vals, device=device)
            except Exception as exc:  # noqa: BLE001
                cu_reason = str(exc)
    err = lambda v, r: _spmm_opt_alg2_reference_error(v, r, value_dtype) if r is not None else None  # noqa: E731
    return {
        "parameters": {"n_rows": n_rows, "n_cols": n_cols, "nnz": nnz, "n_dense_cols": n_dense_cols,
                       "value_dtype": str(value_dtype), "index_dtype": str(index_dtype)},
        "performance": {"base_ms": base_ms, "opt_ms": opt_ms, "opt_alg2_ms": alg2_ms, "torch_ms": torch_ms,
                        "cusparse_ms": cu_ms},
        "verification": {"base_vs_torch_err": err(base_values, torch_ref),
                         "opt_vs_torch_err": err(opt_values, torch_ref),
                         "opt_alg2_vs_torch_err": err(alg2_values, torch_ref),
                         "base_vs_cusparse_err": err(base_values, cu_ref),
                         "opt_vs_cusparse_err": err(opt_values, cu_ref),
                         "opt_alg2_vs_cusparse_err": err(alg2_values, cu_ref)},
        "backend_status": {"cusparse_unavailable_reason": cu_reason},
        "samples": {"base_triton": base_values, "opt_triton": opt_values, "opt_alg2_triton": alg2_values,
                    "torch_ref": torch_ref, "cusparse_ref": cu_ref},
    }


def _sampled_dot(indices, indptr, x, y, data, alpha, beta):
    """PyTorch SDDMM reference: alpha * <x[row(p)], y[col(p)]> + beta * data[p]
    for every stored position p (a gather of both rows and a row-wise dot)."""
    rows = torch.repeat_interleave(torch.arange(indptr.numel() - 1, device=x.device, dtype=torch.int64),
                                   indptr[1:] - indptr[:-1])
    out = alpha * (x.index_select(0, rows) * y.index_select(0, indices.to(torch.int64))).sum(dim=1)
    if data is not None and beta != 0.0:
        out = out + beta * data
    return out


def benchmark_sddmm_case(n_rows=1024, n_cols=1024, nnz=16384, k_dim=64, value_dtype=torch.float32, warmup=10,
                         iters=30, alpha=1.0, beta=0.0, run_cusparse=False):
    """CSR SDDMM (``flagsparse_sddmm_csr`` on a prepared pattern) against a
    PyTorch sampled-dot reference (sddmm_csr.py:472-568)."""
    from .sddmm_csr import SUPPORTED_SDDMM_VALUE_DTYPES, flagsparse_sddmm_csr, prepare_sddmm_csr

    if value_dtype not in SUPPORTED_SDDMM_VALUE_DTYPES:
        raise TypeError("value_dtype must be torch.float32 or torch.float64")
    device = torch.device("cuda")
    data, indices, indptr = _build_random_csr(n_rows, n_cols, nnz, value_dtype, torch.int32, device)
    x = _build_random_dense((n_rows, k_dim), value_dtype, device)
    y = _build_random_dense((n_cols, k_dim), value_dtype, device)
    prepared = prepare_sddmm_csr(indices, indptr, (n_rows, n_cols), k_hint=k_dim)
    ours, ours_ms = _benchmark_cuda_op(
        lambda: flagsparse_sddmm_csr(data=data, x=x, y=y, alpha=alpha, beta=beta, prepared=prepared,
                                     return_time=False), warmup=warmup, iters=iters)
    ip64 = indptr.to(torch.int64)
    ref, pt_ms = _benchmark_cuda_op(lambda: _sampled_dot(indices, ip64, x, y, data, alpha, beta), warmup=warmup,
                                    iters=iters)
    atol, rtol = _tolerance_for_dtype(value_dtype)
    match = bool(torch.allclose(ours, ref, atol=atol, rtol=rtol))
    max_abs = float(torch.max(torch.abs(ours - ref)).item()) if ours.numel() > 0 else 0.0
    cu_ms = cu_reason = cu_match = None
    if run_cusparse:
        if cp is None:
            cu_reason = "CuPy is not available"
        else:
            try:
                def cupy_sampled_dot():
                    xs = cp.asarray(x)[cp.asarray(torch.repeat_interleave(
                        torch.arange(n_rows, device=device), ip64[1:] - ip64[:-1]))]
                    ys = cp.asarray(y)[cp.asarray(indices.to(torch.int64))]
                    v = alpha * (xs * ys).sum(axis=1)
                    return torch.as_tensor(v + beta * cp.asarray(data) if beta != 0.0 else v, device=device)

                ref_cu, cu_ms = _benchmark_cuda_op(cupy_sampled_dot, warmup=warmup, iters=iters)
                cu_match = bool(torch.allclose(ours, ref_cu, atol=atol, rtol=rtol))
            except Exception as exc:  # noqa: BLE001
                cu_reason = str(exc)
    return {
        "parameters": {"n_rows": n_rows, "n_cols": n_cols, "nnz": nnz, "k_dim": k_dim,
                       "value_dtype": str(value_dtype), "warmup": warmup, "iters": iters, "alpha": alpha,
                       "beta": beta},
        "performance": {"triton_ms": ours_ms, "pytorch_ms": pt_ms, "cusparse_ms": cu_ms,
                        "triton_speedup_vs_pytorch": pt_ms / ours_ms if ours_ms > 0 else None,
                        "triton_speedup_vs_cusparse": cu_ms / ours_ms if (cu_ms and ours_ms > 0) else None},
        "verification": {"triton_match_pytorch": match, "triton_max_abs_error": max_abs,
                         "cusparse_match_pytorch": cu_match},
        "backend_status": {"cusparse_unavailable_reason": cu_reason},
        "samples": {"triton": ours, "pytorch": ref},
    }
