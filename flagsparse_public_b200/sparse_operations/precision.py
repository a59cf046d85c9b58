"""Precision form of CSR SpMV / SpMM: half-precision storage, float32 results.

Values and the dense operand are stored in bfloat16 or float16 (half the
bytes of the float32 form), products are accumulated in float32 and written
as float32.  Rows longer than ``compensate_above`` nonzeros (4096 by default)
accumulate with error-free transformations -- TwoProduct by fused multiply-add
and TwoSum (Ogita, Rump & Oishi, "Accurate sum and dot product", SIAM J. Sci.
Comput. 26(6), 2005: the Dot2 algorithm) -- so their result is as accurate as
a float64 accumulation rounded to float32.

FlagSparse's own operators compute half types in float32 and round the result
back to the half type (``spmv_csr.py:116-117``); this form keeps float32
output.  ``return_error=True`` states the result's condition-scaled error
against a float64 product of the same half-precision inputs:
max |y - y64| / sum_k |a_k x_k|.
"""

from ._common import *
from .. import _native as _nat
from .. import _plan
from .. import _structured
from .spmv_csr import _prepare_spmv_csr_matrix

MIXED_VALUE_DTYPES = (torch.bfloat16, torch.float16)
COMPENSATE_ABOVE = 4096
LAYOUTS = ("auto", "csr", "structured")


class PreparedCsrMixed:
    """Validated half-precision CSR, its cached launch plans and (layout
    "auto" / "structured") its structured form."""

    __slots__ = ("data", "kernel_indices", "kernel_indptr", "shape", "n_rows", "n_cols", "max_row_nnz",
                 "compensate_above", "layout", "_stats", "_plans", "_struct")

    def __init__(self, data, kernel_indices, kernel_indptr, shape, n_rows, n_cols, max_row_nnz, compensate_above,
                 layout="auto"):
        self.data = data
        self.kernel_indices = kernel_indices
        self.kernel_indptr = kernel_indptr
        self.shape = (int(shape[0]), int(shape[1]))
        self.n_rows = int(n_rows)
        self.n_cols = int(n_cols)
        self.max_row_nnz = int(max_row_nnz)
        self.compensate_above = int(compensate_above)
        self.layout = layout
        self._stats = None
        self._plans = {}
        self._struct = None


def prepare_csr_mixed(data, indices, indptr, shape, compensate_above=COMPENSATE_ABOVE, layout="auto"):
    """Validate a bfloat16 / float16 CSR matrix for the precision form.

    ``layout``: "csr" runs the products on the CSR kernels; "structured" on the
    structured form (runs of consecutive columns on the tensor cores, long
    rows in compensated chunks); "auto" builds the structured form and uses it
    when runs and long rows hold at least half of the nonzeros."""
    if torch.is_tensor(data) and data.dtype not in MIXED_VALUE_DTYPES:
        raise TypeError("precision form needs bfloat16 or float16 values")
    if int(compensate_above) < 0:
        raise ValueError("compensate_above must be non-negative")
    if layout not in LAYOUTS:
        raise ValueError(f"layout must be one of {LAYOUTS}")
    data, kidx, kptr, n_rows, n_cols, _lens, max_row, stats = _prepare_spmv_csr_matrix(data, indices, indptr, shape,
                                                                                        return_stats=True)
    p = PreparedCsrMixed(data, kidx, kptr, shape, n_rows, n_cols, max_row, compensate_above, layout)
    p._stats = stats
    if layout != "csr":
        _structured_form(p)
    return p


def _structured_form(prepared):
    """The structured form when this matrix runs on it, else None.  Rows of
    more than the structured form's long-row threshold accumulate compensated
    there, so a compensation threshold below it keeps the CSR kernels."""
    if prepared._struct is None:
        use = False
        if prepared.layout != "csr" and prepared.n_rows > 0 and prepared.compensate_above >= _structured.LONG_MIN:
            form = _structured.build(prepared.data, prepared.kernel_indices, prepared.kernel_indptr,
                                     prepared.n_rows, prepared.n_cols)
            use = form if (prepared.layout == "structured" or form.worthwhile()) else False
        prepared._struct = use
    return prepared._struct or None


def _stats(prepared):
    if prepared._stats is None:
        prepared._stats = _plan.matrix_stats(prepared.kernel_indptr, prepared.n_rows, prepared.n_cols)
    return prepared._stats


def _acc_mode(prepared):
    # compensation only matters when some row is longer than the threshold
    return _nat.ACC_COMP if prepared.max_row_nnz > prepared.compensate_above else _nat.ACC_NATIVE


def _mixed_plan(prepared, kind, n_dense=0, operands=None):
    """Cached plan per (kind, width); SpMM plans go through the plan selector
    when the operands (B, C) are given."""
    key = (kind, int(n_dense))
    plan = prepared._plans.get(key)
    if plan is None:
        st = _stats(prepared)
        if kind == "spmv":
            plan = _plan.default_spmv_plan(st, prepared.data.dtype)
        elif operands is not None:
            B, C = operands
            plan = _plan.chosen_spmm_plan(st, prepared.data, prepared.kernel_indices, prepared.kernel_indptr,
                                          prepared.n_rows, prepared.n_cols, B, C, _acc_mode(prepared))
        else:
            plan = _plan.default_spmm_plan(st, n_dense, prepared.data.dtype)
        plan.comp_threshold = prepared.compensate_above
        prepared._plans[key] = plan
    return plan


def _resolve(data, indices, indptr, shape, prepared, compensate_above, layout="auto"):
    if prepared is None:
        if any(a is None for a in (data, indices, indptr, shape)):
            raise ValueError("data, indices, indptr, and shape are required when prepared is not provided")
        # a one-shot call runs one product: building the structured form costs
        # more than it saves, so "auto" keeps the CSR kernels here
        layout = "csr" if layout == "auto" else layout
        prepared = prepare_csr_mixed(data, indices, indptr, shape, compensate_above=compensate_above, layout=layout)
    elif not isinstance(prepared, PreparedCsrMixed):
        raise TypeError("prepared must be a PreparedCsrMixed instance")
    return prepared


def _check_dense(t, name, prepared, ndim):
    if t is None or not torch.is_tensor(t):
        raise TypeError(f"{name} must be a torch.Tensor")
    if t.ndim != ndim:
        raise ValueError(f"{name} must be a {ndim}D tensor")
    if not t.is_cuda or t.device != prepared.data.device:
        raise ValueError(f"{name} must be a CUDA tensor on the sparse matrix's device")
    if t.dtype != prepared.data.dtype:
        raise TypeError(f"{name} dtype must match sparse matrix dtype")
    if t.shape[0] != prepared.n_cols:
        raise ValueError(f"{name}.shape[0] must be n_cols={prepared.n_cols}, got {t.shape[0]}")
    return t.contiguous()


def _error_vs_fp64(prepared, dense, result):
    a64 = torch.sparse_csr_tensor(prepared.kernel_indptr.to(torch.int64), prepared.kernel_indices.to(torch.int64),
                                  prepared.data.to(torch.float64), size=prepared.shape)
    d64 = dense.to(torch.float64)
    exact = (a64 @ d64) if dense.ndim == 2 else (a64 @ d64.unsqueeze(1)).squeeze(1)
    aabs = torch.sparse_csr_tensor(prepared.kernel_indptr.to(torch.int64), prepared.kernel_indices.to(torch.int64),
                                   prepared.data.to(torch.float64).abs(), size=prepared.shape)
    mag = (aabs @ d64.abs()) if dense.ndim == 2 else (aabs @ d64.abs().unsqueeze(1)).squeeze(1)
    diff = (result.to(torch.float64) - exact).abs()
    err = torch.where(mag > 0, diff / mag, diff)
    return float(err.max().item()) if err.numel() else 0.0


def flagsparse_spmv_csr_mixed(data=None, indices=None, indptr=None, x=None, shape=None, prepared=None, out=None,
                              compensate_above=COMPENSATE_ABOVE, return_time=False, return_error=False, layout="auto"):
    """y = A x with half-precision A and x, float32 accumulation and result."""
    prepared = _resolve(data, indices, indptr, shape, prepared, compensate_above, layout)
    x = _check_dense(x, "x", prepared, 1)
    if out is not None and (out.dtype != torch.float32 or out.shape != (prepared.n_rows,) or not out.is_contiguous()
                            or out.device != prepared.data.device):
        raise ValueError("out must be a contiguous float32 CUDA tensor of shape (n_rows,)")
    y = out if out is not None else torch.empty(prepared.n_rows, dtype=torch.float32, device=prepared.data.device)
    t0 = None
    if return_time:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
    if prepared.n_rows:
        form = _structured_form(prepared)
        if form is not None:
            _structured.spmv(form, prepared.data, prepared.kernel_indices, prepared.kernel_indptr, prepared.n_rows,
                             prepared.n_cols, x, y)
        else:
            _plan.run_spmv(prepared.data, prepared.kernel_indices, prepared.kernel_indptr, prepared.n_rows,
                           prepared.n_cols, x, y, _acc_mode(prepared), _mixed_plan(prepared, "spmv"))
    res = [y]
    if return_time:
        torch.cuda.synchronize()
        res.append((time.perf_counter() - t0) * 1000.0)
    if return_error:
        res.append(_error_vs_fp64(prepared, x, y))
    return res[0] if len(res) == 1 else tuple(res)


def flagsparse_spmm_csr_mixed(data=None, indices=None, indptr=None, B=None, shape=None, prepared=None, out=None,
                              compensate_above=COMPENSATE_ABOVE, return_time=False, return_error=False, layout="auto"):
    """C = A B with half-precision A and B (row-major), float32 accumulation and result."""
    prepared = _resolve(data, indices, indptr, shape, prepared, compensate_above, layout)
    B = _check_dense(B, "B", prepared, 2)
    n_dense = int(B.shape[1])
    if out is not None and (out.dtype != torch.float32 or out.shape != (prepared.n_rows, n_dense)
                            or not out.is_contiguous() or out.device != prepared.data.device):
        raise ValueError("out must be a contiguous float32 CUDA tensor of shape (n_rows, n_dense)")
    C = out if out is not None else torch.empty((prepared.n_rows, n_dense), dtype=torch.float32,
                                                device=prepared.data.device)
    t0 = None
    if return_time:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
    if prepared.n_rows and n_dense:
        form = _structured_form(prepared)
        if form is not None and _structured.spmm_supported(form, B, C):
            _structured.spmm(form, prepared.data, prepared.kernel_indices, prepared.kernel_indptr, prepared.n_rows,
                             prepared.n_cols, B, C)
        else:
            _plan.run_spmm(prepared.data, prepared.kernel_indices, prepared.kernel_indptr, prepared.n_rows,
                           prepared.n_cols, B, C, _acc_mode(prepared), _mixed_plan(prepared, "spmm", n_dense, (B, C)))
    res = [C]
    if return_time:
        torch.cuda.synchronize()
        res.append((time.perf_counter() - t0) * 1000.0)
    if return_error:
        res.append(_error_vs_fp64(prepared, B, C))
    return res[0] if len(res) == 1 else tuple(res)
