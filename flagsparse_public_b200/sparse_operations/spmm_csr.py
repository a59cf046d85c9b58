"""CSR SpMM: FlagSparse's ``spmm_csr`` operator API on sm_100a kernels.

Public names, defaults, exception types and messages follow FlagSparse
``sparse_operations/spmm_csr.py``: ``flagsparse_spmm_csr`` (ALG1,
:2088-2157), ``prepare_spmm_csr_opt`` / ``flagsparse_spmm_csr_opt``
(:480-522, :2160-2214), the ``PreparedCsrSpmmOpt`` slots (:337-392) and the
error-metric helpers (:6-90).  Products run in ``libflagsparse_b200.so``:
row-group kernels for even row lengths, merge-path kernels (rows + nonzeros
balanced, split rows finished from per-unit carries) for skewed ones.

Numerics kept from the reference: ALG1 accumulates float32 in float64 and
float16/bfloat16 in float32 (``:544-551``) -- in registers, with no widened
copies of A and B; the opt path accumulates in the value precision (``:631``).
"""

import math

from ._common import *
from .. import _native as _nat
from .. import _plan

SUPPORTED_SPMM_VALUE_DTYPES = SUPPORTED_VALUE_DTYPES


def _spmm_relative_threshold(value_dtype):
    if value_dtype == torch.float16:
        return 5e-3
    if value_dtype == torch.bfloat16:
        return 1e-2
    if value_dtype in (torch.float32, torch.complex64):
        return 1e-6
    if value_dtype in (torch.float64, torch.complex128):
        return 1e-12
    return 1e-6


def _spmm_coo_reference_tolerance(value_dtype):
    if value_dtype == torch.float16:
        return 2e-3, 2e-3
    if value_dtype == torch.bfloat16:
        return 1e-1, 1e-1
    if value_dtype in (torch.float32, torch.complex64):
        return 1e-4, 1e-2
    if value_dtype in (torch.float64, torch.complex128):
        return 1e-12, 1e-10
    return 1e-6, 1e-5


def _spmm_error_metrics(candidate, reference):
    if candidate.shape != reference.shape:
        raise ValueError(
            f"candidate and reference must have the same shape, got {candidate.shape} vs {reference.shape}"
        )
    if candidate.numel() == 0:
        return {
            "max_abs_error": 0.0,
            "max_relative_error": 0.0,
            "sum_relative_error": 0.0,
            "reference_max_magnitude": 0.0,
            "reference_sum_magnitude": 0.0,
        }
    if _is_complex_dtype(reference.dtype):
        reference_compare = torch.abs(reference)
        abs_diff = torch.abs(torch.abs(candidate) - reference_compare)
    else:
        reference_compare = torch.abs(reference)
        abs_diff = torch.abs(candidate - reference)
    max_abs_error = float(torch.max(abs_diff).item())
    reference_max_magnitude = float(torch.max(reference_compare).item())
    sum_abs_error = float(torch.sum(abs_diff).item())
    reference_sum_magnitude = float(torch.sum(reference_compare).item())
    if reference_max_magnitude == 0.0:
        max_relative_error = 0.0 if max_abs_error == 0.0 else float("inf")
    else:
        max_relative_error = max_abs_error / reference_max_magnitude
    if reference_sum_magnitude == 0.0:
        sum_relative_error = 0.0 if sum_abs_error == 0.0 else float("inf")
    else:
        sum_relative_error = sum_abs_error / reference_sum_magnitude
    return {
        "max_abs_error": max_abs_error,
        "max_relative_error": max_relative_error,
        "sum_relative_error": sum_relative_error,
        "reference_max_magnitude": reference_max_magnitude,
        "reference_sum_magnitude": reference_sum_magnitude,
    }


def _spmm_validation_metrics(candidate, reference):
    metrics = _spmm_error_metrics(candidate, reference)
    threshold = _spmm_relative_threshold(reference.dtype)
    atol, rtol = _tolerance_for_dtype(reference.dtype)
    metrics.update({
        "relative_threshold": threshold,
        "matches_threshold": metrics["max_relative_error"] <= threshold,
        "strict_allclose_match": torch.allclose(candidate, reference, atol=atol, rtol=rtol),
    })
    return metrics


def _prepare_spmm_csr_matrix(data, indices, indptr, shape, return_stats=False):
    """Validation of FlagSparse ``spmm_csr.py:197-255`` with one kernel and
    one device->host read for all structural checks.  Returns int32 column indices (int64 ones
    converted, as the reference does) and int64 indptr; with ``return_stats``
    also the row-length statistics of the plan heuristics, from the same read."""
    if len(shape) != 2:
        raise ValueError("shape must be a 2-tuple: (n_rows, n_cols)")
    if data.ndim != 1 or indices.ndim != 1 or indptr.ndim != 1:
        raise ValueError("data, indices, and indptr must be 1D tensors")
    n_rows, n_cols = int(shape[0]), int(shape[1])
    if n_rows < 0 or n_cols < 0:
        raise ValueError("shape dimensions must be non-negative")
    if indptr.numel() != n_rows + 1:
        raise ValueError(f"indptr length must be n_rows+1={n_rows + 1}, got {indptr.numel()}")
    if data.numel() != indices.numel():
        raise ValueError("data and indices must have the same length (nnz)")
    if not all(t.is_cuda for t in (data, indices, indptr)):
        raise ValueError("data, indices, and indptr must be CUDA tensors")
    if not all(t.device == data.device for t in (indices, indptr)):
        raise ValueError("data, indices, and indptr must be on the same CUDA device")
    if data.dtype not in SUPPORTED_SPMM_VALUE_DTYPES:
        raise TypeError("data dtype must be one of: float16, bfloat16, float32, float64, complex64, complex128")
    if indices.dtype not in SUPPORTED_INDEX_DTYPES:
        raise TypeError("indices dtype must be torch.int32 or torch.int64")
    if indptr.dtype not in SUPPORTED_INDEX_DTYPES:
        raise TypeError("indptr dtype must be torch.int32 or torch.int64")

    nnz = data.numel()
    data = data.contiguous()
    indices = indices.contiguous()
    indptr = indptr.contiguous()
    # every structural check in one kernel and one device->host read (fsb_csr_check)
    c = _nat.csr_check(indptr, indices, n_rows)
    if c[0] != 0:
        raise ValueError("indptr[0] must be 0")
    if c[1] != nnz:
        raise ValueError(f"indptr[-1] must equal nnz={nnz}, got {c[1]}")
    if c[2]:
        raise ValueError("indptr must be nondecreasing")
    if nnz > 0:
        if c[3] or c[4] >= n_cols:
            raise IndexError("indices out of range for n_cols")
        if c[4] > _INDEX_LIMIT_INT32:
            raise ValueError("column indices exceed the int32 range supported by the Triton kernel")
    row_lengths = (indptr[1:] - indptr[:-1]).to(torch.int64)
    kernel_indices = indices.to(torch.int32) if indices.dtype == torch.int64 else indices
    kernel_indptr = indptr.to(torch.int64)
    max_row_nnz = c[5]
    sum_sq, empty = c[6], c[7]
    if not return_stats:
        return data, kernel_indices, kernel_indptr, n_rows, n_cols, row_lengths, max_row_nnz
    if n_rows == 0:
        stats = _plan.MatrixStats(0, n_cols, 0, 0, 0.0, 0.0, 0)
    else:
        mean = nnz / n_rows
        std = math.sqrt(max(sum_sq / n_rows - mean * mean, 0.0))
        stats = _plan.MatrixStats(n_rows, n_cols, nnz, max_row_nnz, mean, std, empty)
    return data, kernel_indices, kernel_indptr, n_rows, n_cols, row_lengths, max_row_nnz, stats


def _prepare_spmm_csr_inputs(data, indices, indptr, B, shape):
    if B.ndim != 2:
        raise ValueError("B must be a 2D dense tensor")
    data, kernel_indices, kernel_indptr, n_rows, n_cols, _rl, max_row_nnz = _prepare_spmm_csr_matrix(
        data, indices, indptr, shape
    )
    if B.shape[0] != n_cols:
        raise ValueError(f"B.shape[0] must be n_cols={n_cols}, got {B.shape[0]}")
    if not B.is_cuda:
        raise ValueError("B must be a CUDA tensor")
    if B.device != data.device:
        raise ValueError("B must be on the same CUDA device as the sparse matrix")
    if B.dtype != data.dtype:
        raise TypeError("B dtype must match data dtype")
    B = B.contiguous()
    return data, kernel_indices, kernel_indptr, B, n_rows, n_cols, int(B.shape[1]), max_row_nnz


def _select_spmm_alg1_warp_and_factor(n_dense_cols):
    """FlagSparse's ALG1 tile heuristic (``spmm_csr.py:284-296``); kept for the
    launch-config record, the CUDA kernels choose their own column tiles."""
    if n_dense_cols > 64:
        return 32, 4
    if n_dense_cols > 32:
        return 32, 2
    if n_dense_cols > 16:
        return 32, 1
    if n_dense_cols > 8:
        return 16, 1
    if n_dense_cols > 4:
        return 8, 1
    return 4, 1


def _cdiv(a, b):
    return -(-a // b)


def _resolve_spmm_alg1_launch_config(n_dense_cols, max_row_nnz, block_n=None, block_nnz=None, max_segments=None):
    """Validation and record of ALG1 launch knobs (FlagSparse ``spmm_csr.py:299-334``)."""
    warp_size, factor = _select_spmm_alg1_warp_and_factor(n_dense_cols)
    if block_n is None:
        block_n = warp_size * factor
    if block_nnz is None:
        block_nnz = warp_size
    if block_n <= 0 or block_nnz <= 0:
        raise ValueError("block_n and block_nnz must be positive when provided")
    if max_segments is not None and max_segments <= 0:
        raise ValueError("max_segments must be positive when provided")
    required_segments = _cdiv(max_row_nnz, block_nnz) if max_row_nnz > 0 else 0
    if max_segments is not None and required_segments > int(max_segments):
        raise ValueError(
            "row nnz requires more CSR segments than the explicit max_segments override allows: "
            f"required {required_segments}, provided {int(max_segments)}"
        )
    return {
        "block_n": int(block_n),
        "block_nnz": int(block_nnz),
        "max_segments": (None if max_segments is None else int(max_segments)),
        "required_segments": int(required_segments),
        "warp_size": int(warp_size),
        "factor": int(factor),
        "max_row_nnz": int(max_row_nnz),
        "auto_max_segments": max_segments is None,
    }


class PreparedCsrSpmmOpt:
    """Cached CSR metadata for repeated SpMM-opt calls (FlagSparse ``spmm_csr.py:337-392``)."""

    __slots__ = (
        "data",
        "kernel_indices",
        "kernel_indptr",
        "shape",
        "n_rows",
        "n_cols",
        "row_lengths",
        "max_row_nnz",
        "supports_opt",
        "long_row_fallback_only",
        "_bucket_meta",
        "_stats",
        "_plans",
    )

    def __init__(
        self,
        data,
        kernel_indices,
        kernel_indptr,
        shape,
        n_rows,
        n_cols,
        row_lengths,
        max_row_nnz,
        row_buckets=None,
        long_part_rows=None,
        long_part_starts=None,
        long_part_ends=None,
        long_row_ids=None,
        long_row_part_ptr=None,
        long_row_fallback_only=False,
    ):
        self.data = data
        self.kernel_indices = kernel_indices
        self.kernel_indptr = kernel_indptr
        self.shape = (int(shape[0]), int(shape[1]))
        self.n_rows = int(n_rows)
        self.n_cols = int(n_cols)
        self.row_lengths = row_lengths
        self.max_row_nnz = int(max_row_nnz)
        self.supports_opt = data.dtype in (torch.float32, torch.float64)
        given = (row_buckets, long_part_rows, long_part_starts, long_part_ends, long_row_ids, long_row_part_ptr)
        # FlagSparse's bucket lists and long-row split parts describe its own
        # launches; the kernels here never read them, so a prepare that does
        # not pass them builds them on first access only
        self._bucket_meta = None if all(v is None for v in given) else dict(zip(_SPMM_OPT_META_FIELDS, given))
        self.long_row_fallback_only = bool(long_row_fallback_only)
        self._stats = None
        self._plans = {}

    def _meta(self):
        if self._bucket_meta is None:
            row_buckets, long_rows = _build_spmm_opt_buckets(self.row_lengths)
            split = _build_spmm_opt_split_metadata(
                self.kernel_indptr, long_rows, part_block_nnz=_SPMM_OPT_PART_NNZ
            ) if long_rows.numel() > 0 else (
                torch.empty((0,), dtype=long_rows.dtype, device=self.data.device),
                torch.empty((0,), dtype=torch.int64, device=self.data.device),
                torch.empty((0,), dtype=torch.int64, device=self.data.device),
                torch.zeros(1, dtype=torch.int64, device=self.data.device),
            )
            self._bucket_meta = dict(zip(_SPMM_OPT_META_FIELDS, (row_buckets, split[0], split[1], split[2],
                                                                 long_rows, split[3])))
        return self._bucket_meta


_SPMM_OPT_META_FIELDS = ("row_buckets", "long_part_rows", "long_part_starts", "long_part_ends", "long_row_ids",
                         "long_row_part_ptr")


def _meta_property(name):
    def get(self):
        return self._meta()[name]

    def set_(self, value):
        self._meta()[name] = value

    return property(get, set_)


for _name in _SPMM_OPT_META_FIELDS:
    setattr(PreparedCsrSpmmOpt, _name, _meta_property(_name))


_SPMM_OPT_LONG_ROW_THRESHOLD = 2048
_SPMM_OPT_PART_NNZ = 256


def _select_spmm_opt_block_n(n_dense_cols):
    if n_dense_cols <= 8:
        return 8
    if n_dense_cols <= 16:
        return 16
    if n_dense_cols <= 32:
        return 32
    if n_dense_cols <= 64:
        return 64
    return 128


def _build_spmm_opt_split_metadata(kernel_indptr, long_rows, part_block_nnz):
    """Cut each long row into ``part_block_nnz``-nonzero parts, all on the
    device (FlagSparse built the same arrays in a host loop, ``spmm_csr.py:417-441``).
    Returns (part_rows, part_starts, part_ends, row_part_ptr), bit-identical."""
    device = kernel_indptr.device
    row_dtype = long_rows.dtype if long_rows.numel() > 0 else torch.int32
    if long_rows.numel() == 0:
        return (torch.empty(0, dtype=row_dtype, device=device), torch.empty(0, dtype=torch.int64, device=device),
                torch.empty(0, dtype=torch.int64, device=device), torch.zeros(1, dtype=torch.int64, device=device))
    ptr = kernel_indptr.to(torch.int64)
    rows64 = long_rows.to(torch.int64)
    starts = ptr[rows64]
    ends = ptr[rows64 + 1]
    n_parts = (ends - starts + part_block_nnz - 1) // part_block_nnz
    row_part_ptr = torch.zeros(rows64.numel() + 1, dtype=torch.int64, device=device)
    row_part_ptr[1:] = torch.cumsum(n_parts, 0)
    total = int(row_part_ptr[-1].item())
    owner = torch.repeat_interleave(torch.arange(rows64.numel(), device=device), n_parts, output_size=total)
    local = torch.arange(total, device=device) - row_part_ptr[:-1][owner]
    part_starts = starts[owner] + local * part_block_nnz
    part_ends = torch.minimum(part_starts + part_block_nnz, ends[owner])
    return long_rows[owner].to(row_dtype), part_starts, part_ends, row_part_ptr


def _build_spmm_opt_buckets(row_lengths):
    """Launch description of the opt path and the long rows (> 2048 nonzeros).

    FlagSparse launched one kernel per row-length bucket (``spmm_csr.py:444-477``);
    here one launch covers all rows, so the bucket list describes that launch.
    """
    device = row_lengths.device
    n = int(row_lengths.numel())
    row_index_dtype = torch.int32 if n - 1 <= _INDEX_LIMIT_INT32 else torch.int64
    long_rows = torch.nonzero(row_lengths > _SPMM_OPT_LONG_ROW_THRESHOLD, as_tuple=False).flatten().to(
        row_index_dtype)
    buckets = [] if n == 0 else [{"kind": "single_launch", "rows": n}]
    return buckets, long_rows.to(device)


def prepare_spmm_csr_opt(data, indices, indptr, shape):
    """Validated CSR + cached plans; the bucket / split metadata fields
    (FlagSparse ``spmm_csr.py:480-522``) are built on first access."""
    (data, kernel_indices, kernel_indptr, n_rows, n_cols, row_lengths, max_row_nnz,
     stats) = _prepare_spmm_csr_matrix(data, indices, indptr, shape, return_stats=True)
    p = PreparedCsrSpmmOpt(
        data=data,
        kernel_indices=kernel_indices,
        kernel_indptr=kernel_indptr,
        shape=shape,
        n_rows=n_rows,
        n_cols=n_cols,
        row_lengths=row_lengths,
        max_row_nnz=max_row_nnz,
        long_row_fallback_only=False,
    )
    p._stats = stats
    return p


def _spmm_plan_for(holder, kind, n_dense, operands=None):
    """Cached plan on a prepared object for (kind, n_dense).  With
    ``operands`` = (B, C, acc_mode) the first call per width goes through the
    plan selector (learned / autotune / heuristic); without, the heuristic."""
    key = (kind, int(n_dense))
    plan = holder._plans.get(key)
    if plan is None:
        if holder._stats is None:
            holder._stats = _plan.matrix_stats(holder.kernel_indptr, holder.n_rows, holder.n_cols)
        if operands is not None and getattr(holder, "kernel_indices", None) is not None:
            B, C, acc = operands
            plan = _plan.chosen_spmm_plan(holder._stats, holder.data, holder.kernel_indices, holder.kernel_indptr,
                                          holder.n_rows, holder.n_cols, B, C, acc)
        else:
            plan = _plan.default_spmm_plan(holder._stats, n_dense, holder.data.dtype)
        holder._plans[key] = plan
    return plan


class _Alg1Holder:
    """Plan cache of a one-shot ALG1 call."""

    __slots__ = ("kernel_indptr", "n_rows", "n_cols", "data", "_stats", "_plans")

    def __init__(self, data, kernel_indptr, n_rows, n_cols, max_row_nnz, nnz):
        self.data = data
        self.kernel_indptr = kernel_indptr
        self.n_rows = n_rows
        self.n_cols = n_cols
        mean = nnz / max(n_rows, 1)
        self._stats = _plan.MatrixStats(n_rows, n_cols, nnz, max_row_nnz, mean, 0.0, 0)
        self._plans = {}


def _alg1_acc_mode(dtype):
    return _nat.ACC_WIDE if dtype == torch.float32 else _nat.ACC_NATIVE


def _triton_spmm_csr_impl(data, indices, indptr, B, n_rows, n_dense_cols, block_n, block_nnz, max_row_nnz=None,
                          out=None, plan=None):
    """ALG1 SpMM (FlagSparse ``spmm_csr.py:525-599``) in one CUDA launch.

    ``block_n`` / ``block_nnz`` are the reference's Triton tile sizes; they do
    not change the result.  float32 accumulates in float64 in registers.
    """
    del block_n, block_nnz
    device = data.device
    dtype = data.dtype
    if n_rows == 0 or n_dense_cols == 0 or B.shape[0] == 0:
        return torch.zeros((n_rows, n_dense_cols), dtype=dtype, device=device)
    C = out if out is not None else torch.empty((n_rows, n_dense_cols), dtype=dtype, device=device)
    if plan is None:
        if max_row_nnz is None:
            max_row_nnz = int((indptr[1:] - indptr[:-1]).max().item())
        holder = _Alg1Holder(data, indptr, n_rows, B.shape[0], max_row_nnz, data.numel())
        plan = _spmm_plan_for(holder, "alg1", n_dense_cols)
    _plan.run_spmm(data, indices, indptr, n_rows, B.shape[0], B, C, _alg1_acc_mode(dtype), plan)
    return C


def _check_opt_operand(prepared, B):
    """FlagSparse's checks of the opt paths' dense operand (``spmm_csr.py:1998-2011``)."""
    if not prepared.supports_opt:
        raise TypeError("spmm opt only supports float32 and float64")
    if not B.is_cuda:
        raise ValueError("B must be a CUDA tensor")
    if B.device != prepared.data.device:
        raise ValueError("B must be on the same CUDA device as the sparse matrix")
    if B.dtype != prepared.data.dtype:
        raise TypeError("B dtype must match sparse matrix dtype")
    if B.shape[0] != prepared.n_cols:
        raise ValueError(f"B.shape[0] must be n_cols={prepared.n_cols}, got {B.shape[0]}")
    if B.ndim != 2:
        raise ValueError("B must be a 2D dense tensor")
    return B.contiguous()


def _triton_spmm_csr_impl_opt_prepared(prepared, B, out=None):
    B = _check_opt_operand(prepared, B)
    n_dense = int(B.shape[1])
    C = out if out is not None else torch.empty((prepared.n_rows, n_dense), dtype=B.dtype, device=B.device)
    if prepared.n_rows == 0 or n_dense == 0:
        return C.zero_(), False
    plan = _spmm_plan_for(prepared, "opt", n_dense, (B, C, _nat.ACC_NATIVE))
    _plan.run_spmm(prepared.data, prepared.kernel_indices, prepared.kernel_indptr, prepared.n_rows,
                   prepared.n_cols, B, C, _nat.ACC_NATIVE, plan)
    return C, False


# Diagnose-only forms (FlagSparse ``spmm_csr.py:1998-2086``): fixed-order
# accumulation in fsb_spmm_csr_diag, for comparing the opt path's rounding
# with float64 and compensated sums.  Rows of at most this many nonzeros take
# the candidate form's compensated short-row arithmetic (FlagSparse
# ``_candidate_bucket_uses_stable_short_kernel``, ``:1871-1874``).
_DIAG_CANDIDATE_SHORT_MAX = 256


def _run_spmm_diag(prepared, B, mode_short, mode_long, short_max):
    B = _check_opt_operand(prepared, B)
    n_dense = int(B.shape[1])
    C = torch.zeros((prepared.n_rows, n_dense), dtype=B.dtype, device=B.device)
    if prepared.n_rows == 0 or n_dense == 0:
        return C
    cm = _nat.make_csr(prepared.data, prepared.kernel_indices, prepared.kernel_indptr, prepared.n_rows,
                       prepared.n_cols)
    rc = _nat.library().fsb_spmm_csr_diag(cm, _nat.ptr(B), int(B.stride(0)), n_dense, _nat.ptr(C), int(C.stride(0)),
                                          int(mode_short), int(mode_long), int(short_max),
                                          _nat.stream_handle(B.device))
    _nat.check(rc, "fsb_spmm_csr_diag")
    _plan.LAUNCHES["count"] += 1
    return C


def _triton_spmm_csr_impl_opt_prepared_stable(prepared, B):
    """The stable form: every element accumulated in float64 in nonzero order
    and stored in the value type (FlagSparse ``:2059-2081``, its
    ``_spmm_csr_stable_vector_*`` kernels, ``:1023-1106``)."""
    return _run_spmm_diag(prepared, B, _nat.DIAG_WIDE, _nat.DIAG_WIDE, -1), False


def _flagsparse_spmm_csr_opt_stable_for_diagnose(prepared, B):
    C_out, _ = _triton_spmm_csr_impl_opt_prepared_stable(prepared, B)
    return C_out


def _triton_spmm_csr_impl_opt_prepared_candidate(prepared, B):
    """The candidate form: rows of at most 256 nonzeros with Kahan's sum in
    float64 (FlagSparse's ``_spmm_csr_candidate_stable_short_*`` kernels,
    ``:1540-1634``), longer rows accumulated in the value precision in order."""
    C = _run_spmm_diag(prepared, B, _nat.DIAG_KAHAN_WIDE, _nat.DIAG_NATIVE, _DIAG_CANDIDATE_SHORT_MAX)
    return C, False


def _flagsparse_spmm_csr_opt_candidate_for_diagnose(prepared, B):
    C_out, _ = _triton_spmm_csr_impl_opt_prepared_candidate(prepared, B)
    return C_out


def _flagsparse_spmm_csr_opt_kahan_for_diagnose(prepared, B):
    """Kahan's compensated sum in the value precision on every row (the
    arithmetic of FlagSparse's ``_spmm_csr_stable_batched_*`` kernels,
    ``:923-1020``)."""
    return _run_spmm_diag(prepared, B, _nat.DIAG_KAHAN, _nat.DIAG_KAHAN, -1)


def flagsparse_spmm_csr(
    data,
    indices,
    indptr,
    B,
    shape,
    block_n=None,
    block_nnz=None,
    max_segments=None,
    out=None,
    return_time=False,
):
    """CSR SpMM C = A @ B (ALG1 semantics of FlagSparse ``spmm_csr.py:2088-2157``).

    A is given as CSR arrays; B is a dense CUDA tensor (n_cols, n_dense_cols).
    """
    if block_n is not None and block_n <= 0:
        raise ValueError("block_n must be positive when provided")
    if block_nnz is not None and block_nnz <= 0:
        raise ValueError("block_nnz must be positive when provided")
    if max_segments is not None and max_segments <= 0:
        raise ValueError("max_segments must be positive when provided")
    data, kernel_indices, kernel_indptr, B, n_rows, _, n_dense_cols, max_row_nnz = _prepare_spmm_csr_inputs(
        data, indices, indptr, B, shape
    )
    launch = _resolve_spmm_alg1_launch_config(n_dense_cols, max_row_nnz, block_n=block_n, block_nnz=block_nnz,
                                              max_segments=max_segments)
    if out is not None:
        if not out.is_cuda:
            raise ValueError("out must be a CUDA tensor")
        if out.device != data.device:
            raise ValueError("out must be on the same CUDA device as the inputs")
        if out.shape != (n_rows, n_dense_cols) or out.dtype != data.dtype:
            raise ValueError("out shape/dtype must match result")
    direct = out is not None and out.is_contiguous()
    t0 = None
    if return_time:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
    C = _triton_spmm_csr_impl(data, kernel_indices, kernel_indptr, B, n_rows, n_dense_cols,
                              block_n=launch["block_n"], block_nnz=launch["block_nnz"], max_row_nnz=max_row_nnz,
                              out=out if direct else None)
    elapsed_ms = None
    if return_time:
        torch.cuda.synchronize()
        elapsed_ms = (time.perf_counter() - t0) * 1000.0
    if out is not None:
        if C.data_ptr() != out.data_ptr():
            out.copy_(C)
        C = out
    if return_time:
        return C, elapsed_ms
    return C


def flagsparse_spmm_csr_opt(data=None, indices=None, indptr=None, B=None, shape=None, prepared=None, out=None,
                            return_time=False):
    """CSR SpMM-opt: float32/float64 with value-precision accumulation."""
    if prepared is not None and not isinstance(prepared, PreparedCsrSpmmOpt):
        raise TypeError("prepared must be a PreparedCsrSpmmOpt instance")
    if prepared is None:
        if any(arg is None for arg in (data, indices, indptr, shape)):
            raise ValueError("data, indices, indptr, and shape are required when prepared is not provided")
        prepared = prepare_spmm_csr_opt(data, indices, indptr, shape)
    elif shape is not None:
        resolved_shape = (int(shape[0]), int(shape[1]))
        if resolved_shape != prepared.shape:
            raise ValueError(f"shape {resolved_shape} does not match prepared.shape {prepared.shape}")
    if B is None:
        raise ValueError("B is required")
    if not prepared.supports_opt:
        raise TypeError("flagsparse_spmm_csr_opt only supports float32 and float64")
    if not B.is_cuda:
        raise ValueError("B must be a CUDA tensor")
    if B.device != prepared.data.device:
        raise ValueError("B must be on the same CUDA device as sparse matrix data")
    if out is not None:
        if not out.is_cuda:
            raise ValueError("out must be a CUDA tensor")
        if out.device != prepared.data.device:
            raise ValueError("out must be on the same CUDA device as sparse matrix data")
        if out.shape != (prepared.n_rows, int(B.shape[1])) or out.dtype != prepared.data.dtype:
            raise ValueError("out shape/dtype must match result")
    direct = out is not None and out.is_contiguous()
    t0 = None
    if return_time:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
    C, _long_row_fallback_used = _triton_spmm_csr_impl_opt_prepared(prepared, B, out=out if direct else None)
    elapsed_ms = None
    if return_time:
        torch.cuda.synchronize()
        elapsed_ms = (time.perf_counter() - t0) * 1000.0
    if out is not None:
        if C.data_ptr() != out.data_ptr():
            out.copy_(C)
        C = out
    if return_time:
        return C, elapsed_ms
    return C


def _spmm_opt_reference_error(candidate, reference, value_dtype):
    atol, rtol = _spmm_coo_reference_tolerance(value_dtype)
    if candidate.numel() == 0:
        return 0.0
    diff = torch.abs(candidate - reference)
    denom = atol + rtol * torch.abs(reference)
    return float(torch.max(diff / denom).item())
