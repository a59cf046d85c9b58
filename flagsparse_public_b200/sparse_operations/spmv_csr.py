"""CSR SpMV: FlagSparse's ``spmv_csr`` operator API on sm_100a kernels.

Public names, keyword defaults, exception types and messages follow FlagSparse
``sparse_operations/spmv_csr.py`` (``prepare_spmv_csr`` :570-649,
``flagsparse_spmv_csr`` :796-872, COO->CSR :875-1016).  The private hooks
FlagSparse's own tests patch (``_triton_spmv_csr_impl_prepared``,
``_run_spmv_prepared``, ``_run_spmv_prepared_with_fallback``,
``_INDEX_LIMIT_INT32``) keep their names; behind them the products run in the
CUDA kernels of ``libflagsparse_b200.so`` (row groups or merge path), not in
Triton.

Numerics kept from the reference: the plain path computes float32 input with
float64 accumulation and float16/bfloat16 with float32 accumulation
(``spmv_csr.py:116-121``) -- in registers, without the reference's float64
copies of the matrix and of x; the ``use_opt`` path accumulates float32 in
float32 (``spmv_csr.py:246``).
"""

import ctypes
import math

from ._common import *
from .. import _native as _nat
from .. import _plan

SUPPORTED_SPMV_VALUE_DTYPES = (
    torch.float16,
    torch.bfloat16,
    torch.float32,
    torch.float64,
    torch.complex64,
    torch.complex128,
)

SPMV_OP_NON = 0
SPMV_OP_TRANS = 1
SPMV_OP_CONJ_TRANS = 2
SPMV_OP_NAMES = {SPMV_OP_NON: "non", SPMV_OP_TRANS: "trans", SPMV_OP_CONJ_TRANS: "conj"}
_SPMV_OP_NAME_TO_CODE = {name: code for code, name in SPMV_OP_NAMES.items()}

# Row-length tiers of FlagSparse's CSR-vector buckets (spmv_csr.py:128-153):
# (upper bound of the tier, lanes of the tier).  Used only to reproduce the
# per-row truncation an explicit ``max_segments`` implies on the opt path.
_SPMV_OPT_TIERS_F32 = ((64, 32), (512, 256), (4096, 512), (None, 1024))
_SPMV_OPT_TIERS_F64 = ((64, 32), (256, 64), (2048, 128), (8192, 256), (None, 512))


def _normalize_spmv_op(op=None, transpose=False):
    if op is None:
        return SPMV_OP_TRANS if bool(transpose) else SPMV_OP_NON
    if isinstance(op, str):
        token = op.strip().lower()
        if token not in _SPMV_OP_NAME_TO_CODE:
            raise ValueError("op must be one of: 0=non, 1=trans, 2=conj")
        return _SPMV_OP_NAME_TO_CODE[token]
    try:
        op_code = int(op)
    except (TypeError, ValueError) as exc:
        raise ValueError("op must be one of: 0=non, 1=trans, 2=conj") from exc
    if op_code not in SPMV_OP_NAMES:
        raise ValueError("op must be one of: 0=non, 1=trans, 2=conj")
    return op_code


def _spmv_op_to_name(op):
    return SPMV_OP_NAMES[_normalize_spmv_op(op)]


def _spmv_op_transposes(op):
    return _normalize_spmv_op(op) in (SPMV_OP_TRANS, SPMV_OP_CONJ_TRANS)


class PreparedCsrSpmv:
    """Cached CSR metadata and kernel plans for repeated SpMV calls.

    Constructor keywords and attributes are FlagSparse's (``spmv_csr.py:55-122``);
    ``opt_buckets`` holds the launch plan descriptions of this implementation.
    """

    __slots__ = (
        "data",
        "kernel_indices",
        "kernel_indptr",
        "shape",
        "n_rows",
        "n_cols",
        "block_nnz",
        "max_segments",
        "max_row_nnz",
        "opt_buckets",
        "supports_opt",
        "transpose",
        "op",
        "index_fallback_policy",
        "index_fallback_applied",
        "index_fallback_reason",
        "_baseline_compute_dtype",
        "_baseline_data",
        "_explicit_max_segments",
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
        block_nnz,
        max_segments,
        max_row_nnz,
        opt_buckets,
        transpose=False,
        op=None,
        index_fallback_policy="auto",
        index_fallback_applied=False,
        index_fallback_reason=None,
    ):
        self.data = data
        self.kernel_indices = kernel_indices
        self.kernel_indptr = kernel_indptr
        self.shape = (int(shape[0]), int(shape[1]))
        self.n_rows = n_rows
        self.n_cols = n_cols
        self.block_nnz = block_nnz
        self.max_segments = max_segments
        self.max_row_nnz = max_row_nnz
        self.opt_buckets = opt_buckets
        self.supports_opt = data.dtype in (torch.float32, torch.float64) and kernel_indices.dtype == torch.int32
        self.op = _normalize_spmv_op(op, transpose=transpose)
        self.transpose = _spmv_op_transposes(self.op)
        self.index_fallback_policy = str(index_fallback_policy).lower()
        self.index_fallback_applied = bool(index_fallback_applied)
        self.index_fallback_reason = index_fallback_reason
        if data.dtype in (torch.float16, torch.bfloat16):
            self._baseline_compute_dtype = torch.float32
        elif data.dtype == torch.float32:
            self._baseline_compute_dtype = torch.float64
        else:
            self._baseline_compute_dtype = data.dtype
        self._baseline_data = None
        self._explicit_max_segments = None
        self._stats = None
        self._plans = {}


def _spmv_stats(prepared):
    if prepared._stats is None:
        prepared._stats = _plan.matrix_stats(prepared.kernel_indptr, prepared.n_rows, prepared.n_cols)
    return prepared._stats


def _spmv_plan(prepared, kind, row_cap=0):
    """Kernel plan of ``prepared`` for ``kind`` ('plain' / 'opt'), cached."""
    key = (kind, int(row_cap))
    plan = prepared._plans.get(key)
    if plan is None:
        plan = _plan.default_spmv_plan(_spmv_stats(prepared), prepared.data.dtype, row_cap=row_cap)
        prepared._plans[key] = plan
    return plan


def _build_spmv_opt_buckets(n_rows, max_row_nnz, row_index_dtype, max_segments=None, fp64=False):
    """Plan description of the opt path (FlagSparse kept per-tier row lists
    here, built from the row lengths; this one takes the row count).

    The kernels of this implementation need no row lists: one launch covers
    all rows (row groups sized from the mean row length, or merge-path tiles
    for skewed rows).  The returned list describes that launch.
    """
    del row_index_dtype, max_segments, fp64
    n_rows = int(n_rows)
    if n_rows == 0:
        return []
    return [{"kind": "single_launch", "rows": n_rows, "max_row_nnz": int(max_row_nnz)}]


def _normalize_spmv_index_fallback_policy(index_fallback_policy):
    policy = str(index_fallback_policy).lower()
    if policy not in ("auto", "strict"):
        raise ValueError("index_fallback_policy must be 'auto' or 'strict'")
    return policy


def _spmv_dtype_error_message():
    return "data dtype must be one of: " + ", ".join(
        str(dtype).replace("torch.", "") for dtype in SUPPORTED_SPMV_VALUE_DTYPES
    )


def _transpose_csr_for_spmv(data, indices, indptr, shape):
    """CSR of A^T: a stable sort of the nonzeros by column (FlagSparse
    ``spmv_csr.py:456-494``); output index/indptr dtypes follow the same rules
    (``:487-488``) so the structure is bit-identical."""
    n_rows, n_cols = int(shape[0]), int(shape[1])
    nnz = data.numel()
    device = data.device
    out_index_dtype = indices.dtype if n_rows <= _INDEX_LIMIT_INT32 else torch.int64
    out_indptr_dtype = indptr.dtype if nnz <= _INDEX_LIMIT_INT32 else torch.int64
    if nnz == 0:
        return (
            data,
            torch.empty(0, dtype=out_index_dtype, device=device),
            torch.zeros(n_cols + 1, dtype=out_indptr_dtype, device=device),
            (n_cols, n_rows),
        )
    counts = (indptr[1:] - indptr[:-1]).to(torch.int64)
    row_ids = torch.repeat_interleave(torch.arange(n_rows, dtype=torch.int64, device=device), counts,
                                      output_size=nnz)
    cols = indices.to(torch.int64)
    sorted_cols, order = _plan.stable_sort(cols, key_bound=n_cols)
    t_indptr = _plan.sorted_keys_to_offsets(sorted_cols, n_cols)
    return (
        data[order].contiguous(),
        row_ids[order].to(out_index_dtype).contiguous(),
        t_indptr.to(out_indptr_dtype).contiguous(),
        (n_cols, n_rows),
    )


def _prepare_spmv_csr_matrix(data, indices, indptr, shape, index_fallback_policy="auto", return_stats=False):
    _normalize_spmv_index_fallback_policy(index_fallback_policy)
    if not all(torch.is_tensor(t) for t in (data, indices, indptr)):
        raise TypeError("data, indices, indptr must all be torch.Tensor")
    if data.ndim != 1 or indices.ndim != 1 or indptr.ndim != 1:
        raise ValueError("data, indices, indptr must be 1D tensors")
    n_rows, n_cols = int(shape[0]), int(shape[1])
    if indptr.numel() != n_rows + 1:
        raise ValueError(f"indptr length must be n_rows+1={n_rows + 1}, got {indptr.numel()}")
    if data.numel() != indices.numel():
        raise ValueError("data and indices must have the same length (nnz)")
    if not all(t.is_cuda for t in (data, indices, indptr)):
        raise ValueError("data, indices, indptr must be CUDA tensors")
    if not all(t.device == data.device for t in (indices, indptr)):
        raise ValueError("data, indices, indptr must be on the same CUDA device")
    if data.dtype not in SUPPORTED_SPMV_VALUE_DTYPES:
        raise TypeError(_spmv_dtype_error_message())
    if indices.dtype not in SUPPORTED_INDEX_DTYPES:
        raise TypeError("indices dtype must be torch.int32 or torch.int64")
    if indptr.dtype not in SUPPORTED_INDEX_DTYPES:
        raise TypeError("indptr dtype must be torch.int32 or torch.int64")

    data = data.contiguous()
    indices = indices.contiguous()
    indptr = indptr.contiguous()
    nnz = data.numel()

    # All structural checks in one kernel and one device->host read
    # (fsb_csr_check), raised in FlagSparse's order.
    c = _nat.csr_check(indptr, indices, n_rows)
    if c[0] != 0:
        raise ValueError("indptr must start at zero")
    if c[1] != nnz:
        raise ValueError("indptr[-1] must equal nnz")
    if c[2]:
        raise ValueError("indptr must be non-decreasing")
    if nnz > 0 and (c[3] or c[4] >= n_cols):
        raise IndexError("indices out of range for n_cols")
    max_row_nnz = c[5]
    # row lengths are not materialised: the kernels read the row offsets
    if not return_stats:
        return data, indices, indptr, n_rows, n_cols, None, max_row_nnz
    if n_rows == 0:
        stats = _plan.MatrixStats(0, n_cols, 0, 0, 0.0, 0.0, 0)
    else:
        mean = nnz / n_rows
        std = math.sqrt(max(c[6] / n_rows - mean * mean, 0.0))
        stats = _plan.MatrixStats(n_rows, n_cols, nnz, max_row_nnz, mean, std, c[7])
    return data, indices, indptr, n_rows, n_cols, None, max_row_nnz, stats


def _validate_spmv_x(x, prepared):
    if x is None or not torch.is_tensor(x):
        raise TypeError("x must be a torch.Tensor")
    if x.ndim != 1:
        raise ValueError("x must be a 1D tensor")
    if not x.is_cuda:
        raise ValueError("x must be a CUDA tensor")
    if x.dtype != prepared.data.dtype:
        raise TypeError("x dtype must match sparse matrix dtype")
    if x.numel() != prepared.n_cols:
        raise ValueError(f"x length must be n_cols={prepared.n_cols}, got {x.numel()}")
    if x.device != prepared.data.device:
        raise ValueError("x must be on the same device as sparse matrix data")
    return x.contiguous()


def prepare_spmv_csr(
    data,
    indices,
    indptr,
    shape,
    block_nnz=256,
    max_segments=None,
    transpose=False,
    op=None,
    index_fallback_policy="auto",
):
    index_fallback_policy = _normalize_spmv_index_fallback_policy(index_fallback_policy)
    op_code = _normalize_spmv_op(op, transpose=transpose)
    if op is not None and bool(transpose) and op_code == SPMV_OP_NON:
        raise ValueError("transpose=True conflicts with op=non")
    transpose = _spmv_op_transposes(op_code)
    if transpose:
        data, indices, indptr, *_ = _prepare_spmv_csr_matrix(
            data, indices, indptr, shape, index_fallback_policy=index_fallback_policy
        )
        if op_code == SPMV_OP_CONJ_TRANS and _is_complex_dtype(data.dtype):
            data = data.conj().resolve_conj()
        data, indices, indptr, shape = _transpose_csr_for_spmv(data, indices, indptr, shape)
    (data, kernel_indices, kernel_indptr, n_rows, n_cols, _row_lengths, max_row_nnz,
     stats) = _prepare_spmv_csr_matrix(
        data, indices, indptr, shape, index_fallback_policy=index_fallback_policy, return_stats=True
    )
    block_nnz_use = block_nnz
    if max_segments is None:
        max_segments_use = max((max_row_nnz + block_nnz_use - 1) // block_nnz_use, 1)
        while max_segments_use > 2048 and block_nnz_use < 65536:
            block_nnz_use *= 2
            max_segments_use = max((max_row_nnz + block_nnz_use - 1) // block_nnz_use, 1)
    else:
        max_segments_use = max_segments
    row_index_dtype = torch.int32 if n_rows <= _INDEX_LIMIT_INT32 else torch.int64
    opt_buckets = _build_spmv_opt_buckets(
        n_rows, max_row_nnz=max_row_nnz, row_index_dtype=row_index_dtype, max_segments=max_segments,
        fp64=data.dtype == torch.float64,
    )
    prepared = PreparedCsrSpmv(
        data=data,
        kernel_indices=kernel_indices,
        kernel_indptr=kernel_indptr,
        shape=shape,
        n_rows=n_rows,
        n_cols=n_cols,
        block_nnz=block_nnz_use,
        max_segments=max_segments_use,
        max_row_nnz=max_row_nnz,
        opt_buckets=opt_buckets,
        transpose=transpose,
        op=op_code,
        index_fallback_policy=index_fallback_policy,
    )
    prepared._explicit_max_segments = max_segments
    prepared._stats = stats
    return prepared


def _get_spmv_baseline_data(prepared):
    """(compute dtype, data) of the plain path.  The kernels widen in registers,
    so no widened copy of the matrix is made (FlagSparse ``:652-661`` cached one)."""
    return prepared._baseline_compute_dtype, prepared.data


def _plain_row_cap(prepared):
    cap = int(prepared.block_nnz) * int(prepared.max_segments)
    return cap if cap < int(prepared.max_row_nnz) else 0


def _triton_spmv_csr_impl_prepared(prepared, x, out=None):
    """Plain SpMV (FlagSparse ``spmv_csr.py:664-708``): one launch of the CUDA
    kernels with the reference's accumulation widths and per-row segment cap."""
    dtype = prepared.data.dtype
    y = out if out is not None else torch.empty(prepared.n_rows, dtype=dtype, device=prepared.data.device)
    if prepared.n_rows == 0:
        return y
    acc = _nat.ACC_WIDE if dtype == torch.float32 else _nat.ACC_NATIVE
    row_cap = _plain_row_cap(prepared)
    plan = _spmv_plan(prepared, "plain", row_cap)
    _plan.run_spmv(prepared.data, prepared.kernel_indices, prepared.kernel_indptr, prepared.n_rows,
                   prepared.n_cols, x, y, acc, plan)
    return y


def _opt_row_cap_tiers(prepared):
    """Per-tier caps when an explicit max_segments was given to prepare_spmv_csr."""
    ms = prepared._explicit_max_segments
    if ms is None:
        return None
    tiers = _SPMV_OPT_TIERS_F64 if prepared.data.dtype == torch.float64 else _SPMV_OPT_TIERS_F32
    return [(bound, int(ms) * lanes) for bound, lanes in tiers]


def _triton_spmv_csr_impl_opt_prepared(prepared, x, out=None):
    """Opt SpMV (FlagSparse ``spmv_csr.py:393-440``): native-precision
    accumulation, all rows in one launch."""
    dtype = prepared.data.dtype
    y = out if out is not None else torch.empty(prepared.n_rows, dtype=dtype, device=prepared.data.device)
    if prepared.n_rows == 0:
        return y
    tiers = _opt_row_cap_tiers(prepared)
    if tiers is not None and prepared.max_row_nnz > min(cap for _, cap in tiers):
        # An explicit max_segments truncates each row to max_segments x (its
        # tier's lanes) nonzeros; rows are grouped by tier and capped per group.
        lens = prepared.kernel_indptr[1:] - prepared.kernel_indptr[:-1]
        lower = 0
        for bound, cap in tiers:
            sel = lens > lower if bound is None else ((lens > lower) & (lens <= bound) if lower else lens <= bound)
            rows = torch.nonzero(sel).flatten()
            if rows.numel():
                _run_rows_subset(prepared, x, y, rows, cap)
            if bound is not None:
                lower = bound
        return y
    plan = _spmv_plan(prepared, "opt")
    _plan.run_spmv(prepared.data, prepared.kernel_indices, prepared.kernel_indptr, prepared.n_rows,
                   prepared.n_cols, x, y, _nat.ACC_NATIVE, plan)
    return y


def _run_rows_subset(prepared, x, y, rows, cap):
    """SpMV over a subset of rows (row ids ``rows``) with a per-row cap."""
    ptr = prepared.kernel_indptr.to(torch.int64)
    starts = ptr[rows]
    ends = torch.minimum(ptr[rows + 1], starts + cap)
    lens = ends - starts
    sub_ptr = torch.zeros(rows.numel() + 1, dtype=torch.int64, device=ptr.device)
    sub_ptr[1:] = torch.cumsum(lens, 0)
    total = int(sub_ptr[-1].item())
    gather = torch.repeat_interleave(starts - sub_ptr[:-1], lens, output_size=total) + torch.arange(
        total, device=ptr.device)
    sub_y = torch.empty(rows.numel(), dtype=y.dtype, device=y.device)
    plan = _plan.KernelPlan(_nat.ALGO_ROWS, lanes=32)
    _plan.run_spmv(prepared.data[gather], prepared.kernel_indices[gather], sub_ptr, rows.numel(), prepared.n_cols,
                   x, sub_y, _nat.ACC_NATIVE, plan)
    y[rows] = sub_y


def _spmv_uses_int64_indices(prepared):
    return prepared.kernel_indices.dtype == torch.int64 or prepared.kernel_indptr.dtype == torch.int64


def _spmv_int32_fallback_blocker(prepared):
    if prepared.kernel_indices.dtype == torch.int64 and prepared.kernel_indices.numel() > 0:
        min_index = int(prepared.kernel_indices.min().item())
        max_index = int(prepared.kernel_indices.max().item())
        if min_index < 0 or max_index > _INDEX_LIMIT_INT32:
            return f"column index range [{min_index}, {max_index}] cannot fit int32 for shape={prepared.shape}"
    if prepared.kernel_indptr.dtype == torch.int64 and prepared.kernel_indptr.numel() > 0:
        max_offset = int(prepared.kernel_indptr[-1].item())
        if max_offset > _INDEX_LIMIT_INT32:
            return f"CSR nnz offset {max_offset} cannot fit int32 for shape={prepared.shape}"
    if prepared.n_rows > _INDEX_LIMIT_INT32:
        return f"row count {prepared.n_rows} cannot fit int32 row metadata"
    return None


def _spmv_prepared_with_int32_indices(prepared, reason):
    blocker = _spmv_int32_fallback_blocker(prepared)
    if blocker is not None:
        raise RuntimeError(f"native int64 CSR SpMV failed and int32 fallback is unsafe: {blocker}")
    kernel_indices = prepared.kernel_indices.to(torch.int32)
    kernel_indptr = prepared.kernel_indptr.to(torch.int32)
    max_row_nnz = prepared.max_row_nnz
    row_index_dtype = torch.int32 if prepared.n_rows <= _INDEX_LIMIT_INT32 else torch.int64
    opt_buckets = _build_spmv_opt_buckets(
        prepared.n_rows, max_row_nnz=max_row_nnz, row_index_dtype=row_index_dtype,
        max_segments=prepared.max_segments, fp64=prepared.data.dtype == torch.float64,
    )
    fallback = PreparedCsrSpmv(
        data=prepared.data,
        kernel_indices=kernel_indices,
        kernel_indptr=kernel_indptr,
        shape=prepared.shape,
        n_rows=prepared.n_rows,
        n_cols=prepared.n_cols,
        block_nnz=prepared.block_nnz,
        max_segments=prepared.max_segments,
        max_row_nnz=max_row_nnz,
        opt_buckets=opt_buckets,
        transpose=prepared.transpose,
        op=prepared.op,
        index_fallback_policy=prepared.index_fallback_policy,
        index_fallback_applied=True,
        index_fallback_reason=str(reason),
    )
    fallback._explicit_max_segments = prepared._explicit_max_segments
    return fallback


def _run_spmv_prepared(prepared, x, use_opt=False, out=None):
    impl = _triton_spmv_csr_impl_opt_prepared if use_opt and prepared.supports_opt else _triton_spmv_csr_impl_prepared
    return impl(prepared, x) if out is None else impl(prepared, x, out=out)


def _run_spmv_prepared_with_fallback(prepared, x, use_opt=False, out=None):
    # ``out`` is passed only when given: the hook keeps FlagSparse's signature
    kw = {} if out is None else {"out": out}
    try:
        return _run_spmv_prepared(prepared, x, use_opt=use_opt, **kw)
    except Exception as exc:
        if prepared.index_fallback_policy != "auto" or not _spmv_uses_int64_indices(prepared):
            raise
        fallback_prepared = _spmv_prepared_with_int32_indices(prepared, exc)
        return _run_spmv_prepared(fallback_prepared, x, use_opt=use_opt, **kw)


def _direct_out(out, prepared, x):
    """``out`` itself as the kernel's output when it has exactly the result's
    layout and shares no memory with the operands; otherwise None and the
    result is computed separately and copied into ``out`` (FlagSparse's
    behaviour, ``spmv_csr.py:861-869``), which keeps y = A y correct."""
    if (out is None or not torch.is_tensor(out) or not out.is_cuda or out.device != prepared.data.device
            or out.dtype != prepared.data.dtype or tuple(out.shape) != (prepared.n_rows,)
            or not out.is_contiguous()):
        return None
    a0 = out.data_ptr()
    a1 = a0 + out.numel() * out.element_size()
    for t in (x, prepared.data, prepared.kernel_indices, prepared.kernel_indptr):
        b0 = t.data_ptr()
        if t.numel() and a0 < b0 + t.numel() * t.element_size() and b0 < a1:
            return None
    return out


def flagsparse_spmv_csr(
    data=None,
    indices=None,
    indptr=None,
    x=None,
    shape=None,
    block_nnz=256,
    max_segments=None,
    out=None,
    return_time=False,
    use_opt=False,
    prepared=None,
    transpose=None,
    op=None,
    index_fallback_policy="auto",
):
    """CSR SpMV y = op(A) @ x on the sm_100a kernels.

    data, indices, indptr: CSR arrays; x: dense vector; shape: (n_rows, n_cols).
    prepared: cached metadata from prepare_spmv_csr for steady-state runs.
    op: 0/'non' for A @ x, 1/'trans' for A.T @ x, 2/'conj' for A.conj().T @ x.
    use_opt: float32/float64 with int32 indices accumulate in the value precision.
    """
    op_explicit = op is not None
    op_code = _normalize_spmv_op(op, transpose=False if transpose is None else bool(transpose))
    if op_explicit and transpose is not None and bool(transpose) != _spmv_op_transposes(op_code):
        raise ValueError("transpose conflicts with op")
    if prepared is None:
        if any(arg is None for arg in (data, indices, indptr, shape)):
            raise ValueError("data, indices, indptr, and shape are required when prepared is not provided")
        if op_code == SPMV_OP_NON and max_segments is None and not return_time:
            y = _spmv_csr_checked(data, indices, indptr, x, shape, use_opt, index_fallback_policy)
            if y is not None:
                return _spmv_write_out(y, out)
        prepared = prepare_spmv_csr(
            data, indices, indptr, shape, block_nnz=block_nnz, max_segments=max_segments, op=op_code,
            index_fallback_policy=index_fallback_policy,
        )
    else:
        if op_explicit and op_code != prepared.op:
            raise ValueError(
                f"op={_spmv_op_to_name(op_code)} does not match prepared.op={_spmv_op_to_name(prepared.op)}"
            )
        if not op_explicit and transpose is not None and bool(transpose) != prepared.transpose:
            raise ValueError(
                f"transpose={bool(transpose)} does not match prepared.transpose={prepared.transpose}"
            )
    x = _validate_spmv_x(x, prepared)
    t0 = None
    if return_time:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
    y = _run_spmv_prepared_with_fallback(prepared, x, use_opt=use_opt, out=_direct_out(out, prepared, x))
    elapsed_ms = None
    if return_time:
        torch.cuda.synchronize()
        elapsed_ms = (time.perf_counter() - t0) * 1000.0
    y = _spmv_write_out(y, out)
    if return_time:
        return y, elapsed_ms
    return y


def _spmv_write_out(y, out):
    if out is not None and y is not out:
        if not out.is_cuda:
            raise ValueError("out must be a CUDA tensor")
        if out.device != y.device:
            raise ValueError("out must be on the same CUDA device as the result")
        if out.shape != y.shape or out.dtype != y.dtype:
            raise ValueError("out shape/dtype must match result")
        out.copy_(y)
        y = out
    return y


def _spmv_csr_checked(data, indices, indptr, x, shape, use_opt, index_fallback_policy):
    """One-shot y = A x in one native call (fsb_spmv_csr_checked): the
    structural check, its single device->host read, the heuristic plan and
    the product.  Returns None when the call needs the general route: int64
    column indices (FlagSparse's int32 index fallback applies there), an x
    the prepared route would reject, or anything the argument checks below do
    not cover -- that route then raises FlagSparse's errors in its order."""
    _normalize_spmv_index_fallback_policy(index_fallback_policy)
    if not all(torch.is_tensor(t) for t in (data, indices, indptr, x)) or len(shape) != 2:
        return None
    n_rows, n_cols = int(shape[0]), int(shape[1])
    dtype = data.dtype
    if (data.ndim != 1 or indices.ndim != 1 or indptr.ndim != 1 or x.ndim != 1 or indptr.numel() != n_rows + 1
            or data.numel() != indices.numel() or indices.dtype != torch.int32
            or indptr.dtype not in SUPPORTED_INDEX_DTYPES or dtype not in SUPPORTED_SPMV_VALUE_DTYPES
            or x.dtype != dtype or x.numel() != n_cols or not data.is_cuda
            or not all(t.device == data.device for t in (indices, indptr, x))):
        return None
    data, indices, indptr, x = data.contiguous(), indices.contiguous(), indptr.contiguous(), x.contiguous()
    if use_opt and dtype in (torch.float32, torch.float64):
        acc = _nat.ACC_NATIVE
    else:
        acc = _nat.ACC_WIDE if dtype == torch.float32 else _nat.ACC_NATIVE
    y = torch.empty(n_rows, dtype=dtype, device=data.device)
    cm = _nat.make_csr(data, indices, indptr, n_rows, n_cols)
    out_code = _nat.dtype_code(dtype)
    lib = _nat.library()
    nbytes = int(lib.fsb_spmv_csr_checked_workspace_bytes(cm, acc, out_code))
    ws = torch.empty(nbytes, dtype=torch.uint8, device=data.device)
    fig = (ctypes.c_int64 * 8)()
    fig[7] = -1  # empty-row count: >= 0 once the figures were read
    plan = _nat.FsbPlan()
    rc = lib.fsb_spmv_csr_checked(cm, _nat.ptr(x), _nat.ptr(y), out_code, acc, _nat.ptr(ws), nbytes, fig, plan,
                                  _nat.stream_handle(data.device))
    if rc == _nat.FSB_ERR_INVALID and fig[7] >= 0:
        # FlagSparse's messages, in its order (spmv_csr.py:524-537)
        if fig[0] != 0:
            raise ValueError("indptr must start at zero")
        if fig[1] != data.numel():
            raise ValueError("indptr[-1] must equal nnz")
        if fig[2]:
            raise ValueError("indptr must be non-decreasing")
        raise IndexError("indices out of range for n_cols")
    if rc != _nat.FSB_OK:
        return None  # the general route retries (index fallback) or raises
    _plan.LAUNCHES["count"] += 1 + (0 if n_rows == 0 else (1 if plan.algo == _nat.ALGO_ROWS else 3))
    return y


def _coo_is_sorted_lex(row_i64, col_i64, n_cols):
    """True iff COO entries are in non-decreasing (row, col) order."""
    n = row_i64.numel()
    if n <= 1:
        return True
    key = row_i64 * max(1, int(n_cols)) + col_i64
    return bool((key[1:] >= key[:-1]).all().item())


def coo_to_csr_for_spmv(data, row, col, shape, assume_sorted=False):
    """COO -> CSR (data, int32 column indices, int64 indptr), FlagSparse
    ``spmv_csr.py:885-909``: lexicographic (row, col) order unless already sorted."""
    n_rows, n_cols = int(shape[0]), int(shape[1])
    row64 = row.to(torch.int64)
    col64 = col.to(torch.int64)
    if row64.numel() == 0:
        indptr = torch.zeros(n_rows + 1, dtype=torch.int64, device=data.device)
        return data, col64.to(torch.int32), indptr
    if assume_sorted or _coo_is_sorted_lex(row64, col64, n_cols):
        row_s, col_s, data_s = row64, col64, data
    else:
        key = row64 * max(1, n_cols) + col64
        _, order = _plan.stable_sort(key, key_bound=max(1, n_rows) * max(1, n_cols))
        row_s, col_s, data_s = row64[order], col64[order], data[order]
    # row offsets on the device, no host read: with assume_sorted the whole
    # conversion can be captured in a CUDA graph
    indptr = _plan.sorted_keys_to_offsets(row_s, n_rows)
    return data_s, col_s.to(torch.int32), indptr


def prepare_spmv_coo_tocsr(data, row, col, shape, block_nnz=256, max_segments=None, assume_sorted=False):
    """One-time COO -> CSR + plan; use with ``flagsparse_spmv_coo_tocsr(..., prepared=p)``."""
    if not all(torch.is_tensor(t) for t in (data, row, col)):
        raise TypeError("data, row, col must all be torch.Tensor")
    if not all(t.is_cuda for t in (data, row, col)):
        raise ValueError("data, row, col must all be CUDA tensors")
    if data.ndim != 1 or row.ndim != 1 or col.ndim != 1:
        raise ValueError("data, row, col must all be 1D tensors")
    if data.dtype not in SUPPORTED_SPMV_VALUE_DTYPES:
        raise TypeError(_spmv_dtype_error_message())
    if row.numel() != col.numel() or data.numel() != row.numel():
        raise ValueError("data, row, col must have the same length")
    data_s, indices, indptr = coo_to_csr_for_spmv(data, row, col, shape, assume_sorted=assume_sorted)
    return prepare_spmv_csr(data_s, indices, indptr, shape, block_nnz=block_nnz, max_segments=max_segments)


def flagsparse_spmv_coo_tocsr(
    data=None,
    row=None,
    col=None,
    x=None,
    shape=None,
    block_nnz=256,
    max_segments=None,
    out=None,
    return_time=False,
    use_opt=True,
    prepared=None,
    assume_sorted=False,
):
    """COO SpMV via CSR conversion: y = A @ x (FlagSparse ``spmv_csr.py:947-1016``)."""
    if prepared is not None:
        if x is None:
            raise TypeError("x is required")
        if shape is None:
            shape = prepared.shape
        sh = (int(shape[0]), int(shape[1]))
        if sh != prepared.shape:
            raise ValueError(f"shape {sh} does not match prepared.shape {prepared.shape}")
        return flagsparse_spmv_csr(
            x=x, shape=shape, block_nnz=block_nnz, max_segments=max_segments, out=out, return_time=return_time,
            use_opt=use_opt, prepared=prepared,
        )
    if not all(torch.is_tensor(t) for t in (data, row, col, x)):
        raise TypeError("data, row, col, x must all be torch.Tensor")
    if not all(t.is_cuda for t in (data, row, col, x)):
        raise ValueError("data, row, col, x must all be CUDA tensors")
    if data.ndim != 1 or row.ndim != 1 or col.ndim != 1 or x.ndim != 1:
        raise ValueError("data, row, col, x must all be 1D tensors")
    if data.dtype not in SUPPORTED_SPMV_VALUE_DTYPES:
        raise TypeError(_spmv_dtype_error_message())
    if x.dtype != data.dtype:
        raise TypeError("x dtype must match data dtype")
    data_s, indices, indptr = coo_to_csr_for_spmv(data, row, col, shape, assume_sorted=assume_sorted)
    return flagsparse_spmv_csr(
        data_s, indices, indptr, x, shape, block_nnz=block_nnz, max_segments=max_segments, out=out,
        return_time=return_time, use_opt=use_opt,
    )
