"""COO SpMV without CSR indptr: FlagSparse's ``spmv_coo`` operator API.

Follows FlagSparse ``sparse_operations/spmv_coo.py``:

- ``sort_by_row=True`` (default): lexicographic (row, col) sort and row-run
  offsets ``seg_starts`` (length #runs + 1, ``spmv_coo.py:297-327``); one
  result per run, no atomics.  Here the sort, the run bounds and the row
  offsets stay on the device (the run bounds reach the host only when
  ``seg_starts`` is read) and the runs go through the CSR kernels of
  ``libflagsparse_b200.so`` as rows of the sorted structure.
- ``sort_by_row=False``: one atomic add per nonzero (``:229-294``).

Accumulation is in the value precision (float32 for float32, ``:148``).
"""

from ._common import *
from .. import _native as _nat
from .. import _plan

SUPPORTED_SPMV_COO_VALUE_DTYPES = (torch.float32, torch.float64, torch.complex64, torch.complex128)

SPMV_COO_OP_NON = 0
SPMV_COO_OP_TRANS = 1
SPMV_COO_OP_CONJ_TRANS = 2
SPMV_COO_OP_NAMES = {SPMV_COO_OP_NON: "non", SPMV_COO_OP_TRANS: "trans", SPMV_COO_OP_CONJ_TRANS: "conj"}
_SPMV_COO_OP_NAME_TO_CODE = {name: code for code, name in SPMV_COO_OP_NAMES.items()}


def _spmv_coo_dtype_error_message():
    return "COO SpMV supports float32, float64, complex64, and complex128"


def _normalize_spmv_coo_op(op=None, transpose=False):
    if op is None:
        return SPMV_COO_OP_TRANS if bool(transpose) else SPMV_COO_OP_NON
    if isinstance(op, str):
        token = op.strip().lower()
        if token not in _SPMV_COO_OP_NAME_TO_CODE:
            raise ValueError("op must be one of: 0=non, 1=trans, 2=conj")
        return _SPMV_COO_OP_NAME_TO_CODE[token]
    try:
        op_code = int(op)
    except (TypeError, ValueError) as exc:
        raise ValueError("op must be one of: 0=non, 1=trans, 2=conj") from exc
    if op_code not in SPMV_COO_OP_NAMES:
        raise ValueError("op must be one of: 0=non, 1=trans, 2=conj")
    return op_code


def _spmv_coo_op_to_name(op):
    return SPMV_COO_OP_NAMES[_normalize_spmv_coo_op(op)]


def _spmv_coo_op_transposes(op):
    return _normalize_spmv_coo_op(op) in (SPMV_COO_OP_TRANS, SPMV_COO_OP_CONJ_TRANS)


def _normalize_spmv_coo_index_fallback_policy(index_fallback_policy):
    policy = str(index_fallback_policy).lower()
    if policy not in ("auto", "strict"):
        raise ValueError("index_fallback_policy must be 'auto' or 'strict'")
    return policy


class PreparedCoo:
    """Sorted COO + optional row-run bounds ``seg_starts`` (FlagSparse ``spmv_coo.py:77-128``).

    ``seg_starts`` may be given as a tensor (FlagSparse's constructor) or, from
    ``prepare_spmv_coo``, as ``runs`` = (starts buffer, device run count): the
    run bounds are then read to the host only when ``seg_starts`` / ``n_segs``
    are first accessed, so a prepare records in a CUDA graph.  The products
    run over per-row offsets of the sorted rows, which need no run count."""

    __slots__ = (
        "data",
        "row",
        "col",
        "shape",
        "n_rows",
        "n_cols",
        "nnz",
        "_seg_starts",
        "_runs",
        "_row_ptr",
        "use_seg_kernel",
        "op",
        "transpose",
        "index_fallback_policy",
        "index_fallback_applied",
        "index_fallback_reason",
        "_plan",
    )

    def __init__(
        self,
        data,
        row,
        col,
        shape,
        seg_starts=None,
        transpose=False,
        op=None,
        index_fallback_policy="auto",
        index_fallback_applied=False,
        index_fallback_reason=None,
        runs=None,
    ):
        self.data = data
        self.row = row
        self.col = col
        self.shape = (int(shape[0]), int(shape[1]))
        self.n_rows, self.n_cols = self.shape
        self.nnz = int(data.numel())
        self._seg_starts = seg_starts
        self._runs = runs if seg_starts is None else None
        self._row_ptr = None
        if seg_starts is not None:
            self.use_seg_kernel = int(seg_starts.numel()) - 1 > 0
        else:
            self.use_seg_kernel = self._runs is not None and self.nnz > 0
        self.op = _normalize_spmv_coo_op(op, transpose=transpose)
        self.transpose = _spmv_coo_op_transposes(self.op)
        self.index_fallback_policy = str(index_fallback_policy).lower()
        self.index_fallback_applied = bool(index_fallback_applied)
        self.index_fallback_reason = index_fallback_reason
        self._plan = None

    @property
    def seg_starts(self):
        if self._seg_starts is None and self._runs is not None:
            starts, count = self._runs
            self._seg_starts = starts[: int(count.item())].clone()
            self._runs = None
        return self._seg_starts

    @property
    def n_segs(self):
        seg = self.seg_starts
        return 0 if seg is None else int(seg.numel()) - 1


def _sort_coo_lex_inplace(data, row, col, n_cols, n_rows=None):
    """Lexicographic (row, col) order; indices promoted to a common dtype
    (FlagSparse ``spmv_coo.py:297-309``)."""
    index_dtype = torch.promote_types(row.dtype, col.dtype)
    if data.numel() == 0:
        return data.contiguous(), row.to(index_dtype).contiguous(), col.to(index_dtype).contiguous()
    key = row.to(torch.int64) * max(1, int(n_cols)) + col.to(torch.int64)
    bound = None if n_rows is None else max(1, int(n_rows)) * max(1, int(n_cols))
    _, order = _plan.stable_sort(key, key_bound=bound)
    return data[order].contiguous(), row[order].to(index_dtype).contiguous(), col[order].to(index_dtype).contiguous()


def _seg_starts_from_sorted_rows(row, nnz, device):
    """Boundaries of constant-row runs in sorted COO (FlagSparse ``spmv_coo.py:312-327``)."""
    if nnz == 0:
        return None
    index_dtype = row.dtype if nnz <= _INDEX_LIMIT_INT32 else torch.int64
    return _plan.run_starts(row, index_dtype)


def _prepare_coo_tensors(data, row, col, shape, sort_by_row):
    if not all(torch.is_tensor(t) for t in (data, row, col)):
        raise TypeError("data, row, col must all be torch.Tensor")
    if data.ndim != 1 or row.ndim != 1 or col.ndim != 1:
        raise ValueError("data, row, col must be 1D")
    if not all(t.is_cuda for t in (data, row, col)):
        raise ValueError("data, row, col must be CUDA tensors")
    n_rows, n_cols = int(shape[0]), int(shape[1])
    if data.numel() != row.numel() or data.numel() != col.numel():
        raise ValueError("data, row, col must have the same length")
    if data.dtype not in SUPPORTED_SPMV_COO_VALUE_DTYPES:
        raise TypeError(_spmv_coo_dtype_error_message())
    if row.dtype not in SUPPORTED_INDEX_DTYPES:
        raise TypeError("row dtype must be torch.int32 or torch.int64")
    if col.dtype not in SUPPORTED_INDEX_DTYPES:
        raise TypeError("col dtype must be torch.int32 or torch.int64")
    index_dtype = torch.promote_types(row.dtype, col.dtype)
    if sort_by_row:
        data, kr, kc = _sort_coo_lex_inplace(data, row, col, n_cols, n_rows)
        nnz = data.numel()
        runs = _plan.run_starts_device(kr, kr.dtype if nnz <= _INDEX_LIMIT_INT32 else torch.int64) if nnz else None
    else:
        data = data.contiguous()
        kr = row.to(index_dtype).contiguous()
        kc = col.to(index_dtype).contiguous()
        runs = None
    # the index checks read the device: skipped while a CUDA graph records
    # the prepare (the caller checks the indices before capturing)
    if data.numel() > 0 and not torch.cuda.is_current_stream_capturing():
        lim = torch.stack([kr.min().to(torch.int64), kr.max().to(torch.int64),
                           kc.min().to(torch.int64), kc.max().to(torch.int64)]).tolist()
        if lim[0] < 0 or lim[1] >= n_rows:
            raise IndexError("row indices out of range")
        if lim[2] < 0 or lim[3] >= n_cols:
            raise IndexError("col indices out of range")
    return data, kr, kc, runs


def prepare_spmv_coo(data, row, col, shape, sort_by_row=True, transpose=False, op=None,
                     index_fallback_policy="auto"):
    """Cache sorted COO + row-run ``seg_starts`` when ``sort_by_row``. No ``indptr``."""
    index_fallback_policy = _normalize_spmv_coo_index_fallback_policy(index_fallback_policy)
    op_code = _normalize_spmv_coo_op(op, transpose=transpose)
    if op is not None and bool(transpose) and op_code == SPMV_COO_OP_NON:
        raise ValueError("transpose=True conflicts with op=non")
    transpose = _spmv_coo_op_transposes(op_code)
    if transpose:
        shape = (int(shape[1]), int(shape[0]))
        row, col = col, row
        if op_code == SPMV_COO_OP_CONJ_TRANS and _is_complex_dtype(data.dtype):
            data = data.conj().resolve_conj()
    d, kr, kc, runs = _prepare_coo_tensors(data, row, col, shape, sort_by_row)
    if sort_by_row and runs is None:  # no entries: the one-entry run bound of FlagSparse
        seg = torch.zeros(1, dtype=kr.dtype, device=d.device)
        return PreparedCoo(d, kr, kc, shape, seg_starts=seg, transpose=transpose, op=op_code,
                           index_fallback_policy=index_fallback_policy)
    return PreparedCoo(d, kr, kc, shape, transpose=transpose, op=op_code, index_fallback_policy=index_fallback_policy,
                       runs=runs)


def _validate_x_coo(x, prepared):
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


def _coo_row_ptr(prepared):
    """int64 offsets of the sorted rows (fsb_sorted_keys_to_offsets): every
    row, empty ones included, so no run count is needed on the host."""
    if prepared._row_ptr is None:
        prepared._row_ptr = _plan.sorted_keys_to_offsets(prepared.row, prepared.n_rows)
    return prepared._row_ptr


def _coo_run_plan(prepared):
    """Plan from the sizes the host knows: the longest row is taken as
    unknown (as long as all nonzeros), so short-row matrices go merge path,
    which is balanced whatever the row lengths."""
    if prepared._plan is None:
        n, nnz = prepared.n_rows, prepared.nnz
        stats = _plan.MatrixStats(n, prepared.n_cols, nnz, nnz, nnz / max(n, 1), 0.0, 0)
        prepared._plan = _plan.default_spmv_plan(stats, prepared.data.dtype)
    return prepared._plan


def _triton_spmv_coo_kernel(prepared, x, block_size, num_warps, block_inner):
    """Row-run or atomic COO SpMV (FlagSparse ``spmv_coo.py:423-492``).

    ``block_size`` / ``num_warps`` / ``block_inner`` are FlagSparse's Triton tile
    sizes; they are validated by the caller and do not change the result here.
    """
    del block_size, num_warps, block_inner
    dtype = prepared.data.dtype
    y = torch.zeros(prepared.n_rows, dtype=dtype, device=prepared.data.device)
    if prepared.nnz == 0:
        return y
    if prepared.use_seg_kernel:
        # the row runs as rows of a CSR structure over all rows: each run's
        # sum in entry order, empty rows 0
        _plan.run_spmv(prepared.data, prepared.col, _coo_row_ptr(prepared), prepared.n_rows, prepared.n_cols, x, y,
                       _nat.ACC_NATIVE, _coo_run_plan(prepared))
        return y
    lib = _nat.library()
    row = prepared.row if prepared.row.dtype == prepared.col.dtype else prepared.row.to(prepared.col.dtype)
    rc = lib.fsb_spmv_coo_atomic(_nat.ptr(prepared.data), _nat.ptr(row), _nat.ptr(prepared.col),
                                 _nat.dtype_code(dtype), _nat.dtype_code(prepared.col.dtype), prepared.nnz,
                                 _nat.ptr(x), _nat.ptr(y), _nat.dtype_code(dtype), _nat.stream_handle(y.device))
    _nat.check(rc, "fsb_spmv_coo_atomic")
    return y


def _spmv_coo_uses_int64_indices(prepared):
    return (
        prepared.row.dtype == torch.int64
        or prepared.col.dtype == torch.int64
        or (prepared.seg_starts is not None and prepared.seg_starts.dtype == torch.int64)
    )


def _spmv_coo_int32_fallback_blocker(prepared):
    for name, tensor in (("row", prepared.row), ("col", prepared.col)):
        if tensor.numel() > 0:
            min_index = int(tensor.min().item())
            max_index = int(tensor.max().item())
            if min_index < 0 or max_index > _INDEX_LIMIT_INT32:
                return f"{name} index range [{min_index}, {max_index}] cannot fit int32 for shape={prepared.shape}"
    if prepared.seg_starts is not None and prepared.seg_starts.numel() > 0:
        max_offset = int(prepared.seg_starts[-1].item())
        if max_offset > _INDEX_LIMIT_INT32:
            return f"COO nnz offset {max_offset} cannot fit int32 for shape={prepared.shape}"
    if prepared.n_rows > _INDEX_LIMIT_INT32 or prepared.n_cols > _INDEX_LIMIT_INT32:
        return f"shape {prepared.shape} cannot fit int32 row/col metadata"
    return None


def _spmv_coo_prepared_with_int32_indices(prepared, reason):
    blocker = _spmv_coo_int32_fallback_blocker(prepared)
    if blocker is not None:
        raise RuntimeError(f"native int64 COO SpMV failed and int32 fallback is unsafe: {blocker}")
    seg_starts = None if prepared.seg_starts is None else prepared.seg_starts.to(torch.int32).contiguous()
    return PreparedCoo(
        data=prepared.data,
        row=prepared.row.to(torch.int32).contiguous(),
        col=prepared.col.to(torch.int32).contiguous(),
        shape=prepared.shape,
        seg_starts=seg_starts,
        transpose=prepared.transpose,
        op=prepared.op,
        index_fallback_policy=prepared.index_fallback_policy,
        index_fallback_applied=True,
        index_fallback_reason=str(reason),
    )


def _run_spmv_coo_prepared_with_fallback(prepared, x, block_size, num_warps, block_inner):
    try:
        return _triton_spmv_coo_kernel(prepared, x, block_size=block_size, num_warps=num_warps,
                                       block_inner=block_inner)
    except Exception as exc:
        if prepared.index_fallback_policy != "auto" or not _spmv_coo_uses_int64_indices(prepared):
            raise
        fallback_prepared = _spmv_coo_prepared_with_int32_indices(prepared, exc)
        return _triton_spmv_coo_kernel(fallback_prepared, x, block_size=block_size, num_warps=num_warps,
                                       block_inner=block_inner)


def flagsparse_spmv_coo(
    data=None,
    row=None,
    col=None,
    x=None,
    shape=None,
    out=None,
    return_time=False,
    prepared=None,
    sort_by_row=True,
    block_size=256,
    num_warps=4,
    block_inner=128,
    transpose=None,
    op=None,
    index_fallback_policy="auto",
):
    """COO SpMV with no CSR indptr (FlagSparse ``spmv_coo.py:575-663``)."""
    op_explicit = op is not None
    op_code = _normalize_spmv_coo_op(op, transpose=False if transpose is None else bool(transpose))
    if op_explicit and transpose is not None and bool(transpose) != _spmv_coo_op_transposes(op_code):
        raise ValueError("transpose conflicts with op")
    if prepared is None:
        if any(a is None for a in (data, row, col, x, shape)):
            raise ValueError("data, row, col, x, shape required when prepared is None")
        prepared = prepare_spmv_coo(data, row, col, shape, sort_by_row=sort_by_row, op=op_code,
                                    index_fallback_policy=index_fallback_policy)
    else:
        if x is None:
            raise TypeError("x is required when prepared is set")
        if op_explicit and op_code != prepared.op:
            raise ValueError(
                f"op={_spmv_coo_op_to_name(op_code)} does not match prepared.op={_spmv_coo_op_to_name(prepared.op)}"
            )
        if not op_explicit and transpose is not None and bool(transpose) != prepared.transpose:
            raise ValueError(
                f"transpose={bool(transpose)} does not match prepared.transpose={prepared.transpose}"
            )
        if shape is None:
            shape = prepared.shape
        sh = (int(shape[0]), int(shape[1]))
        if sh != prepared.shape:
            raise ValueError(f"shape {sh} does not match prepared.shape {prepared.shape}")
    x = _validate_x_coo(x, prepared)
    if num_warps not in (1, 2, 4, 8, 16, 32):
        raise ValueError("num_warps must be a power of 2 in [1, 32]")
    if block_inner <= 0 or (block_inner & (block_inner - 1)) != 0:
        raise ValueError("block_inner must be a positive power of 2")
    t0 = None
    if return_time:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
    y = _run_spmv_coo_prepared_with_fallback(prepared, x, block_size=block_size, num_warps=num_warps,
                                             block_inner=block_inner)
    elapsed_ms = None
    if return_time:
        torch.cuda.synchronize()
        elapsed_ms = (time.perf_counter() - t0) * 1000.0
    if out is not None:
        if out.shape != y.shape or out.dtype != y.dtype:
            raise ValueError("out shape/dtype must match result")
        out.copy_(y)
        y = out
    if return_time:
        return y, elapsed_ms
    return y
