"""ctypes front end of the CPU oracle (``oracle.c``).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` to check and time against; the library
``flagsparse_public_b200`` never imports it.

Arguments are CPU torch tensors (moved to the host and made contiguous here);
results are CPU torch tensors.  ``threads=None`` uses every host core.
"""

import ctypes
import os
import subprocess

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

F16, BF16, F32, F64, C64, C128, I32, I64 = range(8)
_CODES = {
    torch.float16: F16, torch.bfloat16: BF16, torch.float32: F32, torch.float64: F64,
    torch.complex64: C64, torch.complex128: C128, torch.int32: I32, torch.int64: I64,
}
ACC_NATIVE, ACC_WIDE = 0, 1

_lib = None


def build():
    """Compile liboracle.so with the committed Makefile (gcc, OpenMP)."""
    res = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    return LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = ctypes.CDLL(LIB_PATH)
        vp, i64, i32 = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int
        lib.orc_spmv_csr.argtypes = [vp, vp, vp, i32, i32, i32, i64, vp, vp, i32, i32, i64, i32]
        lib.orc_spmm_csr.argtypes = [vp, vp, vp, i32, i32, i32, i64, vp, i64, i64, vp, i64, i32, i32, i32]
        lib.orc_spmv_csr_exact.argtypes = [vp, vp, vp, i32, i32, i32, i64, vp, vp, vp, vp, i32]
        lib.orc_spmm_csr_exact.argtypes = [vp, vp, vp, i32, i32, i32, i64, vp, i64, i64, vp, vp, vp, i32]
        lib.orc_csr_transpose.argtypes = [vp, i32, vp, i32, i64, i64, i64, vp, vp, vp]
        lib.orc_coo_lex_order.argtypes = [vp, vp, i64, i64, vp]
        lib.orc_seg_starts.argtypes = [vp, i64, vp]
        lib.orc_seg_starts.restype = i64
        lib.orc_split_metadata.argtypes = [vp, vp, i64, i64, vp, vp, vp, vp]
        lib.orc_split_metadata.restype = i64
        lib.orc_merge_partition.argtypes = [vp, i32, i64, i64, i64, i64, i64, vp]
        lib.orc_spmm_diag.argtypes = [vp, vp, vp, i32, i32, i32, i64, vp, i64, i64, vp, i64, i32, i32, i64, i32]
        lib.orc_merge_runs.argtypes = [vp, i32, i64, vp, i64, vp]
        lib.orc_sddmm_csr.argtypes = [vp, i32, vp, i32, i64, vp, i64, vp, i64, i64, vp, vp, i32,
                                      ctypes.c_double, ctypes.c_double, i32]
        _lib = lib
    return _lib


def _host(t):
    return t.detach().to("cpu").contiguous()


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None and t.numel() > 0 else ctypes.c_void_p(0)


def _threads(threads):
    return int(threads) if threads else (os.cpu_count() or 1)


def spmv_csr(data, indices, indptr, x, acc_mode=ACC_WIDE, out_dtype=None, row_cap=0, threads=None):
    """y = A x in the path's compute precision, rows summed in order."""
    data, indices, indptr, x = map(_host, (data, indices, indptr, x))
    n_rows = indptr.numel() - 1
    out_dtype = out_dtype or data.dtype
    y = torch.empty(n_rows, dtype=out_dtype)
    _load().orc_spmv_csr(_p(data), _p(indices), _p(indptr), _CODES[data.dtype], _CODES[indices.dtype],
                         _CODES[indptr.dtype], n_rows, _p(x), _p(y), _CODES[out_dtype], acc_mode, int(row_cap),
                         _threads(threads))
    return y


def spmm_csr(data, indices, indptr, B, acc_mode=ACC_WIDE, out_dtype=None, threads=None):
    """C = A B in the path's compute precision (B row-major)."""
    data, indices, indptr, B = map(_host, (data, indices, indptr, B))
    n_rows = indptr.numel() - 1
    n_dense = B.shape[1]
    out_dtype = out_dtype or data.dtype
    C = torch.empty((n_rows, n_dense), dtype=out_dtype)
    _load().orc_spmm_csr(_p(data), _p(indices), _p(indptr), _CODES[data.dtype], _CODES[indices.dtype],
                         _CODES[indptr.dtype], n_rows, _p(B), B.stride(0) if B.numel() else n_dense, n_dense, _p(C),
                         n_dense, _CODES[out_dtype], acc_mode, _threads(threads))
    return C


def spmm_diag(data, indices, indptr, B, mode_short, mode_long=None, short_max=-1, threads=None):
    """Diagnose-only SpMM arithmetic (orc_spmm_diag): modes 0 native fma,
    1 float64 fma stored in the value type, 2 Kahan, 3 Kahan in float64; rows
    of at most ``short_max`` nonzeros use ``mode_short``, the others
    ``mode_long`` (default: the same)."""
    data, indices, indptr, B = map(_host, (data, indices, indptr, B))
    B = B.contiguous()
    n_rows = indptr.numel() - 1
    n_dense = B.shape[1]
    mode_long = mode_short if mode_long is None else mode_long
    C = torch.empty((n_rows, n_dense), dtype=data.dtype)
    rc = _load().orc_spmm_diag(_p(data), _p(indices), _p(indptr), _CODES[data.dtype], _CODES[indices.dtype],
                               _CODES[indptr.dtype], n_rows, _p(B), n_dense, n_dense, _p(C), n_dense, int(mode_short),
                               int(mode_long), int(short_max), _threads(threads))
    if rc != 0:
        raise TypeError("orc_spmm_diag: float32 / float64 values only")
    return C


def spmv_csr_exact(data, indices, indptr, x, threads=None):
    """FP64 oracle: (y as float64/complex128, sum_k |a_k x_k| per row)."""
    data, indices, indptr, x = map(_host, (data, indices, indptr, x))
    n_rows = indptr.numel() - 1
    re = torch.empty(n_rows, dtype=torch.float64)
    im = torch.empty(n_rows, dtype=torch.float64)
    mag = torch.empty(n_rows, dtype=torch.float64)
    _load().orc_spmv_csr_exact(_p(data), _p(indices), _p(indptr), _CODES[data.dtype], _CODES[indices.dtype],
                               _CODES[indptr.dtype], n_rows, _p(x), _p(re), _p(im), _p(mag), _threads(threads))
    y = torch.complex(re, im) if data.dtype.is_complex else re
    return y, mag


def spmm_csr_exact(data, indices, indptr, B, threads=None):
    """FP64 oracle of C = A B: (C float64/complex128, sum_k |a_k b_k| per entry)."""
    data, indices, indptr, B = map(_host, (data, indices, indptr, B))
    n_rows = indptr.numel() - 1
    n_dense = B.shape[1]
    re = torch.empty((n_rows, n_dense), dtype=torch.float64)
    im = torch.empty((n_rows, n_dense), dtype=torch.float64)
    mag = torch.empty((n_rows, n_dense), dtype=torch.float64)
    _load().orc_spmm_csr_exact(_p(data), _p(indices), _p(indptr), _CODES[data.dtype], _CODES[indices.dtype],
                               _CODES[indptr.dtype], n_rows, _p(B), B.stride(0) if B.numel() else n_dense, n_dense,
                               _p(re), _p(im), _p(mag), _threads(threads))
    C = torch.complex(re, im) if data.dtype.is_complex else re
    return C, mag


def csr_transpose(indptr, indices, n_rows, n_cols):
    """(t_indptr, t_rows, perm), all int64: the stable-by-column transpose."""
    indptr, indices = _host(indptr), _host(indices)
    nnz = indices.numel()
    t_ptr = torch.empty(n_cols + 1, dtype=torch.int64)
    t_rows = torch.empty(nnz, dtype=torch.int64)
    perm = torch.empty(nnz, dtype=torch.int64)
    rc = _load().orc_csr_transpose(_p(indptr), _CODES[indptr.dtype], _p(indices), _CODES[indices.dtype], n_rows,
                                   n_cols, nnz, _p(t_ptr), _p(t_rows), _p(perm))
    if rc:
        raise MemoryError("orc_csr_transpose")
    return t_ptr, t_rows, perm


def coo_lex_order(row, col, n_cols):
    """Stable permutation ordering COO entries by (row, col)."""
    row = _host(row).to(torch.int64)
    col = _host(col).to(torch.int64)
    perm = torch.empty(row.numel(), dtype=torch.int64)
    if _load().orc_coo_lex_order(_p(row), _p(col), row.numel(), n_cols, _p(perm)):
        raise MemoryError("orc_coo_lex_order")
    return perm


def seg_starts(sorted_row):
    row = _host(sorted_row).to(torch.int64)
    seg = torch.empty(row.numel() + 1, dtype=torch.int64)
    n = _load().orc_seg_starts(_p(row), row.numel(), _p(seg))
    return seg[: n + 1] if n > 0 else None


def split_metadata(indptr, long_rows, part_nnz):
    indptr = _host(indptr).to(torch.int64)
    long_rows = _host(long_rows).to(torch.int64)
    lens = indptr[long_rows + 1] - indptr[long_rows] if long_rows.numel() else torch.zeros(0, dtype=torch.int64)
    cap = int(((lens + part_nnz - 1) // part_nnz).sum().item()) if long_rows.numel() else 0
    rows = torch.empty(cap, dtype=torch.int64)
    starts = torch.empty(cap, dtype=torch.int64)
    ends = torch.empty(cap, dtype=torch.int64)
    rpp = torch.empty(long_rows.numel() + 1, dtype=torch.int64)
    n = _load().orc_split_metadata(_p(indptr), _p(long_rows), long_rows.numel(), part_nnz, _p(rows), _p(starts),
                                   _p(ends), _p(rpp))
    return rows[:n], starts[:n], ends[:n], rpp


def merge_runs(indptr, n_rows, coords):
    """(first, last) unit of the split-row run of each unit's open row, -1 when
    the unit's end is not inside a row (int64 [n_units * 2])."""
    indptr, coords = _host(indptr), _host(coords).to(torch.int64)
    n_units = coords.numel() // 2 - 1
    runs = torch.empty(max(n_units, 0) * 2, dtype=torch.int64)
    if n_units > 0:
        _load().orc_merge_runs(_p(indptr), _CODES[indptr.dtype], int(n_rows), _p(coords), n_units, _p(runs))
    return runs


def csr_check(indptr, indices):
    """The structural figures FlagSparse's CSR validation reads one by one
    (``spmv_csr.py:524-541``: indptr[0], indptr[-1], non-decreasing offsets,
    index range; ``row_lengths.max()``) plus the row-length statistics of the
    plan heuristics, as eight integers: row_ptr[0], row_ptr[-1], rows of
    negative length, negative column indices, largest non-negative column
    index, longest row, sum of squared row lengths, empty rows (the last three
    over rows of non-negative length)."""
    p = _host(indptr).to(torch.int64)
    c = _host(indices).to(torch.int64)
    lens = p[1:] - p[:-1]
    ok = lens[lens >= 0]
    nonneg = c[c >= 0]
    return [int(p[0]), int(p[-1]), int((lens < 0).sum()), int((c < 0).sum()),
            int(nonneg.max()) if nonneg.numel() else 0, int(ok.max()) if ok.numel() else 0,
            int((ok * ok).sum()), int((ok == 0).sum())]


def merge_partition(indptr, n_rows, nnz, items, snap=0):
    indptr = _host(indptr)
    total = n_rows + nnz
    n_units = -(-total // items) if total > 0 else 0
    coords = torch.empty((n_units + 1) * 2, dtype=torch.int64)
    _load().orc_merge_partition(_p(indptr), _CODES[indptr.dtype], n_rows, nnz, items, snap, n_units, _p(coords))
    return coords


def sddmm_csr(indices, indptr, x, y, data=None, alpha=1.0, beta=0.0, threads=None):
    """out[p] = alpha * dot(x[row(p)], y[col(p)]) + beta * data[p] on the CSR
    pattern, accumulated in the value precision (float32 / float64)."""
    indices, indptr, x, y = map(_host, (indices, indptr, x, y))
    data = _host(data) if data is not None else None
    n_rows = indptr.numel() - 1
    out = torch.empty(indices.numel(), dtype=x.dtype)
    rc = _load().orc_sddmm_csr(_p(indices), _CODES[indices.dtype], _p(indptr), _CODES[indptr.dtype], n_rows, _p(x),
                               x.stride(0) if x.numel() else x.shape[1], _p(y), y.stride(0) if y.numel() else y.shape[1],
                               x.shape[1], _p(data) if data is not None else None, _p(out), _CODES[x.dtype],
                               float(alpha), float(beta), _threads(threads))
    if rc != 0:
        raise TypeError("sddmm oracle: values must be float32 or float64")
    return out


def struct_rows(indices, indptr, long_min, min_run):
    """Per-row descriptors of the structured form (pure Python, small cases):
    the row's longest run of consecutive columns -- (first column, offset in
    the row, length), the first run on ties, (0, 0, 0) when shorter than
    min_run -- or (0, 0, -1) for rows of more than long_min nonzeros."""
    indices, indptr = _host(indices).tolist(), _host(indptr).tolist()
    out = []
    for r in range(len(indptr) - 1):
        s, e = indptr[r], indptr[r + 1]
        if e - s > long_min:
            out.append((0, 0, -1))
            continue
        best_len, best_start, start = 0, 0, 0
        for k in range(1, e - s + 1):
            if k == e - s or indices[s + k] != indices[s + k - 1] + 1:
                if k - start > best_len:
                    best_len, best_start = k - start, start
                start = k
        if best_len >= min_run and best_len > 0:
            out.append((indices[s + best_start], best_start, best_len))
        else:
            out.append((0, 0, 0))
    t = torch.tensor(out, dtype=torch.int32).view(-1, 3)
    return t[:, 0].contiguous(), t[:, 1].contiguous(), t[:, 2].contiguous()


def struct_tiles(run_col, run_off, run_len, tile_rows=128, span_max=256):
    """Tile spans of the structured form: per tile of tile_rows rows, the
    smallest run column; runs ending more than span_max columns past it are
    dropped (length and offset set to 0); width rounded up to 16.  Returns
    (tile_base, tile_span, run_off, run_len) (the last two updated)."""
    run_col = _host(run_col).tolist()
    run_off, run_len = _host(run_off).clone(), _host(run_len).clone()
    n = len(run_col)
    bases, spans = [], []
    for t0 in range(0, max(n, 1), tile_rows):
        rows = [r for r in range(t0, min(n, t0 + tile_rows)) if int(run_len[r]) > 0]
        if not rows:
            bases.append(0)
            spans.append(0)
            continue
        lo = min(run_col[r] for r in rows)
        hi = lo
        for r in rows:
            end = run_col[r] + int(run_len[r])
            if end - lo > span_max:
                run_len[r] = 0
                run_off[r] = 0
            else:
                hi = max(hi, end)
        bases.append(lo)
        spans.append((hi - lo + 15) // 16 * 16)
    return (torch.tensor(bases, dtype=torch.int64), torch.tensor(spans, dtype=torch.int32), run_off, run_len)
