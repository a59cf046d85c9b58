"""Seeded synthetic CSR matrices: the workload families of the benchmarks.

Every generator is deterministic for a given (seed, device type) and returns
``(data, indices, indptr, shape)`` with int32 column indices and int64 row
offsets (columns sorted and distinct within a row).  The families:

* ``poisson_uniform``  -- row lengths Poisson(mean), columns uniform
  (SpMV config: 16384 x 16384, mean 16, float32).
* ``zipf_powerlaw``    -- row lengths Zipf(alpha) scaled to a target mean and
  capped, columns uniform (SpMM config: 262144 x 262144, alpha 1.8, mean ~12,
  cap 20000).
* ``banded_plus_random`` -- a dense band of width 64 around the diagonal plus
  4 uniform off-band columns per row, a fraction of rows replaced by long rows
  (precision config: 1,048,576 rows, 1 % of rows with 8192 nonzeros).
* ``block_diagonal``   -- dense 16 x 16 blocks on the diagonal (BSR family).
* ``block_sparse``     -- k dense 16 x 16 blocks per block row, the diagonal
  block among them (BSR family with 16 k nonzeros per row).
* ``rectangular``      -- random 2:1 rectangular with uniform columns.

Values are U(-1, 1); dense operands N(0, 1).
"""

import math

import torch


def _gen(seed, device):
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    return g


def _uniform_values(g, n, dtype, device):
    return (torch.rand(n, generator=g, device=device, dtype=torch.float32) * 2 - 1).to(dtype)


def _rows_from_lengths(lengths, device):
    n_rows = lengths.numel()
    indptr = torch.zeros(n_rows + 1, dtype=torch.int64, device=device)
    indptr[1:] = torch.cumsum(lengths.to(torch.int64), 0)
    nnz = int(indptr[-1].item())
    row_of = torch.repeat_interleave(torch.arange(n_rows, device=device), lengths.to(torch.int64), output_size=nnz)
    return indptr, row_of, nnz


def _distinct_sorted_columns(g, row_of, lengths, n_cols, device, low=None, high=None):
    """Uniform columns, distinct within each row, sorted per row.

    Draws with replacement, then redraws the duplicates of each row until none
    remain (rows never ask for more columns than exist).  ``low``/``high``
    (per-nonzero tensors) restrict the draw to [low, high).
    """
    nnz = row_of.numel()
    if nnz == 0:
        return torch.empty(0, dtype=torch.int64, device=device)
    if low is None:
        cols = torch.randint(0, n_cols, (nnz,), generator=g, device=device)
    else:
        span = (high - low).to(torch.float64)
        cols = low + (torch.rand(nnz, generator=g, device=device, dtype=torch.float64) * span).to(torch.int64)
    for _ in range(64):
        key = row_of * n_cols + cols
        key, order = torch.sort(key)
        cols = cols[order]
        dup = torch.zeros(nnz, dtype=torch.bool, device=device)
        dup[1:] = key[1:] == key[:-1]
        n_dup = int(dup.sum().item())
        if n_dup == 0:
            return cols
        if low is None:
            cols[dup] = torch.randint(0, n_cols, (n_dup,), generator=g, device=device)
        else:
            # rows keep their positions under the sort (row_of is sorted), so
            # the per-position bounds still line up
            lo, hi = low[dup], high[dup]
            cols[dup] = lo + (torch.rand(n_dup, generator=g, device=device, dtype=torch.float64) *
                              (hi - lo).to(torch.float64)).to(torch.int64)
    raise RuntimeError("could not draw distinct columns")


def poisson_uniform(n_rows=16384, n_cols=16384, mean=16.0, seed=0, dtype=torch.float32, device="cuda"):
    g = _gen(seed, device)
    lengths = torch.poisson(torch.full((n_rows,), float(mean), device=device), generator=g).to(torch.int64)
    lengths = lengths.clamp_(max=n_cols)
    indptr, row_of, nnz = _rows_from_lengths(lengths, device)
    cols = _distinct_sorted_columns(g, row_of, lengths, n_cols, device)
    data = _uniform_values(g, nnz, dtype, device)
    return data, cols.to(torch.int32), indptr, (n_rows, n_cols)


def zipf_lengths(n_rows, alpha, mean, cap, g, device):
    """Zipf(alpha) lengths by inverse transform of the continuous power law,
    floored, capped at ``cap`` and scaled so the realised mean is ~``mean``."""
    u = torch.rand(n_rows, generator=g, device=device, dtype=torch.float64).clamp_(min=1e-12)
    raw = torch.floor(u.pow(-1.0 / (alpha - 1.0))).clamp_(max=float(cap))
    scale = mean / float(raw.mean().item())
    lengths = torch.round(raw * scale).clamp_(min=0, max=float(cap)).to(torch.int64)
    return lengths


def zipf_powerlaw(n_rows=262144, n_cols=262144, alpha=1.8, mean=12.0, cap=20000, seed=0, dtype=torch.float32,
                  device="cuda"):
    g = _gen(seed, device)
    lengths = zipf_lengths(n_rows, alpha, mean, min(cap, n_cols), g, device)
    indptr, row_of, nnz = _rows_from_lengths(lengths, device)
    cols = _distinct_sorted_columns(g, row_of, lengths, n_cols, device)
    data = _uniform_values(g, nnz, dtype, device)
    return data, cols.to(torch.int32), indptr, (n_rows, n_cols)


def banded_plus_random(n_rows=1048576, band=64, off_band=4, long_rate=0.01, long_len=8192, seed=0,
                       dtype=torch.bfloat16, device="cuda"):
    """Square matrix: columns [r - band/2, r + band/2) clipped to the matrix plus
    ``off_band`` uniform columns outside the band; a ``long_rate`` fraction of
    rows holds ``long_len`` nonzeros (the band plus uniform columns)."""
    n = n_rows
    g = _gen(seed, device)
    r = torch.arange(n, device=device)
    lo = (r - band // 2).clamp(min=0)
    hi = (r + band // 2).clamp(max=n)
    band_len = hi - lo
    is_long = torch.rand(n, generator=g, device=device) < long_rate
    extra = torch.where(is_long, torch.full_like(band_len, long_len) - band_len,
                        torch.full_like(band_len, off_band)).clamp(min=0)
    extra = torch.minimum(extra, n - band_len)
    lengths = band_len + extra
    indptr, row_of, nnz = _rows_from_lengths(lengths, device)
    # band part: position within row < band_len
    pos = torch.arange(nnz, device=device) - indptr[:-1][row_of]
    in_band = pos < band_len[row_of]
    cols = torch.empty(nnz, dtype=torch.int64, device=device)
    cols[in_band] = lo[row_of[in_band]] + pos[in_band]
    # off-band part: uniform over the columns outside [lo, hi): draw in
    # [0, n - band_len) and shift past the band.
    ob_rows = row_of[~in_band]
    width = (n - band_len[ob_rows])
    draw_hi = width
    draw_lo = torch.zeros_like(draw_hi)
    drawn = _distinct_sorted_columns(g, ob_rows, None, max(n, 1), device, low=draw_lo, high=draw_hi)
    # _distinct_sorted_columns sorted per row; map past the band
    ob_lo = lo[ob_rows]
    drawn = torch.where(drawn >= ob_lo, drawn + band_len[ob_rows], drawn)
    cols[~in_band] = drawn
    key = row_of * n + cols
    key, order = torch.sort(key)
    cols = cols[order]
    data = _uniform_values(g, nnz, dtype, device)
    return data, cols.to(torch.int32), indptr, (n, n)


def block_diagonal(n_blocks=1024, block=16, seed=0, dtype=torch.bfloat16, device="cuda"):
    """Dense ``block`` x ``block`` blocks on the diagonal, as CSR."""
    g = _gen(seed, device)
    n = n_blocks * block
    r = torch.arange(n, device=device)
    lengths = torch.full((n,), block, dtype=torch.int64, device=device)
    indptr, row_of, nnz = _rows_from_lengths(lengths, device)
    pos = torch.arange(nnz, device=device) - indptr[:-1][row_of]
    cols = (row_of // block) * block + pos
    del r
    data = _uniform_values(g, nnz, dtype, device)
    return data, cols.to(torch.int32), indptr, (n, n)


def block_sparse(n_block_rows=1024, blocks_per_row=2, block=16, seed=0, dtype=torch.float32, device="cuda"):
    """Square BSR-structured matrix as CSR: each block row holds
    ``blocks_per_row`` dense ``block`` x ``block`` blocks, the diagonal block
    and uniform distinct other block columns (sorted)."""
    g = _gen(seed, device)
    nb = int(n_block_rows)
    k = max(1, min(int(blocks_per_row), nb))
    # block columns per block row: the diagonal plus k - 1 distinct others
    bcol = torch.empty((nb, k), dtype=torch.int64, device=device)
    bcol[:, 0] = torch.arange(nb, device=device)
    if k > 1:
        brow_of = torch.repeat_interleave(torch.arange(nb, device=device), k - 1)
        lens = torch.full((nb,), k - 1, dtype=torch.int64, device=device)
        others = _distinct_sorted_columns(g, brow_of, lens, max(nb - 1, 1), device)
        others = others.view(nb, k - 1)
        others = torch.where(others >= torch.arange(nb, device=device)[:, None], others + 1, others)
        bcol[:, 1:] = others
    bcol, _ = torch.sort(bcol, dim=1)
    n = nb * block
    lengths = torch.full((n,), k * block, dtype=torch.int64, device=device)
    indptr, row_of, nnz = _rows_from_lengths(lengths, device)
    pos = torch.arange(nnz, device=device) - indptr[:-1][row_of]
    br = row_of // block
    cols = bcol[br, pos // block] * block + pos % block
    data = _uniform_values(g, nnz, dtype, device)
    return data, cols.to(torch.int32), indptr, (n, n)


def rectangular(n_rows=20000, mean=8.0, ratio=2, seed=0, dtype=torch.float32, device="cuda"):
    """n_rows x (n_rows / ratio) with Poisson row lengths and uniform columns."""
    n_cols = max(1, n_rows // ratio)
    return poisson_uniform(n_rows, n_cols, mean=min(mean, n_cols), seed=seed, dtype=dtype, device=device)


def dense_operand(n_rows, n_cols, seed, dtype=torch.float32, device="cuda"):
    g = _gen(seed, device)
    return torch.randn((n_rows, n_cols), generator=g, device=device, dtype=torch.float32).to(dtype)


def dense_vector(n, seed, dtype=torch.float32, device="cuda"):
    g = _gen(seed, device)
    return torch.randn(n, generator=g, device=device, dtype=torch.float32).to(dtype)


def useful_bytes_spmv(nnz, n_rows, n_cols, value_bytes, index_bytes, x_bytes=None, y_bytes=None):
    """values + column indices + x reads + y writes (row offsets excluded)."""
    x_bytes = value_bytes if x_bytes is None else x_bytes
    y_bytes = value_bytes if y_bytes is None else y_bytes
    return nnz * (value_bytes + index_bytes) + n_cols * x_bytes + n_rows * y_bytes


def useful_bytes_spmm(nnz, n_rows, n_cols, n_dense, value_bytes, index_bytes, b_bytes=None, c_bytes=None):
    """values + column indices + B reads + C writes (row offsets excluded)."""
    b_bytes = value_bytes if b_bytes is None else b_bytes
    c_bytes = value_bytes if c_bytes is None else c_bytes
    return nnz * (value_bytes + index_bytes) + n_cols * n_dense * b_bytes + n_rows * n_dense * c_bytes


def log_uniform_int(g, lo, hi, device):
    u = torch.rand(1, generator=g, device=device, dtype=torch.float64).item()
    return int(round(math.exp(math.log(lo) + u * (math.log(hi) - math.log(lo)))))
