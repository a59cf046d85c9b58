"""Structured form of a half-precision CSR matrix: runs of consecutive columns
and long rows (the host side of csrc/fsb_struct.cu).

Built once per matrix on the device and kept beside the caller's CSR arrays,
which stay as they are:

* per row, the row's longest run of consecutive columns (fsb_struct_rows),
  or a mark for rows of more than LONG_MIN nonzeros;
* per tile of 128 rows, the column span of the tile's runs (fsb_struct_tiles);
* the long rows: their indices, chunks of CHUNK_NNZ nonzeros (SpMM) and their
  nonzeros regrouped by blocks of XBLOCK columns of x, with 16-bit offsets
  inside the block (SpMV; a stable device sort keeps each row's column order).

The precision form (sparse_operations/precision.py) runs its products through
fsb_struct_spmv / fsb_struct_spmm when runs and long rows hold most of the
nonzeros (``worthwhile``): run values are then read without column indices,
the band's B rows are staged once per tile for the tensor cores, and the long
rows gather x from shared memory.
"""

import torch

from . import _native as nat
from . import _plan

LONG_MIN = 1024  # rows with more nonzeros take the long-row kernels
# SpMM long-row tiles: rows per group and columns per block (the compiled
# shape, two shared-memory stages)
LT_ROWS = 512
LT_COLS = 1024
MIN_RUN = 16  # shorter runs of consecutive columns count as none
CHUNK_NNZ = 1024  # SpMM: nonzeros per chunk of a long row
XBLOCK = 65536  # SpMV: columns of x per shared-memory block (128 KB of 16-bit values)
TILE_ROWS = 128
SPMM_WIDTHS = (16, 32, 64)  # dense widths of the tensor-core band tiles
WORTHWHILE = 0.5  # runs + long rows must hold at least this share of the nonzeros


class StructuredForm:
    """Device descriptors of one matrix and the C struct pointing at them."""

    __slots__ = ("run_col", "run_off", "run_len", "tile_base", "tile_span", "max_span", "long_rows", "chunk_row",
                 "chunk_ptr", "seg_ptr", "seg_val", "seg_off", "n_long", "n_chunks", "xblock", "n_xblocks",
                 "run_nnz", "long_nnz", "nnz", "lt_groups", "lt_col_blocks", "lt_rec_cap", "lt_rows", "lt_rec", "lt_seg_start",
                 "lt_seg_len", "lt_row_start", "_c", "_ws")

    def worthwhile(self):
        return self.nnz > 0 and (self.run_nnz + self.long_nnz) >= WORTHWHILE * self.nnz

    def stats(self):
        return {"run_nnz": self.run_nnz, "long_nnz": self.long_nnz, "nnz": self.nnz, "long_rows": self.n_long,
                "chunks": self.n_chunks, "max_span": self.max_span, "xblocks": self.n_xblocks}

    def moved_bytes(self, n_rows, n_cols, value_bytes, ptr_bytes, n_dense=0):
        """Algorithmic bytes of one structured product: run values without
        indices, scattered nonzeros with their indices, per-row descriptors
        (run column, offset, length) and row offsets, the long rows' prepared
        stream (SpMM: 32-bit records and per-segment row starts; SpMV: values
        and 16-bit offsets), the dense operand read once and the result
        written once (SpMV: n_dense = 0)."""
        short_scatter = self.nnz - self.run_nnz - self.long_nnz
        b = self.run_nnz * value_bytes + short_scatter * (value_bytes + 4) + n_rows * (12 + ptr_bytes)
        if n_dense:
            if self.lt_rec is not None:
                b += self.lt_rec.numel() * 4 + self.lt_row_start.numel() * 2 + self.lt_seg_start.numel() * 12
            else:
                b += self.long_nnz * (value_bytes + 4)
            b += n_cols * n_dense * value_bytes + n_rows * n_dense * 4
        else:
            b += self.long_nnz * (value_bytes + 2) + (self.n_xblocks * self.n_long + 1) * 8
            b += n_cols * value_bytes + n_rows * 4
        return int(b)

    def c_struct(self):
        if self._c is None:
            s = nat.FsbStruct()
            s.run_col, s.run_off, s.run_len = (t.data_ptr() for t in (self.run_col, self.run_off, self.run_len))
            s.tile_base, s.tile_span = self.tile_base.data_ptr(), self.tile_span.data_ptr()
            s.max_span, s.chunk_nnz = self.max_span, CHUNK_NNZ
            s.n_long = self.n_long
            s.long_rows = self.long_rows.data_ptr() if self.n_long else 0
            s.n_chunks = self.n_chunks
            s.chunk_row = self.chunk_row.data_ptr() if self.n_long else 0
            s.chunk_ptr = self.chunk_ptr.data_ptr() if self.n_long else 0
            s.xblock, s.n_xblocks = self.xblock, self.n_xblocks
            s.seg_ptr = self.seg_ptr.data_ptr() if self.n_long else 0
            s.seg_val = self.seg_val.data_ptr() if self.n_long and self.seg_val.numel() else 0
            s.seg_off = self.seg_off.data_ptr() if self.n_long and self.seg_off.numel() else 0
            if self.lt_rec is not None:
                s.lt_groups, s.lt_col_blocks, s.lt_rec_cap = self.lt_groups, self.lt_col_blocks, self.lt_rec_cap
                s.lt_rows, s.lt_cols = self.lt_rows, LT_COLS
                s.lt_rec = self.lt_rec.data_ptr()
                s.lt_seg_start = self.lt_seg_start.data_ptr()
                s.lt_seg_len = self.lt_seg_len.data_ptr()
                s.lt_row_start = self.lt_row_start.data_ptr()
            self._c = s
        return self._c

    def workspace(self, is_spmm, n_dense, device):
        key = (bool(is_spmm), int(n_dense))
        ws = self._ws.get(key)
        if ws is None:
            nbytes = int(nat.library().fsb_struct_workspace_bytes(int(is_spmm), self.c_struct(), int(n_dense)))
            ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=device)
            self._ws[key] = ws
        return ws


def build(data, indices, indptr, n_rows, n_cols):
    """The structured form of a CSR matrix on its device (several host reads:
    the long-row list and the share statistics)."""
    dev = data.device
    lib = nat.library()
    st = nat.stream_handle(dev)
    n_rows, n_cols = int(n_rows), int(n_cols)
    f = StructuredForm()
    f._c, f._ws = None, {}
    f.nnz = int(data.numel())
    f.run_col = torch.empty(max(n_rows, 1), dtype=torch.int32, device=dev)
    f.run_off = torch.empty_like(f.run_col)
    f.run_len = torch.zeros_like(f.run_col)
    n_tiles = max(1, -(-n_rows // TILE_ROWS))
    f.tile_base = torch.zeros(n_tiles, dtype=torch.int64, device=dev)
    f.tile_span = torch.zeros(n_tiles, dtype=torch.int32, device=dev)
    cm = nat.make_csr(data, indices, indptr, n_rows, n_cols)
    nat.check(lib.fsb_struct_rows(cm, LONG_MIN, MIN_RUN, nat.ptr(f.run_col), nat.ptr(f.run_off), nat.ptr(f.run_len),
                                  st), "fsb_struct_rows")
    nat.check(lib.fsb_struct_tiles(n_rows, nat.ptr(f.run_col), nat.ptr(f.run_off), nat.ptr(f.run_len),
                                   nat.ptr(f.tile_base), nat.ptr(f.tile_span), st), "fsb_struct_tiles")
    rl = f.run_len[:n_rows]
    long_rows = torch.nonzero(rl < 0).flatten()
    lens = indptr[1:] - indptr[:-1]
    long_lens = lens[long_rows]
    stats = torch.stack([rl.clamp(min=0).sum(), long_lens.sum(), f.tile_span.max().to(torch.int64)]).tolist()
    f.run_nnz, f.long_nnz, f.max_span = int(stats[0]), int(stats[1]), int(stats[2])
    f.n_long = int(long_rows.numel())
    f.long_rows = long_rows.to(torch.int32)
    f.xblock = min(XBLOCK, max(8, -(-n_cols // 8) * 8))
    f.n_xblocks = max(1, -(-n_cols // f.xblock))
    f.n_chunks = 0
    f.chunk_row = f.chunk_ptr = f.seg_ptr = f.seg_val = f.seg_off = None
    f.lt_groups = f.lt_col_blocks = f.lt_rec_cap = f.lt_rows = 0
    f.lt_rec = f.lt_seg_start = f.lt_seg_len = f.lt_row_start = None
    if f.n_long:
        # SpMM: chunks of CHUNK_NNZ nonzeros, chunk_ptr[l] = first chunk of long row l
        nch = (long_lens + CHUNK_NNZ - 1) // CHUNK_NNZ
        f.chunk_ptr = torch.zeros(f.n_long + 1, dtype=torch.int64, device=dev)
        f.chunk_ptr[1:] = torch.cumsum(nch, 0)
        f.n_chunks = int(f.chunk_ptr[-1])
        f.chunk_row = torch.repeat_interleave(torch.arange(f.n_long, dtype=torch.int32, device=dev), nch,
                                              output_size=f.n_chunks)
        # SpMV: the long rows' nonzeros by (x block, long row), each row's
        # columns in order inside its segment (stable sort)
        total = f.long_nnz
        off = torch.zeros(f.n_long + 1, dtype=torch.int64, device=dev)
        off[1:] = torch.cumsum(long_lens, 0)
        lpos = torch.repeat_interleave(torch.arange(f.n_long, device=dev), long_lens, output_size=total)
        gidx = torch.arange(total, device=dev) - off[:-1][lpos] + indptr[long_rows].to(torch.int64)[lpos]
        cols = indices[gidx].to(torch.int64)
        blk = cols // f.xblock
        n_seg = f.n_xblocks * f.n_long
        keys, perm = _plan.stable_sort(blk * f.n_long + lpos, key_bound=n_seg)
        # padded to a multiple of 8 elements: the SpMV reads whole 16-byte chunks
        padded = -(-max(total, 1) // 8) * 8
        f.seg_val = torch.zeros(padded, dtype=data.dtype, device=dev)
        f.seg_val[:total] = data[gidx[perm]]
        rel = (cols - blk * f.xblock)[perm]
        f.seg_off = torch.zeros(padded, dtype=torch.int16, device=dev)
        f.seg_off[:total] = torch.where(rel >= 32768, rel - 65536, rel).to(torch.int16)  # uint16 bit patterns
        f.seg_ptr = _plan.sorted_keys_to_offsets(keys, n_seg)
        _build_long_tiles(f, data, gidx, lpos, cols, n_cols)
    return f


def _lt_rec_cap_max(rows, cols, n_dense_max=32):
    """Longest segment (records) whose stages fit in shared memory."""
    stages = 2
    budget = (227 * 1024 - 2048) // stages - cols * n_dense_max * 2 - (rows + 8) * 2
    return max(0, budget // 16 * 4)


def _build_long_tiles(f, data, gidx, lpos, cols, n_cols):
    """SpMM: the long rows' nonzeros as (row group of LT_ROWS, column block
    of LT_COLS) segments of 32-bit records (value bits | column inside the
    block << 16), ordered by row (each row's columns in order: stable sort),
    padded to 4 records, with LT_ROWS + 8 16-bit per-row record starts per
    segment.  Left out (SpMM runs the long rows in chunks) when a segment is
    longer than the shared-memory stages take."""
    dev = data.device
    rows_g, rs_n = LT_ROWS, LT_ROWS + 8
    groups = -(-f.n_long // rows_g)
    blocks = max(1, -(-n_cols // LT_COLS))
    n_seg = groups * blocks
    key = ((lpos // rows_g) * blocks + cols // LT_COLS) * rows_g + lpos % rows_g
    skey, perm = _plan.stable_sort(key, key_bound=n_seg * rows_g)
    offs = _plan.sorted_keys_to_offsets(skey, n_seg * rows_g)  # [n_seg * rows_g + 1]
    first = offs[::rows_g]  # segment boundaries, n_seg + 1 entries
    cnt = first[1:] - first[:-1]
    seg_len = (cnt + 3) // 4 * 4
    cap = int(seg_len.max())
    if cap > _lt_rec_cap_max(rows_g, LT_COLS):
        return
    seg_start = torch.zeros(n_seg, dtype=torch.int64, device=dev)
    seg_start[1:] = torch.cumsum(seg_len, 0)[:-1]
    total_pad = int(seg_len.sum())
    grid = torch.arange(n_seg, device=dev)[:, None] * rows_g + torch.arange(rows_g + 1, device=dev)[None, :]
    rs = offs[grid] - first[:-1][:, None]
    row_start = torch.empty((n_seg, rs_n), dtype=torch.int64, device=dev)
    row_start[:, : rows_g + 1] = rs
    row_start[:, rows_g + 1:] = rs[:, rows_g:]
    seg_of = skey // rows_g
    pos = seg_start[seg_of] + (torch.arange(skey.numel(), device=dev) - first[:-1][seg_of])
    vbits = data[gidx[perm]].view(torch.int16).to(torch.int32) & 0xFFFF
    rec = torch.zeros(max(total_pad, 4), dtype=torch.int32, device=dev)
    rec[pos] = vbits | ((cols[perm] % LT_COLS).to(torch.int32) << 16)
    f.lt_groups, f.lt_col_blocks, f.lt_rec_cap, f.lt_rows = groups, blocks, cap, rows_g
    f.lt_rec = rec
    f.lt_seg_start = seg_start
    f.lt_seg_len = seg_len.to(torch.int32)
    f.lt_row_start = row_start.to(torch.int16).contiguous()  # uint16 bit patterns (starts <= cap < 2^15)


def spmv(form, data, indices, indptr, n_rows, n_cols, x, y):
    """y (float32) = A x through fsb_struct_spmv on torch's current stream."""
    lib = nat.library()
    cm = nat.make_csr(data, indices, indptr, n_rows, n_cols)
    ws = form.workspace(False, 1, data.device)
    rc = lib.fsb_struct_spmv(cm, form.c_struct(), nat.ptr(x), nat.ptr(y), nat.ptr(ws), ws.numel(),
                             nat.stream_handle(data.device))
    nat.check(rc, "fsb_struct_spmv")
    _plan.LAUNCHES["count"] += 3 if form.n_long else 1
    return y


def spmm_supported(form, B, C):
    """Whether fsb_struct_spmm takes these operands (dense width of 16, 32 or
    64; 16-byte aligned B and C rows)."""
    n = int(B.shape[1])
    return (n in SPMM_WIDTHS and B.data_ptr() % 16 == 0 and C.data_ptr() % 16 == 0 and B.stride(0) % 8 == 0
            and C.stride(0) % 4 == 0 and B.stride(1) == 1 and C.stride(1) == 1)


def spmm(form, data, indices, indptr, n_rows, n_cols, B, C):
    """C (float32) = A B through fsb_struct_spmm on torch's current stream."""
    lib = nat.library()
    cm = nat.make_csr(data, indices, indptr, n_rows, n_cols)
    n_dense = int(B.shape[1])
    ws = form.workspace(True, n_dense, data.device)
    rc = lib.fsb_struct_spmm(cm, form.c_struct(), nat.ptr(B), int(B.stride(0)), n_dense, nat.ptr(C),
                             int(C.stride(0)), nat.ptr(ws), ws.numel(), nat.stream_handle(data.device))
    nat.check(rc, "fsb_struct_spmm")
    _plan.LAUNCHES["count"] += 3 if form.n_long else 1
    return C
