"""Block-sparse (BSR, dense 16 x 16 blocks) SpMM on the tensor cores.

FlagSparse multiplies block-structured matrices as plain CSR
(``flagsparse_spmm_csr``, spmm_csr.py:2088-2157): every nonzero is gathered
and multiplied on its own.  When the nonzeros come in dense 16 x 16 blocks,
each block is a small dense contraction; ``flagsparse_spmm_bsr`` runs it as
one tcgen05 tensor-core MMA per block and 128-column tile
(``fsb_bsr_spmm_tc``), bf16 or f16 values and dense operand, fp32
accumulation and fp32 result.

``csr_to_bsr16`` converts a CSR matrix to this form on the device (blocks that
hold any nonzero are stored dense, zero-filled), so a CSR user can switch.
"""

import torch

from . import _native as nat
from . import _plan

BLOCK = 16
BSR_VALUE_DTYPES = (torch.bfloat16, torch.float16)


def block_count(indices, indptr, shape):
    """Number of 16 x 16 blocks holding at least one nonzero (the blocks
    csr_to_bsr16 stores), computed on the device without building them."""
    n_rows, n_cols = int(shape[0]), int(shape[1])
    nnz = int(indices.numel())
    if nnz == 0:
        return 0
    nbc = (n_cols + BLOCK - 1) // BLOCK
    lens = (indptr[1:] - indptr[:-1]).to(torch.int64)
    row = torch.repeat_interleave(torch.arange(n_rows, device=indices.device), lens, output_size=nnz)
    key = (row // BLOCK) * nbc + indices.to(torch.int64) // BLOCK
    return int(torch.unique(key).numel())


def csr_to_bsr16(data, indices, indptr, shape, dtype=None):
    """(block_values [n_blocks, 16, 16], block_col int32, block_row_ptr int64)
    of the 16 x 16 blocks holding the CSR matrix's nonzeros (sorted by block
    row, then block column; integer work on the device, bit-exact)."""
    n_rows, n_cols = int(shape[0]), int(shape[1])
    dev = data.device
    dtype = dtype or data.dtype
    nbr = (n_rows + BLOCK - 1) // BLOCK
    nbc = (n_cols + BLOCK - 1) // BLOCK
    lens = (indptr[1:] - indptr[:-1]).to(torch.int64)
    row = torch.repeat_interleave(torch.arange(n_rows, device=dev), lens, output_size=int(data.numel()))
    col = indices.to(torch.int64)
    key = (row // BLOCK) * nbc + col // BLOCK
    ukeys, inverse = torch.unique(key, sorted=True, return_inverse=True)
    n_blocks = int(ukeys.numel())
    vals = torch.zeros((n_blocks, BLOCK, BLOCK), dtype=dtype, device=dev)
    vals[inverse, row % BLOCK, col % BLOCK] = data.to(dtype)
    brow = ukeys // nbc
    bcol = (ukeys % nbc).to(torch.int32)
    counts = torch.bincount(brow, minlength=nbr)
    bptr = torch.zeros(nbr + 1, dtype=torch.int64, device=dev)
    bptr[1:] = torch.cumsum(counts, 0)
    return vals, bcol, bptr


class PreparedBsr:
    """Validated BSR operands for repeated products."""

    __slots__ = ("block_values", "block_col", "block_row_ptr", "shape", "n_blocks")

    def __init__(self, block_values, block_col, block_row_ptr, shape):
        if block_values.dtype not in BSR_VALUE_DTYPES:
            raise TypeError("BSR values must be bfloat16 or float16")
        if not block_values.is_cuda:
            raise ValueError("BSR operands must be CUDA tensors")
        n_rows, n_cols = int(shape[0]), int(shape[1])
        nbr = (n_rows + BLOCK - 1) // BLOCK
        if block_values.dim() != 3 or tuple(block_values.shape[1:]) != (BLOCK, BLOCK):
            raise ValueError("block_values must have shape (n_blocks, 16, 16)")
        if block_row_ptr.numel() != nbr + 1:
            raise ValueError(f"block_row_ptr must have ceil(n_rows / 16) + 1 = {nbr + 1} entries")
        if block_col.numel() != block_values.shape[0]:
            raise ValueError("block_col must have one entry per block")
        if block_col.numel():
            lo, hi = int(block_col.min().item()), int(block_col.max().item())
            if lo < 0 or hi >= (n_cols + BLOCK - 1) // BLOCK:
                raise IndexError("block_col out of range")
        self.block_values = block_values.contiguous()
        self.block_col = block_col.contiguous()
        self.block_row_ptr = block_row_ptr.contiguous()
        self.shape = (n_rows, n_cols)
        self.n_blocks = int(block_col.numel())


def prepare_spmm_bsr(block_values, block_col, block_row_ptr, shape):
    return PreparedBsr(block_values, block_col, block_row_ptr, shape)


def flagsparse_spmm_bsr(block_values=None, block_col=None, block_row_ptr=None, B=None, shape=None, prepared=None,
                        out=None, staging="auto"):
    """C = A B (fp32) for a BSR matrix of dense 16 x 16 blocks on the tensor
    cores; B row-major with the values' 16-bit type, columns a multiple of 8.
    ``staging``: "tma" (B slices loaded by the Tensor Memory Accelerator),
    "threads" (loaded by the CTA's threads) or "auto" (TMA where a tensor map
    can be encoded for B, else threads)."""
    if staging not in ("auto", "tma", "threads"):
        raise ValueError('staging must be "auto", "tma" or "threads"')
    if prepared is None:
        prepared = PreparedBsr(block_values, block_col, block_row_ptr, shape)
    p = prepared
    if B is None or not torch.is_tensor(B) or B.dim() != 2:
        raise TypeError("B must be a 2D torch.Tensor")
    if B.dtype != p.block_values.dtype:
        raise TypeError("B dtype must match the block values' dtype")
    if B.device != p.block_values.device:
        raise ValueError("B must be on the sparse matrix's device")
    if B.shape[0] != p.shape[1]:
        raise ValueError(f"B.shape[0] must be n_cols={p.shape[1]}")
    B = B.contiguous()
    n_dense = int(B.shape[1])
    if n_dense % 8:
        raise ValueError("the tensor-core BSR path needs B with a multiple of 8 columns")
    C = out if out is not None else torch.empty((p.shape[0], n_dense), dtype=torch.float32, device=B.device)
    if out is not None and (out.dtype != torch.float32 or out.shape != (p.shape[0], n_dense) or not out.is_contiguous()):
        raise ValueError("out must be a contiguous float32 tensor of shape (n_rows, n_dense)")
    lib = nat.library()

    def launch(mode):
        return lib.fsb_bsr_spmm_tc(nat.ptr(p.block_values), nat.dtype_code(p.block_values.dtype),
                                   nat.ptr(p.block_col), nat.dtype_code(p.block_col.dtype), nat.ptr(p.block_row_ptr),
                                   nat.dtype_code(p.block_row_ptr.dtype), p.shape[0], p.shape[1], p.n_blocks,
                                   nat.ptr(B),
                                   int(B.stride(0)), n_dense, nat.ptr(C), int(C.stride(0)), mode,
                                   nat.stream_handle(B.device))

    rc = launch(nat.BSR_STAGE_THREADS if staging == "threads" else nat.BSR_STAGE_TMA)
    if rc == nat.FSB_ERR_UNSUPPORTED and staging == "auto":
        rc = launch(nat.BSR_STAGE_THREADS)
    nat.check(rc, "fsb_bsr_spmm_tc")
    _plan.LAUNCHES["count"] += 1 if p.shape[0] and n_dense else 0
    return C
