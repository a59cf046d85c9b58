"""Tensor-core BSR SpMM (tcgen05) against an FP64 product of the same 16-bit
inputs: fp32 accumulation of exact 16-bit products, condition-scaled error
<= 1e-5."""

import pytest
import torch

from flagsparse_public_b200 import bsr, synthetic

DEV = "cuda"
pytestmark = pytest.mark.gpu


def _check(vals, bcol, bptr, shape, B, C):
    n_rows, n_cols = shape
    nbr = bptr.numel() - 1
    dense = torch.zeros(nbr * 16, ((n_cols + 15) // 16) * 16, dtype=torch.float64)
    v, c, p = vals.double().cpu(), bcol.cpu(), bptr.cpu()
    for br in range(nbr):
        for b in range(int(p[br]), int(p[br + 1])):
            j = int(c[b])
            dense[16 * br:16 * br + 16, 16 * j:16 * j + 16] = v[b]
    A = dense[:n_rows, :n_cols]
    Bd = B.double().cpu()
    ref = A @ Bd
    mag = A.abs() @ Bd.abs()
    err = ((C.double().cpu() - ref).abs() / mag.clamp_min(1e-30)).max().item() if C.numel() else 0.0
    assert err <= 1e-5, err


STAGINGS = ["tma", "threads"]


@pytest.mark.parametrize("staging", STAGINGS)
@pytest.mark.parametrize("n_dense", [8, 32, 128])
def test_block_diagonal_single_tile(n_dense, staging):
    data, indices, indptr, shape = synthetic.block_sparse(8, 1, seed=1, dtype=torch.bfloat16, device=DEV)
    vals, bcol, bptr = bsr.csr_to_bsr16(data, indices, indptr, shape)
    B = synthetic.dense_operand(shape[1], n_dense, seed=2, dtype=torch.bfloat16, device=DEV)
    C = bsr.flagsparse_spmm_bsr(vals, bcol, bptr, B, shape, staging=staging)
    torch.cuda.synchronize()
    _check(vals, bcol, bptr, shape, B, C)


@pytest.mark.parametrize("staging", STAGINGS)
@pytest.mark.parametrize("dtype", [torch.bfloat16, torch.float16])
@pytest.mark.parametrize("n_dense", [16, 136, 256])
def test_block_sparse_many_blocks_per_row(dtype, n_dense, staging):
    data, indices, indptr, shape = synthetic.block_sparse(300, 9, seed=3, dtype=dtype, device=DEV)
    vals, bcol, bptr = bsr.csr_to_bsr16(data, indices, indptr, shape)
    B = synthetic.dense_operand(shape[1], n_dense, seed=4, dtype=dtype, device=DEV)
    C = bsr.flagsparse_spmm_bsr(vals, bcol, bptr, B, shape, staging=staging)
    torch.cuda.synchronize()
    _check(vals, bcol, bptr, shape, B, C)


@pytest.mark.parametrize("staging", STAGINGS)
def test_ragged_shapes_empty_block_rows_and_repeat_calls(staging):
    # 37 x 45: partial last block row and block column; rows 16..31 empty
    data, indices, indptr, shape = synthetic.poisson_uniform(37, 45, mean=9.0, seed=6, dtype=torch.bfloat16,
                                                             device=DEV)
    lens = indptr[1:] - indptr[:-1]
    keep = torch.ones(data.numel(), dtype=torch.bool, device=DEV)
    row = torch.repeat_interleave(torch.arange(37, device=DEV), lens)
    keep &= (row < 16) | (row >= 32)
    counts = torch.bincount(row[keep], minlength=37)
    indptr2 = torch.zeros(38, dtype=torch.int64, device=DEV)
    indptr2[1:] = torch.cumsum(counts, 0)
    vals, bcol, bptr = bsr.csr_to_bsr16(data[keep], indices[keep], indptr2, shape)
    assert int(bptr[2] - bptr[1]) == 0
    B = synthetic.dense_operand(45, 24, seed=7, dtype=torch.bfloat16, device=DEV)
    for _ in range(2):
        C = torch.full((37, 24), float("nan"), device=DEV)
        bsr.flagsparse_spmm_bsr(vals, bcol, bptr, B, shape, out=C, staging=staging)
        torch.cuda.synchronize()
        _check(vals, bcol, bptr, shape, B, C)
        assert torch.all(C[16:32] == 0)


def test_staging_paths_agree_bitwise():
    """Both stagings feed the same MMAs in the same order."""
    data, indices, indptr, shape = synthetic.block_sparse(500, 6, seed=8, dtype=torch.bfloat16, device=DEV)
    vals, bcol, bptr = bsr.csr_to_bsr16(data, indices, indptr, shape)
    B = synthetic.dense_operand(shape[1], 128, seed=9, dtype=torch.bfloat16, device=DEV)
    a = bsr.flagsparse_spmm_bsr(vals, bcol, bptr, B, shape, staging="tma")
    b = bsr.flagsparse_spmm_bsr(vals, bcol, bptr, B, shape, staging="threads")
    torch.cuda.synchronize()
    assert torch.equal(a, b)
