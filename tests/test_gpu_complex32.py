"""complex32 (torch complex32 / chalf: float16 pairs) through the SpMM paths
FlagSparse lists for it -- CSR ALG1 (flagsparse_spmm_csr) with every plan
family and COO SpMM (row runs and atomics) -- against the FP64 oracle of the
same (exactly widened) inputs.  FlagSparse accumulates complex32 in float32
(spmm_csr.py:576-598); so do the kernels here, in registers.

Bound per entry: |c - c64| <= 1e-3 * sum_k |a_k b_k| + 2^-24 (one float16
rounding of each output part, float32 accumulation, the float16 subnormal
spacing for tiny results)."""

import pytest
import torch

import flagsparse_public_b200 as fs
from flagsparse_public_b200 import _native as nat
from flagsparse_public_b200 import _plan
from flagsparse_public_b200.sparse_operations import spmm_coo as mc
from oracle import oracle as orc
from tests.gpu_cases import EDGE_LENGTHS, csr_from_lengths, dense, spmm_plans

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(getattr(torch, "complex32", None) is None, reason="no complex32 in this torch")]
DEV = "cuda"
C32 = getattr(torch, "complex32", None)


def _case(lengths, n_cols, n_dense, seed):
    data64, indices, indptr, (n_rows, n_cols) = csr_from_lengths(lengths, n_cols, seed=seed, dtype=torch.complex64)
    data = data64.to(C32)
    B = dense((n_cols, n_dense), seed + 1, torch.complex64).to(C32)
    exact, mag = orc.spmm_csr_exact(data.to(torch.complex64), indices, indptr, B.to(torch.complex64))
    return data, indices, indptr, n_rows, n_cols, B, exact, mag


def _check(C, exact, mag):
    diff = (C.cpu().to(torch.complex128) - exact.to(torch.complex128)).abs()
    bound = 1e-3 * mag.to(torch.float64) + 2.0 ** -24
    assert bool((diff <= bound).all()), float((diff - bound).max())


@pytest.mark.parametrize("pattern", ["empty_rows", "boundaries", "skewed", "one_row"])
@pytest.mark.parametrize("n_dense", [1, 3, 8, 32, 64])
def test_complex32_all_plans(pattern, n_dense):
    lengths = EDGE_LENGTHS[pattern][::3] if pattern == "skewed" else EDGE_LENGTHS[pattern]
    data, indices, indptr, n_rows, n_cols, B, exact, mag = _case(lengths, 13000, n_dense, 61)
    d = (data.to(DEV), indices.to(DEV), indptr.to(DEV))
    Bd = B.to(DEV)
    for plan in spmm_plans():
        C = torch.empty((n_rows, n_dense), dtype=C32, device=DEV)
        if plan.algo == nat.ALGO_GATHER and not _plan.gather_supported(Bd, C, plan.n_tile):
            continue
        if plan.flags & nat.PLAN_TMA_GATHER:
            assert not _plan.g4_supported(d[0], Bd, C, nat.ACC_NATIVE, n_cols)
            continue
        _plan.run_spmm(*d, n_rows, n_cols, Bd, C, nat.ACC_NATIVE, plan)
        _check(C, exact, mag)


def test_complex32_public_csr_and_coo():
    lengths = [5, 0, 40, 7, 300, 1, 0, 2000, 3]
    data, indices, indptr, n_rows, n_cols, B, exact, mag = _case(lengths, 5000, 24, 63)
    d_data, d_idx, d_ptr, Bd = data.to(DEV), indices.to(DEV), indptr.to(DEV), B.to(DEV)
    C = fs.flagsparse_spmm_csr(d_data, d_idx, d_ptr, Bd, (n_rows, n_cols))
    assert C.dtype == C32
    _check(C, exact, mag)
    # COO: the same entries in shuffled order, row runs and atomics
    rows = torch.repeat_interleave(torch.arange(n_rows), indptr[1:] - indptr[:-1])
    perm = torch.randperm(data.numel(), generator=torch.Generator().manual_seed(64))
    r, c, v = rows[perm].to(DEV), indices[perm].to(DEV), data.to(torch.complex64)[perm].to(C32).to(DEV)
    C2 = fs.flagsparse_spmm_coo(v, r, c, Bd, (n_rows, n_cols))
    assert C2.dtype == C32
    _check(C2, exact, mag)
    C3 = mc._triton_spmm_coo_impl(v, r, c, Bd, n_rows, 24, None, 256, route="atomic")
    assert C3.dtype == C32
    _check(C3, exact, mag)


def test_complex32_opt_path_rejects_like_reference():
    data, indices, indptr, n_rows, n_cols, B, _, _ = _case([3, 4], 50, 8, 65)
    p = fs.prepare_spmm_csr_opt(data.to(DEV), indices.to(DEV), indptr.to(DEV), (n_rows, n_cols))
    with pytest.raises(TypeError, match="only supports float32 and float64"):
        fs.flagsparse_spmm_csr_opt(B=B.to(DEV), prepared=p)
