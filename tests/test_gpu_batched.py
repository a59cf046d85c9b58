"""Batched uneven SpMM (one persistent launch in a CUDA graph) against the
FP64 product of every matrix of the batch."""

import pytest
import torch

from flagsparse_public_b200 import _native as nat
from flagsparse_public_b200 import _plan, batched, synthetic

DEV = "cuda"
pytestmark = pytest.mark.gpu


def _batch(count, seed):
    g = torch.Generator().manual_seed(seed)
    mats = []
    for i in range(count):
        n = int(torch.randint(1, 3000, (1,), generator=g))
        mean = float(torch.rand(1, generator=g) * 30 + 0.5)
        mats.append(synthetic.poisson_uniform(n, n, mean=min(mean, n), seed=seed * 1000 + i, device=DEV))
    # an all-empty matrix and a one-row matrix with a long row
    mats.append((torch.zeros(0, device=DEV), torch.zeros(0, dtype=torch.int32, device=DEV),
                 torch.zeros(5, dtype=torch.int64, device=DEV), (4, 4)))
    mats.append(synthetic.poisson_uniform(1, 5000, mean=1500.0, seed=7, device=DEV))
    return mats


def _check(prep, mats, n_dense):
    for i, m in enumerate(mats):
        ref = torch.sparse_csr_tensor(m[2].cpu(), m[1].long().cpu(), m[0].double().cpu(), size=m[3]) @ \
            prep.b_views[i].double().cpu()
        got = prep.c_views[i].double().cpu()
        mag = (torch.sparse_csr_tensor(m[2].cpu(), m[1].long().cpu(), m[0].double().abs().cpu(), size=m[3]) @
               prep.b_views[i].double().abs().cpu())
        err = ((got - ref).abs() / mag.clamp_min(1e-30)).max().item() if got.numel() else 0.0
        assert err < 1e-5, (i, err)


@pytest.mark.parametrize("n_dense", [32, 8])
def test_batched_graph_matches_each_product(n_dense):
    mats = _batch(40, 1)
    prep = batched.prepare_spmm_csr_batch(mats, n_dense)
    assert prep.timings is not None and prep.plan.algo == nat.ALGO_SEQ
    for i, v in enumerate(prep.b_views):
        v.copy_(synthetic.dense_operand(v.shape[0], n_dense, seed=100 + i, device=DEV))
    prep.run()
    torch.cuda.synchronize()
    _check(prep, mats, n_dense)
    # new operands, same graph
    prep.B.mul_(-0.5)
    prep.run()
    torch.cuda.synchronize()
    _check(prep, mats, n_dense)


def test_persistent_grid_is_bit_identical_to_full_grid():
    mats = _batch(25, 2)
    full = batched.prepare_spmm_csr_batch(mats, 32, plan=_plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=256))
    pers = batched.prepare_spmm_csr_batch(mats, 32, plan=_plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=256,
                                                                          grid_blocks=5))
    B = synthetic.dense_operand(full.n_cols, 32, seed=3, device=DEV)
    full.B.copy_(B)
    pers.B.copy_(B)
    full.run()
    pers.run()
    torch.cuda.synchronize()
    assert torch.equal(full.C, pers.C)
