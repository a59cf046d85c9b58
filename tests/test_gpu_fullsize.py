"""The configured workloads at their full sizes, checked through properties
that do not depend on size, plus exact sampled rows.

* Column checksum: the column sums of C = A B equal (1^T A) B.  With every
  entry of C within eps * sum_k |a_k b_k| of the exact product, the checksum
  of column j is within eps * ((1^T |A|) |B|)_j; eps is the bound of the form
  (float32 accumulation 3e-5, float64 accumulation of float32 data 1e-5).
* Linearity: A (2 B1 - 3 B2) against 2 A B1 - 3 A B2, entrywise within
  eps * (2 |A||B1| + 3 |A||B2|) (x 2 for the two sides).
* Rows against the FP64 oracle, condition-scaled: every row of the
  power-law SpMM and of the Poisson SpMV; sampled rows (a fixed stride plus
  the longest rows) of the larger configurations.
Matrices: the power-law SpMM config (262144 x 262144, Zipf 1.8, mean 12,
N = 64), the Poisson SpMV config (16384 x 16384, mean 16), the banded
precision config (1,048,576 rows, 1 % rows of 8192, bf16 and fp16, SpMM with
N = 32 and SpMV), the
512-matrix batch config (N = 32) and the tensor-core BSR config (65536 block
rows x 4 blocks, N = 128, bf16)."""

import pytest
import torch

import flagsparse_public_b200 as fs
from flagsparse_public_b200 import bsr, synthetic
from oracle import oracle as orc
from tests.numerics import scaled_error

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


def _colsum_check(C, data, indices, B, eps):
    """|colsum(C) - (1^T A) B| <= eps * (1^T |A|) |B| (+ the float64 sum's own rounding)."""
    n_cols = B.shape[0]
    w = torch.zeros(n_cols, dtype=torch.float64, device=DEV).index_add_(0, indices.long(), data.double())
    wa = torch.zeros(n_cols, dtype=torch.float64, device=DEV).index_add_(0, indices.long(), data.double().abs())
    ref = w @ B.double()
    mag = wa @ B.double().abs()
    got = C.double().sum(0)
    err = ((got - ref).abs() - 1e-12 * mag).clamp(min=0) / mag.clamp(min=1e-300)
    assert float(err.max()) <= eps, float(err.max())


def _sampled_rows(indptr_h, step=4096, longest=8):
    n = indptr_h.numel() - 1
    lens = indptr_h[1:] - indptr_h[:-1]
    rows = torch.cat([torch.arange(0, n, step), torch.topk(lens, min(longest, n)).indices])
    return torch.unique(rows)


def _sub_csr(data_h, indices_h, indptr_h, rows):
    parts_d, parts_i, ptr = [], [], [0]
    for r in rows.tolist():
        s, e = int(indptr_h[r]), int(indptr_h[r + 1])
        parts_d.append(data_h[s:e])
        parts_i.append(indices_h[s:e])
        ptr.append(ptr[-1] + e - s)
    return torch.cat(parts_d), torch.cat(parts_i), torch.tensor(ptr, dtype=torch.int64)


@pytest.fixture(scope="module")
def powerlaw():
    data, indices, indptr, shape = synthetic.zipf_powerlaw(262144, 262144, alpha=1.8, mean=12.0, cap=20000, seed=0,
                                                           device=DEV)
    return data, indices, indptr, shape


def test_powerlaw_spmm_full_size(powerlaw):
    data, indices, indptr, shape = powerlaw
    B1 = synthetic.dense_operand(shape[1], 64, seed=1, device=DEV)
    B2 = synthetic.dense_operand(shape[1], 64, seed=2, device=DEV)
    p = fs.prepare_spmm_csr_opt(data, indices, indptr, shape)
    C1 = fs.flagsparse_spmm_csr_opt(B=B1, prepared=p)
    C2 = fs.flagsparse_spmm_csr_opt(B=B2, prepared=p)
    C12 = fs.flagsparse_spmm_csr_opt(B=2 * B1 - 3 * B2, prepared=p)
    _colsum_check(C1, data, indices, B1, 3e-5)
    # linearity, entrywise, condition-scaled by |A| (2|B1| + 3|B2|)
    absA = fs.flagsparse_spmm_csr_opt(data.abs(), indices, indptr, 2 * B1.abs() + 3 * B2.abs(), shape)
    lin = ((C12.double() - (2 * C1.double() - 3 * C2.double())).abs() / absA.double().clamp(min=1e-30))
    assert float(lin.max()) <= 2 * 3e-5 * 1.01
    # every row against the FP64 oracle (3.1 M nonzeros x 64 columns on the host)
    h = [t.cpu() for t in (data, indices, indptr)]
    ex, mag = orc.spmm_csr_exact(*h, B1.cpu())
    assert scaled_error(C1.cpu(), ex, mag) <= 3e-5
    # the FlagSparse-compatible plain form (float64 accumulation): within one
    # float32 rounding of the FP64 result on every row
    Cp = fs.flagsparse_spmm_csr(data, indices, indptr, B1, shape)
    _colsum_check(Cp, data, indices, B1, 1e-5)
    assert scaled_error(Cp.cpu(), ex, mag) <= 1e-5


def test_poisson_spmv_full_size_exact():
    data, indices, indptr, shape = synthetic.poisson_uniform(seed=0, device=DEV)
    x = synthetic.dense_vector(shape[1], seed=1, device=DEV)
    ex, mag = orc.spmv_csr_exact(data.cpu(), indices.cpu(), indptr.cpu(), x.cpu())
    for use_opt, bound in ((False, 1e-5), (True, 3e-5)):
        y = fs.flagsparse_spmv_csr(data, indices, indptr, x, shape, use_opt=use_opt)
        assert scaled_error(y, ex, mag) <= bound


@pytest.fixture(scope="module", params=[torch.bfloat16, torch.float16], ids=["bf16", "f16"])
def banded(request):
    dt = request.param
    data, indices, indptr, shape = synthetic.banded_plus_random(seed=0, dtype=dt, device=DEV)
    p = fs.prepare_csr_mixed(data, indices, indptr, shape)
    h = [t.cpu() for t in (data, indices, indptr)]
    lens = h[2][1:] - h[2][:-1]
    long_rows = torch.nonzero(lens > 4096).flatten()[::64]
    rows = torch.unique(torch.cat([_sampled_rows(h[2], step=4099), long_rows]))
    return dt, data, indices, indptr, shape, p, h, rows, long_rows


def test_banded_precision_spmm_full_size(banded):
    """Precision-form SpMM (N = 32) of the banded-plus-random config: float32
    result, column checksum, sampled and long rows against FP64 of the same
    half-precision inputs (long rows compensated: 2e-7)."""
    dt, data, indices, indptr, shape, p, h, rows, long_rows = banded
    B = synthetic.dense_operand(shape[1], 32, seed=1, dtype=dt, device=DEV)
    C = fs.flagsparse_spmm_csr_mixed(B=B, prepared=p)
    assert C.dtype == torch.float32
    _colsum_check(C, data, indices, B, 3e-5)
    sd, si, sp = _sub_csr(*h, rows)
    ex, mag = orc.spmm_csr_exact(sd, si, sp, B.cpu())
    assert scaled_error(C.cpu()[rows], ex, mag) <= 3e-5
    lr = torch.isin(rows, long_rows)
    assert int(lr.sum()) > 0
    assert scaled_error(C.cpu()[rows][lr], ex[lr], mag[lr]) <= 2e-7


def test_banded_precision_spmv_full_size(banded):
    """Precision-form SpMV of the same config: float32 result, checksum
    sum(y) = (1^T A) x, sampled and long rows against FP64 (long rows
    compensated: 2e-7)."""
    dt, data, indices, indptr, shape, p, h, rows, long_rows = banded
    x = synthetic.dense_vector(shape[1], seed=3, dtype=dt, device=DEV)
    y = fs.flagsparse_spmv_csr_mixed(x=x, prepared=p)
    assert y.dtype == torch.float32
    _colsum_check(y.unsqueeze(1), data, indices, x.unsqueeze(1), 3e-5)
    sd, si, sp = _sub_csr(*h, rows)
    ex, mag = orc.spmv_csr_exact(sd, si, sp, x.cpu())
    assert scaled_error(y.cpu()[rows], ex, mag) <= 3e-5
    lr = torch.isin(rows, long_rows)
    assert scaled_error(y.cpu()[rows][lr], ex[lr], mag[lr]) <= 2e-7


def test_bsr_tensor_core_full_size():
    data, indices, indptr, shape = synthetic.block_sparse(65536, 4, seed=0, dtype=torch.bfloat16, device=DEV)
    vals, bcol, bptr = bsr.csr_to_bsr16(data, indices, indptr, shape)
    B = synthetic.dense_operand(shape[1], 128, seed=1, dtype=torch.bfloat16, device=DEV)
    C = bsr.flagsparse_spmm_bsr(vals, bcol, bptr, B, shape)
    _colsum_check(C, data, indices, B, 3e-5)
    h = [t.cpu() for t in (data, indices, indptr)]
    rows = _sampled_rows(h[2], step=8192)
    sd, si, sp = _sub_csr(*h, rows)
    ex, mag = orc.spmm_csr_exact(sd, si, sp, B.cpu())
    assert scaled_error(C.cpu()[rows], ex, mag) <= 3e-5


def test_batched_512_full_size():
    """The 512-matrix batch config (rows log-uniform in [1024, 65536], Poisson
    lengths with mean U[2, 64], N = 32): column checksum of the stacked
    product and exact sampled rows of every 16th matrix."""
    import math

    import numpy as np

    from flagsparse_public_b200 import batched

    rng = np.random.default_rng(0)
    mats = []
    for _ in range(512):
        n = int(round(math.exp(rng.uniform(math.log(1024), math.log(65536)))))
        mean = float(rng.uniform(2.0, 64.0))
        mats.append(synthetic.poisson_uniform(n, n, mean=mean, seed=int(rng.integers(1 << 30)), device=DEV))
    prep = batched.prepare_spmm_csr_batch(mats, 32)
    prep.B.copy_(synthetic.dense_operand(prep.n_cols, 32, seed=1, device=DEV))
    prep.run()
    torch.cuda.synchronize()
    _colsum_check(prep.C, prep.data, prep.indices, prep.B, 3e-5)
    for i in range(0, 512, 16):
        d, ix, ip, shape = mats[i]
        h = [t.cpu() for t in (d, ix, ip)]
        rows = _sampled_rows(h[2], step=997, longest=4)
        sd, si, sp = _sub_csr(*h, rows)
        ex, mag = orc.spmm_csr_exact(sd, si, sp, prep.b_views[i].cpu())
        assert scaled_error(prep.c_views[i].cpu()[rows], ex, mag) <= 3e-5, i
