"""Precision form: bfloat16 / float16 storage, float32 accumulation and output,
compensated accumulation on rows longer than 4096 nonzeros.

Bounds: against FP64 of the same half-precision inputs the condition-scaled
error stays within float32 accumulation (3e-5; compensated long rows 2e-7);
against FP64 of the float32 data it includes the storage rounding of values
and operands and must stay within 1e-2.
"""

import pytest
import torch

import flagsparse_public_b200 as fs
from flagsparse_public_b200 import synthetic
from oracle import oracle as orc
from tests.numerics import scaled_error

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")


@pytest.fixture(scope="module")
def banded():
    data, indices, indptr, shape = synthetic.banded_plus_random(n_rows=12000, long_rate=0.01, long_len=8192, seed=3,
                                                               dtype=torch.float32, device=DEV)
    x = synthetic.dense_vector(shape[1], seed=4, device=DEV)
    B = synthetic.dense_operand(shape[1], 32, seed=5, device=DEV)
    host = tuple(t.cpu() for t in (data, indices, indptr))
    return data, indices, indptr, shape, x, B, host


@pytest.mark.parametrize("dt", [torch.bfloat16, torch.float16], ids=["bf16", "f16"])
def test_precision_spmv(banded, dt):
    data, indices, indptr, shape, x, _B, host = banded
    y, err = fs.flagsparse_spmv_csr_mixed(data.to(dt), indices, indptr, x.to(dt), shape, return_error=True)
    assert y.dtype == torch.float32
    ex_same, mag_same = orc.spmv_csr_exact(host[0].to(dt), host[1], host[2], x.cpu().to(dt))
    ex_f32, mag_f32 = orc.spmv_csr_exact(*host, x.cpu())
    assert scaled_error(y, ex_same, mag_same) <= 3e-5
    assert abs(err - scaled_error(y, ex_same, mag_same)) <= 1e-7
    lens = host[2][1:] - host[2][:-1]
    long_rows = lens > 4096
    assert int(long_rows.sum()) > 0
    assert scaled_error(y.cpu()[long_rows], ex_same[long_rows], mag_same[long_rows]) <= 2e-7
    assert scaled_error(y, ex_f32, mag_f32) <= 1e-2


@pytest.mark.parametrize("dt", [torch.bfloat16, torch.float16], ids=["bf16", "f16"])
def test_precision_spmm(banded, dt):
    data, indices, indptr, shape, _x, B, host = banded
    prepared = fs.prepare_csr_mixed(data.to(dt), indices, indptr, shape)
    C = fs.flagsparse_spmm_csr_mixed(B=B.to(dt), prepared=prepared)
    assert C.dtype == torch.float32 and C.shape == (shape[0], 32)
    ex_same, mag_same = orc.spmm_csr_exact(host[0].to(dt), host[1], host[2], B.cpu().to(dt))
    ex_f32, mag_f32 = orc.spmm_csr_exact(*host, B.cpu())
    assert scaled_error(C, ex_same, mag_same) <= 3e-5
    lens = host[2][1:] - host[2][:-1]
    long_rows = lens > 4096
    assert scaled_error(C.cpu()[long_rows], ex_same[long_rows], mag_same[long_rows]) <= 2e-7
    assert scaled_error(C, ex_f32, mag_f32) <= 1e-2
    # without compensation the long rows are only float32-accumulated
    plain = fs.prepare_csr_mixed(data.to(dt), indices, indptr, shape, compensate_above=10 ** 9)
    C2 = fs.flagsparse_spmm_csr_mixed(B=B.to(dt), prepared=plain)
    assert scaled_error(C2, ex_same, mag_same) <= 3e-5


def test_precision_api_validation(banded):
    data, indices, indptr, shape, x, B, _ = banded
    with pytest.raises(TypeError, match="bfloat16 or float16"):
        fs.prepare_csr_mixed(data, indices, indptr, shape)
    p = fs.prepare_csr_mixed(data.bfloat16(), indices, indptr, shape)
    with pytest.raises(TypeError, match="dtype must match"):
        fs.flagsparse_spmv_csr_mixed(x=x, prepared=p)
    with pytest.raises(ValueError, match="n_cols"):
        fs.flagsparse_spmm_csr_mixed(B=B[:-1].bfloat16(), prepared=p)
    out = torch.empty(shape[0], device=DEV)
    y, ms = fs.flagsparse_spmv_csr_mixed(x=x.bfloat16(), prepared=p, out=out, return_time=True)
    assert y is out and isinstance(ms, float)


def test_precision_spmm_of_a_block_matrix_runs_on_the_tensor_core_bsr_plan():
    """A bfloat16 matrix of dense 16 x 16 blocks through the public precision
    API: the learned selector picks the tensor-core BSR candidate, and the
    result is within float32 accumulation of FP64 of the same inputs."""
    from flagsparse_public_b200 import _plan, synthetic, tuning

    if _plan.learned_selector(torch.device(DEV)) is None:
        pytest.skip("no selector weights installed")
    data, indices, indptr, shape = synthetic.block_sparse(8192, 6, seed=11, dtype=torch.bfloat16, device=DEV)
    B = synthetic.dense_operand(shape[1], 128, seed=12, dtype=torch.bfloat16, device=DEV)
    prepared = fs.prepare_csr_mixed(data, indices, indptr, shape, layout="csr")
    C, err = fs.flagsparse_spmm_csr_mixed(B=B, prepared=prepared, return_error=True)
    plan = prepared._plans[("spmm", 128)]
    assert isinstance(plan, _plan.BsrPlan), plan.describe()
    assert err <= 1e-5
    f = tuning.raw_features(indices, indptr, shape[0], shape[1], 128, 2)
    assert f[11] == 1.0
