"""SDDMM on sm_100a against FlagSparse's own outputs (golden fixtures) and
FP64: condition-scaled error <= 3e-5 for float32 (float32 accumulation),
1e-12 for float64."""

import os

import pytest
import torch

from flagsparse_public_b200 import flagsparse_sddmm_csr, prepare_sddmm_csr, synthetic
from tests.conftest import GOLDEN_DIR
from tests.test_sddmm_cpu import GOLDEN, exact_sddmm

DEV = "cuda"
pytestmark = pytest.mark.gpu


def _err(out, exact, mag):
    return ((out.double().cpu() - exact).abs() / mag.clamp_min(1e-300)).max().item() if out.numel() else 0.0


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_matches_flagsparse_golden(name):
    c = GOLDEN[name]
    shape = tuple(int(v) for v in c["shape"])
    data = c["data"].to(DEV) if c["has_data"] else None
    out = flagsparse_sddmm_csr(data, c["indices"].to(DEV), c["indptr"].to(DEV), c["x"].to(DEV), c["y"].to(DEV), shape,
                               alpha=c["alpha"], beta=c["beta"] if c["has_data"] else 0.0)
    torch.cuda.synchronize()
    exact, mag = exact_sddmm(c)
    bound = 3e-5 if out.dtype == torch.float32 else 1e-12
    assert _err(out, exact, mag) <= bound
    # and close to FlagSparse's own float32 / float64 result
    ref = c["out"].double()
    assert ((out.double().cpu() - ref).abs() / mag.clamp_min(1e-300)).max().item() <= 2 * bound


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("k", [1, 13, 32, 64, 128, 256, 300])
@pytest.mark.parametrize("ptr_dtype", [torch.int64, torch.int32])
def test_random_patterns_against_fp64(dtype, k, ptr_dtype):
    data, indices, indptr, shape = synthetic.zipf_powerlaw(3000, 2500, mean=6.0, cap=500, seed=k, dtype=dtype,
                                                           device=DEV)
    g = torch.Generator(device=DEV).manual_seed(k)
    x = torch.randn((shape[0], k), generator=g, device=DEV, dtype=torch.float64).to(dtype)
    y = torch.randn((shape[1], k), generator=g, device=DEV, dtype=torch.float64).to(dtype)
    prep = prepare_sddmm_csr(indices, indptr.to(ptr_dtype), shape, k_hint=k)
    out, ms, meta = flagsparse_sddmm_csr(data, x=x, y=y, prepared=prep, alpha=1.5, beta=-0.25, return_time=True,
                                         return_meta=True)
    torch.cuda.synchronize()
    case = {"indptr": indptr.cpu(), "indices": indices.cpu(), "x": x.cpu(), "y": y.cpu(), "alpha": 1.5, "beta": -0.25,
            "has_data": True, "data": data.cpu()}
    exact, mag = exact_sddmm(case)
    assert _err(out, exact, mag) <= (3e-5 if dtype == torch.float32 else 1e-12)
    assert meta["fallback_used"] is False and ms >= 0.0


def test_validation_messages_match_flagsparse():
    ind = torch.tensor([0, 2, 1], dtype=torch.int32, device=DEV)
    ptr = torch.tensor([0, 2, 3], dtype=torch.int64, device=DEV)
    x = torch.randn(2, 4, device=DEV)
    y = torch.randn(3, 4, device=DEV)
    with pytest.raises(TypeError, match="indices dtype must be torch.int32"):
        prepare_sddmm_csr(ind.long(), ptr, (2, 3))
    with pytest.raises(IndexError, match="indices out of range"):
        prepare_sddmm_csr(ind, ptr, (2, 2))
    with pytest.raises(ValueError, match="data is required when beta is non-zero"):
        flagsparse_sddmm_csr(None, ind, ptr, x, y, (2, 3), beta=1.0)
    with pytest.raises(TypeError, match="y dtype must match x dtype"):
        flagsparse_sddmm_csr(None, ind, ptr, x, y.double(), (2, 3))
    with pytest.raises(ValueError, match="x and y must have the same K dimension"):
        flagsparse_sddmm_csr(None, ind, ptr, x, y[:, :3], (2, 3))
    out = flagsparse_sddmm_csr(None, ind, ptr, x[:, :0], y[:, :0], (2, 3))
    assert torch.all(out == 0)
