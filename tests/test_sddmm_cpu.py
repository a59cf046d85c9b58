"""SDDMM golden fixtures (FlagSparse's own kernel) against FP64, and the
host-side validation that runs before any launch."""

import os

import pytest
import torch

from tests.conftest import GOLDEN_DIR

GOLDEN = torch.load(os.path.join(GOLDEN_DIR, "sddmm_golden.pt"), weights_only=True)


def exact_sddmm(case):
    ptr = case["indptr"].long()
    rows = torch.repeat_interleave(torch.arange(ptr.numel() - 1), ptr[1:] - ptr[:-1])
    cols = case["indices"].long()
    prod = case["x"].double()[rows] * case["y"].double()[cols]
    exact = case["alpha"] * prod.sum(1)
    mag = abs(case["alpha"]) * prod.abs().sum(1)
    if case["has_data"]:
        exact = exact + case["beta"] * case["data"].double()
        mag = mag + abs(case["beta"]) * case["data"].double().abs()
    return exact, mag


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_oracle_port_matches_the_golden_outputs(name):
    """The CPU restatement (oracle.sddmm_csr, the bench's CPU baseline) on
    FlagSparse's own fixtures: within one value-precision rounding of the
    reference kernel's output, condition-scaled."""
    from oracle import oracle as orc

    case = GOLDEN[name]
    got = orc.sddmm_csr(case["indices"], case["indptr"], case["x"], case["y"],
                        case["data"] if case["has_data"] else None, case["alpha"], case["beta"], threads=2)
    exact, mag = exact_sddmm(case)
    bound = 3e-5 if case["out"].dtype == torch.float32 else 1e-12
    if got.numel():
        err_ref = ((got.double() - case["out"].double()).abs() / mag.clamp_min(1e-300)).max().item()
        err_exact = ((got.double() - exact).abs() / mag.clamp_min(1e-300)).max().item()
        assert err_ref <= 2 * bound and err_exact <= bound


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_golden_outputs_are_within_fp64_bounds(name):
    case = GOLDEN[name]
    exact, mag = exact_sddmm(case)
    bound = 3e-5 if case["out"].dtype == torch.float32 else 1e-12
    err = ((case["out"].double() - exact).abs() / mag.clamp_min(1e-300)).max().item()
    assert err <= bound


def test_pattern_validation_messages():
    from flagsparse_public_b200 import prepare_sddmm_csr
    ind = torch.tensor([0, 1], dtype=torch.int32)
    ptr = torch.tensor([0, 1, 2], dtype=torch.int64)
    with pytest.raises(ValueError, match="shape must be a 2-tuple"):
        prepare_sddmm_csr(ind, ptr, (2, 2, 2))
    with pytest.raises(ValueError, match=r"indptr length must be n_rows\+1=4"):
        prepare_sddmm_csr(ind, ptr, (3, 2))
    with pytest.raises(ValueError, match="must be CUDA tensors"):
        prepare_sddmm_csr(ind, ptr, (2, 2))
