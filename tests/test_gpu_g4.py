"""The TMA gather4 form of the batched merge-path SpMM (FSB_ALGO_SEQ with
FSB_PLAN_TMA_GATHER) against the FP64 oracle and against the register-staged
form, on skewed matrices whose units span many ring stages.

Bounds (condition-scaled, tests/numerics.py): float32 accumulation 3e-5,
float64 accumulation of float32 values 1e-5, half types one rounding of the
output type.
"""

import pytest
import torch

from flagsparse_public_b200 import _native as nat
from flagsparse_public_b200 import _plan
from oracle import oracle as orc
from tests.gpu_cases import csr_from_lengths, dense
from tests.numerics import REL_BOUND, scaled_error

pytestmark = pytest.mark.gpu
DEV = "cuda"
G4 = nat.PLAN_TMA_GATHER


def _skewed_lengths(n_rows, seed):
    g = torch.Generator().manual_seed(seed)
    lens = torch.poisson(torch.full((n_rows,), 6.0), generator=g).to(torch.int64)
    heavy = torch.randint(0, n_rows, (6,), generator=g)
    lens[heavy] = torch.tensor([3000, 2500, 900, 4100, 1200, 5000])
    lens[::17] = 0
    return lens.tolist()


@pytest.mark.parametrize("dtype,acc,out_dtype,bound", [
    (torch.float32, nat.ACC_NATIVE, torch.float32, 3e-5),
    (torch.float32, nat.ACC_WIDE, torch.float32, REL_BOUND[torch.float32]),
    (torch.bfloat16, nat.ACC_NATIVE, torch.float32, 3e-5),
    (torch.float16, nat.ACC_NATIVE, torch.float16, REL_BOUND[torch.float16]),
])
@pytest.mark.parametrize("n_dense", [16, 64, 128, 200])
def test_g4_matches_oracle_and_seq(dtype, acc, out_dtype, bound, n_dense):
    vw = 16 // torch.empty((), dtype=dtype).element_size()
    if n_dense % vw:
        pytest.skip("n_dense must be a multiple of the 16-byte lane vector")
    lengths = _skewed_lengths(3000, 41)
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths(lengths, 40000, seed=42, dtype=dtype)
    B = dense((n_cols, n_dense), 43, dtype)
    exact, mag = orc.spmm_csr_exact(data, indices, indptr, B)
    d = (data.to(DEV), indices.to(DEV), indptr.to(DEV))
    Bd = B.to(DEV)
    stats = _plan.matrix_stats(d[2], n_rows, n_cols)
    for plan in (_plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=_plan.g4_items_per_unit(stats), flags=G4),
                 _plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=333, flags=G4),
                 _plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=64, flags=G4, grid_blocks=2)):
        C = torch.full((n_rows, n_dense), float("nan"), dtype=out_dtype, device=DEV)
        _plan.run_spmm(*d, n_rows, n_cols, Bd, C, acc, plan)
        assert scaled_error(C, exact, mag) <= bound, plan.describe()
    assert nat.device_error(reset=False) == 0


def test_g4_int64_indices_and_row_map():
    """64-bit column indices and pointers; COO row runs through row_map."""
    lengths = _skewed_lengths(1500, 44)
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths(lengths, 9000, seed=45, index_dtype=torch.int64)
    B = dense((n_cols, 32), 46, torch.float32)
    exact, mag = orc.spmm_csr_exact(data, indices, indptr, B)
    plan = _plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=200, flags=G4)
    C = torch.full((n_rows, 32), float("nan"), device=DEV)
    _plan.run_spmm(data.to(DEV), indices.to(DEV), indptr.to(DEV), n_rows, n_cols, B.to(DEV), C, nat.ACC_WIDE, plan)
    assert scaled_error(C, exact, mag) <= REL_BOUND[torch.float32]
    # the same rows as runs of a row-sorted COO: output row = row_map[run start]
    lens = indptr[1:] - indptr[:-1]
    rows = torch.repeat_interleave(torch.arange(n_rows, dtype=torch.int64), lens)
    runs = torch.nonzero(lens > 0).flatten()
    seg = torch.zeros(runs.numel() + 1, dtype=torch.int64)
    seg[1:] = torch.cumsum(lens[runs], 0)
    C2 = torch.zeros((n_rows, 32), device=DEV)
    _plan.run_spmm(data.to(DEV), indices.to(DEV), seg.to(DEV), runs.numel(), n_cols, B.to(DEV), C2, nat.ACC_WIDE,
                   _plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=200, flags=G4), row_map=rows.to(DEV))
    assert scaled_error(C2, exact, mag) <= REL_BOUND[torch.float32]


def test_g4_agrees_with_register_form_on_power_law():
    from flagsparse_public_b200 import synthetic

    data, indices, indptr, shape = synthetic.zipf_powerlaw(32768, 32768, alpha=1.8, mean=12.0, cap=4000, seed=3,
                                                           device=DEV)
    B = synthetic.dense_operand(shape[1], 64, seed=4, device=DEV)
    stats = _plan.matrix_stats(indptr, shape[0], shape[1])
    c_seq = torch.empty((shape[0], 64), device=DEV)
    c_g4 = torch.empty((shape[0], 64), device=DEV)
    ipu = _plan.seq_items_per_unit(stats)
    _plan.run_spmm(data, indices, indptr, shape[0], shape[1], B, c_seq, nat.ACC_NATIVE,
                   _plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=ipu))
    _plan.run_spmm(data, indices, indptr, shape[0], shape[1], B, c_g4, nat.ACC_NATIVE,
                   _plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=ipu, flags=G4))
    # same units and the same per-lane summation order: identical results
    assert torch.equal(c_seq, c_g4)


def test_g4_rejects_what_it_cannot_stage():
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths([5, 7, 0, 3], 50, seed=47, dtype=torch.float64)
    B = dense((n_cols, 8), 48, torch.float64).to(DEV)
    C = torch.empty((n_rows, 8), dtype=torch.float64, device=DEV)
    plan = _plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=16, flags=G4)
    d = (data.to(DEV), indices.to(DEV), indptr.to(DEV))
    with pytest.raises(ValueError, match="gather4 plan"):
        _plan.run_spmm(*d, n_rows, n_cols, B, C, nat.ACC_NATIVE, plan)
    # the C entry point itself is strict
    plan.ensure_coords(d[2], n_rows, data.numel())
    cm = nat.make_csr(*d, n_rows, n_cols)
    lib = nat.library()
    ws = torch.empty(1 << 16, dtype=torch.uint8, device=DEV)
    rc = lib.fsb_spmm_csr(cm, nat.ptr(B), 8, 8, nat.ptr(C), 8, nat.FSB_F64, nat.ACC_NATIVE, plan.c_plan(),
                          nat.ptr(ws), ws.numel(), nat.stream_handle(torch.device(DEV)))
    assert rc == nat.FSB_ERR_UNSUPPORTED
    # float32 with a fallback-enabled plan runs the register form instead
    data32 = d[0].float()
    B32 = torch.ones((n_cols, 6), device=DEV)  # 6 columns: not a whole number of lane vectors
    C32 = torch.empty((n_rows, 6), device=DEV)
    fb = _plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=16, flags=G4, fallback_ok=True)
    _plan.run_spmm(data32, d[1], d[2], n_rows, n_cols, B32, C32, nat.ACC_NATIVE, fb)
    exact, mag = orc.spmm_csr_exact(data.float(), indices, indptr, B32.cpu())
    assert scaled_error(C32, exact, mag) <= 3e-5
