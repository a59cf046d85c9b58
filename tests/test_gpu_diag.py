"""The diagnose-only SpMM forms (fsb_spmm_csr_diag; FlagSparse's stable and
candidate paths, spmm_csr.py:922-1249, :1501-1634, :1998-2086) against the
oracle's restatement of the same arithmetic, bit for bit, and against FP64.

Every element is the sequential recurrence over its row's nonzeros with
explicitly rounded operations, so the CUDA result must equal the oracle's
exactly: float64 accumulation stored in the value type, Kahan in the value
precision and in float64, and the per-row mode switch at short_max.
"""

import pytest
import torch

import flagsparse_public_b200 as fs
import flagsparse_public_b200.sparse_operations.spmm_csr as spmm_mod
from flagsparse_public_b200 import _native as nat
from oracle import oracle as orc
from tests.gpu_cases import EDGE_LENGTHS, csr_from_lengths, dense
from tests.numerics import scaled_error

pytestmark = pytest.mark.gpu
DEV = "cuda"

MODES = [(nat.DIAG_NATIVE, nat.DIAG_NATIVE, -1), (nat.DIAG_WIDE, nat.DIAG_WIDE, -1),
         (nat.DIAG_KAHAN, nat.DIAG_KAHAN, -1), (nat.DIAG_KAHAN_WIDE, nat.DIAG_KAHAN_WIDE, -1),
         (nat.DIAG_KAHAN_WIDE, nat.DIAG_NATIVE, 64), (nat.DIAG_WIDE, nat.DIAG_KAHAN, 100)]


def _diag(d, i, p, shape, B, mode_short, mode_long, short_max):
    C = torch.full((shape[0], B.shape[1]), float("nan"), dtype=d.dtype, device=DEV)
    cm = nat.make_csr(d, i, p, shape[0], shape[1])
    rc = nat.library().fsb_spmm_csr_diag(cm, nat.ptr(B), int(B.stride(0)), int(B.shape[1]), nat.ptr(C),
                                         int(C.stride(0)), mode_short, mode_long, short_max, nat.stream_handle(DEV))
    nat.check(rc, "fsb_spmm_csr_diag")
    return C


@pytest.mark.parametrize("pattern", ["empty_rows", "boundaries", "long_rows", "skewed", "all_empty"])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("index_dtype,ptr_dtype", [(torch.int32, torch.int64), (torch.int64, torch.int32)],
                         ids=["i32p64", "i64p32"])
def test_diag_forms_equal_oracle_bitwise(pattern, dtype, index_dtype, ptr_dtype):
    d, i, p, shape = csr_from_lengths(EDGE_LENGTHS[pattern], 20000, seed=41, dtype=dtype, index_dtype=index_dtype,
                                      ptr_dtype=ptr_dtype)
    for n_dense in (5, 37):
        B = dense((shape[1], n_dense), seed=42, dtype=dtype)
        dd, di, dp, dB = d.to(DEV), i.to(DEV), p.to(DEV), B.to(DEV)
        for ms, ml, smax in MODES:
            got = _diag(dd, di, dp, shape, dB, ms, ml, smax).cpu()
            ref = orc.spmm_diag(d, i, p, B, ms, ml, smax)
            assert torch.equal(got.view(torch.int64 if dtype == torch.float64 else torch.int32),
                               ref.view(torch.int64 if dtype == torch.float64 else torch.int32)), (ms, ml, smax)


def _cancelling_case():
    """Rows whose terms cancel: large +/- pairs around small values, where
    the value-precision sum loses the small terms."""
    g = torch.Generator().manual_seed(7)
    n_rows, n_cols, per_row = 64, 4096, 250  # short rows: the candidate form compensates them
    rows = []
    for _ in range(n_rows):
        cols = torch.sort(torch.randperm(n_cols, generator=g)[:per_row]).values
        big = torch.randn(per_row // 2, generator=g, dtype=torch.float64) * 1e4
        small = torch.rand(per_row - per_row // 2, generator=g, dtype=torch.float64)
        vals = torch.cat([big, -big + torch.rand(per_row // 2, generator=g, dtype=torch.float64) * 1e-3, small])[
            :per_row]
        vals = vals[torch.randperm(per_row, generator=g)]
        rows.append((cols, vals))
    indptr = torch.tensor([0] + [per_row * (r + 1) for r in range(n_rows)], dtype=torch.int64)
    indices = torch.cat([c for c, _ in rows]).to(torch.int32)
    data = torch.cat([v for _, v in rows]).to(torch.float32)
    return data, indices, indptr, (n_rows, n_cols)


def test_diagnose_entry_points_rank_by_accuracy():
    """FlagSparse's diagnose entry points exist with its signatures; on rows
    with cancellation the float64 (stable) and float64-Kahan (candidate)
    forms are within one float32 rounding of the FP64 result, and no worse
    than the opt path."""
    d, i, p, shape = _cancelling_case()
    B = torch.ones((shape[1], 4), dtype=torch.float32)
    ex, mag = orc.spmm_csr_exact(d, i, p, B)
    prep = fs.prepare_spmm_csr_opt(d.to(DEV), i.to(DEV), p.to(DEV), shape)
    dB = B.to(DEV)
    opt = fs.flagsparse_spmm_csr_opt(B=dB, prepared=prep).cpu()
    stable = spmm_mod._flagsparse_spmm_csr_opt_stable_for_diagnose(prep, dB).cpu()
    cand = spmm_mod._flagsparse_spmm_csr_opt_candidate_for_diagnose(prep, dB).cpu()
    kahan = spmm_mod._flagsparse_spmm_csr_opt_kahan_for_diagnose(prep, dB).cpu()
    C2, used = spmm_mod._triton_spmm_csr_impl_opt_prepared_stable(prep, dB)
    assert used is False and torch.equal(C2.cpu(), stable)
    e_opt, e_stable, e_cand, e_kahan = (scaled_error(c, ex, mag) for c in (opt, stable, cand, kahan))
    # one float32 rounding of the FP64 result: |c - ex| <= 2^-24 |ex| <= 2^-24 mag
    assert e_stable <= 2.0 ** -24 * 1.0001
    assert e_cand <= 2.0 ** -24 * 1.0001
    assert e_stable <= e_opt and e_cand <= e_opt
    assert e_kahan <= e_opt * 1.0001 + 1e-12
    # the stable form equals the oracle's float64-accumulate restatement
    assert torch.equal(stable, orc.spmm_diag(d, i, p, B, nat.DIAG_WIDE))


def test_diag_rejects_half_types_and_bad_modes():
    d, i, p, shape = csr_from_lengths([3, 4], 8, seed=1, dtype=torch.float16)
    B = torch.ones((8, 2), dtype=torch.float16, device=DEV)
    cm = nat.make_csr(d.to(DEV), i.to(DEV), p.to(DEV), 2, 8)
    C = torch.empty((2, 2), dtype=torch.float16, device=DEV)
    rc = nat.library().fsb_spmm_csr_diag(cm, nat.ptr(B), 2, 2, nat.ptr(C), 2, 0, 0, -1, nat.stream_handle(DEV))
    assert rc == nat.FSB_ERR_UNSUPPORTED
    d32, B32, C32 = d.float().to(DEV), B.float(), C.float()
    cm = nat.make_csr(d32, i.to(DEV), p.to(DEV), 2, 8)
    rc = nat.library().fsb_spmm_csr_diag(cm, nat.ptr(B32), 2, 2, nat.ptr(C32), 2, 7, 0, -1, nat.stream_handle(DEV))
    assert rc == nat.FSB_ERR_INVALID
    prep = fs.prepare_spmm_csr_opt(d.to(DEV), i.to(DEV), p.to(DEV), (2, 8))
    with pytest.raises(TypeError, match="spmm opt only supports"):
        spmm_mod._flagsparse_spmm_csr_opt_stable_for_diagnose(prep, B)
