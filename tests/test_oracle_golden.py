"""Pin the CPU oracle to FlagSparse's own outputs (golden vectors).

The fixtures in tests/golden were produced by FlagSparse's Triton kernels and
integer helpers (tests/golden/make_golden.py).  Integer structure must match
bit for bit; floating-point results must agree with the reference within the
rounding of the path's compute precision, and both must sit within the stated
bound of the FP64 oracle.
"""

import pytest
import torch

from oracle import oracle as orc
from tests.conftest import load_golden
from tests.numerics import REL_BOUND, scaled_error

ACC_WIDE, ACC_NATIVE = orc.ACC_WIDE, orc.ACC_NATIVE


def _plain_acc(dtype):
    return ACC_WIDE if dtype == torch.float32 else ACC_NATIVE


@pytest.mark.parametrize("name", ["spmv_plain_f32", "spmv_plain_f64", "spmv_plain_f16", "spmv_plain_bf16",
                                  "spmv_plain_c64", "spmv_plain_c128", "spmv_opt_f32", "spmv_opt_f64"])
def test_oracle_spmv_matches_reference(name):
    g = load_golden(name)
    dtype = g["data"].dtype
    acc = ACC_NATIVE if g["use_opt"] else _plain_acc(dtype)
    y = orc.spmv_csr(g["data"], g["indices"], g["indptr"], g["x"], acc_mode=acc)
    exact, mag = orc.spmv_csr_exact(g["data"], g["indices"], g["indptr"], g["x"])
    bound = REL_BOUND[dtype]
    assert scaled_error(g["y"], exact, mag) <= bound, "reference itself outside the FP64 bound"
    assert scaled_error(y, exact, mag) <= bound
    # oracle vs reference: same compute precision, different summation order
    assert scaled_error(y, g["y"], mag) <= 2 * bound


def test_oracle_spmv_plain_f32_is_rounded_fp64():
    """Plain float32 computes in float64 and rounds once (spmv_csr.py:116-121)."""
    g = load_golden("spmv_plain_f32")
    y = orc.spmv_csr(g["data"], g["indices"], g["indptr"], g["x"], acc_mode=ACC_WIDE)
    exact, _ = orc.spmv_csr_exact(g["data"], g["indices"], g["indptr"], g["x"])
    assert torch.equal(y, exact.to(torch.float32))
    assert torch.equal(g["y"], exact.to(torch.float32))


def test_oracle_spmv_capped_window_matches_reference():
    g = load_golden("spmv_plain_capped")
    cap = g["block_nnz"] * g["max_segments"]
    y = orc.spmv_csr(g["data"], g["indices"], g["indptr"], g["x"], acc_mode=ACC_WIDE, row_cap=cap)
    assert torch.equal(y, g["y"])
    full = orc.spmv_csr(g["data"], g["indices"], g["indptr"], g["x"], acc_mode=ACC_WIDE)
    assert not torch.equal(full, g["y"]), "fixture must contain truncated rows"


def test_oracle_transpose_bit_exact():
    g = load_golden("transpose_c64")
    n_rows, n_cols = g["shape"]
    t_ptr, t_rows, perm = orc.csr_transpose(g["indptr"], g["indices"], n_rows, n_cols)
    assert torch.equal(t_ptr, g["t_indptr"].to(torch.int64))
    assert torch.equal(t_rows, g["t_indices"].to(torch.int64))
    assert torch.equal(g["data"][perm], g["t_data"])


def test_oracle_coo_to_csr_bit_exact():
    g = load_golden("coo_to_csr")
    perm = orc.coo_lex_order(g["row"], g["col"], g["shape"][1])
    assert torch.equal(g["col"][perm].to(torch.int32), g["out_indices"])
    assert torch.equal(g["data"][perm], g["out_data"])
    counts = torch.bincount(g["row"], minlength=g["shape"][0])
    indptr = torch.cat([torch.zeros(1, dtype=torch.int64), torch.cumsum(counts, 0)])
    assert torch.equal(indptr, g["out_indptr"])


@pytest.mark.parametrize("name", ["spmv_coo_seg_f32", "spmv_coo_seg_c128", "spmv_coo_atomic_f64"])
def test_oracle_spmv_coo_matches_reference(name):
    g = load_golden(name)
    n_rows, n_cols = g["shape"]
    if g["sort_by_row"]:
        perm = orc.coo_lex_order(g["row"], g["col"], n_cols)
        assert torch.equal(g["row"][perm], g["sorted_row"])
        assert torch.equal(g["col"][perm], g["sorted_col"])
        assert torch.equal(g["data"][perm], g["sorted_data"])
        assert torch.equal(orc.seg_starts(g["sorted_row"]), g["seg_starts"].to(torch.int64))
    perm = orc.coo_lex_order(g["row"], g["col"], n_cols)
    rows, cols, data = g["row"][perm], g["col"][perm], g["data"][perm]
    indptr = torch.cat([torch.zeros(1, dtype=torch.int64), torch.cumsum(torch.bincount(rows, minlength=n_rows), 0)])
    y = orc.spmv_csr(data, cols, indptr, g["x"], acc_mode=ACC_NATIVE)
    exact, mag = orc.spmv_csr_exact(data, cols, indptr, g["x"])
    bound = REL_BOUND[data.dtype]
    assert scaled_error(g["y"], exact, mag) <= bound
    assert scaled_error(y, g["y"], mag) <= 2 * bound


@pytest.mark.parametrize("name,acc", [("spmm_alg1_f32", ACC_WIDE), ("spmm_alg1_f64", ACC_NATIVE),
                                      ("spmm_alg1_f16", ACC_NATIVE), ("spmm_alg1_c64", ACC_NATIVE),
                                      ("spmm_opt_split_f32", ACC_NATIVE), ("spmm_alg2_f64", ACC_NATIVE),
                                      ("spmm_long_row_f32", ACC_WIDE)])
def test_oracle_spmm_matches_reference(name, acc):
    g = load_golden(name)
    C = orc.spmm_csr(g["data"], g["indices"], g["indptr"], g["B"], acc_mode=acc)
    exact, mag = orc.spmm_csr_exact(g["data"], g["indices"], g["indptr"], g["B"])
    bound = REL_BOUND[g["data"].dtype]
    assert scaled_error(g["C"], exact, mag) <= bound
    assert scaled_error(C, exact, mag) <= bound
    assert scaled_error(C, g["C"], mag) <= 2 * bound
    if acc == ACC_WIDE:
        assert torch.equal(C, exact.to(C.dtype)) or scaled_error(C, g["C"], mag) <= 1e-7


def test_oracle_split_metadata_bit_exact():
    g = load_golden("spmm_opt_split_f32")
    rows, starts, ends, rpp = orc.split_metadata(g["indptr"], g["long_rows"], 256)
    assert torch.equal(rows, g["part_rows"].to(torch.int64))
    assert torch.equal(starts, g["part_starts"])
    assert torch.equal(ends, g["part_ends"])
    assert torch.equal(rpp, g["row_part_ptr"])


def test_oracle_spmm_coo_coalesce_and_product():
    g = load_golden("spmm_coo_f32")
    n_rows, n_cols = g["shape"]
    perm = orc.coo_lex_order(g["row"], g["col"], n_cols)
    rows, cols, data = g["row"][perm], g["col"][perm], g["data"][perm].to(torch.float64)
    key = rows * n_cols + cols
    first = torch.ones_like(key, dtype=torch.bool)
    first[1:] = key[1:] != key[:-1]
    assert torch.equal(rows[first], g["coalesced_row"])
    assert torch.equal(cols[first], g["coalesced_col"])
    group = torch.cumsum(first.to(torch.int64), 0) - 1
    summed = torch.zeros(int(first.sum()), dtype=torch.float64).index_add_(0, group, data)
    assert torch.allclose(summed, g["coalesced_data"].to(torch.float64), rtol=1e-6, atol=1e-7)
    indptr = torch.cat([torch.zeros(1, dtype=torch.int64), torch.cumsum(torch.bincount(rows, minlength=n_rows), 0)])
    C = orc.spmm_csr(g["data"][perm], cols, indptr, g["B"], acc_mode=ACC_WIDE)
    exact, mag = orc.spmm_csr_exact(g["data"][perm], cols, indptr, g["B"])
    assert scaled_error(g["C"], exact, mag) <= 1e-5
    assert scaled_error(C, g["C"], mag) <= 2e-5


def test_oracle_merge_partition_properties():
    g = load_golden("spmv_plain_f32")
    indptr = g["indptr"]
    n_rows = indptr.numel() - 1
    nnz = int(indptr[-1])
    for items, snap in ((64, 0), (100, 0), (128, 16), (1000, 40)):
        c = orc.merge_partition(indptr, n_rows, nnz, items, snap).view(-1, 2)
        assert int(c[0, 0]) == 0 and int(c[0, 1]) == 0
        assert int(c[-1, 0]) == n_rows and int(c[-1, 1]) == nnz
        assert bool((c[1:, 0] >= c[:-1, 0]).all()) and bool((c[1:, 1] >= c[:-1, 1]).all())
        d = c.sum(1)
        # snapping moves a boundary back by less than one short row
        assert bool(((d[1:] - d[:-1]) <= items + snap).all())
        # consumed row ends never run ahead of the nonzeros they close
        i, j = c[:, 0], c[:, 1]
        closed = indptr[i.clamp(max=n_rows)]
        assert bool((closed <= j).all())
        if snap == 0:
            assert bool((d[:-1] == torch.arange(d.numel() - 1) * items).all())
