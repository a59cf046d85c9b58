"""The drop-in operators on the golden inputs reproduce FlagSparse's outputs.

Structure (transposes, COO orderings, row runs) must be bit-identical; values
must match FlagSparse's within the rounding of the path's compute precision
and sit within the stated bound of the FP64 oracle.
"""

import pytest
import torch

import flagsparse_public_b200 as fs
import flagsparse_public_b200.sparse_operations.spmv_coo as spmv_coo_mod
import flagsparse_public_b200.sparse_operations.spmv_csr as spmv_mod
from oracle import oracle as orc
from tests.conftest import load_golden
from tests.numerics import REL_BOUND, scaled_error, ulp_distance_f32

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _cuda(g, *keys):
    return [g[k].to(DEV) for k in keys]


@pytest.mark.parametrize("name", ["spmv_plain_f32", "spmv_plain_f64", "spmv_plain_f16", "spmv_plain_bf16",
                                  "spmv_plain_c64", "spmv_plain_c128", "spmv_opt_f32", "spmv_opt_f64"])
def test_spmv_golden(name):
    g = load_golden(name)
    data, indices, indptr, x = _cuda(g, "data", "indices", "indptr", "x")
    y = fs.flagsparse_spmv_csr(data, indices, indptr, x, shape=g["shape"], use_opt=g["use_opt"])
    exact, mag = orc.spmv_csr_exact(g["data"], g["indices"], g["indptr"], g["x"])
    bound = REL_BOUND[g["data"].dtype]
    assert scaled_error(y, exact, mag) <= bound
    assert scaled_error(y, g["y"], mag) <= 2 * bound
    if name == "spmv_plain_f32":
        # float64 accumulation rounded once: the reference's result up to one ulp
        assert ulp_distance_f32(y.cpu(), g["y"]) <= 1


def test_spmv_capped_golden():
    g = load_golden("spmv_plain_capped")
    data, indices, indptr, x = _cuda(g, "data", "indices", "indptr", "x")
    y = fs.flagsparse_spmv_csr(data, indices, indptr, x, shape=g["shape"], block_nnz=g["block_nnz"],
                               max_segments=g["max_segments"])
    assert ulp_distance_f32(y.cpu(), g["y"]) <= 1


@pytest.mark.parametrize("op", ["trans", "conj"])
def test_transpose_golden(op):
    g = load_golden("transpose_c64")
    data, indices, indptr = _cuda(g, "data", "indices", "indptr")
    p = fs.prepare_spmv_csr(data, indices, indptr, g["shape"], op=op)
    expect_data = g["t_data"].conj() if op == "conj" else g["t_data"]
    assert torch.equal(p.kernel_indices.cpu(), g["t_indices"])
    assert torch.equal(p.kernel_indptr.cpu(), g["t_indptr"])
    assert torch.equal(p.data.cpu(), expect_data)
    assert p.shape == tuple(g["t_shape"])


def test_coo_to_csr_golden():
    g = load_golden("coo_to_csr")
    d, i, p = spmv_mod.coo_to_csr_for_spmv(*_cuda(g, "data", "row", "col"), g["shape"])
    assert torch.equal(d.cpu(), g["out_data"]) and torch.equal(i.cpu(), g["out_indices"])
    assert torch.equal(p.cpu(), g["out_indptr"])


@pytest.mark.parametrize("name", ["spmv_coo_seg_f32", "spmv_coo_seg_c128", "spmv_coo_atomic_f64"])
def test_spmv_coo_golden(name):
    g = load_golden(name)
    data, row, col, x = _cuda(g, "data", "row", "col", "x")
    p = fs.prepare_spmv_coo(data, row, col, g["shape"], sort_by_row=g["sort_by_row"])
    if g["sort_by_row"]:
        assert torch.equal(p.row.cpu(), g["sorted_row"]) and torch.equal(p.col.cpu(), g["sorted_col"])
        assert torch.equal(p.seg_starts.cpu(), g["seg_starts"])
    y = fs.flagsparse_spmv_coo(x=x, prepared=p)
    perm = orc.coo_lex_order(g["row"], g["col"], g["shape"][1])
    rows, cols, vals = g["row"][perm], g["col"][perm], g["data"][perm]
    indptr = torch.cat([torch.zeros(1, dtype=torch.int64),
                        torch.cumsum(torch.bincount(rows, minlength=g["shape"][0]), 0)])
    exact, mag = orc.spmv_csr_exact(vals, cols, indptr, g["x"])
    bound = REL_BOUND[g["data"].dtype]
    assert scaled_error(y, exact, mag) <= bound
    assert scaled_error(y, g["y"], mag) <= 2 * bound


@pytest.mark.parametrize("name", ["spmm_alg1_f32", "spmm_alg1_f64", "spmm_alg1_f16", "spmm_alg1_c64",
                                  "spmm_long_row_f32"])
def test_spmm_alg1_golden(name):
    g = load_golden(name)
    data, indices, indptr, B = _cuda(g, "data", "indices", "indptr", "B")
    C = fs.flagsparse_spmm_csr(data, indices, indptr, B, g["shape"])
    exact, mag = orc.spmm_csr_exact(g["data"], g["indices"], g["indptr"], g["B"])
    bound = REL_BOUND[g["data"].dtype]
    assert scaled_error(C, exact, mag) <= bound
    assert scaled_error(C, g["C"], mag) <= 2 * bound
    if g["data"].dtype == torch.float32:
        assert ulp_distance_f32(C.cpu(), g["C"]) <= 1


def test_spmm_opt_split_golden():
    g = load_golden("spmm_opt_split_f32")
    data, indices, indptr, B = _cuda(g, "data", "indices", "indptr", "B")
    p = fs.prepare_spmm_csr_opt(data, indices, indptr, g["shape"])
    assert torch.equal(p.long_row_ids.cpu(), g["long_rows"])
    assert torch.equal(p.long_part_starts.cpu(), g["part_starts"])
    assert torch.equal(p.long_part_ends.cpu(), g["part_ends"])
    assert torch.equal(p.long_row_part_ptr.cpu(), g["row_part_ptr"])
    C = fs.flagsparse_spmm_csr_opt(B=B, prepared=p)
    exact, mag = orc.spmm_csr_exact(g["data"], g["indices"], g["indptr"], g["B"])
    assert scaled_error(C, exact, mag) <= 3e-5
    assert scaled_error(C, g["C"], mag) <= 6e-5


def test_spmm_alg2_golden():
    g = load_golden("spmm_alg2_f64")
    data, indices, indptr, B = _cuda(g, "data", "indices", "indptr", "B")
    C, meta = fs.flagsparse_spmm_csr_opt_alg2(data, indices, indptr, B, g["shape"], return_meta=True)
    exact, mag = orc.spmm_csr_exact(g["data"], g["indices"], g["indptr"], g["B"])
    assert scaled_error(C, exact, mag) <= 1e-12
    assert scaled_error(C, g["C"], mag) <= 2e-12
    assert {h["bucket_label"] for h in meta["bucket_hits"]} == {"short_16", "short_64", "row_256", "seg_1024",
                                                                "seg_long"}


def test_spmm_coo_golden():
    g = load_golden("spmm_coo_f32")
    data, row, col, B = _cuda(g, "data", "row", "col", "B")
    C = fs.flagsparse_spmm_coo(data, row, col, B, g["shape"])
    perm = orc.coo_lex_order(g["row"], g["col"], g["shape"][1])
    rows = g["row"][perm]
    indptr = torch.cat([torch.zeros(1, dtype=torch.int64),
                        torch.cumsum(torch.bincount(rows, minlength=g["shape"][0]), 0)])
    exact, mag = orc.spmm_csr_exact(g["data"][perm], g["col"][perm], indptr, g["B"])
    assert scaled_error(C, exact, mag) <= 1e-5
    assert scaled_error(C, g["C"], mag) <= 2e-5
    # structure helpers of the COO module reproduce the reference on the device too
    d, r, c = spmv_coo_mod._sort_coo_lex_inplace(data, row, col, g["shape"][1])
    assert torch.equal(r.cpu(), g["row"][perm]) and torch.equal(c.cpu(), g["col"][perm])
