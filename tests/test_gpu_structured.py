"""The structured form of the precision SpMV / SpMM (csrc/fsb_struct.cu,
flagsparse_public_b200/_structured.py) against the oracle.

* Integer structure, bit for bit: the per-row run descriptors and per-tile
  spans equal the oracle's restatement (oracle.struct_rows / struct_tiles);
  the long rows' regrouping by x block reproduces every long row's columns
  and values in order.
* Products against FP64 of the same half-precision inputs, condition-scaled:
  rows up to the long-row threshold within 3e-5 (float32 accumulation),
  long rows within 2e-7 (compensated).
Cases: banded-plus-random matrices with long rows (bf16 and fp16), runs too
wide for a tile's span (rows fall back to scattered), a matrix without runs
forced onto the structured form, empty rows and a ragged last tile, a column
count that is not a multiple of 8, int32 row offsets; SpMM widths 16, 32, 64.
"""

import pytest
import torch

import flagsparse_public_b200 as fs
from flagsparse_public_b200 import _structured, synthetic
from oracle import oracle as orc
from tests.gpu_cases import csr_from_lengths
from tests.numerics import scaled_error

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")
SHORT_BOUND = 3e-5
LONG_BOUND = 2e-7


def _case(name, dtype):
    if name == "banded_long":
        d, i, p, shape = synthetic.banded_plus_random(5000, band=64, off_band=4, long_rate=0.02, long_len=3000,
                                                      seed=1, dtype=dtype, device=DEV)
    elif name == "wide_runs":
        d, i, p, shape = synthetic.banded_plus_random(4000, band=200, off_band=3, long_rate=0.01, long_len=1500,
                                                      seed=2, dtype=dtype, device=DEV)
    elif name == "no_runs":
        d, i, p, shape = synthetic.poisson_uniform(3000, 3000, mean=12.0, seed=3, dtype=dtype, device=DEV)
    elif name == "ragged":
        lengths = [0, 70, 0, 0, 5, 1200, 64, 0] * 16 + [17, 0]  # 130 rows: two tiles, the last of 2 rows
        d, i, p, shape = csr_from_lengths(lengths, 4099, seed=4, dtype=dtype)
        d, i, p = d.to(DEV), i.to(DEV), p.to(DEV)
    elif name == "tiled_long":  # long rows sparse over many columns: the SpMM tiles them
        d, i, p, shape = synthetic.banded_plus_random(131072, band=64, off_band=4, long_rate=0.005, long_len=1600,
                                                      seed=6, dtype=dtype, device=DEV)
    elif name == "banded_i32ptr":
        d, i, p, shape = synthetic.banded_plus_random(3000, band=32, off_band=2, long_rate=0.01, long_len=2000,
                                                      seed=5, dtype=dtype, device=DEV)
        p = p.to(torch.int32)
    else:
        raise KeyError(name)
    return d, i, p, shape


CASES = ["banded_long", "wide_runs", "no_runs", "ragged", "banded_i32ptr", "tiled_long"]
DTYPES = [torch.bfloat16, torch.float16]


def _long_mask(p, shape):
    lens = (p[1:] - p[:-1]).cpu()
    return lens > _structured.LONG_MIN


@pytest.mark.parametrize("name", CASES)
def test_struct_descriptors_match_oracle(name):
    d, i, p, shape = _case(name, torch.bfloat16)
    form = _structured.build(d, i, p, shape[0], shape[1])
    rc, ro, rl = orc.struct_rows(i, p, _structured.LONG_MIN, _structured.MIN_RUN)
    base, span, ro2, rl2 = orc.struct_tiles(rc, ro, rl)
    n = shape[0]
    assert torch.equal(form.run_len[:n].cpu(), rl2)
    assert torch.equal(form.run_off[:n].cpu(), ro2)
    keep = rl > 0  # run columns are defined where the row had a run
    assert torch.equal(form.run_col[:n].cpu()[keep], rc[keep])
    assert torch.equal(form.tile_base.cpu(), base)
    assert torch.equal(form.tile_span.cpu(), span)
    assert form.max_span == int(span.max())


@pytest.mark.parametrize("name", ["banded_long", "wide_runs", "ragged"])
def test_struct_long_rows_regrouped_by_x_block(name):
    d, i, p, shape = _case(name, torch.float16)
    form = _structured.build(d, i, p, shape[0], shape[1])
    hp, hi, hd = p.cpu().long(), i.cpu().long(), d.cpu()
    long_rows = torch.nonzero(_long_mask(p, shape)).flatten()
    assert torch.equal(form.long_rows.cpu().long(), long_rows)
    seg_ptr = form.seg_ptr.cpu()
    off = form.seg_off.cpu().to(torch.int32) & 0xFFFF
    vals = form.seg_val.cpu()
    nl = form.n_long
    for l, r in enumerate(long_rows.tolist()):
        cols, vs = [], []
        for b in range(form.n_xblocks):
            s, e = int(seg_ptr[b * nl + l]), int(seg_ptr[b * nl + l + 1])
            cols.append(off[s:e].long() + b * form.xblock)
            vs.append(vals[s:e])
        assert torch.equal(torch.cat(cols), hi[hp[r]:hp[r + 1]])
        assert torch.equal(torch.cat(vs), hd[hp[r]:hp[r + 1]])
    # chunks of the long rows for the SpMM
    lens = (hp[1:] - hp[:-1])[long_rows]
    nch = (lens + _structured.CHUNK_NNZ - 1) // _structured.CHUNK_NNZ
    assert torch.equal(form.chunk_ptr.cpu()[1:], torch.cumsum(nch, 0))


def _check(got, d, i, p, dense, long_mask):
    h = (d.cpu(), i.cpu(), p.cpu())
    if dense.ndim == 1:
        ex, mag = orc.spmv_csr_exact(*h, dense.cpu())
    else:
        ex, mag = orc.spmm_csr_exact(*h, dense.cpu())
    got = got.cpu()
    short = ~long_mask
    assert scaled_error(got[short], ex[short], mag[short]) <= SHORT_BOUND
    if bool(long_mask.any()):
        assert scaled_error(got[long_mask], ex[long_mask], mag[long_mask]) <= LONG_BOUND


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("dtype", DTYPES, ids=["bf16", "f16"])
def test_struct_spmv_matches_fp64(name, dtype):
    d, i, p, shape = _case(name, dtype)
    x = synthetic.dense_vector(shape[1], seed=7, dtype=dtype, device=DEV)
    prep = fs.prepare_csr_mixed(d, i, p, shape, layout="structured")
    y1 = fs.flagsparse_spmv_csr_mixed(x=x, prepared=prep)
    y2 = fs.flagsparse_spmv_csr_mixed(x=x, prepared=prep)
    assert y1.dtype == torch.float32
    assert torch.equal(y1, y2)  # deterministic: fixed summation order
    _check(y1, d, i, p, x, _long_mask(p, shape))


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("dtype", DTYPES, ids=["bf16", "f16"])
@pytest.mark.parametrize("n_dense", [16, 32, 64])
def test_struct_spmm_matches_fp64(name, dtype, n_dense):
    d, i, p, shape = _case(name, dtype)
    B = synthetic.dense_operand(shape[1], n_dense, seed=8, dtype=dtype, device=DEV)
    prep = fs.prepare_csr_mixed(d, i, p, shape, layout="structured")
    C1 = fs.flagsparse_spmm_csr_mixed(B=B, prepared=prep)
    C2 = torch.full_like(C1, float("nan"))
    fs.flagsparse_spmm_csr_mixed(B=B, prepared=prep, out=C2)
    assert torch.equal(C1, C2)
    _check(C1, d, i, p, B, _long_mask(p, shape))


def test_struct_auto_layout_picks_structure_only_where_it_pays():
    d, i, p, shape = _case("banded_long", torch.bfloat16)
    assert fs.prepare_csr_mixed(d, i, p, shape)._struct  # runs + long rows hold the nonzeros
    d, i, p, shape = _case("no_runs", torch.bfloat16)
    assert fs.prepare_csr_mixed(d, i, p, shape)._struct is False
    # a compensation threshold below the long-row threshold keeps the CSR kernels
    d, i, p, shape = _case("banded_long", torch.bfloat16)
    assert fs.prepare_csr_mixed(d, i, p, shape, compensate_above=100)._struct is False


def test_struct_spmm_unsupported_width_falls_back_to_csr():
    d, i, p, shape = _case("banded_long", torch.bfloat16)
    B = synthetic.dense_operand(shape[1], 24, seed=9, dtype=torch.bfloat16, device=DEV)
    prep = fs.prepare_csr_mixed(d, i, p, shape, layout="structured")
    C = fs.flagsparse_spmm_csr_mixed(B=B, prepared=prep)
    # CSR kernels: rows up to compensate_above (4096) accumulate plainly
    _check(C, d, i, p, B, torch.zeros(shape[0], dtype=torch.bool))


@pytest.mark.parametrize("name", ["tiled_long", "ragged"])
def test_struct_long_row_tiles_decode_to_the_long_rows(name):
    """The SpMM tiles (row group x column block segments of 32-bit records)
    hold every long-row nonzero once, each row's columns in order."""
    d, i, p, shape = _case(name, torch.bfloat16)
    form = _structured.build(d, i, p, shape[0], shape[1])
    assert form.lt_rec is not None
    # dense long rows over few columns overflow a tile segment: chunks instead
    dd, ii, pp, sh = _case("banded_long", torch.bfloat16)
    assert _structured.build(dd, ii, pp, sh[0], sh[1]).lt_rec is None
    rec = form.lt_rec.cpu().to(torch.int64) & 0xFFFFFFFF
    start, seg_len = form.lt_seg_start.cpu(), form.lt_seg_len.cpu()
    rs = form.lt_row_start.cpu().to(torch.int32) & 0xFFFF
    hp, hi, hd = p.cpu().long(), i.cpu().long(), d.cpu()
    long_rows = form.long_rows.cpu().long().tolist()
    got_cols = {l: [] for l in range(len(long_rows))}
    got_vals = {l: [] for l in range(len(long_rows))}
    for g in range(form.lt_groups):
        for j in range(form.lt_col_blocks):
            seg = g * form.lt_col_blocks + j
            assert int(start[seg]) % 4 == 0 and int(seg_len[seg]) % 4 == 0
            for rig in range(_structured.LT_ROWS):
                lo, hi_ = int(rs[seg, rig]), int(rs[seg, rig + 1])
                l = g * _structured.LT_ROWS + rig
                for k in range(lo, hi_):
                    r = int(rec[int(start[seg]) + k])
                    got_cols[l].append(j * _structured.LT_COLS + (r >> 16))
                    got_vals[l].append(r & 0xFFFF)
    for l, row in enumerate(long_rows):
        s, e = int(hp[row]), int(hp[row + 1])
        assert got_cols[l] == hi[s:e].tolist()
        assert got_vals[l] == (hd[s:e].view(torch.int16).to(torch.int32) & 0xFFFF).tolist()
