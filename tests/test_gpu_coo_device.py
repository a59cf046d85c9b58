"""COO prepare on the device: the duplicate merge (fsb_coo_coalesce) equals
torch's coalesce -- which FlagSparse calls, spmm_coo.py:35-51 -- bit for bit,
and the COO SpMV / SpMM prepare and product record in a CUDA graph (no host
read: run bounds, row offsets and the plan stay on the device) with replays
equal to the eager calls and to FlagSparse's fixtures."""

import pytest
import torch

import flagsparse_public_b200 as fs
import flagsparse_public_b200.sparse_operations.spmm_coo as spmm_coo_mod
from tests.conftest import load_golden

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")

DTYPES = [torch.float32, torch.float64, torch.float16, torch.bfloat16, torch.complex64, torch.complex128]


def _bits(t):
    if t.dtype.is_complex:
        t = torch.view_as_real(t)
    return t.contiguous().view({2: torch.int16, 4: torch.int32, 8: torch.int64}[t.element_size()])


def _dup_coo(n_rows, n_cols, nnz, dtype, seed):
    g = torch.Generator().manual_seed(seed)
    row = torch.randint(0, n_rows, (nnz,), generator=g)
    col = torch.randint(0, n_cols, (nnz,), generator=g)
    vals = torch.randn(nnz, generator=g, dtype=torch.float64) * 10.0 ** torch.randint(-3, 4, (nnz,), generator=g)
    vals[::11] = -0.0  # signed zeros: a sum from +0 turns a lone -0 into +0 unless nnz < 2
    if dtype.is_complex:
        vals = torch.complex(vals, torch.randn(nnz, generator=g, dtype=torch.float64))
    return vals.to(dtype).to(DEV), row.to(DEV), col.to(DEV)


def _torch_coalesce(vals, row, col, shape):
    t = torch.sparse_coo_tensor(torch.stack([row.long(), col.long()]), vals, size=shape).coalesce()
    return t.values(), t.indices()[0], t.indices()[1]


@pytest.mark.parametrize("dtype", DTYPES, ids=lambda d: str(d).replace("torch.", ""))
@pytest.mark.parametrize("case", [(40, 30, 2000), (1000, 1000, 5000), (7, 5, 1), (7, 5, 2), (3, 3, 0)],
                         ids=["dense_dups", "sparse", "one", "two", "empty"])
def test_device_coalesce_equals_torch(dtype, case):
    n_rows, n_cols, nnz = case
    vals, row, col = _dup_coo(n_rows, n_cols, nnz, dtype, seed=nnz + n_rows)
    got = spmm_coo_mod._coalesce_coo_entries(vals, row, col, (n_rows, n_cols))
    if nnz == 0:
        assert all(t.numel() == 0 for t in got)
        return
    ref = _torch_coalesce(vals, row, col, (n_rows, n_cols))
    assert torch.equal(got[1], ref[1]) and torch.equal(got[2], ref[2])
    assert got[0].dtype == ref[0].dtype and torch.equal(_bits(got[0]), _bits(ref[0]))


def test_device_coalesce_golden():
    g = load_golden("spmm_coo_f32")
    d, r, c = spmm_coo_mod._coalesce_coo_entries(g["data"].to(DEV), g["row"].to(DEV), g["col"].to(DEV), g["shape"])
    assert torch.equal(r.cpu(), g["coalesced_row"]) and torch.equal(c.cpu(), g["coalesced_col"])
    assert torch.equal(d.cpu(), g["coalesced_data"])


def test_device_coalesce_records_in_a_graph():
    vals, row, col = _dup_coo(200, 150, 6000, torch.float32, seed=3)
    eager = spmm_coo_mod._coalesce_coo_device(vals, row, col, (200, 150))
    torch.cuda.synchronize()
    gr = torch.cuda.CUDAGraph()
    with torch.cuda.graph(gr):
        cap = spmm_coo_mod._coalesce_coo_device(vals, row, col, (200, 150))
    gr.replay()
    torch.cuda.synchronize()
    m = int(eager[3].item())
    assert int(cap[3].item()) == m
    for a, b in zip(eager[:3], cap[:3]):
        assert torch.equal(a[:m], b[:m])


def _capture(fn):
    fn()  # eager first: loads every kernel the call uses
    torch.cuda.synchronize()
    gr = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        fn()
    torch.cuda.current_stream().wait_stream(s)
    holder = {}
    with torch.cuda.graph(gr):
        holder["out"] = fn()
    gr.replay()
    torch.cuda.synchronize()
    return gr, holder["out"]


@pytest.mark.parametrize("name", ["spmv_coo_seg_f32", "spmv_coo_seg_c128"])
def test_coo_spmv_prepare_records_in_a_graph(name):
    g = load_golden(name)
    data, row, col, x = (g[k].to(DEV) for k in ("data", "row", "col", "x"))
    shape = g["shape"]
    eager = fs.flagsparse_spmv_coo(x=x, prepared=fs.prepare_spmv_coo(data, row, col, shape))

    def call():
        p = fs.prepare_spmv_coo(data, row, col, shape)
        return p, fs.flagsparse_spmv_coo(x=x, prepared=p)

    _gr, (p, y) = _capture(call)
    assert torch.equal(y, eager)
    # the run bounds reach the host only now, after the replay
    assert torch.equal(p.seg_starts.cpu(), g["seg_starts"]) and p.n_segs == g["seg_starts"].numel() - 1
    assert torch.equal(p.row.cpu(), g["sorted_row"]) and torch.equal(p.col.cpu(), g["sorted_col"])


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64, torch.complex64])
def test_coo_spmm_one_shot_records_in_a_graph(dtype):
    vals, row, col = _dup_coo(3000, 2000, 40000, dtype, seed=9)
    B = torch.randn(2000, 24, dtype=torch.float64, device=DEV).to(dtype)
    eager = fs.flagsparse_spmm_coo(vals, row, col, B, (3000, 2000))
    _gr, C = _capture(lambda: fs.flagsparse_spmm_coo(vals, row, col, B, (3000, 2000)))
    assert torch.equal(C, eager)
    # the products sum duplicates as separate nonzeros: within one rounding of
    # the product of the coalesced matrix
    wide = torch.complex128 if dtype.is_complex else torch.float64
    d, r, c = spmm_coo_mod._coalesce_coo_entries(vals, row, col, (3000, 2000))
    A = torch.zeros((3000, 2000), dtype=wide, device=DEV)
    A[r, c] = d.to(wide)
    ref = A @ B.to(wide)
    err = (C.to(wide) - ref).abs().max() / ref.abs().max()
    assert float(err) < (1e-5 if dtype != torch.float64 else 1e-12)


def test_coo_spmv_sizes_need_no_host_read():
    """A large skewed COO matrix prepared inside a capture: nothing in the
    prepare or the product synchronises (the capture would fail)."""
    vals, row, col = _dup_coo(50000, 50000, 400000, torch.float32, seed=5)
    row[:20000] = 7  # one long row
    x = torch.randn(50000, device=DEV)
    eager = fs.flagsparse_spmv_coo(vals, row, col, x, (50000, 50000))
    _gr, y = _capture(lambda: fs.flagsparse_spmv_coo(vals, row, col, x, (50000, 50000)))
    assert torch.equal(y, eager)
