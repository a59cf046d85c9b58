"""Host-side logic of the drop-in operators, on CPU tensors (no kernel runs).

Covers the integer preparation steps that must reproduce FlagSparse's
structure bit for bit (golden fixtures), the validation errors raised before
any device work, the int64 -> int32 fallback policy (failure injected on the
host, as FlagSparse's own tests do) and the default kernel plans.
"""

import pytest
import torch

import flagsparse_public_b200.sparse_operations.spmm_coo as spmm_coo_mod
import flagsparse_public_b200.sparse_operations.spmm_csr as spmm_mod
import flagsparse_public_b200.sparse_operations.spmv_coo as spmv_coo_mod
import flagsparse_public_b200.sparse_operations.spmv_csr as spmv_mod
from flagsparse_public_b200 import _native as nat
from flagsparse_public_b200 import _plan
from tests.conftest import load_golden


def test_transpose_structure_matches_reference():
    g = load_golden("transpose_c64")
    td, ti, tp, tshape = spmv_mod._transpose_csr_for_spmv(g["data"], g["indices"], g["indptr"], g["shape"])
    assert tshape == tuple(g["t_shape"])
    assert ti.dtype == g["t_indices"].dtype and tp.dtype == g["t_indptr"].dtype
    assert torch.equal(ti, g["t_indices"])
    assert torch.equal(tp, g["t_indptr"])
    assert torch.equal(td, g["t_data"])


def test_coo_to_csr_matches_reference():
    g = load_golden("coo_to_csr")
    d, i, p = spmv_mod.coo_to_csr_for_spmv(g["data"], g["row"], g["col"], g["shape"])
    assert torch.equal(d, g["out_data"]) and torch.equal(i, g["out_indices"]) and torch.equal(p, g["out_indptr"])
    assert i.dtype == torch.int32 and p.dtype == torch.int64


@pytest.mark.parametrize("name", ["spmv_coo_seg_f32", "spmv_coo_seg_c128"])
def test_coo_sort_and_row_runs_match_reference(name):
    g = load_golden(name)
    d, r, c = spmv_coo_mod._sort_coo_lex_inplace(g["data"], g["row"], g["col"], g["shape"][1])
    assert torch.equal(d, g["sorted_data"]) and torch.equal(r, g["sorted_row"]) and torch.equal(c, g["sorted_col"])
    seg = spmv_coo_mod._seg_starts_from_sorted_rows(r, d.numel(), d.device)
    assert torch.equal(seg, g["seg_starts"]) and seg.dtype == g["seg_starts"].dtype


def test_split_metadata_matches_reference_host_loop():
    g = load_golden("spmm_opt_split_f32")
    rl = g["indptr"][1:] - g["indptr"][:-1]
    _buckets, long_rows = spmm_mod._build_spmm_opt_buckets(rl)
    assert torch.equal(long_rows, g["long_rows"])
    rows, starts, ends, rpp = spmm_mod._build_spmm_opt_split_metadata(g["indptr"], long_rows, 256)
    assert torch.equal(rows, g["part_rows"]) and rows.dtype == g["part_rows"].dtype
    assert torch.equal(starts, g["part_starts"]) and torch.equal(ends, g["part_ends"])
    assert torch.equal(rpp, g["row_part_ptr"])


def test_coalesce_matches_reference():
    g = load_golden("spmm_coo_f32")
    d, r, c = spmm_coo_mod._coalesce_coo_entries(g["data"], g["row"], g["col"], g["shape"])
    assert torch.equal(r, g["coalesced_row"]) and torch.equal(c, g["coalesced_col"])
    assert torch.equal(d, g["coalesced_data"])


def _cpu_csr():
    data = torch.tensor([1.0, 2.0, 3.0])
    indices = torch.tensor([0, 1, 1], dtype=torch.int32)
    indptr = torch.tensor([0, 2, 3], dtype=torch.int64)
    return data, indices, indptr


def test_validation_errors_before_device_work():
    data, indices, indptr = _cpu_csr()
    with pytest.raises(ValueError, match="must be CUDA tensors"):
        spmv_mod.prepare_spmv_csr(data, indices, indptr, (2, 2))
    with pytest.raises(ValueError, match="indptr length"):
        spmv_mod.prepare_spmv_csr(data, indices, indptr[:-1], (2, 2))
    with pytest.raises(TypeError, match="must all be torch.Tensor"):
        spmv_mod.prepare_spmv_csr([1.0], indices, indptr, (2, 2))
    with pytest.raises(ValueError, match="index_fallback_policy"):
        spmv_mod.prepare_spmv_csr(data, indices, indptr, (2, 2), index_fallback_policy="bad")
    with pytest.raises(ValueError, match="op must be one of"):
        spmv_mod.flagsparse_spmv_csr(data, indices, indptr, data[:2], (2, 2), op="bogus")
    with pytest.raises(ValueError, match="conflicts with op"):
        spmv_mod.flagsparse_spmv_csr(data, indices, indptr, data[:2], (2, 2), op="non", transpose=True)
    with pytest.raises(ValueError, match="must be CUDA tensors"):
        spmm_mod.flagsparse_spmm_csr(data, indices, indptr, torch.randn(2, 4), (2, 2))
    with pytest.raises(ValueError, match="shape must be a 2-tuple"):
        spmm_mod.flagsparse_spmm_csr(data, indices, indptr, torch.randn(2, 4), (2,))
    with pytest.raises(ValueError, match="block_n must be positive"):
        spmm_mod.flagsparse_spmm_csr(data, indices, indptr, torch.randn(2, 4), (2, 2), block_n=0)
    with pytest.raises(ValueError, match="CUDA tensors"):
        spmm_coo_mod.flagsparse_spmm_coo(data, indices, indices, torch.randn(2, 4), (2, 2))
    with pytest.raises(ValueError, match="CUDA tensors"):
        spmv_coo_mod.prepare_spmv_coo(data, indices, indices, (2, 2))


def test_op_normalisation():
    assert spmv_mod._normalize_spmv_op(None, transpose=True) == spmv_mod.SPMV_OP_TRANS
    assert spmv_mod._normalize_spmv_op("conj") == spmv_mod.SPMV_OP_CONJ_TRANS
    assert spmv_mod._normalize_spmv_op(1) == spmv_mod.SPMV_OP_TRANS
    assert spmv_coo_mod._normalize_spmv_coo_op(" NON ") == 0
    with pytest.raises(ValueError):
        spmv_coo_mod._normalize_spmv_coo_op(3)


def _prepared_cpu(index_dtype, policy="auto"):
    data, indices, indptr = _cpu_csr()
    return spmv_mod.PreparedCsrSpmv(
        data=data, kernel_indices=indices.to(index_dtype), kernel_indptr=indptr.to(index_dtype), shape=(2, 2),
        n_rows=2, n_cols=2, block_nnz=256, max_segments=1, max_row_nnz=2, opt_buckets=[],
        index_fallback_policy=policy)


def test_int64_failure_falls_back_to_int32(monkeypatch):
    seen = []

    def fake_run(prepared, x, use_opt=False):
        seen.append(prepared.kernel_indices.dtype)
        if prepared.kernel_indices.dtype == torch.int64:
            raise RuntimeError("forced int64 launch failure")
        return torch.zeros(prepared.n_rows)

    monkeypatch.setattr(spmv_mod, "_run_spmv_prepared", fake_run)
    y = spmv_mod._run_spmv_prepared_with_fallback(_prepared_cpu(torch.int64), torch.zeros(2))
    assert seen == [torch.int64, torch.int32] and y.numel() == 2


def test_strict_policy_reraises(monkeypatch):
    def fake_run(prepared, x, use_opt=False):
        raise RuntimeError("forced int64 launch failure")

    monkeypatch.setattr(spmv_mod, "_run_spmv_prepared", fake_run)
    with pytest.raises(RuntimeError, match="forced int64 launch failure"):
        spmv_mod._run_spmv_prepared_with_fallback(_prepared_cpu(torch.int64, "strict"), torch.zeros(2))


def test_fallback_refused_when_index_exceeds_int32(monkeypatch):
    limit = spmv_mod._INDEX_LIMIT_INT32
    prepared = spmv_mod.PreparedCsrSpmv(
        data=torch.ones(1), kernel_indices=torch.tensor([limit + 1], dtype=torch.int64),
        kernel_indptr=torch.tensor([0, 1], dtype=torch.int64), shape=(1, limit + 2), n_rows=1, n_cols=limit + 2,
        block_nnz=256, max_segments=1, max_row_nnz=1, opt_buckets=[], transpose=False,
        index_fallback_policy="auto")

    def fail_launch(_prepared, _x, use_opt=False):
        raise RuntimeError("forced native int64 failure")

    monkeypatch.setattr(spmv_mod, "_run_spmv_prepared", fail_launch)
    with pytest.raises(RuntimeError, match="int32 fallback is unsafe"):
        spmv_mod._run_spmv_prepared_with_fallback(prepared, torch.empty(0), use_opt=False)


def test_coo_fallback_policy(monkeypatch):
    data = torch.tensor([1.0, 2.0])
    row = torch.tensor([0, 1], dtype=torch.int64)
    col = torch.tensor([1, 0], dtype=torch.int64)
    p = spmv_coo_mod.PreparedCoo(data, row, col, (2, 2), seg_starts=torch.tensor([0, 1, 2]))
    calls = []

    def fake(prepared, x, block_size, num_warps, block_inner):
        calls.append(prepared.row.dtype)
        if prepared.row.dtype == torch.int64:
            raise RuntimeError("forced")
        return torch.zeros(2)

    monkeypatch.setattr(spmv_coo_mod, "_triton_spmv_coo_kernel", fake)
    spmv_coo_mod._run_spmv_coo_prepared_with_fallback(p, torch.zeros(2), 256, 4, 128)
    assert calls == [torch.int64, torch.int32]


def test_default_plans():
    flat = _plan.MatrixStats(16384, 16384, 262144, 35, 16.0, 4.0, 0)
    p = _plan.default_spmv_plan(flat, torch.float32)
    assert p.algo == nat.ALGO_ROWS and p.lanes == 8
    skew = _plan.MatrixStats(262144, 262144, 3_100_000, 7200, 11.9, 80.0, 10)
    assert _plan.default_spmv_plan(skew, torch.float32).algo == nat.ALGO_MERGE
    mm = _plan.default_spmm_plan(skew, 64, torch.float32)
    assert mm.algo == nat.ALGO_SEQ and mm.items_per_unit == 256
    assert _plan.default_spmm_plan(skew, 4, torch.float32).algo == nat.ALGO_SEQ
    banded = _plan.MatrixStats(1 << 20, 1 << 20, 156_953_476, 8192, 149.7, 780.0, 0)
    assert _plan.default_spmm_plan(banded, 32, torch.bfloat16).items_per_unit == 1024
    g = _plan.KernelPlan(nat.ALGO_GATHER, items_per_unit=256, fallback_ok=True)
    assert g.as_flat().algo == nat.ALGO_FLAT
    long_skew = _plan.MatrixStats(1 << 20, 1 << 20, 156_953_476, 8192, 149.7, 780.0, 0)
    p = _plan.default_spmv_plan(long_skew, torch.bfloat16)
    assert p.algo == nat.ALGO_ROWS and p.lanes == 32
    assert _plan.default_spmv_plan(long_skew, torch.float32).lanes == 32
    capped = _plan.default_spmv_plan(skew, torch.float32, row_cap=32)
    assert capped.algo == nat.ALGO_ROWS and capped.row_cap == 32


def test_batch_stacking_is_block_diagonal():
    from flagsparse_public_b200 import batched, synthetic
    mats = [synthetic.poisson_uniform(r, c, mean=m, seed=s, device="cpu")
            for r, c, m, s in ((7, 5, 2.0, 1), (1, 9, 4.0, 2), (12, 12, 3.0, 3), (4, 3, 1.0, 4))]
    mats.append((torch.zeros(0), torch.zeros(0, dtype=torch.int32), torch.zeros(3, dtype=torch.int64), (2, 6)))
    data, indices, indptr, row_off, col_off = batched.stack_csr(mats)
    assert row_off == [0, 7, 8, 20, 24, 26] and col_off == [0, 5, 14, 26, 29, 35]
    assert indices.dtype == torch.int32 and indptr.dtype == torch.int64
    got = torch.sparse_csr_tensor(indptr, indices.long(), data, size=(26, 35)).to_dense()
    want = torch.block_diag(*[torch.sparse_csr_tensor(m[2], m[1].long(), m[0], size=m[3]).to_dense() for m in mats])
    assert torch.equal(got, want)


def test_csr_to_bsr16_blocks_match_dense():
    from flagsparse_public_b200 import bsr, synthetic
    data, indices, indptr, shape = synthetic.poisson_uniform(37, 50, mean=6.0, seed=5, device="cpu")
    vals, bcol, bptr = bsr.csr_to_bsr16(data, indices, indptr, shape, dtype=torch.float64)
    dense = torch.sparse_csr_tensor(indptr, indices.long(), data.double(), size=shape).to_dense()
    rebuilt = torch.zeros(48, 64, dtype=torch.float64)
    for br in range(bptr.numel() - 1):
        for b in range(int(bptr[br]), int(bptr[br + 1])):
            c = int(bcol[b])
            rebuilt[16 * br:16 * br + 16, 16 * c:16 * c + 16] = vals[b]
    assert torch.equal(rebuilt[:37, :50], dense) and rebuilt[37:].abs().sum() == 0
    assert bptr[0] == 0 and bptr[-1] == vals.shape[0] and bptr.numel() == 4
    for br in range(3):  # block columns sorted within each block row
        seg = bcol[int(bptr[br]):int(bptr[br + 1])]
        assert torch.all(seg[1:] > seg[:-1])


def test_prepare_sort_wrappers_on_host_tensors():
    """stable_sort / run_starts on host tensors: torch's stable sort and the
    nonzero-based run starts FlagSparse uses, dtype and empty cases included."""
    import torch

    from flagsparse_public_b200 import _plan

    g = torch.Generator().manual_seed(3)
    for dtype in (torch.int32, torch.int64):
        keys = torch.randint(0, 50, (1000,), generator=g).to(dtype)
        k, o = _plan.stable_sort(keys, key_bound=50)
        rk, ro = torch.sort(keys, stable=True)
        assert torch.equal(k, rk) and torch.equal(o, ro)
        for out_dtype in (torch.int32, torch.int64):
            st = _plan.run_starts(k, out_dtype)
            assert st.dtype == out_dtype
            ref = torch.cat([torch.zeros(1, dtype=out_dtype),
                             (torch.nonzero(k[1:] != k[:-1]).flatten() + 1).to(out_dtype),
                             torch.tensor([k.numel()], dtype=out_dtype)])
            assert torch.equal(st, ref)
    assert _plan.run_starts(torch.empty(0, dtype=torch.int64), torch.int32) is None
    assert torch.equal(_plan.run_starts(torch.tensor([7]), torch.int64), torch.tensor([0, 1]))
