"""Every kernel family of the C ABI against the FP64 oracle.

Each launch goes through ``fsb_spmv_csr`` / ``fsb_spmm_csr`` with an explicit
plan (row groups of 1..32 lanes, merge-path tiles/units of several sizes,
column tiles), on matrices that stress row-boundary handling: empty rows,
rows of 1/31/32/33/4095/4097 nonzeros, heavy skew, all-empty matrices.

Bounds (condition-scaled, see tests/numerics.py): float32 with float64
accumulation within 1e-5 and within one float32 rounding of the FP64 result;
float32 accumulation within 3e-5; float64 within 1e-12; half types within
one rounding of the output type.
"""

import pytest
import torch

from flagsparse_public_b200 import _native as nat
from flagsparse_public_b200 import _plan
from oracle import oracle as orc
from tests.gpu_cases import EDGE_LENGTHS, csr_from_lengths, dense, spmm_plans, spmv_plans
from tests.numerics import REL_BOUND, scaled_error, ulp_distance_f32

pytestmark = pytest.mark.gpu
DEV = "cuda"

NATIVE_F32_BOUND = 3e-5

# (value dtype, acc mode, output dtype, bound)
SPMV_MODES = [
    (torch.float32, nat.ACC_WIDE, torch.float32, REL_BOUND[torch.float32]),
    (torch.float32, nat.ACC_NATIVE, torch.float32, NATIVE_F32_BOUND),
    (torch.float64, nat.ACC_NATIVE, torch.float64, REL_BOUND[torch.float64]),
    (torch.float16, nat.ACC_NATIVE, torch.float16, REL_BOUND[torch.float16]),
    (torch.bfloat16, nat.ACC_NATIVE, torch.bfloat16, REL_BOUND[torch.bfloat16]),
    (torch.bfloat16, nat.ACC_NATIVE, torch.float32, NATIVE_F32_BOUND),
    (torch.complex64, nat.ACC_NATIVE, torch.complex64, NATIVE_F32_BOUND),
    (torch.complex64, nat.ACC_WIDE, torch.complex64, REL_BOUND[torch.complex64]),
    (torch.complex128, nat.ACC_NATIVE, torch.complex128, REL_BOUND[torch.complex128]),
]


def _mode_id(m):
    return f"{str(m[0])[6:]}-{['native', 'wide', 'comp'][m[1]]}-{str(m[2])[6:]}"


@pytest.mark.parametrize("pattern", sorted(EDGE_LENGTHS))
@pytest.mark.parametrize("mode", SPMV_MODES, ids=_mode_id)
def test_spmv_all_plans_edge_patterns(pattern, mode):
    dtype, acc, out_dtype, bound = mode
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths(EDGE_LENGTHS[pattern], 13000, seed=5, dtype=dtype)
    x = dense((n_cols,), 6, dtype)
    exact, mag = orc.spmv_csr_exact(data, indices, indptr, x)
    d_data, d_idx, d_ptr, d_x = data.to(DEV), indices.to(DEV), indptr.to(DEV), x.to(DEV)
    for plan in spmv_plans(dtype):
        y = torch.full((n_rows,), float("nan"), dtype=out_dtype, device=DEV)
        _plan.run_spmv(d_data, d_idx, d_ptr, n_rows, n_cols, d_x, y, acc, plan)
        err = scaled_error(y, exact, mag)
        assert err <= bound, (plan.describe(), err)
        if dtype == torch.float32 and acc == nat.ACC_WIDE:
            assert ulp_distance_f32(y.cpu(), exact.to(torch.float32)) <= 1, plan.describe()


@pytest.mark.parametrize("index_dtype,ptr_dtype", [(torch.int32, torch.int32), (torch.int32, torch.int64),
                                                   (torch.int64, torch.int32), (torch.int64, torch.int64)])
def test_spmv_index_widths(index_dtype, ptr_dtype):
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths(EDGE_LENGTHS["skewed"], 20000, seed=7,
                                                               index_dtype=index_dtype, ptr_dtype=ptr_dtype)
    x = dense((n_cols,), 8, torch.float32)
    exact, mag = orc.spmv_csr_exact(data, indices, indptr, x)
    for plan in spmv_plans(torch.float32):
        y = torch.empty(n_rows, dtype=torch.float32, device=DEV)
        _plan.run_spmv(data.to(DEV), indices.to(DEV), indptr.to(DEV), n_rows, n_cols, x.to(DEV), y, nat.ACC_WIDE,
                       plan)
        assert scaled_error(y, exact, mag) <= 1e-5


def test_spmv_unaligned_views_use_scalar_path():
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths([5, 9, 17, 33, 64, 3], 100, seed=9)
    # shift the arrays by one element so 16-byte vector loads are not allowed
    data_u = torch.cat([torch.zeros(1), data]).to(DEV)[1:]
    idx_u = torch.cat([torch.zeros(1, dtype=torch.int32), indices]).to(DEV)[1:]
    x = dense((n_cols,), 10, torch.float32)
    exact, mag = orc.spmv_csr_exact(data, indices, indptr, x)
    for lanes in (2, 4, 32):
        y = torch.empty(n_rows, device=DEV)
        _plan.run_spmv(data_u, idx_u, indptr.to(DEV), n_rows, n_cols, x.to(DEV), y, nat.ACC_WIDE,
                       _plan.KernelPlan(nat.ALGO_ROWS, lanes=lanes))
        assert scaled_error(y, exact, mag) <= 1e-5


def test_spmv_row_cap_truncates_like_reference_window():
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths([10, 40, 70, 0, 33], 200, seed=11)
    x = dense((n_cols,), 12, torch.float32)
    ref = orc.spmv_csr(data, indices, indptr, x, acc_mode=orc.ACC_WIDE, row_cap=32)
    y = torch.empty(n_rows, device=DEV)
    _plan.run_spmv(data.to(DEV), indices.to(DEV), indptr.to(DEV), n_rows, n_cols, x.to(DEV), y, nat.ACC_WIDE,
                   _plan.KernelPlan(nat.ALGO_ROWS, lanes=8, row_cap=32))
    assert ulp_distance_f32(y.cpu(), ref) <= 1


def test_spmv_row_map_runs():
    """Row runs of sorted COO: row_ptr = run offsets, output row = row_map[start]."""
    rows = torch.tensor([1, 1, 4, 4, 4, 7, 9, 9], dtype=torch.int32)
    cols = torch.tensor([0, 5, 1, 2, 9, 3, 0, 8], dtype=torch.int32)
    vals = dense((8,), 13, torch.float64)
    x = dense((10,), 14, torch.float64)
    seg = torch.tensor([0, 2, 5, 6, 8], dtype=torch.int32)
    ref = torch.zeros(10, dtype=torch.float64).index_add_(0, rows.long(), vals * x[cols.long()])
    for plan in spmv_plans(torch.float64):
        y = torch.zeros(10, dtype=torch.float64, device=DEV)
        _plan.run_spmv(vals.to(DEV), cols.to(DEV), seg.to(DEV), 4, 10, x.to(DEV), y, nat.ACC_NATIVE, plan,
                       row_map=rows.to(DEV))
        assert torch.allclose(y.cpu(), ref, rtol=1e-13, atol=1e-14), plan.describe()


@pytest.mark.parametrize("vdtype", [torch.bfloat16, torch.float16, torch.float32])
def test_spmv_compensated_long_rows(vdtype):
    """COMP accumulation: rows > threshold carry a TwoSum/TwoProduct error term."""
    lengths = [8192] * 8 + [68] * 200 + [5000, 9000]
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths(lengths, 12000, seed=15, dtype=vdtype)
    x = dense((n_cols,), 16, vdtype)
    exact, mag = orc.spmv_csr_exact(data, indices, indptr, x)
    for plan in (_plan.KernelPlan(nat.ALGO_ROWS, lanes=32, comp_threshold=4096),
                 _plan.KernelPlan(nat.ALGO_MERGE, items_per_unit=1024, comp_threshold=4096)):
        y = torch.empty(n_rows, dtype=torch.float32, device=DEV)
        _plan.run_spmv(data.to(DEV), indices.to(DEV), indptr.to(DEV), n_rows, n_cols, x.to(DEV), y, nat.ACC_COMP,
                       plan)
        lens = (indptr[1:] - indptr[:-1])
        long_rows = lens > 4096
        err_long = scaled_error(y.cpu()[long_rows], exact[long_rows], mag[long_rows])
        assert err_long <= 2e-7, (plan.describe(), err_long)
        assert scaled_error(y, exact, mag) <= NATIVE_F32_BOUND


SPMM_MODES = [
    (torch.float32, nat.ACC_WIDE, torch.float32, REL_BOUND[torch.float32]),
    (torch.float32, nat.ACC_NATIVE, torch.float32, NATIVE_F32_BOUND),
    (torch.float64, nat.ACC_NATIVE, torch.float64, REL_BOUND[torch.float64]),
    (torch.float16, nat.ACC_NATIVE, torch.float16, REL_BOUND[torch.float16]),
    (torch.bfloat16, nat.ACC_NATIVE, torch.float32, NATIVE_F32_BOUND),
    (torch.complex64, nat.ACC_NATIVE, torch.complex64, NATIVE_F32_BOUND),
    (torch.complex64, nat.ACC_WIDE, torch.complex64, REL_BOUND[torch.complex64]),
    (torch.complex128, nat.ACC_NATIVE, torch.complex128, REL_BOUND[torch.complex128]),
]


@pytest.mark.parametrize("pattern", ["empty_rows", "boundaries", "skewed", "all_empty", "one_row"])
@pytest.mark.parametrize("n_dense", [1, 3, 8, 32, 64, 96])
@pytest.mark.parametrize("mode", SPMM_MODES, ids=_mode_id)
def test_spmm_all_plans(pattern, n_dense, mode):
    dtype, acc, out_dtype, bound = mode
    lengths = EDGE_LENGTHS[pattern]
    if pattern == "skewed":
        lengths = lengths[::3]
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths(lengths, 13000, seed=17, dtype=dtype)
    B = dense((n_cols, n_dense), 18, dtype)
    exact, mag = orc.spmm_csr_exact(data, indices, indptr, B)
    d = (data.to(DEV), indices.to(DEV), indptr.to(DEV))
    Bd = B.to(DEV)
    for plan in spmm_plans():
        C = torch.full((n_rows, n_dense), float("nan"), dtype=out_dtype, device=DEV)
        if plan.algo == nat.ALGO_GATHER and not _plan.gather_supported(Bd, C, plan.n_tile):
            continue
        if plan.flags & nat.PLAN_TMA_GATHER and not _plan.g4_supported(d[0], Bd, C, acc, n_cols):
            continue
        _plan.run_spmm(*d, n_rows, n_cols, Bd, C, acc, plan)
        err = scaled_error(C, exact, mag)
        assert err <= bound, (plan.describe(), err)


def test_spmm_strided_output_and_operand():
    """ldb / ldc larger than the dense width (views into wider buffers)."""
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths([3, 0, 40, 7, 300], 500, seed=19)
    Bw = dense((n_cols, 80), 20, torch.float32)
    B = Bw[:, :64]
    exact, mag = orc.spmm_csr_exact(data, indices, indptr, B.contiguous())
    Cw = torch.zeros((n_rows, 72), device=DEV)
    C = Cw[:, :64]
    lib = nat.library()
    # the struct holds raw pointers: keep the device tensors alive across the call
    d_data, d_idx, d_ptr = data.to(DEV), indices.to(DEV), indptr.to(DEV)
    cm = nat.make_csr(d_data, d_idx, d_ptr, n_rows, n_cols)
    Bd = Bw.to(DEV)
    cp = _plan.KernelPlan(nat.ALGO_ROWS, lanes=32).c_plan()
    rc = lib.fsb_spmm_csr(cm, nat.ptr(Bd), 80, 64, nat.ptr(Cw), 72, nat.FSB_F32, nat.ACC_WIDE, cp, None, 0,
                          nat.stream_handle(torch.device(DEV)))
    nat.check(rc, "fsb_spmm_csr")
    assert scaled_error(C, exact, mag) <= 1e-5
    assert bool((Cw[:, 64:] == 0).all()), "columns beyond n_dense were written"


def test_spmm_compensated_long_rows():
    lengths = [8192] * 4 + [68] * 100 + [6000]
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths(lengths, 12000, seed=21, dtype=torch.bfloat16)
    B = dense((n_cols, 32), 22, torch.bfloat16)
    exact, mag = orc.spmm_csr_exact(data, indices, indptr, B)
    lens = indptr[1:] - indptr[:-1]
    long_rows = lens > 4096
    for plan in (_plan.KernelPlan(nat.ALGO_ROWS, lanes=32, comp_threshold=4096),
                 _plan.KernelPlan(nat.ALGO_MERGE, items_per_unit=256, snap=64, comp_threshold=4096)):
        C = torch.empty((n_rows, 32), dtype=torch.float32, device=DEV)
        _plan.run_spmm(data.to(DEV), indices.to(DEV), indptr.to(DEV), n_rows, n_cols, B.to(DEV), C, nat.ACC_COMP,
                       plan)
        err_long = scaled_error(C.cpu()[long_rows], exact[long_rows], mag[long_rows])
        assert err_long <= 2e-7, (plan.describe(), err_long)


def test_merge_partition_kernel_matches_oracle():
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths(EDGE_LENGTHS["skewed"], 20000, seed=23)
    nnz = data.numel()
    for items, snap in ((128, 0), (256, 64), (1024, 0), (77, 30)):
        plan = _plan.KernelPlan(nat.ALGO_MERGE, items_per_unit=items, snap=snap)
        plan.ensure_coords(indptr.to(DEV), n_rows, nnz)
        ref = orc.merge_partition(indptr, n_rows, nnz, items, snap)
        assert torch.equal(plan.coords.cpu(), ref)


def test_bounded_wait_times_out_and_context_survives():
    """A wait on an mbarrier nothing completes gives up, records a status, and
    the device keeps working (no trap, no hang)."""
    lib = nat.library()
    assert nat.device_error(reset=True) in (0, nat.FSB_ERR_TIMEOUT)
    rc = lib.fsb_selftest_wait_timeout(20_000_000, nat.stream_handle(torch.device(DEV)))  # 20 ms
    nat.check(rc, "fsb_selftest_wait_timeout")
    torch.cuda.synchronize()
    assert nat.device_error(reset=True) == nat.FSB_ERR_TIMEOUT
    assert nat.device_error(reset=False) == 0
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths([5, 0, 40, 3], 300, seed=31)
    B = dense((n_cols, 64), 32, torch.float32)
    exact, mag = orc.spmm_csr_exact(data, indices, indptr, B)
    C = torch.empty((n_rows, 64), device=DEV)
    _plan.run_spmm(data.to(DEV), indices.to(DEV), indptr.to(DEV), n_rows, n_cols, B.to(DEV), C, nat.ACC_WIDE,
                   _plan.KernelPlan(nat.ALGO_GATHER, items_per_unit=16))
    assert scaled_error(C, exact, mag) <= 1e-5
    assert nat.device_error(reset=False) == 0


def test_gather_plan_rejects_unaligned_operands():
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths([5, 7], 50, seed=33)
    B = dense((n_cols, 6), 34, torch.float32).to(DEV)
    C = torch.empty((n_rows, 6), device=DEV)
    with pytest.raises(ValueError, match="16-byte aligned"):
        _plan.run_spmm(data.to(DEV), indices.to(DEV), indptr.to(DEV), n_rows, n_cols, B, C, nat.ACC_NATIVE,
                       _plan.KernelPlan(nat.ALGO_GATHER, items_per_unit=16))


def test_merge_runs_kernel_matches_oracle():
    """fsb_merge_runs (binary searches) equals the oracle's linear walk."""
    for pattern, items, snap in (("skewed", 128, 0), ("skewed", 77, 30), ("long_rows", 256, 64),
                                 ("empty_rows", 4, 0), ("boundaries", 33, 0), ("all_empty", 8, 0)):
        data, indices, indptr, (n_rows, n_cols) = csr_from_lengths(EDGE_LENGTHS[pattern], 20000, seed=29)
        dptr = indptr.to(DEV)
        plan = _plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=items, snap=snap)
        plan.ensure_coords(dptr, n_rows, data.numel())
        plan.ensure_runs(dptr, n_rows, 8)
        ref = orc.merge_runs(indptr, n_rows, plan.coords.cpu())
        assert torch.equal(plan.runs.cpu()[: ref.numel()], ref), (pattern, items, snap)


def test_csr_check_kernel_matches_oracle():
    """fsb_csr_check's eight figures equal the oracle's, valid and malformed
    structures alike (decreasing offsets, negative and out-of-range columns,
    empty matrices), int32 and int64 offsets and indices."""
    cases = []
    for pattern in ("skewed", "empty_rows", "long_rows", "all_empty"):
        _d, indices, indptr, _shape = csr_from_lengths(EDGE_LENGTHS[pattern], 20000, seed=31)
        cases.append((indptr, indices))
    _d, indices, indptr, _shape = csr_from_lengths(EDGE_LENGTHS["skewed"], 20000, seed=32)
    bad_ptr = indptr.clone()
    bad_ptr[3] = bad_ptr[5] + 2  # rows 2 and 3 change length, one negative
    bad_col = indices.to(torch.int64)
    bad_col[::97] = -3
    bad_col[5] = 1 << 40
    cases += [(bad_ptr, indices), (indptr, bad_col), (bad_ptr + 1, indices),
              (torch.zeros(1, dtype=torch.int64), torch.zeros(0, dtype=torch.int64)),
              (torch.tensor([0, 0, 0]), torch.zeros(0, dtype=torch.int32))]
    for k, (p, c) in enumerate(cases):
        for pt, it in ((torch.int64, torch.int64), (torch.int32, torch.int32), (torch.int64, torch.int32)):
            if it == torch.int32 and c.numel() and int(c.to(torch.int64).abs().max()) >= 2**31:
                continue
            hp, hc = p.to(pt), c.to(it)
            got = nat.csr_check(hp.to(DEV), hc.to(DEV), hp.numel() - 1)
            assert got == orc.csr_check(hp, hc), (k, pt, it)


def _spmm_two_kernel(d, n_rows, n_cols, B, C, acc, plan):
    """The same SEQ plan with split rows finished by the separate fix-up
    kernel (no unit runs in the C plan)."""
    cm = nat.make_csr(d[0], d[1], d[2], n_rows, n_cols)
    cp = nat.make_plan(plan.algo, items_per_unit=plan.items_per_unit, n_tile=plan.n_tile, coords=plan.coords,
                       n_units=plan.n_units, comp_threshold=plan.comp_threshold, grid_blocks=plan.grid_blocks,
                       flags=plan.flags)
    out = nat.dtype_code(C.dtype)
    ws, nbytes = _plan._workspace(True, cm, B.shape[1], acc, out, cp, B.device)
    rc = nat.library().fsb_spmm_csr(cm, nat.ptr(B), int(B.stride(0)), int(B.shape[1]), nat.ptr(C), int(C.stride(0)),
                                    out, int(acc), cp, nat.ptr(ws), nbytes, nat.stream_handle(B.device))
    nat.check(rc, "fsb_spmm_csr (two-kernel)")


SEQ_FINISH_PLANS = [(16, 0, 0, 0, 0), (100, 0, 0, 0, 0), (256, 128, 0, 0, 0), (2048, 0, 0, 0, 0),
                    (128, 64, 32, 0, 0), (77, 0, 8, 0, 0), (16, 0, 0, 1, 0), (64, 0, 0, 3, 0),
                    (128, 64, 0, 0, 0), (64, 64, 0, 2, 0)]


@pytest.mark.parametrize("pattern", ["skewed", "long_rows", "boundaries", "empty_rows"])
@pytest.mark.parametrize("n_dense", [1, 8, 64, 96])
@pytest.mark.parametrize("mode", [SPMM_MODES[0], SPMM_MODES[1], SPMM_MODES[2], SPMM_MODES[5], SPMM_MODES[-1]],
                         ids=_mode_id)
def test_seq_in_kernel_finish_equals_fixup_kernel(pattern, n_dense, mode):
    """Split rows finished inside k_spmm_seq (tickets, last unit sums in unit
    order) equal the two-kernel form bit for bit, on two calls in a row, and
    leave every ticket counter at zero."""
    dtype, acc, out_dtype, _ = mode
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths(EDGE_LENGTHS[pattern], 13000, seed=31, dtype=dtype)
    d = (data.to(DEV), indices.to(DEV), indptr.to(DEV))
    Bd = dense((n_cols, n_dense), 32, dtype).to(DEV)
    for items, snap, n_tile, grid, flags in SEQ_FINISH_PLANS:
        plan = _plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=items, snap=snap, n_tile=n_tile, grid_blocks=grid,
                                flags=flags)
        ref = torch.full((n_rows, n_dense), float("nan"), dtype=out_dtype, device=DEV)
        plan.ensure_coords(d[2], n_rows, data.numel())
        _spmm_two_kernel(d, n_rows, n_cols, Bd, ref, acc, plan)
        for _ in range(2):
            C = torch.full((n_rows, n_dense), float("nan"), dtype=out_dtype, device=DEV)
            _plan.run_spmm(*d, n_rows, n_cols, Bd, C, acc, plan)
            assert torch.equal(C, ref), (pattern, n_dense, items, snap, n_tile, grid, flags)
        assert plan.in_kernel_finish() and int(plan.tickets.abs().sum()) == 0


def test_seq_in_kernel_finish_compensated_rows():
    """Compensated (s, c) partials of long bf16 rows finish in the kernel with
    the two-kernel form's bits."""
    lengths = [8192] * 4 + [68] * 100 + [6000]
    data, indices, indptr, (n_rows, n_cols) = csr_from_lengths(lengths, 12000, seed=33, dtype=torch.bfloat16)
    d = (data.to(DEV), indices.to(DEV), indptr.to(DEV))
    Bd = dense((n_cols, 32), 34, torch.bfloat16).to(DEV)
    for items, snap in ((256, 64), (1024, 0), (97, 0)):
        plan = _plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=items, snap=snap, comp_threshold=4096)
        plan.ensure_coords(d[2], n_rows, data.numel())
        ref = torch.empty((n_rows, 32), dtype=torch.float32, device=DEV)
        _spmm_two_kernel(d, n_rows, n_cols, Bd, ref, nat.ACC_COMP, plan)
        C = torch.empty_like(ref)
        _plan.run_spmm(*d, n_rows, n_cols, Bd, C, nat.ACC_COMP, plan)
        assert torch.equal(C, ref), (items, snap)


@pytest.mark.parametrize("captured", [False, True], ids=["eager", "graph"])
def test_overlapped_launch_chain_equals_plain(captured):
    """Back-to-back row SpMVs launched with programmatic dependent launch
    (FSB_PLAN_OVERLAP_LAUNCH), each reading the previous one's output
    (x_{k+1} = A x_k), equal the same chain launched plainly, bit for bit:
    every CTA waits for its predecessor before reading."""
    from flagsparse_public_b200 import synthetic

    d, i, p, shape = synthetic.poisson_uniform(8192, 8192, mean=16.0, seed=11, device=DEV)
    d = d * 0.25
    x0 = synthetic.dense_vector(shape[1], seed=12, device=DEV)
    steps = 12

    def chain(flags):
        plan = _plan.KernelPlan(nat.ALGO_ROWS, lanes=8, flags=flags)
        bufs = [x0.clone()] + [torch.empty_like(x0) for _ in range(steps)]

        def run():
            for k in range(steps):
                _plan.run_spmv(d, i, p, shape[0], shape[1], bufs[k], bufs[k + 1], nat.ACC_NATIVE, plan)

        if captured:
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                run()
            torch.cuda.current_stream().wait_stream(s)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                run()
            for b in bufs[1:]:
                b.fill_(float("nan"))
            g.replay()
        else:
            run()
        torch.cuda.synchronize()
        return torch.stack(bufs[1:])

    plain = chain(0)
    overlapped = chain(nat.PLAN_OVERLAP_LAUNCH)
    assert torch.isfinite(plain).all()
    assert torch.equal(plain, overlapped)


@pytest.mark.parametrize("n_dense", [32, 64, 128])
def test_gather_floor_probe_gathers_every_row(n_dense):
    """fsb_gather_floor reads each nonzero's B row once: the sum of its
    per-thread sums equals the sum of the gathered rows (every variant)."""
    g = torch.Generator().manual_seed(71)
    nnz, n_cols = 100_003, 5000
    col = torch.randint(0, n_cols, (nnz,), generator=g, dtype=torch.int32)
    B = torch.rand((n_cols, n_dense), generator=g, dtype=torch.float64)
    expect = float(B[col.long()].sum())
    lib = nat.library()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    out = torch.empty(sms * 16 * 128, device=DEV)
    dc, dB = col.to(DEV), B.float().to(DEV)
    for variant in range(nat.GATHER_FLOOR_VARIANTS):
        out.fill_(float("nan"))
        used = out[: sms * {0: 16, 1: 8, 2: 4, 3: 12}[variant] * 128]
        rc = lib.fsb_gather_floor(nat.ptr(dc), nnz, nat.ptr(dB), n_dense, n_dense, nat.ptr(out), out.numel(),
                                  variant, nat.stream_handle(torch.device(DEV)))
        nat.check(rc, "fsb_gather_floor")
        torch.cuda.synchronize()
        assert abs(float(used.double().sum()) - expect) <= 1e-5 * expect
    # unsupported widths and too small an output are rejected before any launch
    assert lib.fsb_gather_floor(nat.ptr(dc), nnz, nat.ptr(dB), 48, 48, nat.ptr(out), out.numel(), 0,
                                nat.stream_handle(torch.device(DEV))) == nat.FSB_ERR_UNSUPPORTED
    assert lib.fsb_gather_floor(nat.ptr(dc), nnz, nat.ptr(dB), n_dense, n_dense, nat.ptr(out), 128, 0,
                                nat.stream_handle(torch.device(DEV))) == nat.FSB_ERR_INVALID
