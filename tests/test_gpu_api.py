"""FlagSparse's own accuracy and API tests, run against this implementation.

Mirrors FlagSparse tests/pytest/test_spmv_csr_accuracy.py,
test_spmv_coo_accuracy.py, test_spmm_csr_accuracy.py,
test_spmm_coo_accuracy.py, test_spmm_csr_opt_alg2_accuracy.py and the API
validation cases of tests/test_spmm.py:714-836 (same shapes, dtypes, ops,
tolerances, exception types and message patterns), seeded.  Failure injection
is done on the host by patching the private hooks, as in the reference.
"""

import pytest
import torch

import flagsparse_public_b200 as fs
import flagsparse_public_b200.sparse_operations.spmm_csr as spmm_mod
import flagsparse_public_b200.sparse_operations.spmv_coo as spmv_coo_mod
import flagsparse_public_b200.sparse_operations.spmv_csr as spmv_mod

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda")

SPMV_MN_SHAPES = [(1, 32), (160, 1024), (128, 256)]
MNK_SHAPES = [(8, 4, 16), (64, 16, 96)]
SPMV_DTYPES = [torch.float16, torch.bfloat16, torch.float32, torch.float64, torch.complex64, torch.complex128]


@pytest.fixture(autouse=True)
def _seed():
    torch.manual_seed(1234)


def _random_dense(shape, dtype):
    if dtype.is_complex:
        comp = torch.float32 if dtype == torch.complex64 else torch.float64
        return torch.complex(torch.randn(shape, dtype=comp, device=DEV), torch.randn(shape, dtype=comp, device=DEV))
    return torch.randn(shape, dtype=dtype, device=DEV)


def _reference_dtype(dtype):
    return {torch.float16: torch.float32, torch.bfloat16: torch.float32, torch.float32: torch.float64,
            torch.complex64: torch.complex128}.get(dtype, dtype)


def _tol_spmv(dtype):
    if dtype == torch.float16:
        return 5e-3, 5e-3
    if dtype == torch.bfloat16:
        return 1e-1, 1e-1
    if dtype in (torch.float32, torch.complex64):
        return 1e-4, 1e-4
    return 1e-10, 1e-8


def _random_csr_mn(M, N, dtype, index_dtype):
    p = min(0.25, max(0.06, 32.0 / max(M * N, 1)))
    mask = torch.rand(M, N, device=DEV) < p
    if int(mask.sum().item()) == 0:
        mask[0, 0] = True
    dense = torch.where(mask, _random_dense((M, N), dtype), torch.zeros((), dtype=dtype, device=DEV))
    rows, cols = torch.nonzero(mask, as_tuple=True)
    data = dense[rows, cols].contiguous()
    indptr = torch.zeros(M + 1, dtype=torch.int64, device=DEV)
    indptr[1:] = torch.cumsum(torch.bincount(rows, minlength=M), dim=0)
    return data, cols.to(index_dtype).contiguous(), indptr.to(index_dtype), dense


def _apply_op(dense, op):
    return {"non": dense, "trans": dense.t(), "conj": dense.conj().t()}[op]


@pytest.mark.parametrize("M, N", SPMV_MN_SHAPES)
@pytest.mark.parametrize("dtype", SPMV_DTYPES, ids=lambda d: str(d)[6:])
@pytest.mark.parametrize("index_dtype", [torch.int32, torch.int64], ids=["int32", "int64"])
@pytest.mark.parametrize("op", ["non", "trans", "conj"])
@pytest.mark.parametrize("use_opt", [False, True], ids=["plain", "opt"])
def test_spmv_csr_matches_dense_reference(M, N, dtype, index_dtype, op, use_opt):
    data, indices, indptr, dense = _random_csr_mn(M, N, dtype, index_dtype)
    x = _random_dense((M if op != "non" else N,), dtype)
    ref_dtype = _reference_dtype(dtype)
    ref = (_apply_op(dense, op).to(ref_dtype) @ x.to(ref_dtype)).to(dtype)
    out = fs.flagsparse_spmv_csr(data, indices, indptr, x, shape=(M, N), op=op, use_opt=use_opt)
    rtol, atol = _tol_spmv(dtype)
    assert out.dtype == dtype and out.shape == ref.shape
    assert torch.allclose(out.to(ref_dtype), ref.to(ref_dtype), rtol=rtol, atol=atol)


def test_spmv_csr_prepared_out_and_time():
    data, indices, indptr, dense = _random_csr_mn(160, 1024, torch.float32, torch.int32)
    x = torch.randn(1024, device=DEV)
    prepared = fs.prepare_spmv_csr(data, indices, indptr, (160, 1024))
    out = torch.empty(160, device=DEV)
    y, ms = fs.flagsparse_spmv_csr(x=x, prepared=prepared, out=out, return_time=True, use_opt=True)
    assert y is out and isinstance(ms, float)
    assert torch.allclose(y.double(), dense.double() @ x.double(), rtol=1e-4, atol=1e-4)


def test_spmv_csr_prepared_transpose_mismatch_rejected():
    data, indices, indptr, _ = _random_csr_mn(8, 10, torch.float32, torch.int32)
    prepared = spmv_mod.prepare_spmv_csr(data, indices, indptr, (8, 10), transpose=True)
    with pytest.raises(ValueError, match="does not match prepared.transpose"):
        fs.flagsparse_spmv_csr(x=torch.randn(8, device=DEV), prepared=prepared, transpose=False)


def test_spmv_csr_prepared_op_mismatch_rejected():
    data, indices, indptr, _ = _random_csr_mn(8, 10, torch.complex64, torch.int32)
    prepared = spmv_mod.prepare_spmv_csr(data, indices, indptr, (8, 10), op="conj")
    with pytest.raises(ValueError, match="does not match prepared.op"):
        fs.flagsparse_spmv_csr(x=_random_dense((8,), torch.complex64), prepared=prepared, op="trans")


def test_spmv_csr_int64_auto_fallback_to_int32(monkeypatch):
    data, indices, indptr, dense = _random_csr_mn(12, 9, torch.float32, torch.int64)
    x = torch.randn(9, device=DEV)
    ref = dense.double() @ x.double()
    state = {"forced_once": False}
    original = spmv_mod._triton_spmv_csr_impl_prepared

    def fail_int64_once(prepared, x_in):
        if prepared.kernel_indices.dtype == torch.int64 and not state["forced_once"]:
            state["forced_once"] = True
            raise RuntimeError("forced int64 launch failure")
        return original(prepared, x_in)

    monkeypatch.setattr(spmv_mod, "_triton_spmv_csr_impl_prepared", fail_int64_once)
    out = fs.flagsparse_spmv_csr(data, indices, indptr, x, shape=(12, 9), index_fallback_policy="auto")
    assert state["forced_once"]
    assert torch.allclose(out.double(), ref, rtol=1e-4, atol=1e-4)


def test_spmv_csr_int64_strict_no_fallback(monkeypatch):
    data, indices, indptr, _ = _random_csr_mn(12, 9, torch.float32, torch.int64)

    def fail_int64(prepared, x_in):
        raise RuntimeError("forced int64 launch failure")

    monkeypatch.setattr(spmv_mod, "_triton_spmv_csr_impl_prepared", fail_int64)
    with pytest.raises(RuntimeError, match="forced int64 launch failure"):
        fs.flagsparse_spmv_csr(data, indices, indptr, torch.randn(9, device=DEV), shape=(12, 9),
                               index_fallback_policy="strict")


def test_spmv_csr_explicit_max_segments_truncates_like_reference():
    """An explicit max_segments window shorter than a row truncates that row."""
    g = torch.Generator(device="cpu").manual_seed(3)
    lengths = torch.tensor([5, 70, 20, 100, 0])
    indptr = torch.zeros(6, dtype=torch.int64)
    indptr[1:] = torch.cumsum(lengths, 0)
    indices = torch.cat([torch.sort(torch.randperm(128, generator=g)[:n]).values for n in lengths.tolist()])
    data = torch.rand(int(indptr[-1]), generator=g)
    x = torch.randn(128, generator=g)
    y = fs.flagsparse_spmv_csr(data.to(DEV), indices.to(torch.int32).to(DEV), indptr.to(DEV), x.to(DEV),
                               shape=(5, 128), block_nnz=16, max_segments=2)
    ref = torch.stack([(data[s:min(e, s + 32)].double() * x[indices[s:min(e, s + 32)]].double()).sum()
                       for s, e in zip(indptr[:-1].tolist(), indptr[1:].tolist())]).float()
    assert torch.allclose(y.cpu(), ref, rtol=1e-6, atol=1e-6)
    # opt path: rows are capped at max_segments x (their tier's lanes)
    y_opt = fs.flagsparse_spmv_csr(data.to(DEV), indices.to(torch.int32).to(DEV), indptr.to(torch.int32).to(DEV),
                                   x.to(DEV), shape=(5, 128), max_segments=1, use_opt=True)
    cap = lambda n: 32 if n <= 64 else 256  # noqa: E731
    ref_opt = torch.stack([(data[s:min(e, s + cap(e - s))].double() * x[indices[s:min(e, s + cap(e - s))]].double())
                           .sum() for s, e in zip(indptr[:-1].tolist(), indptr[1:].tolist())]).float()
    assert torch.allclose(y_opt.cpu(), ref_opt, rtol=1e-5, atol=1e-5)


# ------------------------------------------------------------- COO SpMV ----
SPMV_COO_DTYPES = (torch.float32, torch.float64, torch.complex64, torch.complex128)


def _random_coo_mn(M, N, dtype):
    p = min(0.25, max(0.06, 32.0 / max(M * N, 1)))
    mask = torch.rand(M, N, device=DEV) < p
    if int(mask.sum().item()) == 0:
        mask[0, 0] = True
    dense = torch.where(mask, _random_dense((M, N), dtype), torch.zeros((), dtype=dtype, device=DEV))
    return dense.to_sparse_coo().coalesce(), dense


@pytest.mark.parametrize("M, N", SPMV_MN_SHAPES)
@pytest.mark.parametrize("dtype", SPMV_COO_DTYPES, ids=lambda d: str(d)[6:])
@pytest.mark.parametrize("index_dtype", [torch.int32, torch.int64], ids=["int32", "int64"])
@pytest.mark.parametrize("op", ["non", "trans", "conj"])
@pytest.mark.parametrize("sort_by_row", [True, False], ids=["rowrun", "atomic"])
def test_spmv_coo_matches_dense_reference(M, N, dtype, index_dtype, op, sort_by_row):
    Asp, dense = _random_coo_mn(M, N, dtype)
    idx = Asp.indices()
    row, col = idx[0].to(index_dtype).contiguous(), idx[1].to(index_dtype).contiguous()
    x = _random_dense((M if op != "non" else N,), dtype)
    ref_dtype = _reference_dtype(dtype)
    ref = (_apply_op(dense, op).to(ref_dtype) @ x.to(ref_dtype)).to(dtype)
    out = fs.flagsparse_spmv_coo(Asp.values(), row, col, x, shape=(M, N), op=op, sort_by_row=sort_by_row)
    rtol, atol = (1e-4, 1e-4) if dtype in (torch.float32, torch.complex64) else (1e-10, 1e-8)
    assert torch.allclose(out.to(ref_dtype), ref.to(ref_dtype), rtol=rtol, atol=atol)


def test_spmv_coo_prepared_transpose_mismatch_rejected():
    Asp, _ = _random_coo_mn(8, 10, torch.float32)
    idx = Asp.indices()
    prepared = fs.prepare_spmv_coo(Asp.values(), idx[0].to(torch.int32), idx[1].to(torch.int32), (8, 10),
                                   transpose=True)
    with pytest.raises(ValueError, match="does not match prepared.transpose"):
        fs.flagsparse_spmv_coo(x=torch.randn(8, device=DEV), prepared=prepared, transpose=False)


def test_spmv_coo_int64_auto_fallback_to_int32(monkeypatch):
    Asp, dense = _random_coo_mn(12, 9, torch.float32)
    idx = Asp.indices()
    x = torch.randn(9, device=DEV)
    state = {"forced_once": False}
    original = spmv_coo_mod._triton_spmv_coo_kernel

    def fail_int64_once(prepared, x_in, block_size, num_warps, block_inner):
        if prepared.row.dtype == torch.int64 and not state["forced_once"]:
            state["forced_once"] = True
            raise RuntimeError("forced int64 launch failure")
        return original(prepared, x_in, block_size, num_warps, block_inner)

    monkeypatch.setattr(spmv_coo_mod, "_triton_spmv_coo_kernel", fail_int64_once)
    out = fs.flagsparse_spmv_coo(Asp.values(), idx[0].contiguous(), idx[1].contiguous(), x, shape=(12, 9))
    assert state["forced_once"]
    assert torch.allclose(out.double(), dense.double() @ x.double(), rtol=1e-4, atol=1e-4)


def test_spmv_coo_argument_validation():
    Asp, _ = _random_coo_mn(8, 10, torch.float32)
    idx = Asp.indices()
    with pytest.raises(ValueError, match="num_warps"):
        fs.flagsparse_spmv_coo(Asp.values(), idx[0], idx[1], torch.randn(10, device=DEV), shape=(8, 10), num_warps=3)
    with pytest.raises(ValueError, match="block_inner"):
        fs.flagsparse_spmv_coo(Asp.values(), idx[0], idx[1], torch.randn(10, device=DEV), shape=(8, 10),
                               block_inner=100)
    with pytest.raises(TypeError, match="COO SpMV supports"):
        fs.flagsparse_spmv_coo(Asp.values().half(), idx[0], idx[1], torch.randn(10, device=DEV).half(),
                               shape=(8, 10))


@pytest.mark.parametrize("M, N", SPMV_MN_SHAPES)
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64], ids=["float32", "float64"])
def test_spmv_coo_tocsr_matches_torch(M, N, dtype):
    Asp, _ = _random_coo_mn(M, N, dtype)
    idx = Asp.indices()
    x = torch.randn(N, dtype=dtype, device=DEV)
    ref = torch.sparse.mm(Asp, x.unsqueeze(1)).squeeze(1)
    out = fs.flagsparse_spmv_coo_tocsr(Asp.values(), idx[0].contiguous(), idx[1].contiguous(), x, shape=(M, N))
    rtol, atol = (1e-4, 1e-4) if dtype == torch.float32 else (1e-10, 1e-8)
    assert torch.allclose(out, ref, rtol=rtol, atol=atol)
    prepared = fs.prepare_spmv_coo_tocsr(Asp.values(), idx[0], idx[1], (M, N))
    out2 = fs.flagsparse_spmv_coo_tocsr(x=x, prepared=prepared)
    assert torch.allclose(out2, ref, rtol=rtol, atol=atol)


# ------------------------------------------------------------- CSR SpMM ----
def _tol_spmm(dtype):
    if dtype == torch.bfloat16:
        return 1e-1, 1e-1
    if dtype == torch.float16:
        return 5e-3, 5e-3
    if dtype == torch.float32:
        return 1e-4, 1e-4
    return 1e-10, 1e-8


def _random_csr_mk(M, K, dtype, p_lo=0.06, p_hi=0.25, base=32.0):
    p = min(p_hi, max(p_lo, base / max(M * K, 1)))
    mask = torch.rand(M, K, device=DEV) < p
    if int(mask.sum().item()) == 0:
        mask[0, 0] = True
    vals = _random_dense((M, K), dtype) * mask.to(dtype=dtype)
    return vals.to_sparse_csr(), vals


def _csr_ref(data, indices, indptr, B, shape, dtype):
    dense = torch.sparse_csr_tensor(indptr.to(torch.int64), indices.to(torch.int64), data.to(_reference_dtype(dtype)),
                                    size=shape, device=DEV).to_dense()
    return (dense @ B.to(_reference_dtype(dtype))).to(dtype)


@pytest.mark.parametrize("M, N, K", MNK_SHAPES)
@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16, torch.float32, torch.float64, torch.complex64],
                         ids=lambda d: str(d)[6:])
def test_spmm_csr_matches_torch(M, N, K, dtype):
    Asp, _ = _random_csr_mk(M, K, dtype)
    data, indices, indptr = Asp.values(), Asp.col_indices(), Asp.crow_indices()
    B = _random_dense((K, N), dtype)
    ref = _csr_ref(data, indices, indptr, B, (M, K), dtype)
    out = fs.flagsparse_spmm_csr(data, indices, indptr, B, (M, K))
    rtol, atol = _tol_spmm(dtype) if not dtype.is_complex else (1e-4, 1e-4)
    assert torch.allclose(out, ref, rtol=rtol, atol=atol)


@pytest.mark.parametrize("M, N, K", MNK_SHAPES)
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64], ids=["float32", "float64"])
def test_spmm_csr_opt_matches_torch(M, N, K, dtype):
    Asp, _ = _random_csr_mk(M, K, dtype)
    data, indices, indptr = Asp.values(), Asp.col_indices(), Asp.crow_indices()
    B = torch.randn(K, N, dtype=dtype, device=DEV)
    ref = _csr_ref(data, indices, indptr, B, (M, K), dtype)
    prepared = fs.prepare_spmm_csr_opt(data, indices, indptr, (M, K))
    out = fs.flagsparse_spmm_csr_opt(B=B, prepared=prepared)
    rtol, atol = _tol_spmm(dtype)
    assert torch.allclose(out, ref, rtol=rtol, atol=atol)


@pytest.mark.parametrize("M, N, K", MNK_SHAPES)
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64], ids=["float32", "float64"])
@pytest.mark.parametrize("dense_cols", [1, 8, 32, 96])
@pytest.mark.parametrize("index_dtype", [torch.int32, torch.int64], ids=["int32", "int64"])
def test_spmm_csr_opt_alg2_matches_torch(M, N, K, dtype, dense_cols, index_dtype):
    Asp, _ = _random_csr_mk(M, K, dtype, p_lo=0.08, p_hi=0.35, base=48.0)
    data = Asp.values()
    indices, indptr = Asp.col_indices().to(index_dtype), Asp.crow_indices().to(index_dtype)
    B = torch.randn(K, dense_cols, dtype=dtype, device=DEV)
    ref = _csr_ref(data, indices, indptr, B, (M, K), dtype)
    out = fs.flagsparse_spmm_csr_opt_alg2(data, indices, indptr, B, (M, K))
    rtol, atol = _tol_spmm(dtype)
    assert torch.allclose(out, ref, rtol=rtol, atol=atol)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64], ids=["float32", "float64"])
def test_spmm_csr_opt_alg2_prepared_out_and_meta(dtype):
    M, K, N = 16, 32, 24
    Asp, _ = _random_csr_mk(M, K, dtype, p_lo=0.08, p_hi=0.35, base=48.0)
    data = Asp.values()
    indices, indptr = Asp.col_indices().to(torch.int64), Asp.crow_indices().to(torch.int64)
    B = torch.randn(K, N, dtype=dtype, device=DEV)
    prepared = fs.prepare_spmm_csr_opt_alg2(data, indices, indptr, (M, K))
    out_buf = torch.empty((M, N), dtype=dtype, device=DEV)
    out, meta = fs.flagsparse_spmm_csr_opt_alg2(B=B, prepared=prepared, out=out_buf, return_meta=True)
    ref = _csr_ref(data, indices, indptr, B, (M, K), dtype)
    rtol, atol = _tol_spmm(dtype)
    assert out is out_buf
    assert torch.allclose(out, ref, rtol=rtol, atol=atol)
    assert meta["device_name"]
    assert isinstance(meta["sm_count"], int) and isinstance(meta["warp_size"], int)
    assert meta["max_row_nnz"] == prepared.max_row_nnz
    assert meta["n_dense_cols"] == N
    assert meta["bucket_hits"] and meta["launch_configs"]


def test_spmm_csr_opt_alg2_return_time_and_meta_shapes():
    M, K, N = 8, 16, 7
    Asp, _ = _random_csr_mk(M, K, torch.float32, p_lo=0.08, p_hi=0.35, base=48.0)
    out, elapsed_ms, meta = fs.flagsparse_spmm_csr_opt_alg2(
        data=Asp.values(), indices=Asp.col_indices(), indptr=Asp.crow_indices(), B=torch.randn(K, N, device=DEV),
        shape=(M, K), return_time=True, return_meta=True)
    assert out.shape == (M, N) and isinstance(elapsed_ms, float) and meta["n_dense_cols"] == N


@pytest.mark.parametrize("M, N, K", MNK_SHAPES)
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64], ids=["float32", "float64"])
def test_spmm_coo_matches_torch(M, N, K, dtype):
    Asp, _ = _random_csr_mk(M, K, dtype)
    Acoo = Asp.to_sparse_coo().coalesce()
    idx = Acoo.indices()
    B = torch.randn(K, N, dtype=dtype, device=DEV)
    ref = torch.sparse.mm(Acoo.double(), B.double()).to(dtype)
    out = fs.flagsparse_spmm_coo(Acoo.values(), idx[0].contiguous(), idx[1].contiguous(), B, (M, K))
    rtol, atol = _tol_spmm(dtype)
    assert torch.allclose(out, ref, rtol=rtol, atol=atol)


def test_spmm_coo_duplicates_and_atomic_route():
    rows = torch.tensor([0, 2, 2, 0, 1, 2], device=DEV)
    cols = torch.tensor([1, 0, 0, 1, 3, 2], device=DEV)
    vals = torch.randn(6, device=DEV)
    B = torch.randn(4, 5, device=DEV)
    dense = torch.zeros(3, 4, dtype=torch.float64, device=DEV).index_put_((rows, cols), vals.double(),
                                                                          accumulate=True)
    ref = (dense @ B.double()).float()
    out = fs.flagsparse_spmm_coo(vals, rows, cols, B, (3, 4))
    assert torch.allclose(out, ref, rtol=1e-6, atol=1e-6)
    import flagsparse_public_b200.sparse_operations.spmm_coo as mc
    out_atomic = mc._run_spmm_coo_route(vals, rows, cols, B, (3, 4), route="atomic")
    assert torch.allclose(out_atomic, ref, rtol=1e-6, atol=1e-6)


# -------------------------------------------- API validation (test_spmm.py) --
def _api_inputs():
    data = torch.tensor([1.0, 2.0, 3.0], dtype=torch.float32, device=DEV)
    indices = torch.tensor([0, 1, 1], dtype=torch.int32, device=DEV)
    indptr = torch.tensor([0, 2, 3], dtype=torch.int64, device=DEV)
    B = torch.randn((2, 4), dtype=torch.float32, device=DEV)
    return data, indices, indptr, B


def _long_row_case():
    indices = torch.cat([torch.arange(1536), torch.tensor([7, 129, 511, 1024])]).to(torch.int32).to(DEV)
    data = torch.randn(1540, device=DEV)
    indptr = torch.tensor([0, 1536, 1540], dtype=torch.int64, device=DEV)
    B = torch.randn(2048, 48, device=DEV)
    return data, indices, indptr, B, (2, 2048)


NEGATIVE_CASES = [
    ("shape must be 2D", lambda d, i, p, B: fs.flagsparse_spmm_csr(d, i, p, B, (2,)), ValueError),
    ("B must be 2D", lambda d, i, p, B: fs.flagsparse_spmm_csr(d, i, p, B[0], (2, 2)), ValueError),
    ("dtype mismatch", lambda d, i, p, B: fs.flagsparse_spmm_csr(d, i, p, B.to(torch.float64), (2, 2)), TypeError),
    ("shape mismatch", lambda d, i, p, B: fs.flagsparse_spmm_csr(d, i, p, torch.randn((3, 4), device=DEV), (2, 2)),
     ValueError),
    ("indptr length mismatch", lambda d, i, p, B: fs.flagsparse_spmm_csr(d, i, p[:-1], B, (2, 2)), ValueError),
    ("indptr must start at 0", lambda d, i, p, B: fs.flagsparse_spmm_csr(
        d, i, torch.tensor([1, 2, 3], dtype=torch.int64, device=DEV), B, (2, 2)), ValueError),
    ("indptr last must equal nnz", lambda d, i, p, B: fs.flagsparse_spmm_csr(
        d, i, torch.tensor([0, 2, 2], dtype=torch.int64, device=DEV), B, (2, 2)), ValueError),
    ("indptr monotonic", lambda d, i, p, B: fs.flagsparse_spmm_csr(
        d, i, torch.tensor([0, 3, 2], dtype=torch.int64, device=DEV), B, (2, 2)), ValueError),
    ("indices out of range", lambda d, i, p, B: fs.flagsparse_spmm_csr(
        d, torch.tensor([0, 3, 1], dtype=torch.int32, device=DEV), p, B, (2, 2)), IndexError),
    ("block_n positive", lambda d, i, p, B: fs.flagsparse_spmm_csr(d, i, p, B, (2, 2), block_n=0), ValueError),
    ("block_nnz positive", lambda d, i, p, B: fs.flagsparse_spmm_csr(d, i, p, B, (2, 2), block_nnz=0), ValueError),
    ("max_segments positive", lambda d, i, p, B: fs.flagsparse_spmm_csr(d, i, p, B, (2, 2), max_segments=0),
     ValueError),
    ("out shape mismatch", lambda d, i, p, B: fs.flagsparse_spmm_csr(
        d, i, p, B, (2, 2), out=torch.empty((3, 4), device=DEV)), ValueError),
    ("out device mismatch", lambda d, i, p, B: fs.flagsparse_spmm_csr(d, i, p, B, (2, 2), out=torch.empty((2, 4))),
     ValueError),
]


@pytest.mark.parametrize("name,fn,exc", NEGATIVE_CASES, ids=[c[0] for c in NEGATIVE_CASES])
def test_spmm_api_negative_cases(name, fn, exc):
    with pytest.raises(exc):
        fn(*_api_inputs())


def test_spmm_api_segment_overflow_override():
    d, i, p, B, shape = _long_row_case()
    with pytest.raises(ValueError):
        fs.flagsparse_spmm_csr(d, i, p, B, shape, block_nnz=128, max_segments=4)


def test_spmm_api_positive_cases():
    d, i, p, B = _api_inputs()
    dense = torch.tensor([[1.0, 2.0], [0.0, 3.0]], dtype=torch.float64, device=DEV)
    out = torch.empty((2, 4), device=DEV)
    res = fs.flagsparse_spmm_csr(d, i, p, B, (2, 2), out=out)
    assert res.data_ptr() == out.data_ptr()
    assert torch.allclose(res.double(), dense @ B.double(), rtol=1e-6, atol=1e-6)
    empty = fs.flagsparse_spmm_csr(torch.tensor([], device=DEV), torch.tensor([], dtype=torch.int32, device=DEV),
                                   torch.zeros(3, dtype=torch.int64, device=DEV), B, (2, 2))
    assert empty.shape == (2, 4) and bool((empty == 0).all())
    r0 = fs.flagsparse_spmm_csr(d, i, p, torch.empty((2, 0), device=DEV), (2, 2))
    assert r0.shape == (2, 0)
    Bt = torch.randn(4, 2, device=DEV).transpose(0, 1)
    assert not Bt.is_contiguous()
    r1 = fs.flagsparse_spmm_csr(d, i, p, Bt, (2, 2))
    assert torch.allclose(r1.double(), dense @ Bt.double(), rtol=1e-6, atol=1e-6)
    ld, li, lp, lB, lshape = _long_row_case()
    r2 = fs.flagsparse_spmm_csr(ld, li, lp, lB, lshape)
    ref = _csr_ref(ld, li, lp, lB, lshape, torch.float32)
    assert torch.allclose(r2, ref, rtol=1e-5, atol=1e-5)


def test_spmm_opt_type_checks():
    d, i, p, B = _api_inputs()
    with pytest.raises(TypeError, match="PreparedCsrSpmmOpt"):
        fs.flagsparse_spmm_csr_opt(B=B, prepared=object())
    prepared = fs.prepare_spmm_csr_opt(d.half(), i, p, (2, 2))
    with pytest.raises(TypeError, match="only supports float32 and float64"):
        fs.flagsparse_spmm_csr_opt(B=B.half(), prepared=prepared)


def test_sorted_coo_to_csr_is_graph_capturable():
    """With assume_sorted the COO -> CSR conversion reads nothing back to the
    host, so it can be captured in a CUDA graph; the replay equals eager mode
    and cumsum(bincount)."""
    from flagsparse_public_b200.sparse_operations.spmv_csr import coo_to_csr_for_spmv
    from flagsparse_public_b200 import synthetic
    data, indices, indptr, shape = synthetic.zipf_powerlaw(5000, 4000, mean=6.0, cap=400, seed=11, device="cuda")
    row = torch.repeat_interleave(torch.arange(shape[0], device="cuda"), indptr[1:] - indptr[:-1]).to(torch.int32)
    eager = coo_to_csr_for_spmv(data, row, indices, shape, assume_sorted=True)
    assert torch.equal(eager[2], indptr)
    coo_to_csr_for_spmv(data, row, indices, shape, assume_sorted=True)  # warm-up outside capture
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        captured = coo_to_csr_for_spmv(data, row, indices, shape, assume_sorted=True)
    g.replay()
    torch.cuda.synchronize()
    assert all(torch.equal(a, b) for a, b in zip(eager, captured))
    ref = torch.zeros(shape[0] + 1, dtype=torch.int64, device="cuda")
    ref[1:] = torch.cumsum(torch.bincount(row.long(), minlength=shape[0]), 0)
    assert torch.equal(captured[2], ref)


def _malformed(kind):
    d = torch.tensor([1.0, 2.0, 3.0], device=DEV)
    i = torch.tensor([0, 1, 2], dtype=torch.int32, device=DEV)
    p = torch.tensor([0, 2, 3], device=DEV)
    if kind == "start":
        p = torch.tensor([1, 2, 3], device=DEV)
    elif kind == "end":
        p = torch.tensor([0, 2, 2], device=DEV)
    elif kind == "decreasing":
        d = torch.tensor([1.0, 2.0], device=DEV)
        i = torch.tensor([0, 1], dtype=torch.int32, device=DEV)
        p = torch.tensor([0, 3, 2], device=DEV)
    elif kind == "negative_col":
        i = torch.tensor([0, -1, 2], dtype=torch.int32, device=DEV)
    elif kind == "col_too_large":
        i = torch.tensor([0, 1, 3], dtype=torch.int32, device=DEV)
    return d, i, p, (2, 3)


# FlagSparse's messages (spmv_csr.py:524-537, spmm_csr.py:228-237), raised
# from the one-read structural check
SPMV_MALFORMED = [("start", ValueError, "start at zero"), ("end", ValueError, "must equal nnz"),
                  ("decreasing", ValueError, "non-decreasing"), ("negative_col", IndexError, "out of range"),
                  ("col_too_large", IndexError, "out of range")]
SPMM_MALFORMED = [("start", ValueError, "must be 0"), ("end", ValueError, "must equal nnz"),
                  ("decreasing", ValueError, "nondecreasing"), ("negative_col", IndexError, "out of range"),
                  ("col_too_large", IndexError, "out of range")]


@pytest.mark.parametrize("kind,exc,msg", SPMV_MALFORMED)
def test_spmv_rejects_malformed_structure(kind, exc, msg):
    d, i, p, shape = _malformed(kind)
    with pytest.raises(exc, match=msg):
        fs.flagsparse_spmv_csr(d, i, p, torch.ones(3, device=DEV), shape)


@pytest.mark.parametrize("kind,exc,msg", SPMM_MALFORMED)
def test_spmm_rejects_malformed_structure(kind, exc, msg):
    d, i, p, shape = _malformed(kind)
    with pytest.raises(exc, match=msg):
        fs.flagsparse_spmm_csr(d, i, p, torch.ones(3, 4, device=DEV), shape)


def test_prepared_stats_from_the_validation_read():
    """The plan statistics a prepare takes from its single read equal a
    separate computation over the row lengths."""
    from flagsparse_public_b200 import _plan, synthetic

    d, i, p, shape = synthetic.zipf_powerlaw(5000, 5000, alpha=1.8, mean=12.0, cap=3000, seed=3, device=DEV)
    for prep in (fs.prepare_spmv_csr(d, i, p, shape), fs.prepare_spmm_csr_opt(d, i, p, shape)):
        got, ref = prep._stats, _plan.matrix_stats(p, shape[0], shape[1])
        assert (got.n_rows, got.nnz, got.max_row, got.empty_rows) == (ref.n_rows, ref.nnz, ref.max_row,
                                                                      ref.empty_rows)
        assert got.mean_row == pytest.approx(ref.mean_row, rel=1e-12)
        assert got.std_row == pytest.approx(ref.std_row, rel=1e-9)


ONESHOT_CASES = [("poisson", torch.float32, torch.int64, True), ("poisson", torch.float32, torch.int32, False),
                 ("skewed", torch.float32, torch.int64, True), ("skewed", torch.float64, torch.int32, False),
                 ("poisson", torch.bfloat16, torch.int64, False), ("skewed", torch.float16, torch.int64, True),
                 ("poisson", torch.complex64, torch.int64, False), ("dense_rows", torch.float32, torch.int64, True),
                 ("empty", torch.float32, torch.int64, True)]


def _oneshot_matrix(kind, dtype, ptr_dtype):
    from flagsparse_public_b200 import synthetic

    if kind == "poisson":
        d, i, p, shape = synthetic.poisson_uniform(3000, 2000, mean=16.0, seed=5, device=DEV)
    elif kind == "skewed":  # short rows on average, a few very long: merge path
        d, i, p, shape = synthetic.zipf_powerlaw(6000, 6000, alpha=1.8, mean=6.0, cap=4000, seed=6, device=DEV)
    elif kind == "dense_rows":
        d, i, p, shape = synthetic.poisson_uniform(500, 4000, mean=300.0, seed=7, device=DEV)
    else:  # rows without nonzeros only
        n = 40
        d, i = torch.zeros(0, device=DEV), torch.zeros(0, dtype=torch.int32, device=DEV)
        p, shape = torch.zeros(n + 1, dtype=torch.int64, device=DEV), (n, 30)
    if dtype.is_complex:
        d = torch.complex(d, -0.5 * d)
    return d.to(dtype), i.to(torch.int32), p.to(ptr_dtype), shape


@pytest.mark.parametrize("kind,dtype,ptr_dtype,use_opt", ONESHOT_CASES)
def test_spmv_oneshot_native_route_equals_prepared(kind, dtype, ptr_dtype, use_opt):
    """The one-shot call (fsb_spmv_csr_checked: check, one read, plan, product
    in one native call) returns bit for bit what prepare + run returns, with
    the plan the prepared route's heuristic picks."""
    from flagsparse_public_b200 import _native as nat
    from flagsparse_public_b200 import _plan

    d, i, p, shape = _oneshot_matrix(kind, dtype, ptr_dtype)
    x = _random_dense((shape[1],), dtype)
    before = _plan.LAUNCHES["count"]
    y1 = fs.flagsparse_spmv_csr(d, i, p, x, shape, use_opt=use_opt)
    assert _plan.LAUNCHES["count"] > before
    prep = fs.prepare_spmv_csr(d, i, p, shape)
    y2 = fs.flagsparse_spmv_csr(x=x, prepared=prep, use_opt=use_opt)
    assert y1.dtype == y2.dtype and torch.equal(y1, y2)
    # the native plan equals the prepared heuristic's
    cm = nat.make_csr(d, i, p, shape[0], shape[1])
    acc = nat.ACC_NATIVE if (use_opt and dtype in (torch.float32, torch.float64)) else (
        nat.ACC_WIDE if dtype == torch.float32 else nat.ACC_NATIVE)
    nbytes = int(nat.library().fsb_spmv_csr_checked_workspace_bytes(cm, acc, nat.dtype_code(dtype)))
    ws = torch.empty(nbytes, dtype=torch.uint8, device=DEV)
    fig = (nat.ctypes.c_int64 * 8)()
    plan = nat.FsbPlan()
    y3 = torch.empty_like(y1)
    rc = nat.library().fsb_spmv_csr_checked(cm, nat.ptr(x), nat.ptr(y3), nat.dtype_code(dtype), acc, nat.ptr(ws),
                                            nbytes, fig, plan, nat.stream_handle(DEV))
    nat.check(rc, "fsb_spmv_csr_checked")
    assert list(fig) == orc_csr_check(p, i)
    ref = _plan.default_spmv_plan(prep._stats, dtype)
    assert plan.algo == ref.algo and plan.flags == ref.flags
    if ref.algo == nat.ALGO_ROWS:
        assert plan.lanes == ref.lanes
    else:
        assert plan.items_per_unit == ref.items_per_unit
    assert torch.equal(y3, y1)


def orc_csr_check(p, i):
    from oracle import oracle as orc

    return orc.csr_check(p.cpu(), i.cpu())


@pytest.mark.parametrize("index_dtype", [torch.int32, torch.int64], ids=["i32", "i64"])
@pytest.mark.parametrize("kind,exc,msg", SPMV_MALFORMED)
def test_spmv_malformed_both_routes(kind, exc, msg, index_dtype):
    """int32 indices take the one-call native route, int64 the prepared
    route; both raise FlagSparse's error."""
    d, i, p, shape = _malformed(kind)
    with pytest.raises(exc, match=msg):
        fs.flagsparse_spmv_csr(d, i.to(index_dtype), p, torch.ones(3, device=DEV), shape)
