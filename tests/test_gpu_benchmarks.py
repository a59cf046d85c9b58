"""FlagSparse's benchmark entry points for the SpMV / SpMM path
(benchmarks.py:345-507, spmm_csr.py:2226-2573, spmm_csr_opt_alg2.py:862-972):
same arguments and result dictionaries, this package's kernels timed and
checked against the PyTorch reference.  CuPy is absent here, so the cuSPARSE
leg reports FlagSparse's "not available" reason."""

import pytest
import torch

import flagsparse_public_b200 as fs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64, torch.complex64])
@pytest.mark.parametrize("op", ["non", "trans", "conj"])
def test_benchmark_spmv_case(dtype, op):
    r = fs.benchmark_spmv_case(n_rows=3000, n_cols=2000, nnz=40000, value_dtype=dtype, warmup=2, iters=3, op=op)
    assert set(r) == {"parameters", "performance", "verification", "backend_status", "samples"}
    assert r["parameters"]["op"] == op and r["parameters"]["transpose"] == (op != "non")
    assert r["verification"]["triton_match_reference"] is True
    assert r["performance"]["triton_ms"] > 0
    assert r["samples"]["triton"].shape[0] == (2000 if op != "non" else 3000)
    assert r["backend_status"]["cusparse_unavailable_reason"] == "CuPy/cuSPARSE is not available"


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64, torch.float16])
def test_benchmark_spmm_case(dtype):
    r = fs.benchmark_spmm_case(n_rows=2048, n_cols=1024, nnz=30000, n_dense_cols=32, value_dtype=dtype, warmup=2,
                               iters=3)
    v = r["verification"]
    assert v["triton_match_reference"] is True and v["triton_strict_allclose_match"] is True
    assert r["parameters"]["format"] == "csr" and r["backend_status"]["flagsparse_internal_route"] == "csr-alg1"
    assert r["performance"]["triton_ms"] > 0 and r["performance"]["triton_first_call_ms"] > 0
    assert r["samples"]["triton"].shape == (2048, 32)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_benchmark_spmm_opt_and_alg2_cases(dtype):
    r = fs.benchmark_spmm_opt_case(n_rows=2048, n_cols=2048, nnz=40000, n_dense_cols=64, value_dtype=dtype,
                                   warmup=2, iters=3)
    assert r["verification"]["status"] == "PASS" and r["verification"]["base_ok"]
    assert r["performance"]["opt_ms"] > 0 and r["performance"]["pt_ms"] is not None
    r2 = fs.benchmark_spmm_opt_alg2_case(n_rows=2048, n_cols=2048, nnz=40000, n_dense_cols=64, value_dtype=dtype,
                                         warmup=2, iters=3)
    v = r2["verification"]
    assert max(v["base_vs_torch_err"], v["opt_vs_torch_err"], v["opt_alg2_vs_torch_err"]) <= 1.0
    assert v["opt_vs_cusparse_err"] is None
    with pytest.raises(TypeError, match="only supports float32 and float64"):
        fs.benchmark_spmm_opt_case(value_dtype=torch.float16)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_benchmark_sddmm_case(dtype):
    r = fs.benchmark_sddmm_case(n_rows=1500, n_cols=900, nnz=20000, k_dim=64, value_dtype=dtype, warmup=2, iters=3,
                                alpha=1.5, beta=0.5, run_cusparse=True)
    # FlagSparse's own check is allclose in the value type (atol 1e-6, rtol
    # 1e-5 for float32), which two float32 dot products of 64 terms summed in
    # different orders can miss near cancellation: float32 is held to an
    # absolute bound instead (entries are O(10))
    if dtype == torch.float64:
        assert r["verification"]["triton_match_pytorch"] is True
    else:
        assert r["verification"]["triton_max_abs_error"] <= 1e-4
    assert r["performance"]["triton_ms"] > 0 and r["performance"]["pytorch_ms"] > 0
    assert r["backend_status"]["cusparse_unavailable_reason"] == "CuPy is not available"
    assert r["samples"]["triton"].shape == (20000,)
    with pytest.raises(TypeError):
        fs.benchmark_sddmm_case(value_dtype=torch.float16)
