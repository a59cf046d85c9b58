"""Selector device side against the CPU oracle: structure features, the
network's forward / backward / Adam kernels, the autotuner and the shipped
learned selector."""

import os

import numpy as np
import pytest
import torch

from flagsparse_public_b200 import _native as nat
from flagsparse_public_b200 import _plan, synthetic, tuning
from oracle import mlp as omlp

DEV = "cuda"
pytestmark = pytest.mark.gpu


def _host_sums(indices, indptr, n_rows, n_cols):
    lens = (indptr[1:] - indptr[:-1]).to(torch.float64)
    row = torch.repeat_interleave(torch.arange(n_rows, dtype=torch.float64), (indptr[1:] - indptr[:-1]))
    band = ((indices.to(torch.float64) - row * (n_cols / n_rows)).abs() / n_cols).sum()
    starts = torch.repeat_interleave(indptr[:-1].long(), (indptr[1:] - indptr[:-1]))
    pos = torch.arange(indices.numel()) - starts
    aligned = int(((indices.long() & 15) == (pos & 15)).sum())
    return lens.sum().item(), (lens * lens).sum().item(), int(lens.max().item()), int((lens == 0).sum().item()), \
        band.item(), aligned


@pytest.mark.parametrize("idx_dtype,ptr_dtype", [(torch.int32, torch.int64), (torch.int64, torch.int32)])
def test_features_kernel_matches_host_sums(idx_dtype, ptr_dtype):
    data, indices, indptr, (n_rows, n_cols) = synthetic.zipf_powerlaw(5000, 3000, mean=7.0, cap=900, seed=4,
                                                                       device="cpu")
    indices, indptr = indices.to(idx_dtype), indptr.to(ptr_dtype)
    out = torch.zeros(6, dtype=torch.float64, device=DEV)
    ptr_d, idx_d = indptr.to(DEV), indices.to(DEV)  # kept alive across the launch
    rc = nat.library().fsb_csr_features(nat.ptr(ptr_d), nat.dtype_code(ptr_dtype), nat.ptr(idx_d),
                                        nat.dtype_code(idx_dtype), n_rows, n_cols, nat.ptr(out),
                                        nat.stream_handle(torch.device(DEV)))
    torch.cuda.synchronize()
    nat.check(rc, "fsb_csr_features")
    s, sq, mx, empty, band, aligned = _host_sums(indices.long(), indptr.long(), n_rows, n_cols)
    got = out.cpu()
    assert got[0].item() == s and got[1].item() == sq and got[3].item() == empty
    assert got[5].item() == aligned
    assert int(got.view(torch.int64)[2].item()) == mx
    assert got[4].item() == pytest.approx(band, rel=1e-12)


def test_features_kernel_keeps_device_tensors_alive():
    data, indices, indptr, (n_rows, n_cols) = synthetic.poisson_uniform(2000, 2000, mean=5.0, seed=1, device=DEV)
    f = tuning.raw_features(indices, indptr, n_rows, n_cols, 32)
    assert f.shape == (tuning.N_FEATURES,) and np.all(np.isfinite(f))
    assert f[10] == pytest.approx(5.0)


DIMS = (16, 64, 64, len(tuning.SPMM_CANDIDATES))


def _rand_problem(seed, n):
    rng = np.random.default_rng(seed)
    p = rng.normal(0, 0.2, omlp.param_count(*DIMS)).astype(np.float32)
    X = rng.normal(0, 1, (n, DIMS[0])).astype(np.float32)
    T = rng.normal(0, 1, (n, DIMS[3])).astype(np.float32)
    M = (rng.random((n, DIMS[3])) < 0.85).astype(np.float32)
    return p, X, T, M


def _to(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


@pytest.mark.parametrize("n", [1, 37, 1000])
def test_mlp_forward_and_backward_match_oracle(n):
    p, X, T, M = _rand_problem(n, n)
    mlp = tuning.Mlp(_to(p), *DIMS)
    cache = torch.empty((n, mlp.cache_width()), dtype=torch.float32, device=DEV)
    Y = mlp.forward(_to(X), cache).cpu().numpy()
    Yo, _ = omlp.forward(X, p, DIMS)
    np.testing.assert_allclose(Y, Yo, rtol=1e-4, atol=1e-5)
    inv = 1.0 / M.sum()
    deltas = torch.empty_like(cache)
    lt = torch.empty(n, dtype=torch.float32, device=DEV)
    grad = torch.empty(p.size, dtype=torch.float32, device=DEV)
    mlp.backward(_to(X), cache, _to(T), _to(M), inv, deltas, lt, grad)
    go, Lo = omlp.backward(X, p, DIMS, T, M, inv)
    assert float(lt.sum().item()) * inv == pytest.approx(Lo, rel=1e-4)
    g = grad.cpu().numpy()
    np.testing.assert_allclose(g, go, rtol=2e-3, atol=1e-5 * np.abs(go).max())


def test_adam_training_follows_oracle_trajectory():
    n = 64
    p, X, T, M = _rand_problem(7, n)
    Xd, Td, Md = _to(X), _to(T), _to(M)
    mlp = tuning.Mlp(_to(p), *DIMS)
    po = p.astype(np.float64)
    m1o, m2o = np.zeros_like(po), np.zeros_like(po)
    inv = 1.0 / M.sum()
    cache = torch.empty((n, mlp.cache_width()), dtype=torch.float32, device=DEV)
    deltas, lt = torch.empty_like(cache), torch.empty(n, dtype=torch.float32, device=DEV)
    grad = torch.empty(p.size, dtype=torch.float32, device=DEV)
    m1 = torch.zeros(p.size, dtype=torch.float32, device=DEV)
    m2 = torch.zeros(p.size, dtype=torch.float32, device=DEV)
    import ctypes
    for step in range(1, 21):
        mlp.forward(Xd, cache)
        mlp.backward(Xd, cache, Td, Md, inv, deltas, lt, grad)
        rc = nat.library().fsb_adam_step(nat.ptr(mlp.params), nat.ptr(grad), nat.ptr(m1), nat.ptr(m2), p.size,
                                         ctypes.c_float(1e-3), ctypes.c_float(0.9), ctypes.c_float(0.999),
                                         ctypes.c_float(1e-8), step, ctypes.c_float(1e-4),
                                         nat.stream_handle(torch.device(DEV)))
        nat.check(rc, "fsb_adam_step")
        go, _ = omlp.backward(X, po, DIMS, T, M, inv)
        po, m1o, m2o = omlp.adam_step(po, go, m1o, m2o, 1e-3, 0.9, 0.999, 1e-8, step, 1e-4)
    got = mlp.params.cpu().numpy()
    # Adam moves every parameter by about lr per step whatever the gradient's
    # size, so a parameter whose gradient sits near zero can step either way
    # on float32 rounding: 20 steps of lr 1e-3 bound any difference by 2e-2.
    # Nearly all parameters follow the float64 path to 2e-4, none drifts far.
    diff = np.abs(got - po)
    assert diff.max() < 2e-3
    assert np.mean(diff < 2e-4) > 0.999
    assert omlp.loss(X, got, DIMS, T, M, inv) < omlp.loss(X, p, DIMS, T, M, inv)


def test_train_mlp_is_deterministic_and_learns():
    n = 256
    _, X, T, M = _rand_problem(3, n)
    a, la = tuning.train_mlp(_to(X), _to(T), _to(M), steps=150, seed=5)
    b, lb = tuning.train_mlp(_to(X), _to(T), _to(M), steps=150, seed=5)
    assert torch.equal(a.params, b.params)
    assert la[-1] < 0.5 * la[0]


def test_autotuner_picks_the_fastest_and_caches():
    data, indices, indptr, (n_rows, n_cols) = synthetic.zipf_powerlaw(20000, 20000, mean=9.0, cap=3000, seed=2,
                                                                       device=DEV)
    B = synthetic.dense_operand(n_cols, 32, seed=3, device=DEV)
    C = torch.empty((n_rows, 32), device=DEV)
    tuner = tuning.Autotuner(reps=2)
    plan, times = tuner.tune(data, indices, indptr, n_rows, n_cols, B, C, nat.ACC_NATIVE)
    best = min(times, key=times.get)
    assert tuning.SPMM_CANDIDATES[tuning.CANDIDATE_NAMES.index(best)][1]().key() == plan.key()
    plan2, times2 = tuner.tune(data, indices, indptr, n_rows, n_cols, B, C, nat.ACC_NATIVE)
    assert times2 is times and plan2.key() == plan.key()
    _plan.run_spmm(data, indices, indptr, n_rows, n_cols, B, C, nat.ACC_NATIVE, plan)
    ref = torch.sparse_csr_tensor(indptr, indices.long(), data.double(), size=(n_rows, n_cols)) @ B.double()
    assert float((C.double() - ref).abs().max() / ref.abs().max()) < 1e-5


@pytest.mark.skipif(not os.path.exists(tuning.WEIGHTS_PATH), reason="selector weights not trained yet")
def test_learned_selector_runs_its_pick():
    sel = tuning.LearnedSelector()
    data, indices, indptr, (n_rows, n_cols) = synthetic.poisson_uniform(50000, 50000, mean=20.0, seed=9, device=DEV)
    for n_dense in (1, 32):
        B = synthetic.dense_operand(n_cols, n_dense, seed=1, device=DEV)
        C = torch.empty((n_rows, n_dense), device=DEV)
        plan = sel.select(data, indices, indptr, n_rows, n_cols, B, C, nat.ACC_NATIVE)
        assert sel.last[0] in ("learned", "autotune")
        _plan.run_spmm(data, indices, indptr, n_rows, n_cols, B, C, nat.ACC_NATIVE, plan)
        ref = torch.sparse_csr_tensor(indptr, indices.long(), data.double(), size=(n_rows, n_cols)) @ B.double()
        assert float((C.double() - ref).abs().max() / ref.abs().max()) < 1e-5


def test_bsr_candidate_runs_through_run_spmm():
    """The selector's tensor-core BSR candidate (a BsrPlan) through the plan
    interface: bfloat16 block-sparse matrix against FP64 of the same inputs;
    refused (ValueError) for float32 values and for scattered matrices whose
    16 x 16 blocks would be mostly zeros."""
    data, indices, indptr, (n_rows, n_cols) = synthetic.block_sparse(300, 3, seed=5, dtype=torch.bfloat16,
                                                                     device=DEV)
    B = synthetic.dense_operand(n_cols, 32, seed=6, dtype=torch.bfloat16, device=DEV)
    C = torch.full((n_rows, 32), float("nan"), device=DEV)
    plan = tuning.SPMM_CANDIDATES[tuning.BSR_CANDIDATE][1]()
    _plan.run_spmm(data, indices, indptr, n_rows, n_cols, B, C, nat.ACC_NATIVE, plan)
    A = torch.sparse_csr_tensor(indptr.cpu(), indices.long().cpu(), data.double().cpu(), size=(n_rows, n_cols))
    ref = A @ B.double().cpu()
    mag = A.abs() @ B.double().abs().cpu()
    assert float(((C.cpu().double() - ref).abs() / mag.clamp(min=1e-300)).max()) <= 1e-5
    f = tuning.raw_features(indices, indptr, n_rows, n_cols, 32, 2)
    assert f[11] == 1.0  # every nonzero sits as in an aligned dense 16-column block
    with pytest.raises(ValueError):
        _plan.run_spmm(data.float(), indices, indptr, n_rows, n_cols, B.float(), C, nat.ACC_NATIVE,
                       _plan.BsrPlan())
    sd, si, sp, (sr, sc) = synthetic.poisson_uniform(4000, 4000, mean=8.0, seed=7, dtype=torch.bfloat16, device=DEV)
    Bs = synthetic.dense_operand(sc, 32, seed=8, dtype=torch.bfloat16, device=DEV)
    with pytest.raises(ValueError, match="fill-in"):
        _plan.run_spmm(sd, si, sp, sr, sc, Bs, torch.empty((sr, 32), device=DEV), nat.ACC_NATIVE, _plan.BsrPlan())
