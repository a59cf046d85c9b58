"""Selector host logic and the network oracle, on the CPU."""

import math

import numpy as np
import pytest

from flagsparse_public_b200 import tuning
from oracle import mlp as omlp


def _problem(seed, n=7, dims=(5, 6, 4, 3)):
    rng = np.random.default_rng(seed)
    d_in, h1, h2, d_out = dims
    p = rng.normal(0, 0.5, omlp.param_count(*dims))
    X = rng.normal(0, 1, (n, d_in))
    T = rng.normal(0, 1, (n, d_out))
    M = (rng.random((n, d_out)) < 0.8).astype(np.float64)
    return p, X, T, M, 1.0 / max(M.sum(), 1)


def test_oracle_gradient_matches_finite_differences():
    dims = (5, 6, 4, 3)
    p, X, T, M, inv = _problem(0, dims=dims)
    g, L = omlp.backward(X, p, dims, T, M, inv)
    fd = omlp.finite_difference_grad(X, p, dims, T, M, inv)
    assert L == pytest.approx(omlp.loss(X, p, dims, T, M, inv))
    np.testing.assert_allclose(g, fd, rtol=1e-5, atol=1e-7)


def test_oracle_adam_reduces_loss():
    dims = (5, 8, 8, 3)
    p, X, T, M, inv = _problem(1, n=32, dims=dims)
    m1 = np.zeros_like(p)
    m2 = np.zeros_like(p)
    l0 = omlp.loss(X, p, dims, T, M, inv)
    for step in range(1, 201):
        g, _ = omlp.backward(X, p, dims, T, M, inv)
        p, m1, m2 = omlp.adam_step(p, g, m1, m2, 1e-2, 0.9, 0.999, 1e-8, step)
    assert omlp.loss(X, p, dims, T, M, inv) < 0.5 * l0


def test_targets_and_regret():
    times = np.array([[2.0, 1.0, np.inf, 4.0], [3.0, 3.0, 1.5, 100.0]])
    T, M = tuning.targets_from_times(times)
    np.testing.assert_allclose(T[0], [1.0, 0.0, tuning.TARGET_CLIP, 2.0])
    np.testing.assert_array_equal(M[0], [1, 1, 0, 1])
    assert T[1, 3] == tuning.TARGET_CLIP  # log2(100 / 1.5) > clip
    np.testing.assert_allclose(tuning.regret(times, [1, 0]), [1.0, 2.0])


def test_features_from_sums():
    # 4 rows, lengths 1, 3, 0, 4 -> sum 8, squares 26, max 4, one empty row
    f = tuning.features_from_sums(4, 8, 8.0, 26.0, 4, 1.0, 2.0, 32, 4)
    assert f.shape == (tuning.N_FEATURES,)
    assert f[0] == pytest.approx(math.log2(5))
    assert f[2] == pytest.approx(math.log2(9))
    assert f[3] == pytest.approx(math.log2(3))  # mean 2
    assert f[4] == pytest.approx(math.log2(math.sqrt(26 / 4 - 4) + 1))
    assert f[5] == pytest.approx(math.log2(5))
    assert f[8] == pytest.approx(0.25)
    assert f[9] == pytest.approx(0.25)
    assert f[10] == pytest.approx(5.0)
    assert f[11] == 0.0
    # share of nonzeros placed as in aligned dense 16-column blocks
    assert tuning.features_from_sums(4, 8, 8.0, 26.0, 4, 1.0, 2.0, 32, 2, 6.0)[11] == pytest.approx(0.75)


def test_corpus_specs_are_seeded_and_capped():
    a = tuning.corpus_specs(40, 10, seed=3, nnz_cap=1 << 20)
    b = tuning.corpus_specs(40, 10, seed=3, nnz_cap=1 << 20)
    assert a == b and len(a) == 50
    assert {s["family"] for s in a} == set(tuning.FAMILIES)
    assert sum(s["split"] == "test" for s in a) == 10
    for s in a:
        assert 2.0 <= s["mean"] <= 128.0
        assert s["rows"] * s["mean"] <= (1 << 20) or s["rows"] == 10_000


def test_heuristic_choice_is_a_candidate():
    f = tuning.features_from_sums(262144, 262144, 3.1e6, 0.0, 7000, 0.0, 0.0, 64)
    assert tuning.CANDIDATE_NAMES[tuning.heuristic_choice(f)] == "seq256"


def _heldout():
    import os
    from tests.conftest import GOLDEN_DIR
    z = np.load(os.path.join(GOLDEN_DIR, "selector_heldout.npz"), allow_pickle=False)
    assert tuple(str(s) for s in z["names"]) == tuning.CANDIDATE_NAMES
    return z["features"], z["times"].astype(np.float64), z["n_dense"], z["kind"]


@pytest.mark.parametrize("slice_kind,n_samples", [(1, 1600), (2, 160)], ids=["heldout", "above_2e24_nnz"])
def test_shipped_selector_beats_the_heuristic_on_heldout_matrices(slice_kind, n_samples):
    """What the trained network gains over the method without it, on two
    held-out slices (x 4 dense widths): the 400 corpus matrices of at most
    2^24 nonzeros and 40 matrices above that (up to 2e6 rows x 128).  The
    shipped selector's picks cost within 5 % of exhaustive autotuning, the
    default heuristic's clearly more (timings measured on a B200 over 12
    candidates, the tensor-core BSR path among them for the bfloat16
    block-sparse family; committed as a fixture)."""
    F, times, _, kind = _heldout()
    sel = kind == slice_kind
    F, times = F[sel], times[sel]
    w = np.load(tuning.WEIGHTS_PATH, allow_pickle=False)
    dims = tuple(int(v) for v in w["dims"])
    X = (F - w["mu"]) / w["sigma"]
    pred, _ = omlp.forward(X, w["params"].astype(np.float64), dims)
    ok = tuning.selectable(F, times)
    learned = np.argmin(np.where(ok, pred, np.inf), axis=1)
    heur = np.asarray([tuning.heuristic_choice(f) for f in F])
    best = np.where(np.isfinite(times), times, np.inf).min(axis=1).sum()
    rows = np.arange(len(times))
    learned_total = times[rows, learned].sum()
    heur_total = times[rows, heur].sum()
    assert len(times) == n_samples
    assert learned_total / best <= 1.05
    assert heur_total / best > learned_total / best + 0.05
    assert np.median(tuning.regret(times, learned)) == 1.0


def test_bsr_candidate_wins_the_block_family_and_is_picked():
    """On the held-out bfloat16 block-sparse matrices with at least 8 dense
    columns, the tensor-core BSR candidate is the fastest plan on every
    N = 128 sample and on most others; the selector picks it where it is
    fastest, and its picks cost within 1 % of exhaustive autotuning there,
    where the best CSR plan alone would cost about 4 x."""
    F, times, n_dense, kind = _heldout()
    w = np.load(tuning.WEIGHTS_PATH, allow_pickle=False)
    dims = tuple(int(v) for v in w["dims"])
    block = (F[:, 14] <= 0.25) & (n_dense >= 8)
    assert block.sum() >= 200
    Fb, Tb, Nb = F[block], times[block], n_dense[block]
    pred, _ = omlp.forward((Fb - w["mu"]) / w["sigma"], w["params"].astype(np.float64), dims)
    learned = np.argmin(np.where(tuning.selectable(Fb, Tb), pred, np.inf), axis=1)
    best = np.argmin(np.where(np.isfinite(Tb), Tb, np.inf), axis=1)
    bsr_best = best == tuning.BSR_CANDIDATE
    assert bsr_best[Nb == 128].all()
    assert bsr_best.mean() >= 0.75
    assert np.mean(learned[bsr_best] == tuning.BSR_CANDIDATE) >= 0.95
    rows = np.arange(len(Tb))
    assert Tb[rows, learned].sum() / Tb[rows, best].sum() <= 1.01
    assert Tb[:, :tuning.BSR_CANDIDATE].min(axis=1).sum() / Tb[rows, best].sum() > 3.0
    # no other family ever offers it
    other = F[:, 14] > 0.25
    assert not tuning.selectable(F[other], times[other])[:, tuning.BSR_CANDIDATE].any()


def test_selector_fallback_triggers_outside_training_range():
    w = np.load(tuning.WEIGHTS_PATH, allow_pickle=False)
    z_far = np.abs((np.full(tuning.N_FEATURES, 1e3) - w["mu"]) / w["sigma"])
    assert np.any(z_far > 4.0)
