"""Plan selection for the CSR SpMM kernels: candidates, exhaustive autotuning
and the learned selector.

FlagSparse chooses its SpMM launch parameters by fixed row-length buckets
(``_build_spmm_opt_buckets``, spmm_csr.py:444-477, block sizes from
``_select_spmm_opt_block_n``, :405-414) and, in ALG2, by device-property
heuristics (spmm_csr_opt_alg2.py:175-304).  Here a plan is one of a fixed
list of candidates (``SPMM_CANDIDATES``): warp-per-row and vector-per-row
row groups, the merge-path kernel, and the batched merge-path kernel at four
unit sizes and two column tiles.

* ``Autotuner`` times every candidate on the matrix and dense width at hand
  (CUDA events) and caches the winner -- exhaustive autotuning, the yardstick of
  the selector's regret.
* ``LearnedSelector`` predicts each candidate's time relative to the best
  (log2 ratio) with a small MLP over matrix features (rows, columns, nonzeros,
  row-length mean / spread / maximum, distance from the diagonal, empty rows,
  dense width N), computed on the device (``fsb_csr_features``), and picks
  the lowest prediction.  It falls back to the autotuner when the features
  lie outside the training range (a standardised feature beyond z_limit).
  Near ties are not a reason to fall back: two plans predicted equal cost
  about the same whichever is run (a positive ``margin`` makes the selector
  fall back when its two best predictions differ by less than it).
* ``train_mlp`` trains the network on the GPU with the project's own kernels
  (``fsb_mlp_forward`` / ``fsb_mlp_backward`` / ``fsb_adam_step``), full
  batch, deterministic.
* ``main`` (``python -m flagsparse_public_b200.tuning``) builds the training
  corpus from seeds (five families), times every candidate on it, trains,
  reports regret on the held-out matrices against exhaustive autotuning and
  writes the shipped weights (``selector_weights.npz``).
"""

import argparse
import ctypes
import json
import math
import os
import time

import numpy as np
import torch

from . import _native as nat
from . import _plan
from . import synthetic

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS_PATH = os.path.join(HERE, "selector_weights.npz")

N_FEATURES = 16
HIDDEN = 64
N_VALUES = (1, 8, 32, 128)  # dense widths of the training corpus
TARGET_CLIP = 4.0  # log2 slowdowns above 16x count as 16x in the loss


def _rows(lanes, n_tile=0):
    return lambda: _plan.KernelPlan(nat.ALGO_ROWS, lanes=lanes, n_tile=n_tile)


def _merge(items, snap):
    return lambda: _plan.KernelPlan(nat.ALGO_MERGE, items_per_unit=items, snap=snap)


def _seq(items, n_tile=0):
    return lambda: _plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=items, n_tile=n_tile, snap=_plan.SPMM_SNAP_DEFAULT)


# (name, plan factory); the order is the network's output order.
SPMM_CANDIDATES = (
    ("vector_rows", _rows(1)),
    ("rows8", _rows(8)),
    ("warp_rows", _rows(32)),
    ("warp_rows_t32", _rows(32, 32)),
    ("merge128", _merge(128, 64)),
    ("seq128", _seq(128)),
    ("seq256", _seq(256)),
    ("seq512", _seq(512)),
    ("seq1024", _seq(1024)),
    ("seq256_t32", _seq(256, 32)),
    ("seq1024_t32", _seq(1024, 32)),
    ("bsr16_tc", _plan.BsrPlan),  # half-precision values only; 16 x 16 blocks on the tensor cores
)
BSR_CANDIDATE = len(SPMM_CANDIDATES) - 1
# The BSR candidate is offered to the network only for matrices whose
# nonzeros mostly sit as in aligned dense 16-column blocks (feature 11).
BSR_ALIGNED_MIN = 0.5
CANDIDATE_NAMES = tuple(n for n, _ in SPMM_CANDIDATES)


# ---------------------------------------------------------------- features
def raw_features(indices, indptr, n_rows, n_cols, n_dense, value_bytes=4):
    """Feature vector (float64, N_FEATURES) of a CSR matrix and dense width,
    the structure sums computed on the device by fsb_csr_features."""
    n_rows, n_cols = int(n_rows), int(n_cols)
    out = torch.zeros(6, dtype=torch.float64, device=indptr.device)
    if n_rows > 0:
        lib = nat.library()
        rc = lib.fsb_csr_features(nat.ptr(indptr), nat.dtype_code(indptr.dtype), nat.ptr(indices),
                                  nat.dtype_code(indices.dtype), n_rows, n_cols, nat.ptr(out),
                                  nat.stream_handle(indptr.device))
        nat.check(rc, "fsb_csr_features")
    host = out.cpu()
    s = host.numpy()
    max_len = int(host.view(torch.int64)[2].item())
    return features_from_sums(n_rows, n_cols, float(s[0]), float(s[1]), max_len, float(s[3]), float(s[4]),
                              n_dense, value_bytes, float(s[5]))


def features_from_sums(n_rows, n_cols, sum_len, sum_sq, max_len, empty, band_sum, n_dense, value_bytes=4,
                       aligned=0.0):
    nnz = sum_len
    mean = nnz / max(n_rows, 1)
    var = max(sum_sq / max(n_rows, 1) - mean * mean, 0.0)
    std = math.sqrt(var)
    band = band_sum / max(nnz, 1.0)
    f = np.zeros(N_FEATURES, dtype=np.float64)
    f[0] = math.log2(n_rows + 1)
    f[1] = math.log2(n_cols + 1)
    f[2] = math.log2(nnz + 1)
    f[3] = math.log2(mean + 1)
    f[4] = math.log2(std + 1)
    f[5] = math.log2(max_len + 1)
    f[6] = math.log2((max_len + 1) / (mean + 1))
    f[7] = math.log2(std / (mean + 1e-9) + 1)  # coefficient of variation
    f[8] = band
    f[9] = empty / max(n_rows, 1)
    f[10] = math.log2(n_dense)
    f[11] = aligned / max(nnz, 1.0)  # share of nonzeros placed as in aligned dense 16-column blocks
    f[12] = math.log2(n_dense * value_bytes * n_cols + 1)  # dense operand bytes
    f[13] = math.log2(nnz * n_dense + 1)  # multiply-adds
    f[14] = value_bytes / 8.0
    f[15] = math.log2(n_cols / max(n_rows, 1))
    return f


# --------------------------------------------------------------- autotuner
def _time_ms(fn, reps):
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def time_candidates(data, indices, indptr, n_rows, n_cols, B, C, acc_mode, candidates=SPMM_CANDIDATES, reps=3,
                    slow_ms=5.0):
    """Milliseconds per call of each candidate plan (inf where a plan cannot
    run these operands).  One untimed call first (partition, workspace, first
    touch), then ``reps`` timed calls (one when a call takes > slow_ms)."""
    times = []
    for _name, make in candidates:
        plan = make()
        run = lambda: _plan.run_spmm(data, indices, indptr, n_rows, n_cols, B, C, acc_mode, plan)  # noqa: E731
        try:
            _time_ms(run, 1)  # untimed: one-time costs
            t1 = _time_ms(run, 1)
            times.append(t1 if t1 > slow_ms or reps <= 1 else _time_ms(run, reps))
        except (RuntimeError, ValueError):
            times.append(float("inf"))
    return times


class Autotuner:
    """Exhaustive autotuning over SPMM_CANDIDATES, cached per matrix and
    operand shape."""

    def __init__(self, reps=3):
        self.reps = int(reps)
        self.cache = {}

    @staticmethod
    def key(data, indices, indptr, n_rows, n_cols, n_dense, acc_mode):
        return (indptr.data_ptr(), indices.data_ptr(), data.data_ptr(), int(data.numel()), int(n_rows), int(n_cols),
                int(n_dense), str(data.dtype), int(acc_mode))

    def tune(self, data, indices, indptr, n_rows, n_cols, B, C, acc_mode):
        """(best plan, {name: ms}) for these operands."""
        k = self.key(data, indices, indptr, n_rows, n_cols, B.shape[1], acc_mode)
        hit = self.cache.get(k)
        if hit is None:
            times = time_candidates(data, indices, indptr, n_rows, n_cols, B, C, acc_mode, reps=self.reps)
            best = int(np.argmin(times))
            hit = (best, dict(zip(CANDIDATE_NAMES, times)))
            self.cache[k] = hit
        return SPMM_CANDIDATES[hit[0]][1](), hit[1]


# --------------------------------------------------------------------- MLP
class Mlp:
    """Parameters of the selector network on a device."""

    def __init__(self, params, d_in=N_FEATURES, h1=HIDDEN, h2=HIDDEN, d_out=len(SPMM_CANDIDATES)):
        self.dims = (int(d_in), int(h1), int(h2), int(d_out))
        n = nat.library().fsb_mlp_param_count(*self.dims)
        nat.check(n if n < 0 else 0, "fsb_mlp_param_count")
        if params.numel() != n or params.dtype != torch.float32 or not params.is_cuda:
            raise ValueError(f"expected {n} float32 CUDA parameters")
        self.params = params.contiguous()

    @staticmethod
    def init(seed, device, d_in=N_FEATURES, h1=HIDDEN, h2=HIDDEN, d_out=len(SPMM_CANDIDATES)):
        """He-uniform weights, zero biases (seeded)."""
        g = torch.Generator(device="cpu")
        g.manual_seed(int(seed))
        parts = []
        for fan_in, fan_out in ((d_in, h1), (h1, h2), (h2, d_out)):
            bound = math.sqrt(6.0 / fan_in)
            parts.append((torch.rand((fan_in, fan_out), generator=g) * 2 - 1) * bound)
            parts.append(torch.zeros(fan_out))
        p = torch.cat([t.reshape(-1) for t in parts]).to(torch.float32).to(device)
        return Mlp(p, d_in, h1, h2, d_out)

    def cache_width(self):
        return self.dims[1] + self.dims[2] + self.dims[3]

    def forward(self, X, cache=None):
        X = X.contiguous()
        n = X.shape[0]
        Y = torch.empty((n, self.dims[3]), dtype=torch.float32, device=X.device)
        rc = nat.library().fsb_mlp_forward(nat.ptr(X), n, *self.dims, nat.ptr(self.params), nat.ptr(Y),
                                           nat.ptr(cache) if cache is not None else None,
                                           nat.stream_handle(X.device))
        nat.check(rc, "fsb_mlp_forward")
        return Y

    def backward(self, X, cache, T, M, inv_terms, deltas, loss_terms, grad):
        rc = nat.library().fsb_mlp_backward(nat.ptr(X), X.shape[0], *self.dims, nat.ptr(self.params), nat.ptr(cache),
                                            nat.ptr(T), nat.ptr(M), ctypes.c_float(inv_terms), nat.ptr(deltas),
                                            nat.ptr(loss_terms), nat.ptr(grad), nat.stream_handle(X.device))
        nat.check(rc, "fsb_mlp_backward")


def train_mlp(X, T, M, steps=3000, lr=3e-3, weight_decay=1e-4, seed=0, log_every=0):
    """Full-batch Adam on the GPU with the project's kernels.  X (n, d) inputs,
    T (n, K) targets, M (n, K) 0/1 mask, all float32 CUDA.  Returns (Mlp,
    per-step losses)."""
    X, T, M = X.contiguous(), T.contiguous(), M.contiguous()
    dev = X.device
    mlp = Mlp.init(seed, dev, d_in=X.shape[1], d_out=T.shape[1])
    n = X.shape[0]
    np_ = mlp.params.numel()
    cache = torch.empty((n, mlp.cache_width()), dtype=torch.float32, device=dev)
    deltas = torch.empty_like(cache)
    loss_terms = torch.empty(n, dtype=torch.float32, device=dev)
    grad = torch.empty(np_, dtype=torch.float32, device=dev)
    m1 = torch.zeros(np_, dtype=torch.float32, device=dev)
    m2 = torch.zeros(np_, dtype=torch.float32, device=dev)
    inv_terms = 1.0 / max(float(M.sum().item()), 1.0)
    lib = nat.library()
    stream = nat.stream_handle(dev)
    losses = torch.empty(steps, dtype=torch.float32, device=dev)
    for step in range(1, steps + 1):
        mlp.forward(X, cache)
        mlp.backward(X, cache, T, M, inv_terms, deltas, loss_terms, grad)
        losses[step - 1] = loss_terms.sum() * inv_terms
        rc = lib.fsb_adam_step(nat.ptr(mlp.params), nat.ptr(grad), nat.ptr(m1), nat.ptr(m2), np_,
                               ctypes.c_float(lr), ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8),
                               step, ctypes.c_float(weight_decay), stream)
        nat.check(rc, "fsb_adam_step")
        if log_every and step % log_every == 0:
            print(f"step {step}: loss {float(losses[step - 1].item()):.5f}", flush=True)
    return mlp, losses.cpu().numpy()


def targets_from_times(times):
    """(log2(t / t_best) clipped, 0/1 mask of runnable candidates) per row."""
    t = np.asarray(times, dtype=np.float64)
    ok = np.isfinite(t) & (t > 0)
    best = np.where(ok, t, np.inf).min(axis=1, keepdims=True)
    rel = np.where(ok, np.log2(np.where(ok, t, 1.0) / best), TARGET_CLIP)
    return np.minimum(rel, TARGET_CLIP).astype(np.float32), ok.astype(np.float32)


# ---------------------------------------------------------------- selector
class LearnedSelector:
    """Selector network with its feature standardisation; falls back to the
    autotuner outside the training range or on a near tie."""

    def __init__(self, path=WEIGHTS_PATH, device="cuda", margin=0.0, z_limit=4.0, autotuner=None):
        z = np.load(path, allow_pickle=False)
        names = tuple(str(s) for s in z["names"])
        if names != CANDIDATE_NAMES:
            raise ValueError("selector weights were trained for another candidate list")
        self.mu = z["mu"].astype(np.float64)
        self.sigma = z["sigma"].astype(np.float64)
        self.lo = z["lo"].astype(np.float64)
        self.hi = z["hi"].astype(np.float64)
        dims = tuple(int(v) for v in z["dims"])
        self.mlp = Mlp(torch.from_numpy(z["params"].astype(np.float32)).to(device), *dims)
        self.margin = float(margin)
        self.z_limit = float(z_limit)
        self.autotuner = autotuner or Autotuner()
        self.last = None

    def standardize(self, f):
        return ((np.asarray(f, dtype=np.float64) - self.mu) / self.sigma).astype(np.float32)

    def predict(self, features):
        X = torch.from_numpy(np.atleast_2d(self.standardize(features))).to(self.mlp.params.device)
        return self.mlp.forward(X).cpu().numpy()

    def choose(self, f, feasible=None):
        """(candidate index, confident?) for one raw feature vector; only
        candidates marked feasible (all by default) can be picked."""
        pred = self.predict(f)[0]
        if feasible is not None:
            pred = np.where(np.asarray(feasible, dtype=bool), pred, np.inf)
        order = np.argsort(pred)
        z = (np.asarray(f) - self.mu) / self.sigma
        in_range = bool(np.all(np.abs(z) <= self.z_limit))
        confident = in_range and (pred[order[1]] - pred[order[0]] >= self.margin)
        return int(order[0]), confident

    def select(self, data, indices, indptr, n_rows, n_cols, B, C, acc_mode):
        """Plan for these operands: the network's pick, or the autotuner's."""
        f = raw_features(indices, indptr, n_rows, n_cols, B.shape[1], data.element_size())
        feasible = np.ones(len(SPMM_CANDIDATES), dtype=bool)
        feasible[BSR_CANDIDATE] = f[11] >= BSR_ALIGNED_MIN and _plan.BsrPlan.supported(data, B, C, acc_mode)
        k, confident = self.choose(f, feasible)
        if confident and k == BSR_CANDIDATE:
            plan = _plan.BsrPlan()
            try:
                plan.prepared(data, indices, indptr, n_rows, n_cols)  # fill-in check, conversion cached
            except ValueError:
                feasible[BSR_CANDIDATE] = False
                k, confident = self.choose(f, feasible)
            else:
                self.last = ("learned", CANDIDATE_NAMES[k])
                return plan
        if confident:
            self.last = ("learned", CANDIDATE_NAMES[k])
            return SPMM_CANDIDATES[k][1]()
        plan, _ = self.autotuner.tune(data, indices, indptr, n_rows, n_cols, B, C, acc_mode)
        self.last = ("autotune", plan.describe())
        return plan


# ----------------------------------------------------------------- corpus
FAMILIES = ("poisson", "zipf", "banded", "block16", "rect2")


def corpus_specs(n_train=2000, n_test=400, seed=0, min_rows=10_000, max_rows=2_000_000, min_mean=2.0,
                 max_mean=128.0, nnz_cap=1 << 24, n_large=0):
    """Seeded matrix specs (family, rows, mean, seed, split), families in
    rotation; rows and mean log-uniform; rows shrunk where rows x mean would
    exceed nnz_cap.  ``n_large`` more held-out specs (split "large") draw
    rows and mean from the same ranges until rows x mean exceeds nnz_cap:
    the sizes above the cap, up to 2e6 rows x 128 nonzeros."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_train + n_test):
        fam = FAMILIES[i % len(FAMILIES)]
        rows = int(round(math.exp(rng.uniform(math.log(min_rows), math.log(max_rows)))))
        mean = float(math.exp(rng.uniform(math.log(min_mean), math.log(max_mean))))
        if rows * mean > nnz_cap:
            rows = max(min_rows, int(nnz_cap / mean))
        specs.append({"family": fam, "rows": rows, "mean": mean, "seed": int(rng.integers(1 << 30)),
                      "split": "train" if i < n_train else "test"})
    big = np.random.default_rng(seed + 1)
    for i in range(n_large):
        while True:
            rows = int(round(math.exp(big.uniform(math.log(min_rows), math.log(max_rows)))))
            mean = float(math.exp(big.uniform(math.log(min_mean), math.log(max_mean))))
            if rows * mean > nnz_cap:
                break
        specs.append({"family": FAMILIES[i % len(FAMILIES)], "rows": rows, "mean": mean,
                      "seed": int(big.integers(1 << 30)), "split": "large"})
    return specs


def value_dtype(spec):
    """Value (and dense operand) type of a corpus matrix: the block-sparse
    family is bfloat16 (the tensor-core BSR candidate's type), the others
    float32."""
    return torch.bfloat16 if spec["family"] == "block16" else torch.float32


def build_matrix(spec, device="cuda", dtype=torch.float32):
    fam, rows, mean, seed = spec["family"], spec["rows"], spec["mean"], spec["seed"]
    if fam == "poisson":
        return synthetic.poisson_uniform(rows, rows, mean=mean, seed=seed, dtype=dtype, device=device)
    if fam == "zipf":
        # row cap well below n_cols keeps distinct-column draws short
        return synthetic.zipf_powerlaw(rows, rows, alpha=1.8, mean=mean, cap=min(20000, max(8, rows // 8)),
                                       seed=seed, dtype=dtype, device=device)
    if fam == "banded":
        band = max(2, int(round(mean)))
        return synthetic.banded_plus_random(rows, band=band, off_band=0, long_rate=0.0, seed=seed, dtype=dtype,
                                            device=device)
    if fam == "block16":
        k = max(1, int(round(mean / 16)))
        return synthetic.block_sparse(max(1, rows // 16), blocks_per_row=k, block=16, seed=seed, dtype=dtype,
                                      device=device)
    if fam == "rect2":
        return synthetic.rectangular(rows, mean=mean, ratio=2, seed=seed, dtype=dtype, device=device)
    raise ValueError(fam)


def collect(specs, device="cuda", n_values=N_VALUES, log=None):
    """Features and per-candidate times (ms, float32 accumulation and result;
    values and B in value_dtype(spec)) for every (matrix, N); returns dict of
    numpy arrays."""
    feats, times, mat, nval = [], [], [], []
    t_start = time.time()
    for i, spec in enumerate(specs):
        vdt = value_dtype(spec)
        data, indices, indptr, (n_rows, n_cols) = build_matrix(spec, device, dtype=vdt)
        for n_dense in n_values:
            B = synthetic.dense_operand(n_cols, n_dense, seed=spec["seed"] + n_dense, dtype=vdt, device=device)
            C = torch.empty((n_rows, n_dense), dtype=torch.float32, device=device)
            feats.append(raw_features(indices, indptr, n_rows, n_cols, n_dense, data.element_size()))
            times.append(time_candidates(data, indices, indptr, n_rows, n_cols, B, C, nat.ACC_NATIVE))
            mat.append(i)
            nval.append(n_dense)
            del B, C
        del data, indices, indptr
        if log and (i + 1) % 50 == 0:
            log(f"{i + 1}/{len(specs)} matrices, {time.time() - t_start:.0f} s")
    return {"features": np.asarray(feats, dtype=np.float64), "times": np.asarray(times, dtype=np.float64),
            "matrix": np.asarray(mat, dtype=np.int64), "n_dense": np.asarray(nval, dtype=np.int64)}


def selectable(features, times):
    """0/1 per (sample, candidate): the candidate ran (finite time) and the
    selector may offer it (the BSR candidate only for half-precision values
    placed mostly as aligned 16-column blocks), as LearnedSelector.select
    decides from the same features."""
    F = np.atleast_2d(np.asarray(features, dtype=np.float64))
    ok = np.isfinite(np.asarray(times, dtype=np.float64))
    ok[:, BSR_CANDIDATE] &= (F[:, 11] >= BSR_ALIGNED_MIN) & (F[:, 14] <= 0.25)
    return ok


def heuristic_choice(features):
    """Candidate index the default heuristic (no selector) would run: the
    batched merge-path kernel with the unit size of seq_items_per_unit."""
    n_rows = 2 ** features[0] - 1
    nnz = 2 ** features[2] - 1
    st = _plan.MatrixStats(int(n_rows), 0, int(nnz), 0, nnz / max(n_rows, 1), 0.0, 0)
    items = _plan.seq_items_per_unit(st)
    return CANDIDATE_NAMES.index(f"seq{items}")


def regret(times, choice):
    """Per-sample time of the chosen candidate over the best (>= 1)."""
    t = np.asarray(times, dtype=np.float64)
    best = np.where(np.isfinite(t), t, np.inf).min(axis=1)
    chosen = t[np.arange(len(t)), np.asarray(choice)]
    return chosen / best


def fit_standardisation(F):
    mu = F.mean(0)
    sigma = F.std(0)
    sigma = np.where(sigma > 1e-9, sigma, 1.0)
    return mu, sigma


def save_weights(path, mlp, mu, sigma, lo, hi, meta):
    np.savez(path, params=mlp.params.cpu().numpy(), dims=np.asarray(mlp.dims, dtype=np.int64), mu=mu, sigma=sigma,
             lo=lo, hi=hi, names=np.asarray(CANDIDATE_NAMES), meta=np.asarray(json.dumps(meta)))


def main(argv=None):
    ap = argparse.ArgumentParser(description="time the corpus, train the selector, report regret")
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--test", type=int, default=400)
    ap.add_argument("--nnz-cap", type=int, default=1 << 24)
    ap.add_argument("--large", type=int, default=0, help="held-out matrices above the nnz cap")
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--dataset", default=None, help="reuse a timing dataset (.npz) instead of timing")
    ap.add_argument("--save-dataset", default=None)
    ap.add_argument("--weights", default=WEIGHTS_PATH)
    ap.add_argument("--report", default=None)
    args = ap.parse_args(argv)
    dev = torch.device("cuda")
    if args.dataset:
        z = np.load(args.dataset, allow_pickle=False)
        data = {k: z[k] for k in ("features", "times", "matrix", "n_dense", "split", "kind")}
    else:
        specs = corpus_specs(args.train, args.test, nnz_cap=args.nnz_cap, n_large=args.large)
        data = collect(specs, dev, log=lambda s: print(s, flush=True))
        kinds = ("train", "test", "large")
        data["kind"] = np.asarray([kinds.index(specs[m]["split"]) for m in data["matrix"]], dtype=np.int8)
        data["split"] = data["kind"] == 0
        if args.save_dataset:
            np.savez_compressed(args.save_dataset, **data, names=np.asarray(CANDIDATE_NAMES))
    F, Tm, is_train = data["features"], data["times"], data["split"].astype(bool)
    kind = data["kind"]
    mu, sigma = fit_standardisation(F[is_train])
    T, M = targets_from_times(Tm)
    X = ((F - mu) / sigma).astype(np.float32)
    to = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    t0 = time.time()
    mlp, losses = train_mlp(to(X[is_train]), to(T[is_train]), to(M[is_train]), steps=args.steps)
    train_s = time.time() - t0
    report = {"samples_train": int(is_train.sum()), "train_seconds": train_s, "final_loss": float(losses[-1])}
    for name, sel in (("test", kind == 1), ("large", kind == 2)):
        if not sel.any():
            continue
        pred = mlp.forward(to(X[sel])).cpu().numpy()
        learned = np.argmin(np.where(selectable(F[sel], Tm[sel]), pred, np.inf), axis=1)
        heur = np.asarray([heuristic_choice(f) for f in F[sel]])
        r_learned = regret(Tm[sel], learned)
        r_heur = regret(Tm[sel], heur)
        total = lambda c: float(np.sum(Tm[sel][np.arange(len(c)), c]))  # noqa: E731
        best_total = float(np.sum(np.where(np.isfinite(Tm[sel]), Tm[sel], np.inf).min(axis=1)))
        report[name] = {
            "samples": int(sel.sum()),
            "total_ms": {"autotune": best_total, "learned": total(learned), "heuristic": total(heur)},
            "learned_over_autotune": total(learned) / best_total,
            "heuristic_over_autotune": total(heur) / best_total,
            "regret_learned": {"mean": float(r_learned.mean()), "median": float(np.median(r_learned)),
                               "p90": float(np.percentile(r_learned, 90)), "max": float(r_learned.max())},
            "regret_heuristic": {"mean": float(r_heur.mean()), "median": float(np.median(r_heur)),
                                 "p90": float(np.percentile(r_heur, 90)), "max": float(r_heur.max())},
            "exact_pick_rate": float(np.mean(r_learned <= 1.0 + 1e-9)),
            "bsr_best": int(np.sum(np.argmin(np.where(np.isfinite(Tm[sel]), Tm[sel], np.inf), axis=1) == BSR_CANDIDATE)),
            "bsr_picked": int(np.sum(learned == BSR_CANDIDATE)),
        }
    print(json.dumps(report, indent=1), flush=True)
    save_weights(args.weights, mlp, mu, sigma, F[is_train].min(0), F[is_train].max(0),
                 {"report": report, "steps": args.steps})
    if args.report:
        with open(args.report, "w") as fh:
            json.dump(report, fh, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
