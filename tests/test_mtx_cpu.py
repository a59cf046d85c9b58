"""Native Matrix Market parser: bit-exact against FlagSparse's own loader on
the committed cases, against its restatement on a large seeded file
(multithreaded path), and thread-count independent."""

import os

import numpy as np
import pytest
import torch

from flagsparse_public_b200 import mtx
from oracle import mtx as omtx
from tests.conftest import GOLDEN_DIR

MTX_DIR = os.path.join(GOLDEN_DIR, "mtx")
GOLDEN = torch.load(os.path.join(GOLDEN_DIR, "mtx_golden.pt"), weights_only=True)


@pytest.mark.parametrize("name", sorted(GOLDEN))
def test_matches_flagsparse_loader(name):
    g = GOLDEN[name]
    data, indices, indptr, shape = mtx.load_mtx_to_csr(os.path.join(MTX_DIR, name), dtype=torch.float64,
                                                       device="cpu")
    assert shape == tuple(int(v) for v in g["shape"])
    assert torch.equal(indptr, g["indptr"].to(torch.int64))
    assert torch.equal(indices, g["indices"].to(torch.int64))
    assert torch.equal(data, g["data"].to(torch.float64))


def test_rounds_to_dtype_once():
    d32, _, _, _ = mtx.load_mtx_to_csr(os.path.join(MTX_DIR, "general_duplicates.mtx"), dtype=torch.float32,
                                       device="cpu")
    d64, _, _, _ = mtx.load_mtx_to_csr(os.path.join(MTX_DIR, "general_duplicates.mtx"), dtype=torch.float64,
                                       device="cpu")
    assert torch.equal(d32, d64.to(torch.float32))


def _write_random(path, seed, n_rows, n_cols, n_entries, symmetry):
    rng = np.random.default_rng(seed)
    r = rng.integers(1, n_rows + 1, n_entries)
    c = rng.integers(1, n_cols + 1, n_entries)
    r[:50] = r[50:100]  # forced duplicates
    c[:50] = c[50:100]
    v = rng.standard_normal(n_entries)
    with open(path, "w") as fh:
        fh.write(f"%%MatrixMarket matrix coordinate real {symmetry}\n% seeded\n{n_rows} {n_cols} {n_entries}\n")
        fh.write("".join(f"{a} {b} {float(x)!r}\n" for a, b, x in zip(r, c, v)))


@pytest.mark.parametrize("symmetry", ["general", "symmetric", "skew-symmetric"])
def test_large_file_matches_restatement(tmp_path, symmetry):
    p = str(tmp_path / f"big_{symmetry}.mtx")
    n = 30000
    _write_random(p, 7, n, n, 200_000, symmetry)
    vals, idx, ptr, shape = omtx.load(p)
    data, indices, indptr, shape2 = mtx.load_mtx_to_csr(p, dtype=torch.float64, device="cpu")
    assert shape2 == shape
    assert torch.equal(indptr, torch.tensor(ptr, dtype=torch.int64))
    assert torch.equal(indices, torch.tensor(idx, dtype=torch.int64))
    assert torch.equal(data, torch.tensor(vals, dtype=torch.float64))
    one = mtx.load_mtx_to_csr(p, dtype=torch.float64, device="cpu", threads=1)
    assert all(torch.equal(a, b) for a, b in zip(one[:3], (data, indices, indptr)))


def test_malformed_files_raise(tmp_path):
    p = tmp_path / "bad.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 x 1.0\n")
    with pytest.raises(ValueError):
        mtx.load_mtx_to_csr(str(p), device="cpu")
    q = tmp_path / "noheader.mtx"
    q.write_text("% only comments\n")
    with pytest.raises(ValueError, match="Cannot parse .mtx header"):
        mtx.load_mtx_to_csr(str(q), device="cpu")
    with pytest.raises(ValueError):
        mtx.load_mtx_to_csr(str(tmp_path / "missing.mtx"), device="cpu")
