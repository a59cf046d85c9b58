"""Golden SDDMM outputs from FlagSparse's own kernel (_sddmm_csr_real_kernel
through _run_sddmm_prepared, sddmm_csr.py:108-152, :271-348), run on CPU
tensors under TRITON_INTERPRET=1:

    FLAGSPARSE_SRC=<FlagSparse project root> python tests/golden/make_sddmm_golden.py

Writes tests/golden/sddmm_golden.pt: per case the seeded pattern, x, y,
data, alpha, beta and FlagSparse's output.
"""

import importlib
import os
import sys
import types

os.environ.setdefault("TRITON_INTERPRET", "1")

import torch  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
def _src():
    root = os.environ.get("FLAGSPARSE_SRC")
    if not root:
        raise SystemExit("set FLAGSPARSE_SRC to the FlagSparse project root")
    return os.path.join(root, "src", "flagsparse")


SRC = _src()


def load_sddmm():
    pkg = types.ModuleType("flagsparse")
    pkg.__path__ = [SRC]
    sys.modules["flagsparse"] = pkg
    sub = types.ModuleType("flagsparse.sparse_operations")
    sub.__path__ = [os.path.join(SRC, "sparse_operations")]
    sys.modules["flagsparse.sparse_operations"] = sub
    return importlib.import_module("flagsparse.sparse_operations.sddmm_csr")


def pattern(seed, n_rows, n_cols, mean):
    g = torch.Generator().manual_seed(seed)
    lens = torch.poisson(torch.full((n_rows,), float(mean)), generator=g).long().clamp(max=n_cols)
    lens[n_rows // 3] = 0  # an empty row
    cols = [torch.randperm(n_cols, generator=g)[: int(l)].sort().values for l in lens]
    indices = torch.cat(cols).to(torch.int32)
    indptr = torch.zeros(n_rows + 1, dtype=torch.int64)
    indptr[1:] = torch.cumsum(lens, 0)
    return indices, indptr


CASES = [
    # name, seed, n_rows, n_cols, mean, k, dtype, with data, alpha, beta
    ("f32_k64_data", 1, 40, 30, 5, 64, torch.float32, True, 2.0, 0.5),
    ("f64_k17_nodata", 2, 25, 50, 7, 17, torch.float64, False, 1.0, 0.0),
    ("f32_k1_data", 3, 33, 12, 4, 1, torch.float32, True, 1.0, -1.0),
    ("f64_k200_data", 4, 20, 20, 6, 200, torch.float64, True, -0.5, 2.0),
    ("f32_k96_nodata", 5, 64, 48, 9, 96, torch.float32, False, 0.75, 0.0),
]


def main():
    mod = load_sddmm()
    out = {}
    for name, seed, n_rows, n_cols, mean, k, dtype, with_data, alpha, beta in CASES:
        g = torch.Generator().manual_seed(seed + 100)
        indices, indptr = pattern(seed, n_rows, n_cols, mean)
        nnz = int(indices.numel())
        x = torch.randn((n_rows, k), generator=g, dtype=torch.float64).to(dtype)
        y = torch.randn((n_cols, k), generator=g, dtype=torch.float64).to(dtype)
        data = (torch.rand(nnz, generator=g, dtype=torch.float64) * 2 - 1).to(dtype) if with_data else None
        prepared = mod.SDDMMPrepared(indices, indptr, (n_rows, n_cols), mod._build_row_ids(indptr), 64, 4)
        res, _ = mod._run_sddmm_prepared(prepared, x, y, data, alpha, beta, None)
        out[name] = {"indices": indices, "indptr": indptr, "shape": torch.tensor([n_rows, n_cols]), "x": x, "y": y,
                     "data": data if data is not None else torch.empty(0, dtype=dtype), "has_data": with_data,
                     "alpha": alpha, "beta": beta, "out": res.clone()}
        print(name, nnz)
    torch.save(out, os.path.join(HERE, "sddmm_golden.pt"))


if __name__ == "__main__":
    main()
