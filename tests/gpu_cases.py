"""Matrix cases and launch-plan sweeps shared by the GPU parity tests."""

import torch

from flagsparse_public_b200 import _native as nat
from flagsparse_public_b200 import _plan
from flagsparse_public_b200 import synthetic


def csr_from_lengths(lengths, n_cols, seed, dtype=torch.float32, index_dtype=torch.int32, ptr_dtype=torch.int64,
                     device="cpu"):
    """CSR with the given row lengths: sorted distinct uniform columns, U(-1,1) values."""
    lengths = torch.as_tensor(lengths, dtype=torch.int64)
    if lengths.numel() and int(lengths.max()) > n_cols:
        raise ValueError(f"a row of {int(lengths.max())} distinct columns needs n_cols >= that, got {n_cols}")
    g = torch.Generator().manual_seed(seed)
    n_rows = lengths.numel()
    indptr = torch.zeros(n_rows + 1, dtype=torch.int64)
    indptr[1:] = torch.cumsum(lengths, 0)
    cols = []
    for ln in lengths.tolist():
        cols.append(torch.sort(torch.randperm(n_cols, generator=g)[:ln]).values)
    indices = torch.cat(cols) if cols else torch.empty(0, dtype=torch.int64)
    nnz = int(indptr[-1])
    if dtype.is_complex:
        comp = torch.float32 if dtype == torch.complex64 else torch.float64
        data = torch.complex(torch.rand(nnz, generator=g, dtype=comp) * 2 - 1,
                             torch.rand(nnz, generator=g, dtype=comp) * 2 - 1)
    else:
        data = (torch.rand(nnz, generator=g, dtype=torch.float64) * 2 - 1).to(dtype)
    return (data.to(device), indices.to(index_dtype).to(device), indptr.to(ptr_dtype).to(device), (n_rows, n_cols))


def dense(shape, seed, dtype, device="cpu"):
    g = torch.Generator().manual_seed(seed)
    if dtype.is_complex:
        comp = torch.float32 if dtype == torch.complex64 else torch.float64
        t = torch.complex(torch.randn(shape, generator=g, dtype=comp), torch.randn(shape, generator=g, dtype=comp))
    else:
        t = torch.randn(shape, generator=g, dtype=torch.float64).to(dtype)
    return t.to(device)


# Row-length patterns that stress the kernels' edge handling.
EDGE_LENGTHS = {
    "empty_rows": [0, 0, 3, 0, 1, 0, 0, 7, 0],
    "boundaries": [1, 31, 32, 33, 63, 64, 65, 127, 128, 129],
    "long_rows": [4095, 2, 4097, 0, 5, 9000, 1],
    "one_row": [300],
    "all_empty": [0] * 17,
    "skewed": [2] * 500 + [3000] + [1] * 300 + [12000] + [4] * 200,
}


def spmv_plans(dtype):
    """Every SpMV launch plan family the selector can choose."""
    plans = [_plan.KernelPlan(nat.ALGO_ROWS, lanes=lanes) for lanes in (1, 2, 4, 8, 16, 32)]
    plans += [_plan.KernelPlan(nat.ALGO_MERGE, items_per_unit=128 * ipt) for ipt in (1, 2, 4, 8)]
    return plans


def spmm_plans():
    plans = [_plan.KernelPlan(nat.ALGO_ROWS, lanes=lanes) for lanes in (1, 4, 8, 16, 32)]
    plans += [_plan.KernelPlan(nat.ALGO_ROWS, lanes=32, n_tile=8)]
    plans += [_plan.KernelPlan(nat.ALGO_MERGE, items_per_unit=ipu, snap=snap)
              for ipu, snap in ((32, 0), (64, 16), (128, 64), (512, 0))]
    plans += [_plan.KernelPlan(nat.ALGO_FLAT, items_per_unit=ipu, snap=snap, n_tile=nt)
              for ipu, snap, nt in ((16, 0, 0), (100, 0, 0), (256, 128, 0), (1024, 0, 0), (128, 64, 32))]
    plans += [_plan.KernelPlan(nat.ALGO_GATHER, items_per_unit=ipu, snap=snap, n_tile=nt)
              for ipu, snap, nt in ((16, 0, 0), (100, 0, 0), (256, 128, 0), (2048, 0, 0), (128, 64, 32), (64, 0, 0))]
    plans += [_plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=ipu, snap=snap, n_tile=nt)
              for ipu, snap, nt in ((16, 0, 0), (100, 0, 0), (256, 128, 0), (2048, 0, 0), (128, 64, 32), (77, 0, 8))]
    # persistent grids: one and three CTAs striding over every unit
    plans += [_plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=ipu, grid_blocks=g) for ipu, g in ((16, 1), (64, 3))]
    # snapped units (only rows of at least 64 nonzeros split)
    plans += [_plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=ipu, snap=64) for ipu in (100, 128)]
    # B rows staged by TMA gather4: short units (ring slots reused across
    # units), long units (the ring wraps many times), snapped units, column
    # tiles, one persistent CTA
    plans += [_plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=ipu, snap=snap, n_tile=nt, grid_blocks=g,
                               flags=nat.PLAN_TMA_GATHER)
              for ipu, snap, nt, g in ((16, 0, 0, 0), (100, 0, 0, 0), (256, 128, 0, 0), (2048, 0, 0, 0),
                                       (128, 64, 16, 0), (40, 0, 0, 1))]
    return plans


def c1_matrix(device="cuda", n=16384):
    return synthetic.poisson_uniform(n_rows=n, n_cols=n, mean=16.0, seed=0, dtype=torch.float32, device=device)
