"""Many independent CSR SpMMs in one persistent launch, captured in a CUDA graph.

FlagSparse multiplies one matrix per call (``flagsparse_spmm_csr``,
spmm_csr.py:2088-2157); a batch of uneven matrices costs one host round of
validation, plan lookup and launches per matrix.  Here the batch is stacked
into one block-diagonal CSR matrix -- matrix i's rows follow matrix i-1's,
its column indices are offset by the rows of the dense operands stacked
before it -- so one merge-path partition balances nonzeros across all
matrices and one persistent launch of the batched merge-path kernel (plus
the carry fix-up) computes every product.  The launch pair is captured once
in a CUDA graph; a product of the whole batch is one graph replay.

Dense operands live in stacked buffers: ``b_views[i]`` (n_cols_i x N) and
``c_views[i]`` (n_rows_i x N) are views of them, so filling B and reading C
needs no gather or scatter.  The plan (unit size, persistent grid, column
tile) comes from the autotuner over ``BATCH_CANDIDATES``.
"""

import torch

from . import _native as nat
from . import _plan
from .tuning import time_candidates

SM_COUNT = _plan.SM_COUNT


def _seq(items, grid=0, n_tile=0):
    return lambda: _plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=items, n_tile=n_tile, grid_blocks=grid,
                                    snap=_plan.SPMM_SNAP_DEFAULT)


# (name, factory): unit sizes x {one CTA per 4 units, persistent 8 / 16 CTAs per SM}
BATCH_CANDIDATES = tuple(
    [(f"seq{i}", _seq(i)) for i in (256, 512, 1024)]
    + [(f"seq{i}_p{b}", _seq(i, SM_COUNT * b)) for i in (256, 512, 1024) for b in (8, 16)]
)


def stack_csr(mats):
    """Block-diagonal stacking: (data, indices, indptr, row_off, col_off).
    Column indices of matrix i are offset by col_off[i]; indices are int32
    while the stacked column count fits, row offsets int64."""
    rows = [int(m[3][0]) for m in mats]
    cols = [int(m[3][1]) for m in mats]
    nnzs = [int(m[0].numel()) for m in mats]
    row_off, col_off = [0], [0]
    for r, c in zip(rows, cols):
        row_off.append(row_off[-1] + r)
        col_off.append(col_off[-1] + c)
    dev = mats[0][0].device
    idx_dtype = torch.int32 if col_off[-1] < 2 ** 31 else torch.int64
    data = torch.cat([m[0] for m in mats])
    indices = torch.cat([m[1].to(idx_dtype) + off for m, off in zip(mats, col_off[:-1])])
    nnz_off = 0
    ptrs = []
    for m, nz in zip(mats, nnzs):
        ptrs.append(m[2][:-1].to(torch.int64) + nnz_off)
        nnz_off += nz
    ptrs.append(torch.tensor([nnz_off], dtype=torch.int64, device=dev))
    return data, indices, torch.cat(ptrs), row_off, col_off


class PreparedCsrBatch:
    """A batch of CSR matrices stacked for one launch.

    ``mats``: sequence of (data, indices, indptr, (n_rows, n_cols)) on one CUDA
    device, one value dtype; ``n_dense``: columns of every dense operand.
    """

    def __init__(self, mats, n_dense, acc_mode=nat.ACC_NATIVE, plan=None, tune=True):
        if not mats:
            raise ValueError("empty batch")
        dev = mats[0][0].device
        dtype = mats[0][0].dtype
        if not all(m[0].device == dev and m[0].dtype == dtype for m in mats):
            raise ValueError("all matrices must share one device and value dtype")
        self.n_dense = int(n_dense)
        self.acc_mode = int(acc_mode)
        self.count = len(mats)
        self.data, self.indices, self.indptr, self.row_off, self.col_off = stack_csr(mats)
        self.n_rows, self.n_cols, self.nnz = self.row_off[-1], self.col_off[-1], int(self.data.numel())
        self.B = torch.zeros((self.n_cols, self.n_dense), dtype=dtype, device=dev)
        out_dtype = torch.float32 if dtype in (torch.float16, torch.bfloat16) else dtype
        self.C = torch.zeros((self.n_rows, self.n_dense), dtype=out_dtype, device=dev)
        self.b_views = [self.B[self.col_off[i]:self.col_off[i + 1]] for i in range(self.count)]
        self.c_views = [self.C[self.row_off[i]:self.row_off[i + 1]] for i in range(self.count)]
        self.timings = None
        if plan is None:
            if tune:
                times = time_candidates(self.data, self.indices, self.indptr, self.n_rows, self.n_cols, self.B,
                                        self.C, self.acc_mode, candidates=BATCH_CANDIDATES)
                self.timings = dict(zip((n for n, _ in BATCH_CANDIDATES), times))
                best = min(range(len(times)), key=times.__getitem__)
                plan = BATCH_CANDIDATES[best][1]()
            else:
                plan = BATCH_CANDIDATES[0][1]()
        self.plan = plan
        self.plan.ensure_coords(self.indptr, self.n_rows, self.nnz)
        self.graph = None

    def useful_bytes(self):
        vb = self.data.element_size()
        return (self.nnz * (vb + self.indices.element_size()) + self.n_cols * self.n_dense * self.B.element_size()
                + self.n_rows * self.n_dense * self.C.element_size())

    def _launch(self):
        _plan.run_spmm(self.data, self.indices, self.indptr, self.n_rows, self.n_cols, self.B, self.C, self.acc_mode,
                       self.plan)

    def capture(self):
        """Capture the launch pair in a CUDA graph (one warm-up launch first)."""
        self._launch()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._launch()
        self.graph = g
        return g

    def run(self):
        """C = A B for every matrix of the batch (one graph replay)."""
        if self.graph is None:
            self.capture()
        self.graph.replay()
        return self.c_views


def prepare_spmm_csr_batch(mats, n_dense, acc_mode=nat.ACC_NATIVE, plan=None, tune=True):
    """Stack ``mats`` for batched products with ``n_dense``-column operands."""
    return PreparedCsrBatch(mats, n_dense, acc_mode=acc_mode, plan=plan, tune=tune)
