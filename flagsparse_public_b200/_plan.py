"""Launch plans for the CSR kernels and the calls that run them.

A plan names one kernel family of the C ABI (row groups or merge path) and its
shape (lanes per row, merge-path items per unit, dense-column tile).  Plans
come from the matrix statistics gathered at prepare time (one device->host
read) through ``default_spmv_plan`` / ``default_spmm_plan``, or from the
autotuner and the learned selector (``flagsparse_public_b200.tuning``).
Merge-path partitions are computed on the device once per (matrix, plan) and
cached on the prepared object.
"""

import math
import os

import torch

from . import _native as nat

SPMV_MERGE_THREADS = 128
# SEQ plans move unit boundaries that fall inside rows shorter than this many
# nonzeros back to the row start: only longer rows are split across units
# (power-law SpMM: 169 us snapped against 172 us unsnapped at 128 items).
SPMM_SNAP_DEFAULT = 64

# Kernels launched by run_spmv / run_spmm since import (partition launches
# excluded): one per call for row groups and for the SpMM merge-path kernel
# that finishes split rows itself, two (tiles + carry fix-up) otherwise.
LAUNCHES = {"count": 0}


def _kernels_per_call(plan):
    if plan.algo == nat.ALGO_ROWS or plan.algo == ALGO_BSR:
        return 1
    return 1 if plan.in_kernel_finish() else 2


class MatrixStats:
    """Row-length statistics of a CSR structure (from one host read)."""

    __slots__ = ("n_rows", "n_cols", "nnz", "max_row", "mean_row", "std_row", "empty_rows")

    def __init__(self, n_rows, n_cols, nnz, max_row, mean_row, std_row, empty_rows):
        self.n_rows = int(n_rows)
        self.n_cols = int(n_cols)
        self.nnz = int(nnz)
        self.max_row = int(max_row)
        self.mean_row = float(mean_row)
        self.std_row = float(std_row)
        self.empty_rows = int(empty_rows)

    @property
    def skew(self):
        return self.max_row / max(self.mean_row, 1.0)

    def as_dict(self):
        return {k: getattr(self, k) for k in self.__slots__}


def matrix_stats(row_ptr, n_rows, n_cols):
    n_rows = int(n_rows)
    if n_rows == 0:
        return MatrixStats(0, n_cols, 0, 0, 0.0, 0.0, 0)
    lens = (row_ptr[1:] - row_ptr[:-1]).to(torch.float64)
    vals = torch.stack([lens.max(), lens.mean(), lens.std(unbiased=False), (lens == 0).sum().to(torch.float64),
                        lens.sum()]).tolist()
    return MatrixStats(n_rows, n_cols, int(vals[4]), int(vals[0]), vals[1], vals[2], int(vals[3]))


class KernelPlan:
    """One launch configuration of fsb_spmv_csr / fsb_spmm_csr."""

    __slots__ = ("algo", "lanes", "items_per_unit", "n_tile", "snap", "coords", "n_units", "row_cap",
                 "comp_threshold", "fallback_ok", "grid_blocks", "flags", "runs", "tickets")

    def __init__(self, algo, lanes=32, items_per_unit=0, n_tile=0, snap=0, row_cap=0, comp_threshold=0,
                 fallback_ok=False, grid_blocks=0, flags=0):
        self.algo = int(algo)
        self.lanes = int(lanes)
        self.items_per_unit = int(items_per_unit)
        self.n_tile = int(n_tile)
        self.snap = int(snap)
        self.coords = None
        self.n_units = 0
        self.row_cap = int(row_cap)
        self.comp_threshold = int(comp_threshold)
        self.fallback_ok = bool(fallback_ok)
        self.grid_blocks = int(grid_blocks)
        self.flags = int(flags)
        self.runs = None
        self.tickets = None

    def _seq_registers(self):
        return self.algo == nat.ALGO_SEQ and not (self.flags & nat.PLAN_TMA_GATHER)

    def in_kernel_finish(self):
        """Whether split rows finish inside the SEQ kernel (unit runs + ticket
        counters) rather than in the separate carry fix-up: decided once per
        partition by ensure_runs."""
        return self._seq_registers() and self.runs is not None and self.runs is not False

    def as_flat(self):
        """The register-staged flat plan over the same merge-path units."""
        p = KernelPlan(nat.ALGO_FLAT, items_per_unit=self.items_per_unit, n_tile=self.n_tile, snap=self.snap,
                       row_cap=self.row_cap, comp_threshold=self.comp_threshold)
        p.coords, p.n_units = self.coords, self.n_units
        return p

    def key(self):
        return (self.algo, self.lanes, self.items_per_unit, self.n_tile, self.snap, self.grid_blocks, self.flags)

    def describe(self):
        if self.algo == nat.ALGO_ROWS:
            kind = "warp_rows" if self.lanes == 32 else "vector_rows"
            return {"kind": kind, "lanes": self.lanes, "n_tile": self.n_tile}
        kind = {nat.ALGO_MERGE: "merge_path", nat.ALGO_FLAT: "merge_path_flat",
                nat.ALGO_GATHER: "merge_path_tma_gather", nat.ALGO_SEQ: "merge_path_seq"}[self.algo]
        if self.algo == nat.ALGO_SEQ and self.flags & nat.PLAN_TMA_GATHER:
            kind = "merge_path_seq_gather4"
        d = {"kind": kind, "items_per_unit": self.items_per_unit, "n_tile": self.n_tile,
             "snap": self.snap, "n_units": self.n_units}
        if self.grid_blocks:
            d["grid_blocks"] = self.grid_blocks
        return d

    def copy(self):
        p = KernelPlan(self.algo, self.lanes, self.items_per_unit, self.n_tile, self.snap, self.row_cap,
                       self.comp_threshold, self.fallback_ok, self.grid_blocks, self.flags)
        return p

    def ensure_coords(self, row_ptr, n_rows, nnz):
        """Compute (once) the merge-path unit coordinates on the device."""
        if self.algo == nat.ALGO_ROWS or self.coords is not None:
            return
        n_units = -(-(int(n_rows) + int(nnz)) // self.items_per_unit) if (n_rows + nnz) > 0 else 0
        coords = torch.empty((n_units + 1) * 2, dtype=torch.int64, device=row_ptr.device)
        if n_units > 0:
            lib = nat.library()
            rc = lib.fsb_merge_partition(nat.ptr(row_ptr), nat.dtype_code(row_ptr.dtype), int(n_rows), int(nnz),
                                         self.items_per_unit, self.snap, nat.ptr(coords), n_units,
                                         nat.stream_handle(row_ptr.device))
            nat.check(rc, "fsb_merge_partition")
        self.coords = coords
        self.n_units = n_units

    def ensure_runs(self, row_ptr, n_rows, n_dense):
        """SEQ plans: the unit runs of the partition (once) and, when split
        rows finish in the kernel, zero-filled ticket counters for one per
        unit and column tile of an n_dense-wide call (the kernel returns them
        to zero).  Each unit holding part of a split row takes an atomic
        ticket at its end, which pays off against the separate fix-up launch
        only while such units are few: at most IN_KERNEL_FINISH_MAX of them
        (one host read, once per partition; decided outside stream capture,
        the fix-up runs meanwhile)."""
        if not self._seq_registers():
            return
        if self.runs is None:
            if row_ptr.is_cuda and torch.cuda.is_current_stream_capturing():
                return
            runs = torch.empty(max(self.n_units, 1) * 2, dtype=torch.int64, device=row_ptr.device)
            contributors = 0
            if self.n_units > 0:
                rc = nat.library().fsb_merge_runs(nat.ptr(row_ptr), nat.dtype_code(row_ptr.dtype), int(n_rows),
                                                  nat.ptr(self.coords), self.n_units, nat.ptr(runs),
                                                  nat.stream_handle(row_ptr.device))
                nat.check(rc, "fsb_merge_runs")
                contributors = int((runs.view(-1, 2)[: self.n_units, 0] >= 0).sum())
            self.runs = runs if contributors <= IN_KERNEL_FINISH_MAX else False
        if self.runs is False:
            return
        need = self.n_units * ticket_col_tiles(n_dense, self.n_tile)
        if self.tickets is None or self.tickets.numel() < need:
            self.tickets = torch.zeros(max(need, 1), dtype=torch.int32, device=row_ptr.device)

    def c_plan(self):
        finish = self.in_kernel_finish()
        return nat.make_plan(self.algo, lanes=self.lanes, items_per_unit=self.items_per_unit, n_tile=self.n_tile,
                             coords=self.coords, n_units=self.n_units, row_cap=self.row_cap,
                             comp_threshold=self.comp_threshold, grid_blocks=self.grid_blocks, flags=self.flags,
                             runs=self.runs if finish else None, tickets=self.tickets if finish else None)


# Plan kind (host side only) of the tensor-core BSR candidate.
ALGO_BSR = -1
# Largest fill-in the BSR candidate accepts: stored block entries (256 per
# 16 x 16 block holding a nonzero) per nonzero.
BSR_FILL_MAX = 2.0


class BsrPlan:
    """The tensor-core BSR path as an SpMM plan: the CSR matrix is converted
    once (``bsr.csr_to_bsr16``, cached on the plan for that matrix) and each
    call runs ``fsb_bsr_spmm_tc``.  Runs only half-precision values with a
    same-typed B, a float32 C with a multiple of 8 columns and float32
    accumulation; ValueError otherwise, or when the 16 x 16 blocks would
    store more than BSR_FILL_MAX entries per nonzero."""

    algo = ALGO_BSR
    flags = 0
    n_tile = 0
    items_per_unit = 0
    lanes = 0
    grid_blocks = 0

    def __init__(self):
        self.comp_threshold = 0
        self._form = None  # (matrix key, PreparedBsr)

    def key(self):
        return (ALGO_BSR,)

    def describe(self):
        return {"kind": "bsr16_tcgen05"}

    def copy(self):
        return BsrPlan()

    def in_kernel_finish(self):
        return True

    def ensure_coords(self, row_ptr, n_rows, nnz):
        return

    def ensure_runs(self, row_ptr, n_rows, n_dense):
        return

    @staticmethod
    def supported(values, B, C, acc_mode, row_map=None):
        return (values.dtype in (torch.bfloat16, torch.float16) and B.dtype == values.dtype and
                C.dtype == torch.float32 and C.is_contiguous() and B.shape[1] % 8 == 0 and row_map is None and
                int(acc_mode) == nat.ACC_NATIVE)

    def prepared(self, values, col_idx, row_ptr, n_rows, n_cols):
        from . import bsr

        key = (values.data_ptr(), col_idx.data_ptr(), row_ptr.data_ptr(), int(values.numel()), int(n_rows),
               int(n_cols))
        if self._form is None or self._form[0] != key:
            blocks = bsr.block_count(col_idx, row_ptr, (n_rows, n_cols))
            if blocks * bsr.BLOCK * bsr.BLOCK > BSR_FILL_MAX * max(int(values.numel()), 1):
                raise ValueError(f"BSR fill-in too high: {blocks} blocks for {int(values.numel())} nonzeros")
            vals, bcol, bptr = bsr.csr_to_bsr16(values, col_idx, row_ptr, (n_rows, n_cols))
            self._form = (key, bsr.prepare_spmm_bsr(vals, bcol, bptr, (n_rows, n_cols)))
        return self._form[1]

    def run(self, values, col_idx, row_ptr, n_rows, n_cols, B, C, acc_mode, row_map=None):
        from . import bsr

        if not self.supported(values, B, C, acc_mode, row_map):
            raise ValueError("the BSR plan needs half-precision values and B, a float32 C with a multiple of 8 "
                             "columns and float32 accumulation")
        bsr.flagsparse_spmm_bsr(B=B, prepared=self.prepared(values, col_idx, row_ptr, n_rows, n_cols), out=C)
        return C


# Split rows finish inside the SEQ kernel while at most this many units hold
# parts of them (power-law SpMM: 10 K - 24 K such units, 5 - 10 us faster than
# the separate fix-up; banded matrix: 152 K, 66 us slower).
IN_KERNEL_FINISH_MAX = 32768


def ticket_col_tiles(n_dense, n_tile=0):
    """Upper bound of the column tiles of a SEQ launch: a tile spans
    (lane vector) x (lanes per nonzero) >= min(target width, 32) columns."""
    n_dense = int(n_dense)
    if n_dense <= 0:
        return 1
    width = int(n_tile) if n_tile > 0 else n_dense
    return -(-n_dense // max(1, min(width, 32)))


def _pow2_clamp(v, lo, hi):
    v = max(float(v), 1.0)
    p = 1 << int(round(math.log2(v)))
    return int(min(max(p, lo), hi))


def _vec_elems(dtype):
    return max(1, 16 // dtype.itemsize)


def default_spmv_plan(stats, dtype, row_cap=0):
    """Heuristic SpMV plan: merge path for skewed rows that are short on
    average, else row groups sized so a row's nonzeros take about half a
    16-byte vector per lane (more lanes shorten each row's dependent load
    chain; long average rows keep 16-32 lanes busy even when a few rows are
    much longer: measured faster than merge path there)."""
    if row_cap > 0 or stats.n_rows == 0:
        lanes = _pow2_clamp(stats.mean_row / _vec_elems(dtype), 2, 32) if stats.n_rows else 32
        return KernelPlan(nat.ALGO_ROWS, lanes=lanes, row_cap=row_cap)
    skewed = stats.max_row > 8 * max(stats.mean_row, 1.0) + 256
    if skewed and stats.mean_row < 32:
        ipt = 8 if dtype.itemsize <= 4 else 4
        return KernelPlan(nat.ALGO_MERGE, items_per_unit=SPMV_MERGE_THREADS * ipt)
    lanes = _pow2_clamp(2 * stats.mean_row / _vec_elems(dtype), 2, 32)
    return KernelPlan(nat.ALGO_ROWS, lanes=lanes, flags=nat.PLAN_OVERLAP_LAUNCH)


SM_COUNT = 148  # B200
SEQ_WARPS_PER_SM = 32


def seq_items_per_unit(stats):
    """Merge-path unit size for the batched SpMM kernel: (rows + nonzeros)
    spread over about two waves of resident warps, between 128 and 1024."""
    items = stats.n_rows + stats.nnz
    return _pow2_clamp(items / (SM_COUNT * SEQ_WARPS_PER_SM * 2), 128, 1024)


def default_spmm_plan(stats, n_dense, dtype, row_cap=0):
    """Heuristic SpMM plan: the batched merge-path kernel (nonzero-balanced
    units, rows split across units where long); row groups when a per-row
    segment cap is requested."""
    if row_cap > 0 or stats.n_rows == 0:
        return KernelPlan(nat.ALGO_ROWS, lanes=32, row_cap=row_cap)
    return KernelPlan(nat.ALGO_SEQ, items_per_unit=seq_items_per_unit(stats), snap=SPMM_SNAP_DEFAULT)


# How the prepared SpMM paths pick their plan: "learned" (the shipped
# selector network, falling back to autotuning when unsure), "autotune"
# (time every candidate once per matrix and width) or "heuristic"
# (default_spmm_plan, no timing).
PLAN_SELECTORS = ("learned", "autotune", "heuristic")
_selector_mode = os.environ.get("FSB_PLAN_SELECTOR", "learned")
_selectors = {}
_autotuner = None


def set_plan_selector(mode):
    """Select how prepared SpMM calls choose plans (see PLAN_SELECTORS)."""
    global _selector_mode
    if mode not in PLAN_SELECTORS:
        raise ValueError(f"plan selector must be one of {PLAN_SELECTORS}")
    _selector_mode = mode


def plan_selector():
    return _selector_mode


def _tuner():
    global _autotuner
    if _autotuner is None:
        from . import tuning
        _autotuner = tuning.Autotuner()
    return _autotuner


def learned_selector(device):
    """The shipped selector on ``device`` (None when no weights are installed)."""
    from . import tuning
    key = str(device)
    sel = _selectors.get(key)
    if sel is None:
        if not os.path.exists(tuning.WEIGHTS_PATH):
            return None
        sel = tuning.LearnedSelector(device=device, autotuner=_tuner())
        _selectors[key] = sel
    return sel


def chosen_spmm_plan(stats, data, indices, indptr, n_rows, n_cols, B, C, acc_mode):
    """Plan for a prepared SpMM call by the current selector mode.  Needs the
    operands (the learned selector reads the structure on the device, the
    autotuner runs every candidate into C); not for use inside graph capture."""
    n_dense = int(B.shape[1])
    mode = _selector_mode
    if mode == "heuristic" or stats.n_rows == 0 or n_dense == 0:
        return default_spmm_plan(stats, n_dense, data.dtype)
    if mode == "learned":
        sel = learned_selector(B.device)
        if sel is not None:
            return sel.select(data, indices, indptr, n_rows, n_cols, B, C, acc_mode)
        return default_spmm_plan(stats, n_dense, data.dtype)
    plan, _ = _tuner().tune(data, indices, indptr, n_rows, n_cols, B, C, acc_mode)
    return plan


def sorted_keys_to_offsets(keys, n_bins):
    """int64 offsets[0 .. n_bins] of nondecreasing keys in [0, n_bins):
    cumsum(bincount(keys)) computed without reading anything back to the host
    (fsb_sorted_keys_to_offsets on CUDA tensors; a plain bincount on CPU)."""
    n_bins = int(n_bins)
    if not keys.is_cuda:
        out = torch.zeros(n_bins + 1, dtype=torch.int64, device=keys.device)
        if keys.numel():
            out[1:] = torch.cumsum(torch.bincount(keys.to(torch.int64), minlength=n_bins), dim=0)
        return out
    keys = keys.contiguous()
    out = torch.empty(n_bins + 1, dtype=torch.int64, device=keys.device)
    rc = nat.library().fsb_sorted_keys_to_offsets(nat.ptr(keys), nat.dtype_code(keys.dtype), keys.numel(), n_bins,
                                                  nat.ptr(out), nat.stream_handle(keys.device))
    nat.check(rc, "fsb_sorted_keys_to_offsets")
    return out


_SORT_MAX_KEYS = 2 ** 31 - 1  # fsb_stable_sort / fsb_run_starts limit


def stable_sort(keys, key_bound=None):
    """(sorted keys, int64 permutation) of a 1-D int32 / int64 tensor, equal
    to ``torch.sort(keys, stable=True)``: fsb_stable_sort (LSD radix sort) on
    CUDA tensors, torch on CPU.  ``key_bound``: an exclusive upper bound of
    non-negative keys (fewer radix passes); None sorts the full signed width."""
    if not keys.is_cuda or keys.numel() > _SORT_MAX_KEYS:
        # host tensors, and more keys than the kernels' 32-bit positions hold
        return torch.sort(keys, stable=True)
    keys = keys.contiguous()
    n = keys.numel()
    width = 32 if keys.dtype == torch.int32 else 64
    if keys.dtype not in (torch.int32, torch.int64):
        raise TypeError("stable_sort: keys must be int32 or int64")
    bits = width if key_bound is None else min(width, max(1, (max(int(key_bound), 1) - 1).bit_length()))
    out = torch.empty_like(keys)
    order = torch.empty(n, dtype=torch.int64, device=keys.device)
    if n == 0:
        return out, order
    lib = nat.library()
    code = nat.dtype_code(keys.dtype)
    nbytes = int(lib.fsb_sort_workspace_bytes(n, code, bits))
    ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=keys.device)
    rc = lib.fsb_stable_sort(nat.ptr(keys), code, n, bits, nat.ptr(out), nat.ptr(order), nat.ptr(ws), nbytes,
                             nat.stream_handle(keys.device))
    nat.check(rc, "fsb_stable_sort")
    return out, order


def run_starts_device(sorted_keys, out_dtype):
    """fsb_run_starts without a host read: (starts buffer of n + 1 entries,
    device int64 tensor holding how many of them were written)."""
    keys = sorted_keys.contiguous()
    n = keys.numel()
    lib = nat.library()
    starts = torch.empty(n + 1, dtype=out_dtype, device=keys.device)
    count = torch.zeros(1, dtype=torch.int64, device=keys.device)
    if n == 0:
        return starts, count
    nbytes = int(lib.fsb_run_starts_workspace_bytes(n))
    ws = torch.empty(nbytes, dtype=torch.uint8, device=keys.device)
    rc = lib.fsb_run_starts(nat.ptr(keys), nat.dtype_code(keys.dtype), n, nat.ptr(starts), nat.dtype_code(out_dtype),
                            nat.ptr(count), nat.ptr(ws), nbytes, nat.stream_handle(keys.device))
    nat.check(rc, "fsb_run_starts")
    return starts, count


def coalesce_sorted(sorted_keys, order, values):
    """Distinct keys and their summed values (fsb_coo_coalesce) of stably
    sorted keys; buffers of n entries and the device count of distinct keys
    (no host read)."""
    n = sorted_keys.numel()
    out_keys = torch.empty_like(sorted_keys)
    out_vals = torch.empty_like(values)
    starts, count = run_starts_device(sorted_keys, torch.int64)
    if n:
        rc = nat.library().fsb_coo_coalesce(nat.ptr(sorted_keys), nat.dtype_code(sorted_keys.dtype), nat.ptr(order),
                                            nat.ptr(values), nat.dtype_code(values.dtype), n, nat.ptr(starts),
                                            nat.dtype_code(starts.dtype), nat.ptr(count), nat.ptr(out_keys),
                                            nat.ptr(out_vals), nat.stream_handle(values.device))
        nat.check(rc, "fsb_coo_coalesce")
    return out_keys, out_vals, (count - 1).clamp_(min=0)


def run_starts(sorted_keys, out_dtype):
    """[0, start of every later run of equal keys ..., n] of sorted 1-D keys in
    ``out_dtype`` (int32 / int64): fsb_run_starts on CUDA tensors (one host
    read of the run count), the equivalent torch expression on CPU.  None for
    no keys."""
    n = sorted_keys.numel()
    if n == 0:
        return None
    if not sorted_keys.is_cuda or n > _SORT_MAX_KEYS:
        dev = sorted_keys.device
        breaks = torch.nonzero(sorted_keys[1:] != sorted_keys[:-1], as_tuple=False).flatten().to(out_dtype) + 1
        return torch.cat([torch.zeros(1, dtype=out_dtype, device=dev), breaks,
                          torch.tensor([n], dtype=out_dtype, device=dev)])
    starts, count = run_starts_device(sorted_keys, out_dtype)
    return starts[: int(count.item())].clone()


def _workspace(is_spmm, cm, n_dense, acc_mode, out_code, cp, device):
    lib = nat.library()
    nbytes = int(lib.fsb_workspace_bytes(int(is_spmm), cm, int(n_dense), int(acc_mode), int(out_code), cp))
    if nbytes <= 0:
        return None, 0
    return torch.empty(nbytes, dtype=torch.uint8, device=device), nbytes


def run_spmv(values, col_idx, row_ptr, n_rows, n_cols, x, y, acc_mode, plan, row_map=None):
    """y = A x through fsb_spmv_csr on torch's current stream."""
    if plan.algo == nat.ALGO_MERGE and plan.snap:
        raise ValueError("SpMV merge-path tiles need an unsnapped partition (snap=0)")
    plan.ensure_coords(row_ptr, n_rows, values.numel())
    cm = nat.make_csr(values, col_idx, row_ptr, n_rows, n_cols, row_map)
    cp = plan.c_plan()
    out_code = nat.dtype_code(y.dtype)
    ws, nbytes = _workspace(False, cm, 1, acc_mode, out_code, cp, values.device)
    lib = nat.library()
    rc = lib.fsb_spmv_csr(cm, nat.ptr(x), nat.ptr(y), out_code, int(acc_mode), cp, nat.ptr(ws), nbytes,
                          nat.stream_handle(values.device))
    nat.check(rc, "fsb_spmv_csr")
    LAUNCHES["count"] += _kernels_per_call(plan)
    return y


def gather_supported(B, C, n_tile=0):
    """Whether the TMA bulk-gather plan can run on these operands: 16-byte
    aligned B rows, column tiles and C lane vectors (mirrors the check in
    fsb_spmm_gather.cu)."""
    vb, vc = B.element_size(), C.element_size()
    vw = max(1, 16 // max(vb, vc))
    n_dense = B.shape[1]
    target = n_tile if n_tile > 0 else n_dense
    lpn_log2 = 0
    while (1 << lpn_log2) * vw < target and lpn_log2 < 5:
        lpn_log2 += 1
    tile_bytes = (vw << lpn_log2) * vb
    multi_tile = n_dense > (vw << lpn_log2)
    return (lpn_log2 >= 3 and B.data_ptr() % 16 == 0 and (B.stride(0) * vb) % 16 == 0 and (n_dense * vb) % 16 == 0
            and (not multi_tile or tile_bytes % 16 == 0) and C.data_ptr() % (vw * vc) == 0
            and C.stride(0) % vw == 0 and n_dense % vw == 0)


G4_WARPS_PER_SM = 12  # resident warps of the gather4 SpMM (3 CTAs of 4 warps, 64 KB of rings each)


def g4_items_per_unit(stats, units_per_warp=1):
    """Merge-path unit size for the gather4 SpMM: (rows + nonzeros) over
    units_per_warp units per resident warp (one pipeline fill per unit)."""
    items = stats.n_rows + stats.nnz
    return max(64, -(-items // (SM_COUNT * G4_WARPS_PER_SM * units_per_warp)))


def g4_supported(values, B, C, acc_mode, n_cols):
    """Whether the TMA gather4 form of the SEQ plan can run on these operands
    (mirrors launch_g4 in fsb_spmm_g4.cuh): float32 / float16 / bfloat16
    values with float accumulators, 16-byte aligned B rows, n_dense a multiple
    of the 16-byte lane vector, C lane vectors aligned, n_cols below 2^31."""
    if values.dtype not in (torch.float32, torch.float16, torch.bfloat16) or acc_mode == nat.ACC_COMP:
        return False
    vb, vc = B.element_size(), C.element_size()
    vw = 16 // vb
    n_dense = B.shape[1]
    return (B.data_ptr() % 16 == 0 and (B.stride(0) * vb) % 16 == 0 and n_dense % vw == 0
            and C.data_ptr() % min(16, vw * vc) == 0 and C.stride(0) % vw == 0 and int(n_cols) < 2 ** 31 - 1)


def run_spmm(values, col_idx, row_ptr, n_rows, n_cols, B, C, acc_mode, plan, row_map=None):
    """C = A B through fsb_spmm_csr (B, C row-major with unit column stride)."""
    if isinstance(plan, BsrPlan):
        return plan.run(values, col_idx, row_ptr, n_rows, n_cols, B, C, acc_mode, row_map)
    if plan.algo == nat.ALGO_GATHER and not gather_supported(B, C, plan.n_tile):
        if not plan.fallback_ok:
            raise ValueError("the TMA gather plan needs 16-byte aligned B and C rows")
        plan = plan.as_flat()
    if plan.flags & nat.PLAN_TMA_GATHER and not g4_supported(values, B, C, acc_mode, n_cols):
        if not plan.fallback_ok:
            raise ValueError("the gather4 plan needs float32 / float16 / bfloat16 values, float accumulators and "
                             "16-byte aligned B and C rows")
        plan = plan.copy()
        plan.flags &= ~nat.PLAN_TMA_GATHER
    plan.ensure_coords(row_ptr, n_rows, values.numel())
    n_dense = int(B.shape[1])
    plan.ensure_runs(row_ptr, n_rows, n_dense)
    cm = nat.make_csr(values, col_idx, row_ptr, n_rows, n_cols, row_map)
    cp = plan.c_plan()
    out_code = nat.dtype_code(C.dtype)
    ws, nbytes = _workspace(True, cm, n_dense, acc_mode, out_code, cp, values.device)
    lib = nat.library()
    rc = lib.fsb_spmm_csr(cm, nat.ptr(B), int(B.stride(0)), n_dense, nat.ptr(C), int(C.stride(0)), out_code,
                          int(acc_mode), cp, nat.ptr(ws), nbytes, nat.stream_handle(values.device))
    nat.check(rc, "fsb_spmm_csr")
    LAUNCHES["count"] += _kernels_per_call(plan) if n_dense > 0 and n_rows > 0 else 0
    return C
