#!/usr/bin/env python
"""Benchmark of the CSR SpMV / SpMM hot path on B200.

Default workload (one step = one SpMM over one batch of synthetic input):
power-law CSR SpMM, 262144 x 262144, Zipf(1.8) row lengths scaled to mean ~12
and capped at 20000, uniform columns, U(-1,1) float32 values, int32 indices,
dense B 262144 x 64 float32 N(0,1), C 262144 x 64 float32.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  ``value`` is the useful HBM bytes per second
of the chosen form (launch plan from the selector / heuristic, float32
accumulation), summed over all ranks, with inputs resident in HBM and L2
flushed (256 MiB write) before every timed step; ``plain`` reports the
FlagSparse-compatible plain form (float64 accumulation) the same way; ``e2e``
runs the public API from pinned host buffers (host->device copies of A and B,
prepare, SpMM, device->host copy of C) every step.  ``--impl reference`` times
the CPU restatement of FlagSparse's algorithm (the oracle port) on the host
cores instead.

Multi-GPU: one process per GPU (torchrun), each rank runs the same workload
on its own GPU (replicas; the path needs no data exchange), timed on the
device, max over ranks.
"""

import argparse
import json
import math
import os
import statistics
import sys
import threading
import time

import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

L2_FLUSH_BYTES = 256 << 20
FALLBACK_HBM_GBS = 6650.0


# ----------------------------------------------------------------- setup ----
def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default="spmm_powerlaw", choices=sorted(WORKLOADS))
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--profile", action="store_true",
                    help="only warm-up + timed device steps (for a profiler launch list)")
    ap.add_argument("--form", default=None,
                    help="with --profile: time this extra form of the workload (e.g. spmv_bf16) instead of its step")
    ap.add_argument("--only", action="store_true",
                    help="measure the chosen workload alone (no side configurations, no selector check)")
    ap.add_argument("--plan", default=None,
                    help="force the chosen-form plan: rows:<lanes>[:<n_tile>] | merge:<items>:<snap> | "
                         "flat|gather|seq:<items>:<snap>[:<n_tile>] | g4:<items>[:<snap>[:<n_tile>]]")
    return ap.parse_args(argv)


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def init_dist(world, backend=None):
    """One process per GPU: NCCL where CUDA is present, gloo otherwise (CPU
    tests of the multi-rank path).  Short timeout: ranks that wait on a
    missing peer end with an error instead of hanging."""
    if world > 1:
        import datetime

        import torch.distributed as dist

        backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(value, world):
    if world == 1:
        return value
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_value(units_per_rank, world, max_ms):
    """Whole-job throughput: the units every rank processed over the slowest
    rank's time (weak scaling: each rank runs the full workload)."""
    return units_per_rank * world / (max_ms * 1e-3) / 1e9


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def committed_traffic(kernel_key):
    """DRAM bytes per launch from a committed ncu summary (profiles/*.txt) and
    the file it was read from (an earlier cold-L2 capture of the same
    command, not a measurement of this run); (None, None) when absent."""
    rel = os.path.join("profiles", f"{kernel_key}.txt")
    try:
        for line in open(os.path.join(ROOT, rel)):
            if line.startswith("dram_bytes_per_launch:"):
                return float(line.split(":", 1)[1].split()[0]), rel + " (committed ncu capture, cold L2)"
    except OSError:
        pass
    return None, None


# ---------------------------------------------------------- clock sampling --
class ClockSampler:
    """Samples SM clocks and clock-event reasons of one GPU through NVML."""

    REASONS = {
        "hw_slowdown": 0x8,
        "sw_thermal_slowdown": 0x20,
        "hw_thermal_slowdown": 0x40,
        "hw_power_brake_slowdown": 0x80,
        "sw_power_cap": 0x4,
    }

    def __init__(self, device_index, period_s=0.01):
        self.samples = []
        self.max_mhz = None
        self.ok = False
        self.period = period_s
        self._stop = threading.Event()
        try:
            import pynvml

            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(device_index).uuid)
            if not uuid.startswith("GPU-"):
                uuid = "GPU-" + uuid
            self.h = pynvml.nvmlDeviceGetHandleByUUID(uuid)
            self.nvml = pynvml
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:  # noqa: BLE001 -- clocks are reported as unavailable
            self.ok = False

    def _run(self):
        nv = self.nvml
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((sm, reasons))
            except Exception:  # noqa: BLE001
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *exc):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0}
        sms = [s for s, _ in self.samples]
        active = set()
        for _, r in self.samples:
            for name, bit in self.REASONS.items():
                if r & bit:
                    active.add(name)
        return {"sm_mhz": float(statistics.median(sms)), "sm_max_mhz": self.max_mhz, "reasons": sorted(active),
                "samples": len(sms)}


# --------------------------------------------------------------- workloads --
class SpmmPowerlaw:
    """Power-law CSR SpMM (262144^2, Zipf 1.8, mean ~12, cap 20000, N = 64, fp32)."""

    metric = "CSR SpMM useful HBM throughput (chosen form)"
    e2e_what = ("per step: pinned host A then the dense operand -> device on an upload stream, "
                "prepare_spmm_csr_opt (validation, plan) once A is in, flagsparse_spmm_csr_opt once B is in, "
                "result -> pinned host on a download stream; steps pipelined (a step's uploads overlap the "
                "previous step's product and download), timed from the first upload to the last download")
    unit = "GB/s"

    def __init__(self, n_rows=262144, n_dense=64, seed=0):
        self.n_rows = n_rows
        self.n_dense = n_dense
        self.seed = seed

    def generate(self, device):
        """Seeded inputs only (no kernel of this project runs here)."""
        from flagsparse_public_b200 import synthetic

        data, indices, indptr, shape = synthetic.zipf_powerlaw(self.n_rows, self.n_rows, alpha=1.8, mean=12.0,
                                                               cap=20000, seed=self.seed, dtype=torch.float32,
                                                               device=device)
        B = synthetic.dense_operand(shape[1], self.n_dense, seed=self.seed + 1, dtype=torch.float32, device=device)
        self.A = (data, indices, indptr)
        self.shape = shape
        self.B = B
        self.nnz = data.numel()
        self.useful_bytes = self.nnz * (4 + 4) + shape[1] * self.n_dense * 4 + shape[0] * self.n_dense * 4
        self.flops = 2 * self.nnz * self.n_dense
        lens = (indptr[1:] - indptr[:-1])
        self.row_stats = {"mean_row": float(lens.float().mean()), "max_row": int(lens.max())}

    def build(self, device):
        import flagsparse_public_b200 as fs

        self.generate(device)
        data, indices, indptr = self.A
        self.C = torch.empty((self.shape[0], self.n_dense), dtype=torch.float32, device=device)
        self.prepared = fs.prepare_spmm_csr_opt(data, indices, indptr, self.shape)

    def config(self):
        return {
            "workload": f"csr_spmm_powerlaw_{self.shape[0]}x{self.shape[1]}_zipf1.8_mean12_cap20000_n{self.n_dense}"
                        "_f32_i32",
            "n_rows": self.shape[0], "n_cols": self.shape[1], "nnz": self.nnz, "n_dense": self.n_dense,
            "global_batch": 1, "useful_bytes_per_step": self.useful_bytes, **self.row_stats,
            "l2": "flushed before every timed step (256 MiB write)",
            "parallelism": "replicas",
        }

    def step(self):
        import flagsparse_public_b200 as fs

        fs.flagsparse_spmm_csr_opt(B=self.B, prepared=self.prepared, out=self.C)

    def plain_step(self):
        import flagsparse_public_b200.sparse_operations.spmm_csr as mm

        data, indices, indptr = self.A
        if not hasattr(self, "_alg1_plan"):
            holder = mm._Alg1Holder(data, indptr, self.shape[0], self.shape[1], self.row_stats["max_row"], self.nnz)
            self._alg1_plan = mm._spmm_plan_for(holder, "alg1", self.n_dense)
        mm._triton_spmm_csr_impl(data, indices, indptr, self.B, self.shape[0], self.n_dense, 0, 0,
                                 out=self.C, plan=self._alg1_plan)

    def plan_desc(self):
        from flagsparse_public_b200.sparse_operations.spmm_csr import _spmm_plan_for

        return _spmm_plan_for(self.prepared, "opt", self.n_dense).describe()

    def force_plan(self, plan):
        self.prepared._plans[("opt", self.n_dense)] = plan

    def selector_check(self, flush, steps=20, warmup=5):
        """The plan the learned selector picked for this matrix against
        exhaustive autotuning: every candidate timed with the bench protocol
        (L2 flushed, CUDA events), regret = chosen / best."""
        from flagsparse_public_b200 import _native as nat
        from flagsparse_public_b200 import _plan, tuning
        from flagsparse_public_b200.sparse_operations.spmm_csr import _spmm_plan_for

        data, indices, indptr = self.A
        times = {}
        for name, factory in tuning.SPMM_CANDIDATES:
            plan = factory()
            C = torch.empty_like(self.C)

            def run(plan=plan, C=C):
                _plan.run_spmm(data, indices, indptr, self.shape[0], self.shape[1], self.B, C, nat.ACC_NATIVE, plan)

            try:
                times[name] = _time_form(run, steps, warmup, flush, 1)
            except ValueError:  # a plan that cannot run these operands (BSR on float32 values)
                times[name] = None
        chosen = _spmm_plan_for(self.prepared, "opt", self.n_dense)
        chosen_name = next((n for n, f in tuning.SPMM_CANDIDATES if f().key() == chosen.key()), None)
        chosen_ms = _time_form(self.step, steps, warmup, flush, 1)
        best = min((n for n in times if times[n] is not None), key=times.get)
        return {"mode": _plan.plan_selector(), "chosen": chosen_name or chosen.describe(), "chosen_ms": chosen_ms,
                "autotune_best": best, "autotune_best_ms": times[best], "regret": chosen_ms / times[best],
                "candidates_ms": times,
                "what": "learned selector's plan (prepared path) vs exhaustive autotuning over every candidate "
                        "plan on this matrix, same timing protocol"}

    def gather_floor(self, flush, steps=20, warmup=5):
        """The gather floor of this product: fsb_gather_floor gathers the same
        B rows for the same column-index stream and does nothing else (every
        variant timed with the bench protocol, the fastest kept)."""
        from flagsparse_public_b200 import _native as nat

        lib = nat.library()
        _, indices, _ = self.A
        sms = torch.cuda.get_device_properties(self.B.device).multi_processor_count
        out = torch.empty(sms * 16 * 128, dtype=torch.float32, device=self.B.device)
        stream = nat.stream_handle(self.B.device)
        times = []
        for variant in range(nat.GATHER_FLOOR_VARIANTS):
            def run(variant=variant):
                rc = lib.fsb_gather_floor(nat.ptr(indices), self.nnz, nat.ptr(self.B), int(self.B.stride(0)),
                                          self.n_dense, nat.ptr(out), out.numel(), variant, stream)
                nat.check(rc, "fsb_gather_floor")

            times.append(_time_form(run, steps, warmup, flush, 1))
        best = min(range(len(times)), key=times.__getitem__)
        row_bytes = self.n_dense * 4
        return {"ms": times[best], "variant": best, "variants_ms": times,
                "gathered_rows_per_s": self.nnz / (times[best] * 1e-3),
                "gathered_gbs": self.nnz * row_bytes / (times[best] * 1e-3) / 1e9,
                "what": "fsb_gather_floor: the same B-row gathers (one 256-byte row per nonzero, same column "
                        "stream, L2 flushed) with no other work; the product's speed limit"}

    # end to end through the public API from pinned host memory
    def host_inputs(self):
        data, indices, indptr = self.A
        self.h = [t.cpu().pin_memory() for t in (data, indices, indptr, self.B)]
        self.h_out = torch.empty(self.C.shape, dtype=self.C.dtype).pin_memory()
        self.h2d_bytes = sum(t.numel() * t.element_size() for t in self.h)
        self.d2h_bytes = self.h_out.numel() * self.h_out.element_size()

    def e2e_step(self, device):
        import flagsparse_public_b200 as fs

        # A goes up on the current stream and is prepared (validated, planned)
        # while the dense operand B goes up on a side stream; the product
        # waits for both.  The side stream first waits for everything before
        # this step, so every copy stays inside the timed region.
        cur = torch.cuda.current_stream()
        if getattr(self, "_up", None) is None:
            self._up = torch.cuda.Stream(device=device)
            self._down = torch.cuda.Stream(device=device)
        # uploads run on their own stream, A first then B, without waiting for
        # the previous step's product: the prepare waits for A, the product
        # for B (e2e_start makes the first upload follow the timed region's
        # start)
        with torch.cuda.stream(self._up):
            d = [t.to(device, non_blocking=True) for t in self.h[:3]]
            a_ready = torch.cuda.Event()
            a_ready.record(self._up)
            dB = self.h[3].to(device, non_blocking=True)
        for t in d + [dB]:
            t.record_stream(cur)
        cur.wait_event(a_ready)
        prepared = fs.prepare_spmm_csr_opt(d[0], d[1], d[2], self.shape)
        cur.wait_stream(self._up)
        C = fs.flagsparse_spmm_csr_opt(B=dB, prepared=prepared)
        # the download runs on its own stream, next to the next step's uploads
        self._down.wait_stream(cur)
        with torch.cuda.stream(self._down):
            self.h_out.copy_(C, non_blocking=True)
        C.record_stream(self._down)

    def e2e_check(self):
        """The downloaded result of the last pipelined step equals the resident
        product (same matrix, operand and plan family)."""
        self.step()
        torch.cuda.synchronize()
        if not torch.allclose(self.h_out, self.C.cpu(), rtol=1e-5, atol=1e-6):
            raise RuntimeError("end-to-end result differs from the resident product")

    def e2e_start(self, device):
        """The first upload of a timed sequence follows the work queued so far
        (the timed region's start event)."""
        if getattr(self, "_up", None) is None:
            self._up = torch.cuda.Stream(device=device)
            self._down = torch.cuda.Stream(device=device)
        self._up.wait_stream(torch.cuda.current_stream())

    def e2e_finish(self, device):
        """Join the last step's download before the end of the timed region."""
        if getattr(self, "_down", None) is not None:
            torch.cuda.current_stream().wait_stream(self._down)

    def fp64_error(self):
        """Condition-scaled error of chosen and plain results vs the FP64 oracle."""
        from oracle import oracle as orc
        from tests.numerics import scaled_error

        data, indices, indptr = (t.cpu() for t in self.A)
        exact, mag = orc.spmm_csr_exact(data, indices, indptr, self.B.cpu())
        self.step()
        chosen = scaled_error(self.C.cpu(), exact, mag)
        self.plain_step()
        plain = scaled_error(self.C.cpu(), exact, mag)
        return {"chosen": chosen, "plain": plain, "definition": "max |c - c64| / sum_k |a_k b_k|"}

    def cpu_step_factory(self, threads, sample_rows=None):
        """Oracle port of FlagSparse's plain SpMM (float64 accumulation) on host cores."""
        from oracle import oracle as orc

        data, indices, indptr = (t.cpu() for t in self.A)
        B = self.B.cpu()
        rows = self.shape[0] if sample_rows is None else min(sample_rows, self.shape[0])
        sub_ptr = indptr[: rows + 1].clone()
        k = int(sub_ptr[-1])
        sub = (data[:k], indices[:k], sub_ptr)
        frac_bytes = k * 8 + self.shape[1] * self.n_dense * 4 + rows * self.n_dense * 4

        def run():
            orc.spmm_csr(sub[0], sub[1], sub[2], B, acc_mode=orc.ACC_WIDE, threads=threads)

        return run, frac_bytes, f"rows [0, {rows}) of the workload ({k} nonzeros), N = {self.n_dense}"


class SpmvPoisson:
    """CSR SpMV 16384^2, Poisson(16) rows, fp32 -- L2-resident, timed as a CUDA
    graph of 1000 back-to-back launches per step."""

    metric = "CSR SpMV useful throughput (L2-resident, graph of 1000 launches)"
    unit = "GB/s"
    graph_iters = 1000

    def generate(self, device):
        from flagsparse_public_b200 import synthetic

        data, indices, indptr, shape = synthetic.poisson_uniform(seed=0, device=device)
        self.A = (data, indices, indptr)
        self.shape = shape
        self.x = synthetic.dense_vector(shape[1], seed=1, device=device)
        self.nnz = data.numel()
        self.useful_bytes = (self.nnz * 8 + shape[1] * 4 + shape[0] * 4) * self.graph_iters
        self.flops = 2 * self.nnz * self.graph_iters

    def build(self, device):
        import flagsparse_public_b200 as fs

        self.generate(device)
        data, indices, indptr = self.A
        self.y = torch.empty(self.shape[0], device=device)
        self.prepared = fs.prepare_spmv_csr(data, indices, indptr, self.shape)
        fs.flagsparse_spmv_csr(x=self.x, prepared=self.prepared, out=self.y, use_opt=True)
        fs.flagsparse_spmv_csr(x=self.x, prepared=self.prepared, out=self.y, use_opt=False)
        self.graph = self._capture(use_opt=True)
        self.graph_plain = self._capture(use_opt=False)

    def _capture(self, use_opt):
        import flagsparse_public_b200 as fs

        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            for _ in range(3):
                fs.flagsparse_spmv_csr(x=self.x, prepared=self.prepared, out=self.y, use_opt=use_opt)
        torch.cuda.current_stream().wait_stream(s)
        with torch.cuda.graph(g):
            for _ in range(self.graph_iters):
                fs.flagsparse_spmv_csr(x=self.x, prepared=self.prepared, out=self.y, use_opt=use_opt)
        return g

    plain_desc = "float64 accumulation (FlagSparse plain), graph of 1000"

    def config(self):
        return {"workload": "csr_spmv_poisson16_16384x16384_f32_i32_graph1000", "n_rows": self.shape[0],
                "nnz": self.nnz, "global_batch": self.graph_iters,
                "l2": "L2-resident by design (2.2 MB working set)", "parallelism": "replicas"}

    def step(self):
        self.graph.replay()

    def plain_step(self):
        self.graph_plain.replay()

    def plan_desc(self):
        return self.graph_plan().describe()

    def graph_plan(self):
        from flagsparse_public_b200.sparse_operations.spmv_csr import _spmv_plan

        return _spmv_plan(self.prepared, "opt")

    def force_plan(self, plan):
        self.prepared._plans[("opt", 0)] = plan
        self.graph = self._capture(use_opt=True)

    e2e_what = ("per step: the step's A (values, column indices, row offsets) and x, packed in one pinned host "
                "buffer, -> device in one copy; the one-shot flagsparse_spmv_csr on them (structural check, its "
                "device->host read, plan, product in one native call); y -> pinned host.  Steps back to back on "
                "one stream (a look-ahead upload on a second stream measured slower: copies and the call's "
                "check contend)")

    def host_inputs(self):
        data, indices, indptr = self.A
        parts = [t.cpu() for t in (data, indices, indptr, self.x)]
        self._layout, off = [], 0
        for t in parts:
            nb = t.numel() * t.element_size()
            self._layout.append((off, nb, t.dtype))
            off += (nb + 15) // 16 * 16  # 16-byte aligned sections
        self.h_pack = torch.zeros(off, dtype=torch.uint8).pin_memory()
        for (o, nb, _dt), t in zip(self._layout, parts):
            self.h_pack[o:o + nb].copy_(t.view(torch.uint8))
        self.h_out = torch.empty(self.y.shape, dtype=self.y.dtype).pin_memory()
        self.h2d_bytes = off
        self.d2h_bytes = self.h_out.numel() * self.h_out.element_size()

    def e2e_step(self, device):
        import flagsparse_public_b200 as fs

        buf = self.h_pack.to(device, non_blocking=True)
        d = [buf[o:o + nb].view(dt) for o, nb, dt in self._layout]
        y = fs.flagsparse_spmv_csr(d[0], d[1], d[2], d[3], self.shape, use_opt=True)
        self.h_out.copy_(y, non_blocking=True)

    def e2e_check(self):
        """The last downloaded result equals the resident one-shot product."""
        import flagsparse_public_b200 as fs

        ref = fs.flagsparse_spmv_csr(*self.A, self.x, self.shape, use_opt=True)
        torch.cuda.synchronize()
        if not torch.equal(self.h_out, ref.cpu()):
            raise RuntimeError("end-to-end result differs from the resident product")

    def e2e_breakdown(self, device):
        """Each part of one step alone (us): the packed upload and the result
        download (CUDA events), the one-shot call on resident inputs (host
        wall time: check, read, plan, launch, product) and the product kernel
        (CUDA-graph time per SpMV)."""
        import time

        import flagsparse_public_b200 as fs

        def ev(fn, n=50):
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            for _ in range(n):
                fn()
            e.record()
            torch.cuda.synchronize()
            return s.elapsed_time(e) * 1e3 / n

        dbuf = torch.empty(self.h_pack.shape, dtype=torch.uint8, device=device)
        up = ev(lambda: dbuf.copy_(self.h_pack, non_blocking=True))
        down = ev(lambda: self.h_out.copy_(self.y, non_blocking=True))
        data, indices, indptr = self.A

        def call():
            fs.flagsparse_spmv_csr(data, indices, indptr, self.x, self.shape, use_opt=True)

        for _ in range(5):
            call()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(50):
            call()
        torch.cuda.synchronize()
        call_us = (time.perf_counter() - t0) * 1e6 / 50
        kern = ev(self.step, 5) / self.graph_iters
        return {"upload_us": round(up, 2), "oneshot_call_us": round(call_us, 2), "kernel_us": round(kern, 3),
                "download_us": round(down, 2)}

    def fp64_error(self):
        from oracle import oracle as orc
        from tests.numerics import scaled_error
        import flagsparse_public_b200 as fs

        data, indices, indptr = (t.cpu() for t in self.A)
        exact, mag = orc.spmv_csr_exact(data, indices, indptr, self.x.cpu())
        y1 = fs.flagsparse_spmv_csr(x=self.x, prepared=self.prepared, use_opt=True)
        y2 = fs.flagsparse_spmv_csr(x=self.x, prepared=self.prepared, use_opt=False)
        return {"chosen": scaled_error(y1, exact, mag), "plain": scaled_error(y2, exact, mag),
                "definition": "max |y - y64| / sum_k |a_k x_k|"}

    def cpu_step_factory(self, threads, sample_rows=None):
        from oracle import oracle as orc

        data, indices, indptr = (t.cpu() for t in self.A)
        x = self.x.cpu()
        per_call = self.nnz * 8 + self.shape[1] * 4 + self.shape[0] * 4

        def run():
            for _ in range(100):
                orc.spmv_csr(data, indices, indptr, x, acc_mode=orc.ACC_WIDE, threads=threads)

        return run, per_call * 100, "100 calls of the full SpMV"


class PrecisionBanded:
    """Precision form vs plain: 1,048,576-row banded-plus-random CSR (band 64
    + 4 uniform off-band columns, 1 % of rows with 8192 nonzeros).  Headline:
    bfloat16 SpMM (N = 32, float32 accumulation and output, compensated rows
    > 4096 nonzeros); beside it bfloat16 SpMV, the float16 runs and the
    float32 forms, each with its error against FP64 of the float32 data."""

    metric = "bf16-value CSR SpMM useful throughput (precision form)"
    dtype = "bf16"  # bf16 values and operand, fp32 accumulation
    unit = "GB/s"
    n_dense = 32
    plain_desc = "float32 values, float32 accumulation (same kernels)"

    def __init__(self, n_rows=1048576):
        self.n_rows = n_rows

    def generate(self, device):
        from flagsparse_public_b200 import synthetic

        data, indices, indptr, shape = synthetic.banded_plus_random(self.n_rows, seed=0, dtype=torch.float32,
                                                                   device=device)
        self.A = (data, indices, indptr)
        self.shape = shape
        self.x = synthetic.dense_vector(shape[1], seed=1, device=device)
        self.B = synthetic.dense_operand(shape[1], self.n_dense, seed=2, device=device)
        self.nnz = data.numel()
        n, N = shape[0], self.n_dense
        self.bytes = {
            "spmm_bf16": self.nnz * 6 + n * N * 2 + n * N * 4,
            "spmm_f32": self.nnz * 8 + n * N * 4 + n * N * 4,
            "spmv_bf16": self.nnz * 6 + n * 2 + n * 4,
            "spmv_f32": self.nnz * 8 + n * 4 + n * 4,
        }
        self.useful_bytes = self.bytes["spmm_bf16"]
        self.plain_bytes = self.bytes["spmm_f32"]
        self.flops = 2 * self.nnz * N
        lens = indptr[1:] - indptr[:-1]
        self.row_stats = {"mean_row": float(lens.float().mean()), "max_row": int(lens.max()),
                          "rows_over_4096": int((lens > 4096).sum())}

    def build(self, device):
        import flagsparse_public_b200 as fs

        self.generate(device)
        data, indices, indptr = self.A
        self.half = {}
        for dt in (torch.bfloat16, torch.float16):
            p = fs.prepare_csr_mixed(data.to(dt), indices, indptr, self.shape)
            self.half[dt] = (p, self.x.to(dt), self.B.to(dt))
        self.p32 = fs.prepare_spmv_csr(data, indices, indptr, self.shape)
        self.p32mm = fs.prepare_spmm_csr_opt(data, indices, indptr, self.shape)
        self.C = torch.empty((self.shape[0], self.n_dense), device=device)
        self.y = torch.empty(self.shape[0], device=device)

    def config(self):
        return {"workload": f"csr_banded64_plus4_long1pct8192_{self.shape[0]}_spmm_n{self.n_dense}_bf16",
                "n_rows": self.shape[0], "nnz": self.nnz, "n_dense": self.n_dense, "global_batch": 1,
                "useful_bytes_per_step": self.useful_bytes, **self.row_stats,
                "l2": "inputs larger than L2; flushed before every timed step (256 MiB write)",
                "parallelism": "replicas"}

    def _spmm_half(self, dt):
        import flagsparse_public_b200 as fs

        p, _x, Bh = self.half[dt]
        fs.flagsparse_spmm_csr_mixed(B=Bh, prepared=p, out=self.C)

    def _spmv_half(self, dt):
        import flagsparse_public_b200 as fs

        p, xh, _B = self.half[dt]
        fs.flagsparse_spmv_csr_mixed(x=xh, prepared=p, out=self.y)

    def step(self):
        self._spmm_half(torch.bfloat16)

    def plain_step(self):
        import flagsparse_public_b200 as fs

        fs.flagsparse_spmm_csr_opt(B=self.B, prepared=self.p32mm, out=self.C)

    def speedups(self, extra, ms_step, plain_ms):
        out = {"speedup_spmm_bf16_vs_f32": plain_ms / ms_step}
        if "spmv_bf16" in extra:
            out["speedup_spmv_bf16_vs_f32"] = extra["spmv_f32_fp32acc"]["ms_per_step"] / extra["spmv_bf16"]["ms_per_step"]
        return out

    def extra_forms(self):
        import flagsparse_public_b200 as fs

        return {
            "spmv_bf16": (lambda: self._spmv_half(torch.bfloat16), self.bytes["spmv_bf16"]),
            "spmv_f16": (lambda: self._spmv_half(torch.float16), self.bytes["spmv_bf16"]),
            "spmv_f32_fp32acc": (lambda: fs.flagsparse_spmv_csr(x=self.x, prepared=self.p32, out=self.y,
                                                                use_opt=True), self.bytes["spmv_f32"]),
            "spmv_f32_plain": (lambda: fs.flagsparse_spmv_csr(x=self.x, prepared=self.p32, out=self.y),
                               self.bytes["spmv_f32"]),
            "spmm_f16": (lambda: self._spmm_half(torch.float16), self.bytes["spmm_bf16"]),
            "spmm_f32_fp32acc": (self.plain_step, self.bytes["spmm_f32"]),
        }

    def plan_desc(self):
        from flagsparse_public_b200.sparse_operations.precision import _mixed_plan, _structured_form

        p = self.half[torch.bfloat16][0]
        form = _structured_form(p)
        if form is not None:
            return {"kind": "structured", "band": "tcgen05 tiles of 128 rows (K-major runs x MN-major B span)",
                    "long_rows": "tiles of 512 rows x 1024 columns streamed through shared memory"
                    if form.lt_rec is not None else "chunks of 1024 nonzeros", **form.stats()}
        return _mixed_plan(p, "spmm", self.n_dense).describe()

    def roofline_note(self, out):
        """The structured kernels read run values without indices and the long
        rows as prepared records: the bytes they must move, and the roofline
        fraction against them (the metric's useful bytes count int32 indices
        for every nonzero)."""
        from flagsparse_public_b200.sparse_operations.precision import _structured_form

        p = self.half[torch.bfloat16][0]
        form = _structured_form(p)
        if form is None:
            return {}
        moved = form.moved_bytes(self.shape[0], self.shape[1], 2, p.kernel_indptr.element_size(), self.n_dense)
        achieved = moved / (statistics.mean(out["times"]) * 1e-3) / 1e9
        return {"moved_bytes": moved, "achieved_moved": achieved, "frac_moved": achieved / out["roofline"]["peak"],
                "moved_what": "bytes the structured kernels must move (run values without indices, prepared "
                              "long-row records, B and C once)"}

    def force_plan(self, plan):
        self.half[torch.bfloat16][0]._plans[("spmm", self.n_dense)] = plan

    def host_inputs(self):
        data, indices, indptr = self.A
        self.h = [data.to(torch.bfloat16).cpu().pin_memory(), indices.cpu().pin_memory(), indptr.cpu().pin_memory(),
                  self.B.to(torch.bfloat16).cpu().pin_memory()]
        self.h_out = torch.empty(self.C.shape, dtype=torch.float32).pin_memory()
        self.h2d_bytes = sum(t.numel() * t.element_size() for t in self.h)
        self.d2h_bytes = self.h_out.numel() * self.h_out.element_size()

    def e2e_step(self, device):
        import flagsparse_public_b200 as fs

        d = [t.to(device, non_blocking=True) for t in self.h]
        C = fs.flagsparse_spmm_csr_mixed(d[0], d[1], d[2], d[3], self.shape)
        self.h_out.copy_(C, non_blocking=True)

    def fp64_error(self):
        """Errors vs FP64 of the float32 data (storage rounding + arithmetic),
        and of the same half inputs (arithmetic only), on a row sample."""
        from oracle import oracle as orc
        from tests.numerics import scaled_error

        data, indices, indptr = self.A
        rows = torch.arange(0, self.shape[0], 97, device=data.device)  # ~10.8 K rows incl. long ones
        lens = indptr[rows + 1] - indptr[rows]
        sub_ptr = torch.zeros(rows.numel() + 1, dtype=torch.int64, device=data.device)
        sub_ptr[1:] = torch.cumsum(lens, 0)
        gather = torch.repeat_interleave(indptr[rows] - sub_ptr[:-1], lens) + torch.arange(int(sub_ptr[-1]),
                                                                                             device=data.device)
        sub = (data[gather].cpu(), indices[gather].cpu(), sub_ptr.cpu())
        out = {}
        exact, mag = orc.spmm_csr_exact(*sub, self.B.cpu())
        for dt, name in ((torch.bfloat16, "bf16"), (torch.float16, "f16")):
            self._spmm_half(dt)
            got = self.C[rows].cpu()
            ex_h, mag_h = orc.spmm_csr_exact(sub[0].to(dt), sub[1], sub[2], self.B.cpu().to(dt))
            out[f"spmm_{name}_vs_fp64_of_f32_data"] = scaled_error(got, exact, mag)
            out[f"spmm_{name}_vs_fp64_same_inputs"] = scaled_error(got, ex_h, mag_h)
        self.plain_step()
        out["spmm_f32_fp32acc"] = scaled_error(self.C[rows].cpu(), exact, mag)
        ex_v, mag_v = orc.spmv_csr_exact(*sub, self.x.cpu())
        for dt, name in ((torch.bfloat16, "bf16"), (torch.float16, "f16")):
            self._spmv_half(dt)
            got = self.y[rows].cpu()
            ex_h, mag_h = orc.spmv_csr_exact(sub[0].to(dt), sub[1], sub[2], self.x.cpu().to(dt))
            out[f"spmv_{name}_vs_fp64_of_f32_data"] = scaled_error(got, ex_v, mag_v)
            out[f"spmv_{name}_vs_fp64_same_inputs"] = scaled_error(got, ex_h, mag_h)
        out["definition"] = "max |c - c64| / sum_k |a_k b_k| over every 97th row"
        return out

    def cpu_step_factory(self, threads, sample_rows=None):
        from oracle import oracle as orc

        data, indices, indptr = self.A
        rows = min(self.shape[0], 65536 if sample_rows is None else sample_rows)
        k = int(indptr[rows])
        sub = (data[:k].to(torch.bfloat16).cpu(), indices[:k].cpu(), indptr[: rows + 1].cpu())
        B = self.B.to(torch.bfloat16).cpu()
        nbytes = k * 6 + self.shape[1] * self.n_dense * 2 + rows * self.n_dense * 4

        def run():
            orc.spmm_csr(*sub, B, acc_mode=orc.ACC_NATIVE, out_dtype=torch.float32, threads=threads)

        return run, nbytes, f"rows [0, {rows}) ({k} nonzeros), bf16 inputs, f32 accumulation, N = {self.n_dense}"


class BatchedUneven:
    """512 independent square CSR matrices, rows log-uniform in [1024, 65536],
    Poisson row lengths with mean U[2, 64] per matrix, fp32 values, int32
    indices, each times its own 32-column N(0, 1) operand.  Chosen form: the
    batch stacked block-diagonally, one persistent launch of the batched
    merge-path kernel (plan from the autotuner) replayed from a CUDA graph.
    Plain form: FlagSparse's way, one flagsparse_spmm_csr call per matrix."""

    metric = "batched uneven CSR SpMM useful throughput (512 matrices, one graph launch)"
    unit = "GB/s"
    graph_iters = 1  # one captured launch pair per step
    n_mats = 512
    n_dense = 32

    def specs(self):
        import numpy as np

        rng = np.random.default_rng(0)
        out = []
        for i in range(self.n_mats):
            n = int(round(math.exp(rng.uniform(math.log(1024), math.log(65536)))))
            out.append((n, float(rng.uniform(2.0, 64.0)), int(rng.integers(1 << 30))))
        return out

    def generate(self, device):
        from flagsparse_public_b200 import synthetic

        self.mats = [synthetic.poisson_uniform(n, n, mean=m, seed=s, device=device) for n, m, s in self.specs()]
        self.nnz = sum(int(m[0].numel()) for m in self.mats)
        self.rows = sum(int(m[3][0]) for m in self.mats)
        self.useful_bytes = self.nnz * 8 + 2 * self.rows * self.n_dense * 4
        self.flops = 2 * self.nnz * self.n_dense

    def build(self, device):
        from flagsparse_public_b200 import batched, synthetic

        self.generate(device)
        self.prep = batched.prepare_spmm_csr_batch(self.mats, self.n_dense)
        self.prep.B.copy_(synthetic.dense_operand(self.prep.n_cols, self.n_dense, seed=1, device=device))
        self.prep.capture()
        self.plain_C = [torch.empty_like(c) for c in self.prep.c_views]
        self.seq_plans = [self.prep.plan.copy() for _ in self.mats]

    def config(self):
        return {"workload": "csr_spmm_batched512_rows1024to65536_poisson2to64_n32_f32_i32",
                "matrices": self.n_mats, "n_rows_total": self.rows, "nnz": self.nnz, "n_dense": self.n_dense,
                "global_batch": self.n_mats, "parallelism": "replicas",
                "l2": "inputs larger than L2 (4.3 GB); flushed before every timed step (256 MiB write)",
                "autotune_ms": self.prep.timings if hasattr(self, "prep") else None}

    def step(self):
        self.prep.graph.replay()

    plain_desc = "512 sequential flagsparse_spmm_csr calls (float64 accumulation, FlagSparse plain)"

    def plain_step(self):
        import flagsparse_public_b200 as fs

        for m, b, c in zip(self.mats, self.prep.b_views, self.plain_C):
            fs.flagsparse_spmm_csr(m[0], m[1], m[2], b, m[3], out=c)

    def _seq_each(self):
        from flagsparse_public_b200 import _plan

        for m, b, c, p in zip(self.mats, self.prep.b_views, self.plain_C, self.seq_plans):
            _plan.run_spmm(m[0], m[1], m[2], m[3][0], m[3][1], b, c, 0, p)

    def extra_forms(self):
        return {"sequential_batched_kernel": (self._seq_each, self.useful_bytes)}

    def speedups(self, extra, ms_step, plain_ms):
        return {"speedup_vs_sequential_plain": plain_ms / ms_step,
                "speedup_vs_sequential_same_kernel": extra["sequential_batched_kernel"]["ms_per_step"] / ms_step}

    def plan_desc(self):
        return self.prep.plan.describe()

    def graph_plan(self):
        return self.prep.plan

    def force_plan(self, plan):
        from flagsparse_public_b200 import batched

        self.prep = batched.prepare_spmm_csr_batch(self.mats, self.n_dense, plan=plan)
        self.prep.B.normal_()
        self.prep.capture()

    def host_inputs(self):
        self.h_B = self.prep.B.cpu().pin_memory()
        self.h_C = torch.empty(self.prep.C.shape, dtype=self.prep.C.dtype).pin_memory()
        self.h2d_bytes = self.h_B.numel() * self.h_B.element_size()
        self.d2h_bytes = self.h_C.numel() * self.h_C.element_size()

    e2e_what = ("matrices prepared once (resident); per step every dense operand pinned host -> device, "
                "one batch product, every result -> pinned host")

    def e2e_step(self, device):
        # the matrices are prepared once; each step moves every dense operand
        # in and every product out through the prepared batch
        self.prep.B.copy_(self.h_B, non_blocking=True)
        self.prep.run()
        self.h_C.copy_(self.prep.C, non_blocking=True)

    def fp64_error(self):
        from oracle import oracle as orc
        from tests.numerics import scaled_error

        self.prep.run()
        self.plain_step()
        torch.cuda.synchronize()
        worst = {"chosen": 0.0, "plain": 0.0}
        for i in range(0, self.n_mats, 32):  # every 32nd matrix
            m = self.mats[i]
            data, indices, indptr = (t.cpu() for t in m[:3])
            exact, mag = orc.spmm_csr_exact(data, indices, indptr, self.prep.b_views[i].cpu())
            worst["chosen"] = max(worst["chosen"], scaled_error(self.prep.c_views[i], exact, mag))
            worst["plain"] = max(worst["plain"], scaled_error(self.plain_C[i], exact, mag))
        worst["definition"] = "max |c - c64| / sum_k |a_k b_k| over every 32nd matrix"
        return worst

    def cpu_step_factory(self, threads, sample_rows=None):
        from oracle import oracle as orc

        picks = list(range(0, self.n_mats, 16))  # every 16th matrix
        host = [(tuple(t.cpu() for t in self.mats[i][:3]), self.prep.b_views[i].cpu()) for i in picks]
        nbytes = sum(a[0].numel() * 8 + 2 * b.shape[0] * self.n_dense * 4 for a, b in host)

        def run():
            for (data, indices, indptr), b in host:
                orc.spmm_csr(data, indices, indptr, b, acc_mode=orc.ACC_NATIVE, threads=threads)

        return run, nbytes, f"every 16th matrix ({len(picks)} of {self.n_mats}), N = {self.n_dense}"


class BsrTensorCore:
    """Block-sparse matrix of dense 16 x 16 blocks (65536 block rows = 1,048,576
    rows, 4 blocks per block row: the diagonal block and 3 uniform others;
    64 nonzeros per row), bf16 values, B 1,048,576 x 128 bf16, C fp32.
    Chosen form: BSR on the tensor cores (tcgen05, one 128 x 16 x 16 MMA per
    block).  Plain form: the same matrix as CSR through the CUDA-core SpMM
    (default plan, fp32 accumulation)."""

    metric = "BSR 16x16 SpMM useful throughput (tensor cores)"
    unit = "GB/s"
    dtype = "bf16"  # bf16 blocks and operand, fp32 accumulation in TMEM
    n_block_rows = 65536
    blocks_per_row = 4
    n_dense = 128

    def generate(self, device):
        from flagsparse_public_b200 import bsr, synthetic

        data, indices, indptr, shape = synthetic.block_sparse(self.n_block_rows, self.blocks_per_row, seed=0,
                                                              dtype=torch.bfloat16, device=device)
        self.csr = (data, indices, indptr)
        self.shape = shape
        self.bsr = bsr.csr_to_bsr16(data, indices, indptr, shape)
        self.B = synthetic.dense_operand(shape[1], self.n_dense, seed=1, dtype=torch.bfloat16, device=device)
        self.n_blocks = int(self.bsr[0].shape[0])
        self.nnz = int(data.numel())
        self.useful_bytes = (self.n_blocks * (256 * 2 + 4) + shape[1] * self.n_dense * 2
                             + shape[0] * self.n_dense * 4)
        self.plain_bytes = self.nnz * 6 + shape[1] * self.n_dense * 2 + shape[0] * self.n_dense * 4
        self.flops = 2 * self.n_blocks * 256 * self.n_dense

    def build(self, device):
        from flagsparse_public_b200 import _native as nat
        from flagsparse_public_b200 import _plan, bsr

        self.generate(device)
        self.prepared = bsr.prepare_spmm_bsr(*self.bsr, self.shape)
        self.C = torch.empty((self.shape[0], self.n_dense), dtype=torch.float32, device=device)
        self.C_plain = torch.empty_like(self.C)
        st = _plan.matrix_stats(self.csr[2], self.shape[0], self.shape[1])
        self.plain_plan = _plan.default_spmm_plan(st, self.n_dense, torch.bfloat16)
        self.acc = nat.ACC_NATIVE

    def config(self):
        return {"workload": "bsr16_blocksparse_65536x4blocks_1048576rows_n128_bf16",
                "n_rows": self.shape[0], "n_blocks": self.n_blocks, "nnz": self.nnz, "n_dense": self.n_dense,
                "global_batch": 1, "parallelism": "replicas",
                "l2": "inputs larger than L2 (134 MB blocks + 268 MB B, 537 MB C); flushed before every timed step "
                      "(256 MiB write)",
                "tensor_flops_per_step": self.flops}

    def step(self):
        from flagsparse_public_b200 import bsr

        bsr.flagsparse_spmm_bsr(B=self.B, prepared=self.prepared, out=self.C)

    plain_desc = "same matrix as CSR, CUDA-core SpMM (fp32 accumulation), useful bytes of the CSR form"

    def plain_step(self):
        from flagsparse_public_b200 import _plan

        d, i, p = self.csr
        _plan.run_spmm(d, i, p, self.shape[0], self.shape[1], self.B, self.C_plain, self.acc, self.plain_plan)

    def speedups(self, extra, ms_step, plain_ms):
        return {}

    def plan_desc(self):
        return {"kind": "bsr16_tcgen05", "tile_columns": 128, "mma": "128x16x16 kind::f16, fp32 in TMEM"}

    def force_plan(self, plan):
        self.plain_plan = plan

    def host_inputs(self):
        vals, bcol, bptr = self.bsr
        self.h = [t.cpu().pin_memory() for t in (vals, bcol, bptr, self.B)]
        self.h_out = torch.empty(self.C.shape, dtype=torch.float32).pin_memory()
        self.h2d_bytes = sum(t.numel() * t.element_size() for t in self.h)
        self.d2h_bytes = self.h_out.numel() * 4

    def e2e_step(self, device):
        from flagsparse_public_b200 import bsr

        d = [t.to(device, non_blocking=True) for t in self.h]
        C = bsr.flagsparse_spmm_bsr(d[0], d[1], d[2], d[3], self.shape)
        self.h_out.copy_(C, non_blocking=True)

    def fp64_error(self):
        from oracle import oracle as orc
        from tests.numerics import scaled_error

        self.step()
        self.plain_step()
        torch.cuda.synchronize()
        rows = 4096
        d, i, p = (t.cpu() for t in self.csr)
        end = int(p[rows])
        sub = (d[:end], i[:end], p[:rows + 1])
        exact, mag = orc.spmm_csr_exact(*sub, self.B.cpu())
        return {"chosen": scaled_error(self.C[:rows], exact, mag), "plain": scaled_error(self.C_plain[:rows], exact, mag),
                "definition": "max |c - c64| / sum_k |a_k b_k| over the first 4096 rows (FP64 of the same bf16 inputs)"}

    def cpu_step_factory(self, threads, sample_rows=None):
        from oracle import oracle as orc

        rows = 16384
        d, i, p = (t.cpu() for t in self.csr)
        end = int(p[rows])
        sub = (d[:end], i[:end], p[:rows + 1])
        Bh = self.B.cpu()
        nbytes = end * 6 + rows * self.n_dense * 6

        def run():
            orc.spmm_csr(*sub, Bh, acc_mode=orc.ACC_NATIVE, out_dtype=torch.float32, threads=threads)

        return run, nbytes, f"rows [0, {rows}) as CSR (bf16 inputs, fp32 accumulation), N = {self.n_dense}"


class SddmmPowerlaw:
    """SDDMM on the power-law CSR pattern of the SpMM config (262144^2,
    Zipf(1.8) rows, mean 12): out[p] = alpha * dot(x[row(p)], y[col(p)]) +
    beta * data[p], K = 64, float32 (float32 accumulation, as FlagSparse's
    kernel)."""

    metric = "CSR SDDMM useful HBM throughput"
    unit = "GB/s"
    plain_desc = "one-shot flagsparse_sddmm_csr call (pattern prepared inside every call)"
    k = 64
    alpha, beta = 2.0, 0.5

    def __init__(self, n_rows=262144, seed=0):
        self.n_rows = n_rows
        self.seed = seed

    def generate(self, device):
        """Seeded inputs only (no kernel of this project runs here)."""
        from flagsparse_public_b200 import synthetic

        data, indices, indptr, shape = synthetic.zipf_powerlaw(self.n_rows, self.n_rows, alpha=1.8, mean=12.0,
                                                               cap=20000, seed=self.seed, dtype=torch.float32,
                                                               device=device)
        self.A = (data, indices, indptr)
        self.shape = shape
        self.x = synthetic.dense_operand(shape[0], self.k, seed=self.seed + 1, dtype=torch.float32, device=device)
        self.y = synthetic.dense_operand(shape[1], self.k, seed=self.seed + 2, dtype=torch.float32, device=device)
        self.nnz = data.numel()
        # per position: index, data and output word; x and y rows once each
        self.useful_bytes = self.nnz * 12 + (shape[0] + shape[1]) * self.k * 4
        self.flops = 2 * self.nnz * self.k

    def build(self, device):
        import flagsparse_public_b200 as fs

        self.generate(device)
        data, indices, indptr = self.A
        self.out = torch.empty(self.nnz, dtype=torch.float32, device=device)
        self.prepared = fs.prepare_sddmm_csr(indices, indptr, self.shape, k_hint=self.k)

    def config(self):
        return {"workload": f"csr_sddmm_powerlaw_{self.shape[0]}x{self.shape[1]}_zipf1.8_mean12_cap20000_k{self.k}"
                            "_f32_i32",
                "n_rows": self.shape[0], "n_cols": self.shape[1], "nnz": self.nnz, "k": self.k,
                "alpha": self.alpha, "beta": self.beta, "global_batch": 1,
                "useful_bytes_per_step": self.useful_bytes,
                "l2": "flushed before every timed step (256 MiB write)", "parallelism": "replicas"}

    def step(self):
        import flagsparse_public_b200 as fs

        fs.flagsparse_sddmm_csr(self.A[0], x=self.x, y=self.y, alpha=self.alpha, beta=self.beta,
                                prepared=self.prepared, out=self.out)

    def plain_step(self):
        import flagsparse_public_b200 as fs

        data, indices, indptr = self.A
        fs.flagsparse_sddmm_csr(data, indices, indptr, self.x, self.y, self.shape, alpha=self.alpha, beta=self.beta,
                                out=self.out)

    def speedups(self, extra, ms_step, plain_ms):
        return {}

    def plan_desc(self):
        lanes = 1
        while lanes * 4 < self.k and lanes < 32:
            lanes *= 2
        return {"kind": "sddmm_subgroups", "lanes_per_position": lanes, "positions_per_batch": 4 * (32 // lanes)}

    def force_plan(self, plan):
        raise SystemExit("the SDDMM workload has no launch plans to force")

    def host_inputs(self):
        data, indices, indptr = self.A
        self.h = [t.cpu().pin_memory() for t in (data, indices, indptr, self.x, self.y)]
        self.h_out = torch.empty(self.out.shape, dtype=self.out.dtype).pin_memory()
        self.h2d_bytes = sum(t.numel() * t.element_size() for t in self.h)
        self.d2h_bytes = self.h_out.numel() * self.h_out.element_size()

    def e2e_step(self, device):
        import flagsparse_public_b200 as fs

        d = [t.to(device, non_blocking=True) for t in self.h]
        o = fs.flagsparse_sddmm_csr(d[0], d[1], d[2], d[3], d[4], self.shape, alpha=self.alpha, beta=self.beta)
        self.h_out.copy_(o, non_blocking=True)

    def fp64_error(self):
        from tests.numerics import scaled_error

        self.step()
        data, indices, indptr = (t.cpu() for t in self.A)
        sel = torch.arange(0, self.nnz, 97)
        rows = torch.searchsorted(indptr, sel, right=True) - 1
        xs, ys = self.x.cpu().double()[rows], self.y.cpu().double()[indices.long()[sel]]
        prod = xs * ys
        exact = self.alpha * prod.sum(1) + self.beta * data.double()[sel]
        mag = abs(self.alpha) * prod.abs().sum(1) + abs(self.beta) * data.double()[sel].abs()
        return {"chosen": scaled_error(self.out.cpu()[sel], exact, mag),
                "definition": "max |o - o64| / (|alpha| sum_k |x_k y_k| + |beta data|) over every 97th position"}

    def cpu_step_factory(self, threads, sample_rows=None):
        """Oracle port of FlagSparse's SDDMM kernel (float32 accumulation) on host cores."""
        from oracle import oracle as orc

        data, indices, indptr = (t.cpu() for t in self.A)
        rows = self.shape[0] if sample_rows is None else min(sample_rows, self.shape[0])
        sub_ptr = indptr[: rows + 1].clone()
        k = int(sub_ptr[-1])
        x, y = self.x.cpu(), self.y.cpu()
        nbytes = k * 12 + (rows + self.shape[1]) * self.k * 4

        def run():
            orc.sddmm_csr(indices[:k], sub_ptr, x[:rows], y, data[:k], self.alpha, self.beta, threads=threads)

        return run, nbytes, f"rows [0, {rows}) of the workload ({k} positions), K = {self.k}"


WORKLOADS = {"spmm_powerlaw": SpmmPowerlaw, "spmv_poisson": SpmvPoisson, "precision_banded": PrecisionBanded,
             "batched_uneven": BatchedUneven, "bsr_tensor_core": BsrTensorCore, "sddmm_powerlaw": SddmmPowerlaw}


# ------------------------------------------------------------------ timing --
def time_device_steps(fn, steps, flush):
    """CUDA-event time of each step on the current stream, L2 flushed before each."""
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    for i in range(steps):
        if flush is not None:
            flush.zero_()
        starts[i].record()
        fn()
        ends[i].record()
    torch.cuda.synchronize()
    return [s.elapsed_time(e) for s, e in zip(starts, ends)]


def time_cpu(run, min_seconds=10.0, max_seconds=30.0, min_reps=3):
    run()  # warm-up
    times = []
    t_end = time.perf_counter() + min_seconds
    while (len(times) < min_reps or time.perf_counter() < t_end) and sum(times) < max_seconds:
        t0 = time.perf_counter()
        run()
        times.append(time.perf_counter() - t0)
    return statistics.median(times), len(times)


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# -------------------------------------------------------------------- arms --
def run_reference(args):
    """FlagSparse's algorithm restated for the CPU (oracle port), host cores."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    wl = WORKLOADS[args.workload]()
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    wl.generate(dev)
    threads = cpu_threads()
    run, nbytes, sample = wl.cpu_step_factory(threads)
    for _ in range(max(args.warmup, 1)):
        run()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        run()
        times.append(time.perf_counter() - t0)
    ms = 1000.0 * statistics.mean(times)
    value = nbytes / (ms * 1e-3) / 1e9
    line = {
        "impl": "reference", "metric": wl.metric, "value": value, "unit": wl.unit, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": getattr(wl, "dtype", "f32"), "data": "synthetic",
        "config": wl.config(),
        "cpu_baseline": {"value": value, "unit": wl.unit, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": wl.unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def parse_plan(text):
    from flagsparse_public_b200 import _native as nat
    from flagsparse_public_b200 import _plan

    parts = text.split(":")
    kind, nums = parts[0], [int(v) for v in parts[1:]]
    if kind == "rows":
        return _plan.KernelPlan(nat.ALGO_ROWS, lanes=nums[0], n_tile=nums[1] if len(nums) > 1 else 0)
    if kind == "g4":
        return _plan.KernelPlan(nat.ALGO_SEQ, items_per_unit=nums[0], snap=nums[1] if len(nums) > 1 else 0,
                                n_tile=nums[2] if len(nums) > 2 else 0, flags=nat.PLAN_TMA_GATHER)
    algo = {"merge": nat.ALGO_MERGE, "flat": nat.ALGO_FLAT, "gather": nat.ALGO_GATHER, "seq": nat.ALGO_SEQ}[kind]
    return _plan.KernelPlan(algo, items_per_unit=nums[0], snap=nums[1] if len(nums) > 1 else 0,
                            n_tile=nums[2] if len(nums) > 2 else 0, grid_blocks=nums[3] if len(nums) > 3 else 0)


def _graph_kernels(wl):
    """Kernels one graph replay of a graph-timed workload launches."""
    from flagsparse_public_b200 import _plan

    plan = wl.graph_plan() if hasattr(wl, "graph_plan") else None
    per = _plan._kernels_per_call(plan) if plan is not None else 1
    return wl.graph_iters * per


def _time_form(fn, steps, warmup, flush, world):
    for _ in range(max(warmup, 1)):
        fn()
    torch.cuda.synchronize()
    return max_over_ranks(sum(time_device_steps(fn, steps, flush)), world) / steps


def _e2e(wl, device, steps, warmup, world):
    """End to end through the public API with host buffers (every step's
    host->device copies and its result's device->host copy timed)."""
    wl.host_inputs()
    finish = getattr(wl, "e2e_finish", None)
    start = getattr(wl, "e2e_start", None)
    if start is not None:
        start(device)
    for _ in range(max(1, min(warmup, 3))):
        wl.e2e_step(device)
    if finish is not None:
        finish(device)
    torch.cuda.synchronize()
    barrier(world)
    e_steps = max(3, min(steps, 20))
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    if start is not None:
        start(device)
    for _ in range(e_steps):
        wl.e2e_step(device)
    if finish is not None:
        finish(device)
    e.record()
    torch.cuda.synchronize()
    e_ms = max_over_ranks(s.elapsed_time(e), world) / e_steps
    check = getattr(wl, "e2e_check", None)
    if check is not None:
        check()
    per_step_bytes = wl.useful_bytes / getattr(wl, "graph_iters", 1)
    out = {"value": per_step_bytes * world / (e_ms * 1e-3) / 1e9, "unit": wl.unit, "ms_per_step": e_ms,
           "h2d_bytes_per_step": wl.h2d_bytes, "d2h_bytes_per_step": wl.d2h_bytes,
           "what": getattr(wl, "e2e_what", "pinned host A and dense operand -> device, public one-shot API "
                                           "(prepare + product), result -> pinned host")}
    breakdown = getattr(wl, "e2e_breakdown", None)
    if breakdown is not None:
        out["breakdown"] = breakdown(device)
    return out


def measure(wl, name, args, device, flush, world, rank, steps, warmup, cpu_seconds, with_e2e=True):
    """Every figure of one workload: the chosen form (device time, L2 flushed),
    the plain form, extra forms, end to end, FP64 error, CPU baseline."""
    from flagsparse_public_b200 import _plan

    for _ in range(warmup):
        wl.step()
    torch.cuda.synchronize()
    barrier(world)
    launches0 = _plan.LAUNCHES["count"]
    with ClockSampler(device.index or 0) as clocks:
        times = time_device_steps(wl.step, steps, flush)
    launches = _plan.LAUNCHES["count"] - launches0
    if getattr(wl, "graph_iters", 0):
        # graph replays launch the captured kernels without passing through Python
        launches = steps * _graph_kernels(wl)
    barrier(world)
    ms_step = max_over_ranks(sum(times), world) / steps
    value = aggregate_value(wl.useful_bytes, world, ms_step)
    out = {"ms_per_step": ms_step, "value": value, "unit": wl.unit, "times": times, "launches": launches,
           "clocks": clocks.summary()}
    plain_ms = _time_form(wl.plain_step, steps, warmup, flush, world)
    out["plain"] = {"value": getattr(wl, "plain_bytes", wl.useful_bytes) * world / (plain_ms * 1e-3) / 1e9,
                    "unit": wl.unit, "ms_per_step": plain_ms,
                    "form": getattr(wl, "plain_desc", "float64 accumulation (FlagSparse plain)")}
    extra = {}
    if hasattr(wl, "extra_forms"):
        for fname, (fn, nbytes) in wl.extra_forms().items():
            ms_x = _time_form(fn, steps, warmup, flush, world)
            extra[fname] = {"ms_per_step": ms_x, "value": nbytes * world / (ms_x * 1e-3) / 1e9, "unit": wl.unit}
        extra.update(wl.speedups(extra, ms_step, plain_ms))
    out["forms"] = extra or None
    out["e2e"] = _e2e(wl, device, steps, warmup, world) if with_e2e else None
    out["error_vs_fp64"] = wl.fp64_error() if rank == 0 else None
    cpu = None
    if rank == 0 and world == 1 and cpu_seconds > 0:
        threads = cpu_threads()
        run, nbytes, sample = wl.cpu_step_factory(threads)
        sec, reps = time_cpu(run, min_seconds=cpu_seconds, max_seconds=3 * cpu_seconds)
        cpu = {"value": nbytes / sec / 1e9, "unit": wl.unit, "cores": threads, "kind": "port",
               "sample": f"{sample}; median of {reps} runs", "ms": sec * 1e3}
    out["cpu_baseline"] = cpu
    peak, peak_kind = measured_peak_hbm()
    achieved = wl.useful_bytes / (statistics.mean(times) * 1e-3) / 1e9
    traffic, source = committed_traffic(f"traffic_{name}")
    out["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                       "peak_kind": peak_kind, "traffic": traffic, "traffic_source": source,
                       "what": "useful bytes / mean CUDA-event duration of one product call"}
    if hasattr(wl, "roofline_note"):
        out["roofline"].update(wl.roofline_note(out))
    out["plan"] = wl.plan_desc()
    out["gflops"] = wl.flops * world / (ms_step * 1e-3) / 1e9
    return out


# The configurations measured beside the headline in the default run (one
# JSON line): name -> (workload, steps, CPU-baseline seconds).
SIDE_CONFIGS = (
    ("spmv_poisson", 20, 3.0),
    ("precision_banded", 10, 3.0),
    ("batched_uneven", 10, 3.0),
    ("bsr_tensor_core", 20, 3.0),
    ("sddmm_powerlaw", 20, 3.0),
)


def _compact(m):
    keep = ("ms_per_step", "value", "unit", "plain", "forms", "e2e", "error_vs_fp64", "cpu_baseline", "roofline",
            "plan", "gflops", "launches", "clocks")
    return {k: m[k] for k in keep if k in m}


def run_ours(args):
    rank, world, local_rank = dist_env()
    init_dist(world)
    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=device)
    wl = WORKLOADS[args.workload]()
    wl.build(device)
    if args.plan:
        wl.force_plan(parse_plan(args.plan))

    if args.profile:
        fn = wl.step
        if args.form:
            forms = wl.extra_forms() if hasattr(wl, "extra_forms") else {}
            if args.form not in forms:
                raise SystemExit(f"workload {args.workload} has no form {args.form!r}: {sorted(forms)}")
            fn = forms[args.form][0]
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        times = time_device_steps(fn, args.steps, flush)
        if rank == 0:
            print(json.dumps({"profile_run": True, "ms_per_step": sum(times) / len(times)}), flush=True)
        return 0

    head = measure(wl, args.workload, args, device, flush, world, rank, args.steps, args.warmup,
                   0.0 if args.no_cpu else 10.0, with_e2e=not args.no_e2e)
    selector = wl.selector_check(flush) if hasattr(wl, "selector_check") and rank == 0 and not args.only else None
    if hasattr(wl, "gather_floor") and rank == 0:
        floor = wl.gather_floor(flush)
        floor["product_over_floor"] = head["ms_per_step"] / floor["ms"]
        head["roofline"]["gather_floor"] = floor
    config = {**wl.config(), "plan": head["plan"]}
    del wl
    torch.cuda.empty_cache()

    configs = {}
    if not args.only:
        for name, steps, cpu_s in SIDE_CONFIGS:
            if name == args.workload:
                continue
            side = WORKLOADS[name]()
            side.build(device)
            m = measure(side, name, args, device, flush, world, rank, min(args.steps, steps), max(3, args.warmup),
                        0.0 if args.no_cpu else cpu_s, with_e2e=not args.no_e2e)
            configs[name] = {"metric": side.metric, "dtype": getattr(side, "dtype", "f32"), "config": side.config(),
                             **_compact(m)}
            del side
            torch.cuda.empty_cache()

    if rank == 0:
        line = {
            "metric": WORKLOADS[args.workload].metric, "value": head["value"], "unit": head["unit"],
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": getattr(WORKLOADS[args.workload], "dtype", "f32"),
            "data": "synthetic (seeded generators, no dataset)", "config": config,
            "roofline": head["roofline"], "plain": head["plain"], "forms": head["forms"],
            "error_vs_fp64": head["error_vs_fp64"], "e2e": head["e2e"], "cpu_baseline": head["cpu_baseline"],
            "gpu_launches": head["launches"] + sum(c.get("launches", 0) for c in configs.values()),
            "gpu_launches_headline": head["launches"],
            "clocks": head["clocks"], "gflops": head["gflops"],
            "selector": selector,
            "configs": configs or None,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
