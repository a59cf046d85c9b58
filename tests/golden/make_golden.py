"""Generate golden vectors from FlagSparse's own SpMV/SpMM implementation.

Run where the FlagSparse sources are available, naming the project root:

    FLAGSPARSE_SRC=<FlagSparse project root> python tests/golden/make_golden.py

FlagSparse's package ``__init__`` does not import (its benchmarks module asks
``gather_scatter`` for a name it never defines), so the hot-path submodules are
loaded under stub parent packages, and its Triton kernels run on CPU tensors
under ``TRITON_INTERPRET=1``.  The kernels and the integer helpers are called
below FlagSparse's CUDA-only validators, with the same arguments its
``prepare_*`` functions would build.  Each case is saved with its seeded
inputs to ``tests/golden/<name>.pt`` (a dict of CPU tensors and scalars).

The fixtures pin the oracle (``oracle/``) and the CUDA kernels to the
reference's outputs; the test suite never reads the FlagSparse sources.
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


def load_reference():
    pkg = types.ModuleType("flagsparse")
    pkg.__path__ = [SRC]
    sys.modules["flagsparse"] = pkg
    sub = types.ModuleType("flagsparse.sparse_operations")
    sub.__path__ = [os.path.join(SRC, "sparse_operations")]
    sys.modules["flagsparse.sparse_operations"] = sub
    mods = {}
    for name in ("spmv_csr", "spmv_coo", "spmm_csr", "spmm_csr_opt_alg2", "spmm_coo"):
        mods[name] = importlib.import_module(f"flagsparse.sparse_operations.{name}")
    return mods


def rand_values(g, n, dtype):
    if dtype.is_complex:
        comp = torch.float32 if dtype == torch.complex64 else torch.float64
        return torch.complex(torch.rand(n, generator=g, dtype=comp) * 2 - 1,
                             torch.rand(n, generator=g, dtype=comp) * 2 - 1)
    return (torch.rand(n, generator=g, dtype=torch.float64) * 2 - 1).to(dtype)


def rand_dense(g, shape, dtype):
    if dtype.is_complex:
        comp = torch.float32 if dtype == torch.complex64 else torch.float64
        return torch.complex(torch.randn(shape, generator=g, dtype=comp), torch.randn(shape, generator=g, dtype=comp))
    return torch.randn(shape, generator=g, dtype=torch.float64).to(dtype)


def random_csr(seed, n_rows, n_cols, lengths, dtype, index_dtype=torch.int32, ptr_dtype=torch.int64):
    """CSR with the given row lengths, columns sorted and unique per row."""
    g = torch.Generator().manual_seed(seed)
    cols = []
    for ln in lengths:
        ln = min(int(ln), n_cols)
        cols.append(torch.sort(torch.randperm(n_cols, generator=g)[:ln]).values)
    lens = torch.tensor([c.numel() for c in cols], dtype=torch.int64)
    indptr = torch.zeros(n_rows + 1, dtype=torch.int64)
    indptr[1:] = torch.cumsum(lens, 0)
    indices = torch.cat(cols) if cols else torch.empty(0, dtype=torch.int64)
    data = rand_values(g, int(indptr[-1]), dtype)
    return data, indices.to(index_dtype), indptr.to(ptr_dtype), g


def skewed_lengths(seed, n_rows, mean, long_rows=(), long_len=0):
    g = torch.Generator().manual_seed(seed + 7)
    lens = torch.poisson(torch.full((n_rows,), float(mean)), generator=g).to(torch.int64)
    lens[::11] = 0  # empty rows
    for r in long_rows:
        lens[r] = long_len
    return lens.tolist()


def save(name, **case):
    path = os.path.join(HERE, f"{name}.pt")
    torch.save(case, path)
    print("wrote", path, {k: (tuple(v.shape), str(v.dtype)) if torch.is_tensor(v) else v for k, v in case.items()})


def spmv_cases(R):
    spmv = R["spmv_csr"]
    n_rows, n_cols = 96, 160
    for dtype, idt, pdt, use_opt, tag in (
        (torch.float32, torch.int32, torch.int64, False, "spmv_plain_f32"),
        (torch.float64, torch.int64, torch.int64, False, "spmv_plain_f64"),
        (torch.float16, torch.int32, torch.int32, False, "spmv_plain_f16"),
        (torch.bfloat16, torch.int32, torch.int64, False, "spmv_plain_bf16"),
        (torch.complex64, torch.int32, torch.int64, False, "spmv_plain_c64"),
        (torch.complex128, torch.int64, torch.int32, False, "spmv_plain_c128"),
        (torch.float32, torch.int32, torch.int32, True, "spmv_opt_f32"),
        (torch.float64, torch.int32, torch.int32, True, "spmv_opt_f64"),
    ):
        lens = skewed_lengths(1, n_rows, 12, long_rows=(5, 70), long_len=150)
        data, indices, indptr, g = random_csr(11, n_rows, n_cols, lens, dtype, idt, pdt)
        x = rand_dense(g, (n_cols,), dtype)
        rl = (indptr[1:] - indptr[:-1]).to(torch.int64)
        max_row = int(rl.max())
        block_nnz = 256
        max_segments = max((max_row + block_nnz - 1) // block_nnz, 1)
        buckets = spmv._build_spmv_opt_buckets(rl.to(indptr.dtype), max_row, torch.int32,
                                               fp64=dtype == torch.float64)
        p = spmv.PreparedCsrSpmv(data=data, kernel_indices=indices, kernel_indptr=indptr, shape=(n_rows, n_cols),
                                 n_rows=n_rows, n_cols=n_cols, block_nnz=block_nnz, max_segments=max_segments,
                                 max_row_nnz=max_row, opt_buckets=buckets)
        if use_opt:
            y = spmv._triton_spmv_csr_impl_opt_prepared(p, x)
        else:
            y = spmv._triton_spmv_csr_impl_prepared(p, x)
        save(tag, data=data, indices=indices, indptr=indptr, x=x, y=y, shape=(n_rows, n_cols), use_opt=use_opt)

    # Plain path with a segment window shorter than the longest rows:
    # rows are truncated to block_nnz * max_segments nonzeros.
    lens = skewed_lengths(2, 40, 20, long_rows=(3, 17), long_len=90)
    data, indices, indptr, g = random_csr(12, 40, 128, lens, torch.float32)
    x = rand_dense(g, (128,), torch.float32)
    rl = indptr[1:] - indptr[:-1]
    p = spmv.PreparedCsrSpmv(data=data, kernel_indices=indices, kernel_indptr=indptr, shape=(40, 128), n_rows=40,
                             n_cols=128, block_nnz=16, max_segments=2, max_row_nnz=int(rl.max()), opt_buckets=[])
    y = spmv._triton_spmv_csr_impl_prepared(p, x)
    save("spmv_plain_capped", data=data, indices=indices, indptr=indptr, x=x, y=y, shape=(40, 128), block_nnz=16,
         max_segments=2)

    # Structure: transpose and COO -> CSR.
    lens = skewed_lengths(3, 50, 6)
    data, indices, indptr, g = random_csr(13, 50, 37, lens, torch.complex64, torch.int32, torch.int64)
    td, ti, tp, tshape = spmv._transpose_csr_for_spmv(data, indices, indptr, (50, 37))
    save("transpose_c64", data=data, indices=indices, indptr=indptr, t_data=td, t_indices=ti, t_indptr=tp,
         shape=(50, 37), t_shape=tshape)
    gperm = torch.Generator().manual_seed(14)
    counts = indptr[1:] - indptr[:-1]
    row = torch.repeat_interleave(torch.arange(50), counts)
    perm = torch.randperm(row.numel(), generator=gperm)
    row_u, col_u, data_u = row[perm], indices.to(torch.int64)[perm], data[perm]
    d2, i2, p2 = spmv.coo_to_csr_for_spmv(data_u, row_u, col_u, (50, 37))
    save("coo_to_csr", data=data_u, row=row_u, col=col_u, out_data=d2, out_indices=i2, out_indptr=p2,
         shape=(50, 37))


def spmv_coo_cases(R):
    coo = R["spmv_coo"]
    for dtype, tag, sort_by_row in ((torch.float32, "spmv_coo_seg_f32", True),
                                    (torch.complex128, "spmv_coo_seg_c128", True),
                                    (torch.float64, "spmv_coo_atomic_f64", False)):
        lens = skewed_lengths(4, 60, 5)
        data, indices, indptr, g = random_csr(15, 60, 80, lens, dtype, torch.int64, torch.int64)
        counts = indptr[1:] - indptr[:-1]
        row = torch.repeat_interleave(torch.arange(60), counts)
        perm = torch.randperm(row.numel(), generator=g)
        row, col, data = row[perm], indices[perm], data[perm]
        x = rand_dense(g, (80,), dtype)
        if sort_by_row:
            d, kr, kc = coo._sort_coo_lex_inplace(data, row, col, 80)
            seg = coo._seg_starts_from_sorted_rows(kr, d.numel(), d.device)
        else:
            d, kr, kc, seg = data, row, col, None
        p = coo.PreparedCoo(d, kr, kc, (60, 80), seg_starts=seg)
        y = coo._triton_spmv_coo_kernel(p, x, block_size=256, num_warps=4, block_inner=128)
        case = dict(data=data, row=row, col=col, x=x, y=y, shape=(60, 80), sorted_data=d, sorted_row=kr,
                    sorted_col=kc, sort_by_row=sort_by_row)
        if seg is not None:
            case["seg_starts"] = seg
        save(tag, **case)


def spmm_cases(R):
    mm = R["spmm_csr"]
    alg2 = R["spmm_csr_opt_alg2"]
    for dtype, n_dense, tag in ((torch.float32, 16, "spmm_alg1_f32"), (torch.float64, 7, "spmm_alg1_f64"),
                                (torch.float16, 8, "spmm_alg1_f16"), (torch.complex64, 5, "spmm_alg1_c64")):
        lens = skewed_lengths(5, 48, 6, long_rows=(9,), long_len=40)
        data, indices, indptr, g = random_csr(16, 48, 64, lens, dtype, torch.int32, torch.int64)
        B = rand_dense(g, (64, n_dense), dtype)
        rl = indptr[1:] - indptr[:-1]
        launch = mm._resolve_spmm_alg1_launch_config(n_dense, int(rl.max()))
        C = mm._triton_spmm_csr_impl(data, indices, indptr, B, 48, n_dense, launch["block_n"], launch["block_nnz"])
        save(tag, data=data, indices=indices, indptr=indptr, B=B, C=C, shape=(48, 64))

    # Opt path including the long-row split bucket (> 2048 nonzeros).
    lens = skewed_lengths(6, 24, 10, long_rows=(4,), long_len=2300)
    data, indices, indptr, g = random_csr(17, 24, 2400, lens, torch.float32, torch.int32, torch.int64)
    B = rand_dense(g, (2400, 12), torch.float32)
    rl = indptr[1:] - indptr[:-1]
    buckets, long_rows = mm._build_spmm_opt_buckets(rl)
    lpr, lps, lpe, lrpp = mm._build_spmm_opt_split_metadata(indptr, long_rows, part_block_nnz=256)
    p = mm.PreparedCsrSpmmOpt(data=data, kernel_indices=indices, kernel_indptr=indptr, shape=(24, 2400), n_rows=24,
                              n_cols=2400, row_lengths=rl, max_row_nnz=int(rl.max()), row_buckets=buckets,
                              long_part_rows=lpr, long_part_starts=lps, long_part_ends=lpe, long_row_ids=long_rows,
                              long_row_part_ptr=lrpp, long_row_fallback_only=False)
    block_n = mm._select_spmm_opt_block_n(12)
    C = torch.zeros((24, 12), dtype=torch.float32)
    for bucket in buckets:
        if bucket["kind"] == "split":
            mm._run_spmm_opt_split_bucket(p, B, C, block_n)
        else:
            mm._run_spmm_opt_bucket(p, bucket, B, C, block_n)
    save("spmm_opt_split_f32", data=data, indices=indices, indptr=indptr, B=B, C=C, shape=(24, 2400),
         long_rows=long_rows, part_rows=lpr, part_starts=lps, part_ends=lpe, row_part_ptr=lrpp)

    # alg2 (device-aware buckets), float64, one row in every bucket.
    lens = [0, 3, 16, 17, 40, 64, 65, 200, 256, 257, 700, 1024, 1025, 1300] * 2
    data, indices, indptr, g = random_csr(18, len(lens), 1400, lens, torch.float64, torch.int32, torch.int64)
    B = rand_dense(g, (1400, 9), torch.float64)
    rl = indptr[1:] - indptr[:-1]
    props = {"device_name": "cpu", "warp_size": 32, "sm_count": 148, "max_threads_per_mp": 2048,
             "max_threads_per_block": 1024, "shared_memory_per_block": 49152, "capability": (10, 0)}
    buckets = alg2._build_spmm_opt_alg2_buckets(rl, torch.float64)
    p = alg2.PreparedCsrSpmmOptAlg2(data=data, kernel_indices=indices, kernel_indptr=indptr,
                                    shape=(len(lens), 1400), n_rows=len(lens), n_cols=1400, row_lengths=rl,
                                    max_row_nnz=int(rl.max()), opt_buckets=buckets)
    C = torch.zeros((len(lens), 9), dtype=torch.float64)
    for bucket in buckets:
        alg2._run_spmm_opt_alg2_bucket(p, bucket, B, C, props)
    save("spmm_alg2_f64", data=data, indices=indices, indptr=indptr, B=B, C=C, shape=(len(lens), 1400))

    # Long-row API case of FlagSparse's tests/test_spmm.py:401-413 (row of 1536
    # nonzeros plus a 4-nonzero row, shape (2, 2048), 48 dense columns).
    g = torch.Generator().manual_seed(19)
    indices = torch.cat([torch.arange(1536), torch.tensor([7, 129, 511, 1024])]).to(torch.int32)
    indptr = torch.tensor([0, 1536, 1540], dtype=torch.int64)
    data = rand_values(g, 1540, torch.float32)
    B = rand_dense(g, (2048, 48), torch.float32)
    launch = mm._resolve_spmm_alg1_launch_config(48, 1536)
    C = mm._triton_spmm_csr_impl(data, indices, indptr, B, 2, 48, launch["block_n"], launch["block_nnz"])
    save("spmm_long_row_f32", data=data, indices=indices, indptr=indptr, B=B, C=C, shape=(2, 2048))


def spmm_coo_cases(R):
    mc = R["spmm_coo"]
    lens = skewed_lengths(8, 40, 4)
    data, indices, indptr, g = random_csr(20, 40, 50, lens, torch.float32, torch.int64, torch.int64)
    counts = indptr[1:] - indptr[:-1]
    row = torch.repeat_interleave(torch.arange(40), counts)
    # duplicate a few entries (coalesce sums them) and shuffle
    dup = torch.arange(0, row.numel(), 9)
    row = torch.cat([row, row[dup]])
    col = torch.cat([indices, indices[dup]])
    data = torch.cat([data, rand_values(g, dup.numel(), torch.float32)])
    perm = torch.randperm(row.numel(), generator=g)
    row, col, data = row[perm], col[perm], data[perm]
    B = rand_dense(g, (50, 10), torch.float32)
    (cd, cr, cc, cB, n_rows, n_cols, n_dense, out_dtype, comp_dtype) = mc._prepare_spmm_coo_canonical_prepared(
        data, row.to(torch.int32), col.to(torch.int32), B, 40, 50, 10)
    C = mc._triton_spmm_coo_rowrun_impl(cd, cr, cc, cB, 40, 10, 32, 256, output_dtype=out_dtype)
    coal_d, coal_r, coal_c = mc._coalesce_coo_entries(data, row, col, (40, 50))
    save("spmm_coo_f32", data=data, row=row, col=col, B=B, C=C, shape=(40, 50), coalesced_data=coal_d,
         coalesced_row=coal_r, coalesced_col=coal_c)


def main():
    torch.set_num_threads(max(1, os.cpu_count() or 1))
    R = load_reference()
    spmv_cases(R)
    spmv_coo_cases(R)
    spmm_cases(R)
    spmm_coo_cases(R)


if __name__ == "__main__":
    main()
