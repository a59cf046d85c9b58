// fsb_spmm.cu -- CSR SpMM on sm_100a: C = A B, B and C row-major.
//
// Lane layout.  A dense column tile of LPN * VW columns is covered by LPN lanes
// holding VW consecutive columns each (VW * sizeof(V) = 16 bytes when B and C
// rows are 16-byte aligned, else VW = 1).  A group of G lanes (G a multiple of
// LPN) works on one row; its G / LPN sub-groups take interleaved nonzeros so
// that G / LPN B rows are in flight per step, and meet in a xor butterfly at
// the end of the row.  Column indices and values are read once per group with
// coalesced streaming loads and handed out by warp shuffles; B rows are
// gathered with 16-byte read-only loads (B stays in L2), C rows are written
// with streaming stores.
//
//   * k_spmm_rows  : row groups over rows (G = 32: warp per row; G = LPN:
//                    vector per row).
//   * k_spmm_merge : one warp per merge-path unit (rows + nonzeros balanced);
//                    rows split across units leave a carry / head partial in
//                    scratch that k_spmm_merge_fixup folds in, in unit order.
//
// FlagSparse computes the same products in _spmm_csr_real/complex_kernel
// (spmm_csr.py:92-195), the opt bucket kernels (:602-775), the long-row split
// kernels (:778-919), the alg2 kernels (spmm_csr_opt_alg2.py:338-629) and the
// COO row-run kernels (spmm_coo.py:135-241).
#include "fsb_spmm_common.cuh"
#include "fsb_spmm_seq.cuh"

namespace fsb {

constexpr int kSpmmUnroll = 4;

struct Lanes {
    int G;       // lanes per row group
    int LPN;     // lanes per B row (column tile)
    int lig;     // lane in group
    int sub;     // sub-group (nonzero slot) of this lane
    unsigned mask;
};

template <class V, class A, class I, int VW>
__device__ __forceinline__ void row_segment(const V* __restrict__ val, const I* __restrict__ col,
                                            const V* __restrict__ B, int64_t ldb, int64_t c0, bool col_ok,
                                            int64_t a, int64_t b, A (&acc)[VW], const Lanes& L) {
    const int NPAR = L.G / L.LPN;
    for (int64_t base = a; base < b; base += L.G) {
        const int cnt = (b - base) < (int64_t)L.G ? (int)(b - base) : L.G;
        V v = vzero<V>();
        I c = 0;
        if (L.lig < cnt) {
            v = ld_stream1(val + base + L.lig);
            c = ld_stream1(col + base + L.lig);
        }
        for (int j = 0; j < cnt; j += NPAR * kSpmmUnroll) {
            vec_t<V, VW> bv[kSpmmUnroll];
            V av[kSpmmUnroll];
#pragma unroll
            for (int u = 0; u < kSpmmUnroll; ++u) {
                const int jj = j + u * NPAR + L.sub;
                const V vv = shfl_idx(L.mask, v, jj & (L.G - 1), L.G);
                const I cc = shfl_idx(L.mask, c, jj & (L.G - 1), L.G);
                const bool ok = (jj < cnt) && col_ok;
                av[u] = ok ? vv : vzero<V>();
                if (ok) {
                    bv[u] = ld_ro<V, VW>(B + idx(cc) * ldb + c0);
                } else {
#pragma unroll
                    for (int w = 0; w < VW; ++w) bv[u].v[w] = vzero<V>();
                }
            }
#pragma unroll
            for (int u = 0; u < kSpmmUnroll; ++u)
#pragma unroll
                for (int w = 0; w < VW; ++w) acc[w] = Acc<V, A>::fma(av[u], bv[u].v[w], acc[w]);
        }
    }
}


template <class V, class A, class I, int VW>
__device__ __forceinline__ void row_accumulate(const V* __restrict__ val, const I* __restrict__ col,
                                               const V* __restrict__ B, int64_t ldb, int64_t c0, bool col_ok,
                                               int64_t a, int64_t b, int64_t row_len, int64_t comp_threshold,
                                               A (&acc)[VW], const Lanes& L) {
    if constexpr (is_comp_acc<A>::value) {
        if (row_len > comp_threshold) {
            row_segment<V, comp_t, I, VW>(val, col, B, ldb, c0, col_ok, a, b, acc, L);
        } else {
            float plain[VW];
#pragma unroll
            for (int w = 0; w < VW; ++w) plain[w] = 0.f;
            row_segment<V, float, I, VW>(val, col, B, ldb, c0, col_ok, a, b, plain, L);
#pragma unroll
            for (int w = 0; w < VW; ++w) acc[w] = acc_add(acc[w], comp_t{plain[w], 0.f});
        }
    } else {
        row_segment<V, A, I, VW>(val, col, B, ldb, c0, col_ok, a, b, acc, L);
    }
}

template <class V, class A, class O, class I, class P, int VW>
__global__ void __launch_bounds__(kSpmmThreads)
k_spmm_rows(const V* __restrict__ val, const I* __restrict__ col, const P* __restrict__ ptr,
            const I* __restrict__ row_map, const V* __restrict__ B, int64_t ldb, O* __restrict__ C, int64_t ldc,
            int64_t n_rows, int64_t n_dense, int g_log2, int lpn_log2, int64_t row_cap, int64_t comp_threshold) {
    Lanes L;
    L.G = 1 << g_log2;
    L.LPN = 1 << lpn_log2;
    const int wl = threadIdx.x & 31;
    L.lig = wl & (L.G - 1);
    L.sub = L.lig >> lpn_log2;
    L.mask = segment_mask(wl, L.G);
    const int64_t c0 = (int64_t)blockIdx.y * (L.LPN * VW) + (int64_t)(L.lig & (L.LPN - 1)) * VW;
    const bool col_ok = c0 < n_dense;
    const int64_t stride = ((int64_t)gridDim.x * blockDim.x) >> g_log2;
    for (int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> g_log2; row < n_rows; row += stride) {
        const int64_t s = idx(ptr[row]);
        int64_t e = idx(ptr[row + 1]);
        if (row_cap > 0 && e - s > row_cap) e = s + row_cap;
        A acc[VW];
#pragma unroll
        for (int w = 0; w < VW; ++w) acc[w] = Acc<V, A>::zero();
        row_accumulate<V, A, I, VW>(val, col, B, ldb, c0, col_ok, s, e, e - s, comp_threshold, acc, L);
#pragma unroll
        for (int w = 0; w < VW; ++w) acc[w] = segment_reduce(L.mask, acc[w], L.LPN, L.G);
        if (L.sub == 0 && col_ok) {
            const int64_t out_row = row_map ? idx(row_map[s]) : row;
            store_row<O, A, VW>(C, ldc, out_row, c0, acc);
        }
    }
}

// One warp per (unit, column tile).  unit_coords as in fsb_merge_partition.
template <class V, class A, class O, class I, class P, int VW>
__global__ void __launch_bounds__(kSpmmThreads)
k_spmm_merge(const V* __restrict__ val, const I* __restrict__ col, const P* __restrict__ ptr,
             const I* __restrict__ row_map, const V* __restrict__ B, int64_t ldb, O* __restrict__ C, int64_t ldc,
             int64_t n_rows, int64_t n_dense, int lpn_log2, const int64_t* __restrict__ coords, int64_t n_units,
             int64_t comp_threshold, int64_t* __restrict__ carry_row, A* __restrict__ carry_val,
             A* __restrict__ head_val) {
    const int64_t unit = (int64_t)blockIdx.x * (kSpmmThreads / 32) + (threadIdx.x >> 5);
    if (unit >= n_units) return;
    Lanes L;
    L.G = 32;
    L.LPN = 1 << lpn_log2;
    L.lig = threadIdx.x & 31;
    L.sub = L.lig >> lpn_log2;
    L.mask = 0xffffffffu;
    const int64_t c0 = (int64_t)blockIdx.y * (L.LPN * VW) + (int64_t)(L.lig & (L.LPN - 1)) * VW;
    const bool col_ok = c0 < n_dense;

    const int64_t r0 = coords[2 * unit], k0 = coords[2 * unit + 1];
    const int64_t r1 = coords[2 * unit + 2], k1 = coords[2 * unit + 3];
    const int64_t last = r1 < n_rows ? r1 : r1 - 1;
    int64_t s_next = r0 < n_rows ? idx(ptr[r0]) : k1;
    const bool continued = (r0 < n_rows) && (k0 > s_next);
    bool open = false;
    for (int64_t r = r0; r <= last; ++r) {
        const int64_t rs = s_next;
        const int64_t re_full = idx(ptr[r + 1]);
        s_next = re_full;
        const int64_t a = rs > k0 ? rs : k0;
        const int64_t b = (r < r1) ? re_full : k1;
        if (r == r1 && b <= a) break;  // open row untouched by this unit
        A acc[VW];
#pragma unroll
        for (int w = 0; w < VW; ++w) acc[w] = Acc<V, A>::zero();
        row_accumulate<V, A, I, VW>(val, col, B, ldb, c0, col_ok, a, b, re_full - rs, comp_threshold, acc, L);
#pragma unroll
        for (int w = 0; w < VW; ++w) acc[w] = segment_reduce(L.mask, acc[w], L.LPN, 32);
        if (L.sub == 0 && col_ok) {
            if (r == r1) {
                A* dst = carry_val + unit * n_dense + c0;
#pragma unroll
                for (int w = 0; w < VW; ++w) dst[w] = acc[w];
            } else if (r == r0 && continued) {
                A* dst = head_val + unit * n_dense + c0;
#pragma unroll
                for (int w = 0; w < VW; ++w) dst[w] = acc[w];
            } else {
                const int64_t out_row = row_map ? idx(row_map[rs]) : r;
                store_row<O, A, VW>(C, ldc, out_row, c0, acc);
            }
        }
        if (r == r1) open = true;
    }
    if (blockIdx.y == 0 && L.lig == 0) carry_row[unit] = open ? r1 : -1;
}

// ------------------------------------------------------------ flat units ----
// One warp per (merge-path unit, column tile of LPN * VW columns).  Lane l owns
// columns [c0, c0 + VW) of the tile (16-byte vectors) and sub-group
// s = l / LPN takes every NPAR-th nonzero of the unit's stream (NPAR = 32 /
// LPN), so one warp step advances NPAR nonzeros.  The unit's values and column
// indices stream through a 32-entry register window (the next window is
// prefetched), row ends through a second 32-entry window, and kFlatU steps of
// B rows are gathered before they are accumulated.  When a step crosses the
// current row's end, the sub-groups' partials meet in a xor butterfly and the
// row is flushed: to C, or -- for the unit's first row when it began in an
// earlier unit -- to head_val; the row left open at the unit's end goes to
// carry_val (folded in by k_spmm_merge_fixup, in unit order).
constexpr int kFlatU = 4;

template <class V, class A, class O, class I, class P, int VW, bool ADDR32>
__global__ void __launch_bounds__(kSpmmThreads)
k_spmm_flat(const V* __restrict__ val, const I* __restrict__ col, const P* __restrict__ ptr,
            const I* __restrict__ row_map, const V* __restrict__ B, int64_t ldb, O* __restrict__ C, int64_t ldc,
            int64_t n_rows, int64_t n_dense, int lpn_log2, const int64_t* __restrict__ coords, int64_t n_units,
            int64_t* __restrict__ carry_row, A* __restrict__ carry_val, A* __restrict__ head_val) {
    const int lane = threadIdx.x & 31;
    const int64_t unit = (int64_t)blockIdx.x * (kSpmmThreads / 32) + (threadIdx.x >> 5);
    if (unit >= n_units) return;
    const unsigned full = 0xffffffffu;
    const int LPN = 1 << lpn_log2;
    const int NPAR = 32 >> lpn_log2;
    const int sub = lane >> lpn_log2;
    const int U = NPAR * kFlatU <= 32 ? kFlatU : 32 / NPAR;  // steps per batch, batch stays in one window
    const int64_t c0 = (int64_t)blockIdx.y * (LPN * VW) + (int64_t)(lane & (LPN - 1)) * VW;
    const bool col_ok = c0 < n_dense;

    const int64_t r0 = coords[2 * unit], k0 = coords[2 * unit + 1];
    const int64_t r1 = coords[2 * unit + 2], k1 = coords[2 * unit + 3];
    const int64_t last_row = r1 < n_rows ? r1 : r1 - 1;  // last row this unit touches
    constexpr int64_t kNoEnd = INT64_MAX;

    // Row-end window: lane l holds ptr[rb + l + 1] (rows rb .. rb + 31).
    int64_t rb = r0;
    int64_t e_win = (rb + lane <= last_row) ? idx(ptr[rb + lane + 1]) : kNoEnd;
    int64_t row = r0;
    int64_t row_start = (r0 < n_rows) ? idx(ptr[r0]) : k0;
    const bool continued = (r0 < n_rows) && (k0 > row_start);
    int64_t row_end = (r0 <= last_row) ? __shfl_sync(full, e_win, 0) : kNoEnd;

    // Nonzero windows: lane l holds entry kb + l (current) and kb + 32 + l (next).
    int64_t kb = k0;
    V v_cur = vzero<V>(), v_nxt = vzero<V>();
    I c_cur = 0, c_nxt = 0;
    if (kb + lane < k1) { v_cur = ld_stream1(val + kb + lane); c_cur = ld_stream1(col + kb + lane); }
    if (kb + 32 + lane < k1) { v_nxt = ld_stream1(val + kb + 32 + lane); c_nxt = ld_stream1(col + kb + 32 + lane); }

    A acc[VW];
    zero_acc<A, VW>(acc);

    auto reduce = [&]() {
#pragma unroll
        for (int w = 0; w < VW; ++w) acc[w] = segment_reduce(full, acc[w], LPN, 32);
    };
    auto flush = [&](int64_t r, int64_t r_start) {
        reduce();
        if (sub == 0 && col_ok) {
            if (r == r0 && continued) {
                A* dst = head_val + unit * n_dense + c0;
#pragma unroll
                for (int w = 0; w < VW; ++w) dst[w] = acc[w];
            } else {
                const int64_t out_row = row_map ? idx(row_map[r_start]) : r;
                store_row<O, A, VW>(C, ldc, out_row, c0, acc);
            }
        }
        zero_acc<A, VW>(acc);
    };
    auto advance = [&]() {
        ++row;
        row_start = row_end;
        if (row > last_row) return kNoEnd;
        if (row - rb >= 32) {
            rb += 32;
            e_win = (rb + lane <= last_row) ? idx(ptr[rb + lane + 1]) : kNoEnd;
        }
        return __shfl_sync(full, e_win, (int)(row - rb));
    };

    int64_t k = k0;
    while (k < k1) {
        // a batch covers U steps of NPAR nonzeros, never past the window or k1
        int64_t lim = k1 - k;
        if (kb + 32 - k < lim) lim = kb + 32 - k;
        const int n_here = lim < (int64_t)(NPAR * U) ? (int)lim : NPAR * U;
        const int base = (int)(k - kb);
        vec_t<V, VW> bv[kFlatU];
        V av[kFlatU];
#pragma unroll
        for (int u = 0; u < kFlatU; ++u) {
            if (u < U) {
                const int j = u * NPAR + sub;
                const int src = (base + j) & 31;
                av[u] = shfl_idx(full, v_cur, src, 32);
                const I cc = shfl_idx(full, c_cur, src, 32);
                if (j < n_here && col_ok) {
                    const V* bp = ADDR32 ? B + (int32_t)((int32_t)cc * (int32_t)ldb + (int32_t)c0)
                                         : B + idx(cc) * ldb + c0;
                    bv[u] = ld_ro<V, VW>(bp);
                } else {
#pragma unroll
                    for (int w = 0; w < VW; ++w) bv[u].v[w] = vzero<V>();
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kFlatU; ++u) {
            if (u < U && u * NPAR < n_here) {
                const int64_t step = k + u * NPAR;
                const int64_t my_k = step + sub;
                const int64_t step_last = (step + NPAR < k1 ? step + NPAR : k1) - 1;
                bool done = my_k >= k1;
                while (step_last >= row_end) {
                    if (!done && my_k < row_end) {
#pragma unroll
                        for (int w = 0; w < VW; ++w) acc[w] = Acc<V, A>::fma(av[u], bv[u].v[w], acc[w]);
                        done = true;
                    }
                    flush(row, row_start);
                    row_end = advance();
                }
                if (!done) {
#pragma unroll
                    for (int w = 0; w < VW; ++w) acc[w] = Acc<V, A>::fma(av[u], bv[u].v[w], acc[w]);
                }
            }
        }
        k += n_here;
        if (k == kb + 32) {
            kb += 32;
            v_cur = v_nxt;
            c_cur = c_nxt;
            if (kb + 32 + lane < k1) {
                v_nxt = ld_stream1(val + kb + 32 + lane);
                c_nxt = ld_stream1(col + kb + 32 + lane);
            }
        }
    }
    // Rows ending exactly at k1 (and empty rows) still owned by this unit.
    while (row < r1) {
        flush(row, row_start);
        row_end = advance();
    }
    bool open = false;
    if (r1 < n_rows) {
        const int64_t s1 = row_start > k0 ? row_start : k0;  // row == r1 here
        open = k1 > s1;
        if (open) {
            reduce();
            if (sub == 0 && col_ok) {
                A* dst = carry_val + unit * n_dense + c0;
#pragma unroll
                for (int w = 0; w < VW; ++w) dst[w] = acc[w];
            }
        }
    }
    if (blockIdx.y == 0 && lane == 0) carry_row[unit] = open ? r1 : -1;
}

template <class V, class A, class O, class I, class P>
int launch_spmm_flat(const fsb_csr* Am, const V* val, const I* col, const P* ptr, const I* rmap, const V* B,
                     int64_t ldb, int64_t n_dense, O* C, int64_t ldc, const fsb_plan* plan, void* workspace,
                     int64_t workspace_bytes, cudaStream_t st) {
    const int64_t n_units = plan->n_units;
    if (plan->items_per_unit < 1 || plan->items_per_unit > kMaxItemsPerUnit || n_units != ceil_div(Am->n_rows + Am->nnz, plan->items_per_unit) ||
        !plan->unit_coords) {
        fsb_host::set_error("fsb_spmm_csr: flat plan does not match the matrix");
        return FSB_ERR_INVALID;
    }
    if (plan->row_cap > 0) {
        fsb_host::set_error("fsb_spmm_csr: row_cap needs the rows algorithm");
        return FSB_ERR_INVALID;
    }
    const int64_t need = merge_scratch_bytes(n_units, n_dense, (int)sizeof(A));
    if (!workspace || workspace_bytes < need) {
        fsb_host::set_error("fsb_spmm_csr: workspace %lld bytes < %lld", (long long)workspace_bytes, (long long)need);
        return FSB_ERR_WORKSPACE;
    }
    // 16-byte lane vectors when B and C rows allow that alignment; LPN lanes
    // cover the column tile, NPAR = 32 / LPN nonzeros per warp step.
    constexpr int kMaxBytes = (int)(sizeof(V) > sizeof(O) ? sizeof(V) : sizeof(O));
    constexpr int kVW = 16 / kMaxBytes >= 1 ? 16 / kMaxBytes : 1;
    auto vec_ok = [&](int w) {
        return w == 1 || (((uintptr_t)B) % (w * sizeof(V)) == 0 && ldb % w == 0 && n_dense % w == 0 &&
                          ((uintptr_t)C) % (w * sizeof(O)) == 0 && ldc % w == 0);
    };
    const int vw = (kVW > 1 && vec_ok(kVW)) ? kVW : 1;
    const int64_t target = plan->n_tile > 0 ? plan->n_tile : n_dense;
    int lpn_log2 = 0;
    while ((1LL << lpn_log2) * vw < target && lpn_log2 < 5) ++lpn_log2;
    const int64_t col_tiles = ceil_div(n_dense, (int64_t)vw << lpn_log2);
    const int64_t blocks = ceil_div(n_units, kSpmmThreads / 32);
    if (col_tiles > 65535 || blocks > 0x7fffffffLL) {
        fsb_host::set_error("fsb_spmm_csr: flat grid too large");
        return FSB_ERR_LIMIT;
    }
    // 32-bit B offsets when every element of B is addressable that way
    const bool addr32 = (Am->n_cols * ldb + n_dense) < 0x7fffffffLL;
    MergeScratch ms = merge_scratch_carve(workspace, n_units, n_dense, (int)sizeof(A));
    dim3 g((unsigned)blocks, (unsigned)col_tiles);
    A* cv = static_cast<A*>(ms.carry_val);
    A* hv = static_cast<A*>(ms.head_val);
#define FSB_FLAT(W, A32)                                                                                        \
    k_spmm_flat<V, A, O, I, P, W, A32><<<g, kSpmmThreads, 0, st>>>(val, col, ptr, rmap, B, ldb, C, ldc,        \
                                                                   Am->n_rows, n_dense, lpn_log2,              \
                                                                   plan->unit_coords, n_units, ms.carry_row, cv, hv)
    if (vw == kVW && kVW > 1) {
        if (addr32) FSB_FLAT(kVW, true); else FSB_FLAT(kVW, false);
    } else {
        if (addr32) FSB_FLAT(1, true); else FSB_FLAT(1, false);
    }
#undef FSB_FLAT
    int rc = fsb_host::check_launch("k_spmm_flat");
    if (rc) return rc;
    k_spmm_merge_fixup<A, O, I, P><<<(unsigned)blocks, kSpmmThreads, 0, st>>>(
        ms.carry_row, static_cast<const A*>(ms.carry_val), static_cast<const A*>(ms.head_val), n_units, n_dense, ptr,
        rmap, C, ldc);
    return fsb_host::check_launch("k_spmm_merge_fixup");
}

template <class V, class A, class O, class I, class P, int VW>
int launch_spmm(const fsb_csr* Am, const V* val, const I* col, const P* ptr, const I* rmap, const V* B, int64_t ldb,
                int64_t n_dense, O* C, int64_t ldc, const fsb_plan* plan, void* workspace, int64_t workspace_bytes,
                cudaStream_t st) {
    int ntile = plan->n_tile > 0 ? plan->n_tile : (int)(n_dense < 32 * VW ? n_dense : 32 * VW);
    int lpn = (int)ceil_div(ntile, VW);
    int lpn_log2 = 0;
    while ((1 << lpn_log2) < lpn && lpn_log2 < 5) ++lpn_log2;
    lpn = 1 << lpn_log2;
    const int64_t col_tiles = ceil_div(n_dense, (int64_t)lpn * VW);
    if (col_tiles > 65535) {
        fsb_host::set_error("fsb_spmm_csr: too many column tiles");
        return FSB_ERR_LIMIT;
    }
    const int64_t thr = plan->comp_threshold > 0 ? plan->comp_threshold : 0;
    if (plan->algo == FSB_ALGO_ROWS) {
        int G = plan->lanes;
        if (G < 1 || G > 32 || (G & (G - 1))) {
            fsb_host::set_error("fsb_spmm_csr: lanes=%d is not a power of two in [1, 32]", G);
            return FSB_ERR_INVALID;
        }
        if (G < lpn) G = lpn;
        int g_log2 = 0;
        while ((1 << g_log2) < G) ++g_log2;
        int64_t grid = ceil_div(Am->n_rows, kSpmmThreads / G);
        if (plan->grid_blocks > 0 && grid > plan->grid_blocks) grid = plan->grid_blocks;
        if (grid > 0x7fffffffLL) grid = 0x7fffffffLL;
        dim3 g((unsigned)grid, (unsigned)col_tiles);
        k_spmm_rows<V, A, O, I, P, VW><<<g, kSpmmThreads, 0, st>>>(val, col, ptr, rmap, B, ldb, C, ldc, Am->n_rows,
                                                                   n_dense, g_log2, lpn_log2, plan->row_cap, thr);
        return fsb_host::check_launch("k_spmm_rows");
    }
    if (plan->algo != FSB_ALGO_MERGE) {
        fsb_host::set_error("fsb_spmm_csr: unknown algo %d", plan->algo);
        return FSB_ERR_INVALID;
    }
    const int64_t n_units = plan->n_units;
    if (plan->items_per_unit < 1 || plan->items_per_unit > kMaxItemsPerUnit || n_units != ceil_div(Am->n_rows + Am->nnz, plan->items_per_unit) ||
        !plan->unit_coords) {
        fsb_host::set_error("fsb_spmm_csr: merge plan does not match the matrix");
        return FSB_ERR_INVALID;
    }
    if (plan->row_cap > 0) {
        fsb_host::set_error("fsb_spmm_csr: row_cap needs the rows algorithm");
        return FSB_ERR_INVALID;
    }
    const int64_t need = merge_scratch_bytes(n_units, n_dense, (int)sizeof(A));
    if (!workspace || workspace_bytes < need) {
        fsb_host::set_error("fsb_spmm_csr: workspace %lld bytes < %lld", (long long)workspace_bytes, (long long)need);
        return FSB_ERR_WORKSPACE;
    }
    MergeScratch ms = merge_scratch_carve(workspace, n_units, n_dense, (int)sizeof(A));
    const int64_t blocks = ceil_div(n_units, kSpmmThreads / 32);
    if (blocks > 0x7fffffffLL) {
        fsb_host::set_error("fsb_spmm_csr: too many merge units");
        return FSB_ERR_LIMIT;
    }
    dim3 g((unsigned)blocks, (unsigned)col_tiles);
    k_spmm_merge<V, A, O, I, P, VW><<<g, kSpmmThreads, 0, st>>>(
        val, col, ptr, rmap, B, ldb, C, ldc, Am->n_rows, n_dense, lpn_log2, plan->unit_coords, n_units, thr,
        ms.carry_row, static_cast<A*>(ms.carry_val), static_cast<A*>(ms.head_val));
    int rc = fsb_host::check_launch("k_spmm_merge");
    if (rc) return rc;
    k_spmm_merge_fixup<A, O, I, P><<<(unsigned)blocks, kSpmmThreads, 0, st>>>(
        ms.carry_row, static_cast<const A*>(ms.carry_val), static_cast<const A*>(ms.head_val), n_units, n_dense, ptr,
        rmap, C, ldc);
    return fsb_host::check_launch("k_spmm_merge_fixup");
}

}  // namespace fsb

using namespace fsb;

extern "C" int fsb_spmm_csr(const fsb_csr* A, const void* B, int64_t ldb, int64_t n_dense, void* C, int64_t ldc,
                            int out_dtype, int acc_mode, const fsb_plan* plan, void* workspace,
                            int64_t workspace_bytes, void* stream) {
    if (!A || !plan) {
        fsb_host::set_error("fsb_spmm_csr: null matrix or plan");
        return FSB_ERR_INVALID;
    }
    if (A->n_rows < 0 || A->nnz < 0 || n_dense < 0 || ldb < n_dense || ldc < n_dense) {
        fsb_host::set_error("fsb_spmm_csr: bad sizes");
        return FSB_ERR_INVALID;
    }
    if (A->n_rows == 0 || n_dense == 0) return FSB_OK;
    if (!A->row_ptr || !C || (A->nnz > 0 && (!A->values || !A->col_idx || !B))) {
        fsb_host::set_error("fsb_spmm_csr: null data pointer");
        return FSB_ERR_INVALID;
    }
    if (A->row_map && A->row_map_dtype != A->index_dtype) {
        fsb_host::set_error("fsb_spmm_csr: row_map dtype must equal index dtype");
        return FSB_ERR_INVALID;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (plan->algo == FSB_ALGO_GATHER)
        return spmm_gather_dispatch(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes,
                                    st);
    if (plan->algo == FSB_ALGO_SEQ) {
        switch (A->value_dtype) {
        case FSB_F16: return seq_dispatch_f16(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st);
        case FSB_BF16: return seq_dispatch_bf16(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st);
        case FSB_F32: return seq_dispatch_f32(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st);
        case FSB_F64: return seq_dispatch_f64(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st);
        case FSB_C32: return seq_dispatch_c32(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st);
        case FSB_C64: return seq_dispatch_c64(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st);
        case FSB_C128: return seq_dispatch_c128(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st);
        default:
            fsb_host::set_error("fsb_spmm_csr: value dtype code %d", A->value_dtype);
            return FSB_ERR_UNSUPPORTED;
        }
    }
    return dispatch_vao(A->value_dtype, acc_mode, out_dtype, [&](auto tv, auto ta, auto to) -> int {
        using V = typename decltype(tv)::type;
        using Ac = typename decltype(ta)::type;
        using O = typename decltype(to)::type;
        return dispatch_idx(A->index_dtype, [&](auto ti) -> int {
            using I = typename decltype(ti)::type;
            return dispatch_idx(A->ptr_dtype, [&](auto tp) -> int {
                using P = typename decltype(tp)::type;
                constexpr int VW = VecWidth<V>::value < VecWidth<O>::value ? VecWidth<V>::value
                                                                           : VecWidth<O>::value;
                const V* val = static_cast<const V*>(A->values);
                const I* col = static_cast<const I*>(A->col_idx);
                const P* ptr = static_cast<const P*>(A->row_ptr);
                const I* rmap = static_cast<const I*>(A->row_map);
                const V* Bv = static_cast<const V*>(B);
                O* Cv = static_cast<O*>(C);
                if (plan->algo == FSB_ALGO_FLAT)
                    return launch_spmm_flat<V, Ac, O, I, P>(A, val, col, ptr, rmap, Bv, ldb, n_dense, Cv, ldc, plan,
                                                            workspace, workspace_bytes, st);
                // 16-byte vectors need aligned bases and row strides; the output
                // vector must be a loadable width too.
                const bool vec_ok = VW > 1 && aligned16(Bv) && (ldb % VW == 0) && (n_dense % VW == 0) &&
                                    (((uintptr_t)Cv) % (sizeof(O) * VW) == 0) && (ldc % VW == 0) &&
                                    (sizeof(O) * VW <= 16);
                if (vec_ok)
                    return launch_spmm<V, Ac, O, I, P, (VW > 1 ? VW : 1)>(A, val, col, ptr, rmap, Bv, ldb, n_dense,
                                                                          Cv, ldc, plan, workspace, workspace_bytes,
                                                                          st);
                return launch_spmm<V, Ac, O, I, P, 1>(A, val, col, ptr, rmap, Bv, ldb, n_dense, Cv, ldc, plan,
                                                      workspace, workspace_bytes, st);
            });
        });
    });
}
