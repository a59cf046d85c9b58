// fsb_spmm_seq.cuh -- the batched merge-path SpMM kernel template and its
// launcher (FSB_ALGO_SEQ; instantiated per value type in fsb_spmm_seq_*.cu).
//
// One warp per (merge-path unit, column tile).  The warp walks the unit's
// nonzeros in order, NPAR = 32 / LPN of them per step: sub-group s (LPN lanes)
// takes nonzero k + s and covers the column tile with VW elements per lane
// (16-byte lane vectors where B and C allow), so a step costs each lane one
// vector load of a B-row slice and VW fused multiply-adds.
//
// Batches of U steps (UN = U * NPAR nonzeros, UN divides 32) issue their U
// B loads back to back -- independent, so all are in flight together --
// before the accumulation uses them.  A batch lying inside one row takes the
// unpredicated path; a batch holding row ends is consumed in segments, one
// row each: the sub-groups add their nonzeros of the segment, the row's sum is
// reduced across sub-groups (log2 NPAR xor-shuffles per element) and stored.
// The row flush exists once, outside the unrolled bodies, which keeps the
// kernel small.  B loads carry an L2 evict-last policy: B rows are gathered
// many times while the values and column indices stream through once.
//
// Split rows (rows spread over several units) finish in one of two ways.
// With the plan's unit runs and ticket counters, inside this kernel: each
// unit holding part of such a row stores its partial (the carry at its end,
// the head partial where the row ends), then takes a ticket on the row's
// counter; the unit drawing the last ticket adds the row's partials in unit
// order and stores the row.  Nothing waits, so nothing can hang, and the sums
// are those of the separate fix-up kernel (k_spmm_merge_fixup), which runs
// instead when the plan carries no runs.
#pragma once
#include <type_traits>

#include "fsb_spmm_g4.cuh"

namespace fsb {

// Resident CTAs per SM requested from the compiler (register cap 65536 /
// (128 x blocks)): 8 (64 registers) while a lane's accumulators take at most
// 16 bytes, 6 (80 registers) up to 48 bytes (block-compensated rows add a
// 4-byte partial per element), else 4.  Gathers are latency bound, so
// resident warps are worth more than the few bytes ptxas spills at 64 (fewer
// resident warps with twice or four times the loads per batch measured
// slower on the power-law SpMM: 191 and 229 us against 170 us).
template <class V, class A, int VW> struct SeqMinBlocks {
    static constexpr int acc_bytes =
        (int)sizeof(A) * VW + ((is_comp_acc<A>::value && sizeof(V) == 2) ? 4 * VW : 0);
    static constexpr int value = acc_bytes <= 16 ? 8 : (acc_bytes <= 48 ? 6 : 4);
};

// Steps per batch: 16 B elements per lane in flight at 8 resident CTAs, 32 at
// fewer (fewer warps need more loads each), at most 32 nonzeros per batch.
template <class V, class A, int VW, int NPAR> struct SeqBatch {
    static constexpr int elems = SeqMinBlocks<V, A, VW>::value >= 8 ? 16 : 32;
    static constexpr int by_elems = elems / VW < 1 ? 1 : elems / VW;
    static constexpr int value = by_elems * NPAR > 32 ? 32 / NPAR : by_elems;
};

// Load of a partial written by another CTA in this launch: L2 only (no stale
// L1 line can answer it).
template <class A>
__device__ __forceinline__ A ld_partial(const A* p) {
    using R = typename raw_type<sizeof(A)>::T;
    R r = __ldcg(reinterpret_cast<const R*>(p));
    A out;
    memcpy(&out, &r, sizeof(A));
    return out;
}

// Whole warp, after its lanes stored their partial of a split row: one ticket
// on the row's counter; true on the warp that drew the last of `count`
// tickets, which then resets the counter for the next call.  The lanes'
// stores are ordered before lane 0's ticket by the warp barrier; the ticket is
// an acquire-release atomic, so the finisher's loads after it (and after the
// broadcast) see every contributor's partial.
__device__ __forceinline__ bool seq_take_ticket(int* slot, int count, int lane) {
    __syncwarp();
    int last = 0;
    if (lane == 0) {
        int old;
        asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;" : "=r"(old) : "l"(slot) : "memory");
        last = old == count - 1;
        if (last) *slot = 0;
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    __syncwarp();  // the other lanes' loads follow lane 0's acquire
    return last != 0;
}

// The finishing unit's lanes (sub-group 0) add the split row's partials in
// unit order -- carries of units first .. last - 1, then the head partial of
// unit last, as k_spmm_merge_fixup does -- and store the row.
template <class A, class O, class I, class P, int VW>
__device__ __forceinline__ void seq_finish_row(int64_t first, int64_t last, int64_t row, const A* carry_val,
                                               const A* head_val, int64_t n_dense, int64_t c0, const P* ptr,
                                               const I* row_map, O* C, int64_t ldc) {
    A sum[VW];
    const A* p = carry_val + first * n_dense + c0;
#pragma unroll
    for (int w = 0; w < VW; ++w) sum[w] = ld_partial(p + w);
    for (int64_t u = first + 1; u < last; ++u) {
        p = carry_val + u * n_dense + c0;
#pragma unroll
        for (int w = 0; w < VW; ++w) sum[w] = acc_add(sum[w], ld_partial(p + w));
    }
    p = head_val + last * n_dense + c0;
#pragma unroll
    for (int w = 0; w < VW; ++w) sum[w] = acc_add(sum[w], ld_partial(p + w));
    const int64_t out_row = row_map ? idx(row_map[idx(ptr[row])]) : row;
    store_row<O, A, VW>(C, ldc, out_row, c0, sum);
}

// Whole warp, once at the end of a unit whose partials are stored: tickets
// for the split row the unit continued and ended (its head partial) and for
// the row open at its end (its carry); finishes the rows whose last ticket it
// drew.  Not inlined: kept out of the register allocation of the unit loop.
template <class A, class O, class I, class P, int VW>
__device__ __noinline__ void seq_unit_tickets(int64_t unit, int64_t r0, int64_t r1, bool head, bool open,
                                              int lane, bool finisher_lane, int64_t c0, const int64_t* runs,
                                              int* tix, const A* carry_val, const A* head_val, int64_t n_dense,
                                              const P* ptr, const I* row_map, O* C, int64_t ldc) {
    for (int job = 0; job < 2; ++job) {
        int64_t first = -1, last = -1, row = 0;
        if (job == 0 && head) {
            first = runs[2 * unit - 2];
            last = unit;
            row = r0;
        } else if (job == 1 && open) {
            first = runs[2 * unit];
            last = runs[2 * unit + 1];
            row = r1;
        }
        if (first >= 0 && last > first && seq_take_ticket(tix + first, (int)(last - first + 1), lane) &&
            finisher_lane)
            seq_finish_row<A, O, I, P, VW>(first, last, row, carry_val, head_val, n_dense, c0, ptr, row_map, C, ldc);
    }
}

template <class V, class A, class O, class I, class P, int VW, int LPN_LOG2, bool ADDR32>
__global__ void __launch_bounds__(kSpmmThreads, SeqMinBlocks<V, A, VW>::value)
k_spmm_seq(const V* __restrict__ val, const I* __restrict__ col, const P* __restrict__ ptr,
           const I* __restrict__ row_map, const V* __restrict__ B, int64_t ldb, O* __restrict__ C, int64_t ldc,
           int64_t n_rows, int64_t n_dense, const int64_t* __restrict__ coords, int64_t n_units,
           int64_t comp_threshold, int64_t* __restrict__ carry_row, A* __restrict__ carry_val,
           A* __restrict__ head_val, const int64_t* __restrict__ runs, int* __restrict__ tickets) {
    constexpr int kNoEnd = 0x7fffffff;
    constexpr int LPN = 1 << LPN_LOG2;
    constexpr int NPAR = 32 >> LPN_LOG2;
    constexpr int U = SeqBatch<V, A, VW, NPAR>::value;
    // Compensated rows with 16-bit values: the products are exact in f32, so
    // a batch's products are summed plainly (per lane, at most U of them) and
    // the batch sum enters the (s, c) accumulator through one TwoSum.
    constexpr bool kBlockComp = is_comp_acc<A>::value && sizeof(V) == 2;
    constexpr int UN = U * NPAR;  // nonzeros per batch (divides 32)
    const int lane = threadIdx.x & 31;
    // Persistent when the grid is smaller than the unit count: each warp
    // takes units warp_id, warp_id + total warps, ...
    const int64_t unit_stride = (int64_t)gridDim.x * (kSpmmThreads / 32);
    for (int64_t unit = (int64_t)blockIdx.x * (kSpmmThreads / 32) + (threadIdx.x >> 5); unit < n_units;
         unit += unit_stride) {  // whole warp
        const unsigned full = 0xffffffffu;
        const int sub = lane >> LPN_LOG2;
        const int64_t c0 = (int64_t)blockIdx.y * (LPN * VW) + (int64_t)(lane & (LPN - 1)) * VW;
        const bool col_ok = c0 < n_dense;
        // lanes past the last column read column 0 (a valid address) and store nothing
        const V* Bl = B + (col_ok ? c0 : 0);
        const uint64_t keep_b = policy_evict_last();

        const int64_t r0 = coords[2 * unit], k0 = coords[2 * unit + 1];
        const int64_t r1 = coords[2 * unit + 2], k1 = coords[2 * unit + 3];
        const int64_t last_row = r1 < n_rows ? r1 : r1 - 1;
        const int nk = (int)(k1 - k0);  // unit nonzeros (the host keeps units far below 2^31)

        // Row ends relative to k0; a row ending past the unit reads as kNoEnd.
        auto load_ends = [&](int64_t rbase) -> int {
            const int64_t r = rbase + lane;
            if (r > last_row) return kNoEnd;
            const int64_t e = idx(ptr[r + 1]) - k0;
            return e > (int64_t)kNoEnd ? kNoEnd : (int)e;
        };
        // rows rb .. rb + 31 in e_win, the next 64 prefetched in e_nxt, e_nx2
        int64_t rb = r0;
        int e_win = load_ends(rb);
        int e_nxt = load_ends(rb + 32);
        int e_nx2 = load_ends(rb + 64);
        int64_t row = r0;
        int64_t row_start = (r0 < n_rows) ? idx(ptr[r0]) : k0;  // global start of the current row
        const bool continued = (r0 < n_rows) && (k0 > row_start);
        int row_end = __shfl_sync(full, e_win, 0);
        // FSB_ACC_COMP: compensated accumulation only on rows longer than
        // comp_threshold nonzeros; shorter rows add plainly into the f32 part.
        auto row_is_long = [&]() -> bool {
            if constexpr (!is_comp_acc<A>::value) return false;
            if (row > last_row) return false;
            const int64_t len = (row_end == kNoEnd ? idx(ptr[row + 1]) : k0 + row_end) - row_start;
            return len > comp_threshold;
        };
        bool long_row = row_is_long();

        A acc[VW];
        zero_acc<A, VW>(acc);
        auto fma_vec = [&](V a, const vec_t<V, VW>& b) {
            if constexpr (is_comp_acc<A>::value) {
                if (!long_row) {
#pragma unroll
                    for (int w = 0; w < VW; ++w) acc[w].s = fmaf(to_f32(a), to_f32(b.v[w]), acc[w].s);
                    return;
                }
            }
#pragma unroll
            for (int w = 0; w < VW; ++w) acc[w] = Acc<V, A>::fma(a, b.v[w], acc[w]);
        };
        // Per-batch partial sums of the block-compensated rows.
        float blk[kBlockComp ? VW : 1];
        auto blk_zero = [&]() {
            if constexpr (kBlockComp) {
#pragma unroll
                for (int w = 0; w < VW; ++w) blk[w] = 0.f;
            }
        };
        // One product into the row: the batch partial for block-compensated long
        // rows, else the accumulator.
        auto fma_step = [&](V a, const vec_t<V, VW>& b) {
            if constexpr (kBlockComp) {
                if (long_row) {
                    const float fa = to_f32(a);
#pragma unroll
                    for (int w = 0; w < VW; ++w) blk[w] = fmaf(fa, to_f32(b.v[w]), blk[w]);
                    return;
                }
            }
            fma_vec(a, b);
        };
        auto blk_fold = [&]() {
            if constexpr (kBlockComp) {
                if (long_row) {
#pragma unroll
                    for (int w = 0; w < VW; ++w) acc[w] = comp_add_value(acc[w], blk[w], 0.f);
                }
            }
        };
        auto reduce = [&]() {
            if constexpr (NPAR > 1) {
#pragma unroll
                for (int w = 0; w < VW; ++w) acc[w] = segment_reduce(full, acc[w], LPN, 32);
            }
        };
        // Store the finished current row and move to the next one.
        auto flush = [&]() {
            reduce();
            if (sub == 0 && col_ok) {
                if (row == r0 && continued) {
                    A* dst = head_val + unit * n_dense + c0;
#pragma unroll
                    for (int w = 0; w < VW; ++w) dst[w] = acc[w];
                } else {
                    const int64_t out_row = row_map ? idx(row_map[row_start]) : row;
                    store_row<O, A, VW>(C, ldc, out_row, c0, acc);
                }
            }
            zero_acc<A, VW>(acc);
            ++row;
            row_start = k0 + row_end;
            if (row <= last_row && row - rb >= 32) {
                rb += 32;
                e_win = e_nxt;
                e_nxt = e_nx2;
                e_nx2 = load_ends(rb + 64);
            }
            row_end = row <= last_row ? __shfl_sync(full, e_win, (int)(row - rb)) : kNoEnd;
            long_row = row_is_long();
        };
        auto b_row = [&](I c) -> const V* {
            if constexpr (ADDR32) return Bl + (uint32_t)((uint32_t)c * (uint32_t)ldb);
            else return Bl + idx(c) * ldb;
        };

        // Value / column windows: lane l holds entry kb + l (current) and
        // kb + 32 + l (next), relative to k0.
        int kb = 0;
        V v_cur = vzero<V>(), v_nxt = vzero<V>();
        I c_cur = 0, c_nxt = 0;
        if (lane < nk) { v_cur = ld_stream1(val + k0 + lane); c_cur = ld_stream1(col + k0 + lane); }
        if (32 + lane < nk) { v_nxt = ld_stream1(val + k0 + 32 + lane); c_nxt = ld_stream1(col + k0 + 32 + lane); }

        for (int k = 0; k < nk;) {
            // UN divides 32 and k advances by UN except at the unit end, so a batch
            // never crosses the window: bs + u * NPAR stays below 32
            const int n_here = nk - k < UN ? nk - k : UN;
            const int bs = (k - kb) + sub;
            vec_t<V, VW> bv[U];
            if (n_here == UN) {
#pragma unroll
                for (int u = 0; u < U; ++u) bv[u] = ld_keep<V, VW>(b_row(shfl_idx(full, c_cur, bs + u * NPAR, 32)), keep_b);
            } else {
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const I c = shfl_idx(full, c_cur, (bs + u * NPAR) & 31, 32);
                    if (u * NPAR + sub < n_here) {
                        bv[u] = ld_keep<V, VW>(b_row(c), keep_b);
                    } else {
#pragma unroll
                        for (int w = 0; w < VW; ++w) bv[u].v[w] = vzero<V>();
                    }
                }
            }
            if (n_here == UN && row_end - k >= UN) {
                // common case: the batch lies inside the current row
                blk_zero();
#pragma unroll
                for (int u = 0; u < U; ++u) fma_step(shfl_idx(full, v_cur, bs + u * NPAR, 32), bv[u]);
                blk_fold();
            } else {
                // segments [s, e) of the batch, one row each, flushed in between
                int s = 0;
                for (;;) {
                    const int e = row_end - k;
                    if (e <= s) {
                        flush();
                        continue;
                    }
                    const int ee = e < n_here ? e : n_here;
                    blk_zero();
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const V a = shfl_idx(full, v_cur, (bs + u * NPAR) & 31, 32);
                        const int p = u * NPAR + sub;
                        if (p >= s && p < ee) fma_step(a, bv[u]);
                    }
                    blk_fold();
                    if (ee == n_here) break;
                    s = ee;
                }
            }
            k += n_here;
            if (k - kb == 32) {
                kb += 32;
                v_cur = v_nxt;
                c_cur = c_nxt;
                if (kb + 32 + lane < nk) {
                    v_nxt = ld_stream1(val + k0 + kb + 32 + lane);
                    c_nxt = ld_stream1(col + k0 + kb + 32 + lane);
                }
            }
        }
        while (row < r1) flush();  // rows ending at the unit end, empty rows
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
        if (runs) {
            // the split rows this unit holds parts of: the one it continued
            // and ended (head partial) and the one open at its end (carry)
            seq_unit_tickets<A, O, I, P, VW>(unit, r0, r1, continued && r1 > r0, open, lane, sub == 0 && col_ok, c0,
                                             runs, tickets + (int64_t)blockIdx.y * n_units, carry_val, head_val,
                                             n_dense, ptr, row_map, C, ldc);
        } else if (blockIdx.y == 0 && lane == 0) {
            carry_row[unit] = open ? r1 : -1;
        }
    }
}

// Widest lane vector: 16 bytes of B and of C.
template <class V, class O>
constexpr int seq_max_vw() {
    constexpr int bv = 16 / (int)sizeof(V), bo = 16 / (int)sizeof(O);
    return bv < bo ? bv : bo;
}

template <class V, class A, class O, class I, class P, int VW>
void launch_seq_vw(int lpn_log2, bool addr32, dim3 g, cudaStream_t st, const V* val, const I* col, const P* ptr,
                   const I* rmap, const V* B, int64_t ldb, O* C, int64_t ldc, int64_t n_rows, int64_t n_dense,
                   const int64_t* coords, int64_t n_units, int64_t thr, int64_t* carry_row, A* cv, A* hv,
                   const int64_t* runs, int* tickets) {
#define FSB_SEQ_KERNEL(L, A32)                                                                                  \
    k_spmm_seq<V, A, O, I, P, VW, L, A32><<<g, kSpmmThreads, 0, st>>>(                                          \
        val, col, ptr, rmap, B, ldb, C, ldc, n_rows, n_dense, coords, n_units, thr, carry_row, cv, hv, runs,    \
        tickets)
#define FSB_SEQ_LAUNCH(L)                                                                                         \
    if (lpn_log2 == L) {                                                                                          \
        if (addr32)                                                                                               \
            FSB_SEQ_KERNEL(L, true);                                                                              \
        else                                                                                                      \
            FSB_SEQ_KERNEL(L, false);                                                                             \
        return;                                                                                                   \
    }
    FSB_SEQ_LAUNCH(0)
    FSB_SEQ_LAUNCH(1)
    FSB_SEQ_LAUNCH(2)
    FSB_SEQ_LAUNCH(3)
    FSB_SEQ_LAUNCH(4)
    FSB_SEQ_LAUNCH(5)
#undef FSB_SEQ_LAUNCH
#undef FSB_SEQ_KERNEL
}

template <class V, class A, class O, class I, class P>
int launch_seq(const fsb_csr* Am, const V* val, const I* col, const P* ptr, const I* rmap, const V* B, int64_t ldb,
               int64_t n_dense, O* C, int64_t ldc, const fsb_plan* plan, void* workspace, int64_t workspace_bytes,
               cudaStream_t st) {
    // B rows staged by TMA gather4 (fsb_spmm_g4.cuh); a matrix without
    // nonzeros gathers nothing and takes the plain kernel
    if ((plan->flags & FSB_PLAN_TMA_GATHER) && Am->nnz > 0)
        return launch_g4<V, A, O, I, P>(Am, val, col, ptr, rmap, B, ldb, n_dense, C, ldc, plan, workspace,
                                        workspace_bytes, st);
    const int64_t n_units = plan->n_units;
    if (plan->items_per_unit < 1 || plan->items_per_unit > kMaxItemsPerUnit || n_units != ceil_div(Am->n_rows + Am->nnz, plan->items_per_unit) ||
        !plan->unit_coords || plan->row_cap > 0) {
        fsb_host::set_error("fsb_spmm_csr: seq plan does not match the matrix");
        return FSB_ERR_INVALID;
    }
    // Lane vectors of the widest aligned width (whole vectors: n_dense a
    // multiple of the width); otherwise one element per lane.
    constexpr int kMaxVW = seq_max_vw<V, O>();
    constexpr size_t kCAlign = kMaxVW * sizeof(O) < 16 ? kMaxVW * sizeof(O) : 16;
    const bool wide_ok = ((uintptr_t)B) % (kMaxVW * sizeof(V)) == 0 && ldb % kMaxVW == 0 &&
                         n_dense % kMaxVW == 0 && ((uintptr_t)C) % kCAlign == 0 && ldc % kMaxVW == 0;
    const int vw = wide_ok ? kMaxVW : 1;
    // Lanes per nonzero: the column tile (n_tile, or all of n_dense) in lane
    // vectors, rounded up to a power of two, at most 32.
    const int64_t target = plan->n_tile > 0 ? plan->n_tile : n_dense;
    int lpn_log2 = 0;
    while ((int64_t)(vw << lpn_log2) < target && lpn_log2 < 5) ++lpn_log2;
    const int64_t need = merge_scratch_bytes(n_units, n_dense, (int)sizeof(A));
    if (!workspace || workspace_bytes < need) {
        fsb_host::set_error("fsb_spmm_csr: workspace %lld bytes < %lld", (long long)workspace_bytes, (long long)need);
        return FSB_ERR_WORKSPACE;
    }
    const int64_t col_tiles = ceil_div(n_dense, (int64_t)(vw << lpn_log2));
    const int64_t blocks = ceil_div(n_units, kSpmmThreads / 32);
    if (col_tiles > 65535 || blocks > 0x7fffffffLL) {
        fsb_host::set_error("fsb_spmm_csr: seq grid too large");
        return FSB_ERR_LIMIT;
    }
    // 32-bit B offsets when every row start fits (unsigned arithmetic)
    const bool addr32 = Am->n_cols * ldb + n_dense < 0xffffffffLL;
    MergeScratch ms = merge_scratch_carve(workspace, n_units, n_dense, (int)sizeof(A));
    A* cv = static_cast<A*>(ms.carry_val);
    A* hv = static_cast<A*>(ms.head_val);
    const int64_t thr = plan->comp_threshold > 0 ? plan->comp_threshold : 0;
    // plan->grid_blocks > 0: a persistent grid of that many CTAs per column
    // tile, its warps striding over the units
    const int64_t grid = plan->grid_blocks > 0 && plan->grid_blocks < blocks ? plan->grid_blocks : blocks;
    dim3 g((unsigned)grid, (unsigned)col_tiles);
    // split rows finish inside the kernel when the plan brings the unit runs
    // and enough ticket counters (one per unit and column tile)
    const bool in_kernel = plan->unit_runs && plan->tickets && plan->ticket_slots >= n_units * col_tiles;
    const int64_t* runs = in_kernel ? plan->unit_runs : nullptr;
    int* tickets = in_kernel ? reinterpret_cast<int*>(plan->tickets) : nullptr;
    if (vw == kMaxVW)
        launch_seq_vw<V, A, O, I, P, kMaxVW>(lpn_log2, addr32, g, st, val, col, ptr, rmap, B, ldb, C, ldc, Am->n_rows,
                                             n_dense, plan->unit_coords, n_units, thr, ms.carry_row, cv, hv, runs,
                                             tickets);
    if constexpr (kMaxVW > 1) {
        if (vw == 1)
            launch_seq_vw<V, A, O, I, P, 1>(lpn_log2, addr32, g, st, val, col, ptr, rmap, B, ldb, C, ldc, Am->n_rows,
                                            n_dense, plan->unit_coords, n_units, thr, ms.carry_row, cv, hv, runs,
                                            tickets);
    }
    int rc = fsb_host::check_launch("k_spmm_seq");
    if (rc || in_kernel) return rc;
    k_spmm_merge_fixup<A, O, I, P><<<(unsigned)blocks, kSpmmThreads, 0, st>>>(
        ms.carry_row, static_cast<const A*>(ms.carry_val), static_cast<const A*>(ms.head_val), n_units, n_dense, ptr,
        rmap, C, ldc);
    return fsb_host::check_launch("k_spmm_merge_fixup");
}

// Launch for value type VSel only (each fsb_spmm_seq_*.cu instantiates one).
template <class VSel>
int seq_dispatch_for(const fsb_csr* A, const void* B, int64_t ldb, int64_t n_dense, void* C, int64_t ldc,
                     int out_dtype, int acc_mode, const fsb_plan* plan, void* workspace, int64_t workspace_bytes,
                     cudaStream_t st) {
    return dispatch_vao(A->value_dtype, acc_mode, out_dtype, [&](auto tv, auto ta, auto to) -> int {
        using V = typename decltype(tv)::type;
        using Ac = typename decltype(ta)::type;
        using O = typename decltype(to)::type;
        if constexpr (!std::is_same<V, VSel>::value) {
            return FSB_ERR_UNSUPPORTED;
        } else {
            return dispatch_idx(A->index_dtype, [&](auto ti) -> int {
                using I = typename decltype(ti)::type;
                return dispatch_idx(A->ptr_dtype, [&](auto tp) -> int {
                    using P = typename decltype(tp)::type;
                    return launch_seq<V, Ac, O, I, P>(
                        A, static_cast<const V*>(A->values), static_cast<const I*>(A->col_idx),
                        static_cast<const P*>(A->row_ptr), static_cast<const I*>(A->row_map),
                        static_cast<const V*>(B), ldb, n_dense, static_cast<O*>(C), ldc, plan, workspace,
                        workspace_bytes, st);
                });
            });
        }
    });
}

#define FSB_SEQ_DECL(NAME)                                                                                       \
    int NAME(const fsb_csr* A, const void* B, int64_t ldb, int64_t n_dense, void* C, int64_t ldc, int out_dtype, \
             int acc_mode, const fsb_plan* plan, void* workspace, int64_t workspace_bytes, cudaStream_t st)
FSB_SEQ_DECL(seq_dispatch_f16);
FSB_SEQ_DECL(seq_dispatch_bf16);
FSB_SEQ_DECL(seq_dispatch_f32);
FSB_SEQ_DECL(seq_dispatch_f64);
FSB_SEQ_DECL(seq_dispatch_c32);
FSB_SEQ_DECL(seq_dispatch_c64);
FSB_SEQ_DECL(seq_dispatch_c128);

}  // namespace fsb
