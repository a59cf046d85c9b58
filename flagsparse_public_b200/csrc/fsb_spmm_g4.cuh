// fsb_spmm_g4.cuh -- merge-path SpMM with the B rows staged in shared memory
// by the Tensor Memory Accelerator's row gather (cp.async.bulk.tensor.2d
// .tile::gather4: four rows of a 2-D tensor map, given by four row
// coordinates, in one instruction).  FSB_ALGO_SEQ with FSB_PLAN_TMA_GATHER;
// instantiated per value type in fsb_spmm_seq_*.cu.
//
// The batched merge-path SpMM (k_spmm_seq) keeps its B-row gathers in
// registers, so the rows in flight per SM are bounded by the register file;
// gathers of random B rows are latency bound.  Here each warp owns a ring of
// S stages in shared memory, G nonzeros per stage: the warp's first G / 4
// lanes gather the stage's G B-row slices (one column tile: TW columns, RB
// bytes) with one tile::gather4 each, S - 1 stages ahead of the stage being
// consumed, and the stage's mbarrier counts the bytes in.  The consumer side
// is the merge-path walk of k_spmm_seq: NPAR = 32 / LPN nonzeros per warp
// step, one 16-byte shared-memory load per lane and step, stages inside one
// row take the unpredicated path, stages holding row ends are consumed in row
// segments, split rows leave carries for k_spmm_merge_fixup.
//
// Ring protocol (per warp, no CTA barrier): stage t of the warp's stage
// counter goes to slot t % S with mbarrier phase parity (t / S) & 1.  The
// refill of stage t + S - 1 is issued at the start of iteration t into the
// slot of stage t - 1, whose values the previous iteration's multiply-adds
// consumed.  Stages never cross a unit, so every issued stage is waited for
// before the warp moves on.  Waits are bounded (fsb_tma.cuh); on expiry the
// warp records FSB_ERR_TIMEOUT, marks its remaining units as carrying
// nothing, waits (bounded) for its stages in flight and returns.
//
// Float accumulators only (value precision or float64): compensated rows use
// k_spmm_seq.
#pragma once
#include <type_traits>

#include "fsb_spmm_common.cuh"
#include "fsb_tma.cuh"

namespace fsb {

constexpr int kG4Warps = 4;
constexpr int kG4Threads = 32 * kG4Warps;

// Stage shape by gathered row bytes: G nonzeros per stage (2 KB stages), S
// stages per warp (16 KB rings, 64 KB per CTA: 3 CTAs per SM).
template <int RB> struct G4Shape {
    static constexpr int G = 2048 / RB;
    static constexpr int S = 8;
};

// Dynamic shared memory of one CTA: the warps' rings and their mbarriers.
template <int RB>
constexpr int g4_smem_bytes() {
    return kG4Warps * G4Shape<RB>::S * (G4Shape<RB>::G * RB + 8);
}

__device__ __forceinline__ void tma_gather4(uint32_t dst, const CUtensorMap* map, int x, int y0, int y1, int y2,
                                            int y3, uint32_t bar, uint64_t policy) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7], %8;" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y0), "r"(y1), "r"(y2), "r"(y3), "r"(bar), "l"(policy)
        : "memory");
}

template <class V, class A, class O, class I, class P, int VW, int LPN_LOG2>
__global__ void __launch_bounds__(kG4Threads)
k_spmm_g4(const __grid_constant__ CUtensorMap bmap, const V* __restrict__ val, const I* __restrict__ col,
          const P* __restrict__ ptr, const I* __restrict__ row_map, O* __restrict__ C, int64_t ldc, int64_t n_rows,
          int64_t n_dense, const int64_t* __restrict__ coords, int64_t n_units, int64_t* __restrict__ carry_row,
          A* __restrict__ carry_val, A* __restrict__ head_val, int* __restrict__ err) {
    constexpr int kNoEnd = 0x7fffffff;
    constexpr int LPN = 1 << LPN_LOG2;
    constexpr int NPAR = 32 >> LPN_LOG2;
    constexpr int TW = LPN * VW;              // columns of the tile (the box width)
    constexpr int RB = TW * (int)sizeof(V);  // bytes of one gathered row slice
    constexpr int G = G4Shape<RB>::G;        // nonzeros per stage
    constexpr int S = G4Shape<RB>::S;        // stages per ring
    constexpr int U = G / NPAR;              // warp steps per stage
    constexpr int SB = G * RB;               // bytes per stage
    static_assert(sizeof(V) * VW == 16, "16-byte lane vectors");
    static_assert(G % 4 == 0 && 32 % G == 0 && G % NPAR == 0 && U >= 1, "stage shape");
    extern __shared__ __align__(128) unsigned char g4_smem[];
    const unsigned full_mask = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char* ring = g4_smem + warp * (S * SB);
    uint64_t* full = reinterpret_cast<uint64_t*>(g4_smem + kG4Warps * S * SB) + warp * S;
    if (lane == 0) {
#pragma unroll
        for (int i = 0; i < S; ++i) tma::mbar_init(tma::smem_u32(&full[i]), 1);
        tma::mbar_init_fence();
    }
    __syncwarp();

    const int sub = lane >> LPN_LOG2;
    const int64_t ct = (int64_t)blockIdx.y * TW;  // first column of the tile
    const int64_t c0 = ct + (int64_t)(lane & (LPN - 1)) * VW;
    const bool col_ok = c0 < n_dense;
    const uint64_t keep_b = policy_evict_last();
    uint32_t done = 0;  // stages this warp has consumed: ring slot and phase of the next one

    const int64_t unit_stride = (int64_t)gridDim.x * kG4Warps;
    for (int64_t unit = (int64_t)blockIdx.x * kG4Warps + warp; unit < n_units; unit += unit_stride) {
        const int64_t r0 = coords[2 * unit], k0 = coords[2 * unit + 1];
        const int64_t r1 = coords[2 * unit + 2], k1 = coords[2 * unit + 3];
        const int64_t last_row = r1 < n_rows ? r1 : r1 - 1;
        const int nk = (int)(k1 - k0);  // unit nonzeros (the host keeps units below 2^24 items)
        const int n_st = (nk + G - 1) / G;

        // Producer window: lane l holds the B row of entry pb + l (relative to
        // k0), the next 32 in p_nxt; entries past the unit read row 0.
        int pb = 0;
        int p_cur = lane < nk ? (int)idx(col[k0 + lane]) : 0;
        int p_nxt = 32 + lane < nk ? (int)idx(col[k0 + 32 + lane]) : 0;
        auto issue = [&](int t) {  // whole warp; t increases by one per call
            if (t * G - pb >= 32) {
                pb += 32;
                p_cur = p_nxt;
                p_nxt = pb + 32 + lane < nk ? (int)idx(col[k0 + pb + 32 + lane]) : 0;
            }
            const uint32_t slot = (done + (uint32_t)t) % S;
            const uint32_t bar = tma::smem_u32(&full[slot]);
            const int e = t * G - pb + 4 * lane;  // lane q < G / 4 gathers entries e .. e + 3
            const int y0 = __shfl_sync(full_mask, p_cur, e & 31);
            const int y1 = __shfl_sync(full_mask, p_cur, (e + 1) & 31);
            const int y2 = __shfl_sync(full_mask, p_cur, (e + 2) & 31);
            const int y3 = __shfl_sync(full_mask, p_cur, (e + 3) & 31);
            if (lane == 0) tma::mbar_arrive_expect_tx(bar, SB);
            __syncwarp();
            if (lane < G / 4)
                tma_gather4(tma::smem_u32(ring + slot * SB + lane * 4 * RB), &bmap, (int)ct, y0, y1, y2, y3, bar,
                            keep_b);
        };
        const int n_pre = n_st < S - 1 ? n_st : S - 1;
        for (int t = 0; t < n_pre; ++t) issue(t);

        // Row ends relative to k0; a row ending past the unit reads as kNoEnd.
        auto load_ends = [&](int64_t rbase) -> int {
            const int64_t r = rbase + lane;
            if (r > last_row) return kNoEnd;
            const int64_t e = idx(ptr[r + 1]) - k0;
            return e > (int64_t)kNoEnd ? kNoEnd : (int)e;
        };
        int64_t rb = r0;
        int e_win = load_ends(rb);
        int e_nxt = load_ends(rb + 32);
        int64_t row = r0;
        int64_t row_start = (r0 < n_rows) ? idx(ptr[r0]) : k0;
        const bool continued = (r0 < n_rows) && (k0 > row_start);
        int row_end = __shfl_sync(full_mask, e_win, 0);

        A acc[VW];
        zero_acc<A, VW>(acc);
        auto reduce = [&]() {
            if constexpr (NPAR > 1) {
#pragma unroll
                for (int w = 0; w < VW; ++w) acc[w] = segment_reduce(full_mask, acc[w], LPN, 32);
            }
        };
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
                e_nxt = load_ends(rb + 32);
            }
            row_end = row <= last_row ? __shfl_sync(full_mask, e_win, (int)(row - rb)) : kNoEnd;
        };

        int kb = 0;
        V v_cur = vzero<V>(), v_nxt = vzero<V>();
        if (lane < nk) v_cur = ld_stream1(val + k0 + lane);
        if (32 + lane < nk) v_nxt = ld_stream1(val + k0 + 32 + lane);

        for (int t = 0, k = 0; k < nk; ++t) {
            if (t + S - 1 < n_st) issue(t + S - 1);
            const uint32_t g = done + (uint32_t)t;
            const bool ok = tma::mbar_wait(tma::smem_u32(&full[g % S]), (g / S) & 1u);
            if (!__all_sync(full_mask, ok)) {
                // give up: record, leave no stale carry for the fix-up, wait
                // (bounded) for this unit's stages in flight, then leave
                if (lane == 0) {
                    atomicExch(err, FSB_ERR_TIMEOUT);
                    if (blockIdx.y == 0)
                        for (int64_t u = unit; u < n_units; u += unit_stride) carry_row[u] = -1;
                }
                const int last = t + S - 1 < n_st ? t + S - 1 : n_st - 1;
                for (int q = t; q <= last; ++q) {
                    const uint32_t gq = done + (uint32_t)q;
                    tma::mbar_wait(tma::smem_u32(&full[gq % S]), (gq / S) & 1u);
                }
                return;
            }
            const int n_here = nk - k < G ? nk - k : G;
            const int bs = (k - kb) + sub;
            const unsigned char* sp = ring + (g % S) * SB + sub * RB + (lane & (LPN - 1)) * 16;
            vec_t<V, VW> bv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const uint4 r = *reinterpret_cast<const uint4*>(sp + u * NPAR * RB);
                memcpy(&bv[u], &r, 16);
            }
            if (n_here == G && row_end - k >= G) {
                // the stage lies inside the current row
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const V a = shfl_idx(full_mask, v_cur, bs + u * NPAR, 32);
#pragma unroll
                    for (int w = 0; w < VW; ++w) acc[w] = Acc<V, A>::fma(a, bv[u].v[w], acc[w]);
                }
            } else {
                int s = 0;
                for (;;) {
                    const int e = row_end - k;
                    if (e <= s) {
                        flush();
                        continue;
                    }
                    const int ee = e < n_here ? e : n_here;
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const V a = shfl_idx(full_mask, v_cur, (bs + u * NPAR) & 31, 32);
                        const int p = u * NPAR + sub;
                        if (p >= s && p < ee) {
#pragma unroll
                            for (int w = 0; w < VW; ++w) acc[w] = Acc<V, A>::fma(a, bv[u].v[w], acc[w]);
                        }
                    }
                    if (ee == n_here) break;
                    s = ee;
                }
            }
            k += n_here;
            if (k - kb == 32) {
                kb += 32;
                v_cur = v_nxt;
                if (kb + 32 + lane < nk) v_nxt = ld_stream1(val + k0 + kb + 32 + lane);
            }
        }
        done += (uint32_t)n_st;
        while (row < r1) flush();  // rows ending at the unit end, empty rows
        bool open = false;
        if (r1 < n_rows) {
            const int64_t s1 = row_start > k0 ? row_start : k0;
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
}

template <class V, class A, class O, class I, class P, int VW>
int launch_g4_vw(int lpn_log2, dim3 g, size_t smem, cudaStream_t st, const CUtensorMap& map, const V* val,
                 const I* col, const P* ptr, const I* rmap, O* C, int64_t ldc, int64_t n_rows, int64_t n_dense,
                 const int64_t* coords, int64_t n_units, int64_t* carry_row, A* cv, A* hv, int* err) {
#define FSB_G4_LAUNCH(L)                                                                                         \
    if (lpn_log2 == L) {                                                                                         \
        auto kern = k_spmm_g4<V, A, O, I, P, VW, L>;                                                             \
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {  \
            fsb_host::set_error("fsb_spmm_csr: cannot reserve %d bytes of shared memory", (int)smem);             \
            return FSB_ERR_LAUNCH;                                                                               \
        }                                                                                                        \
        kern<<<g, kG4Threads, smem, st>>>(map, val, col, ptr, rmap, C, ldc, n_rows, n_dense, coords, n_units,    \
                                          carry_row, cv, hv, err);                                               \
        return FSB_OK;                                                                                           \
    }
    // tiles of 64, 128 or 256 bytes per row (4, 8 or 16 lanes of 16 bytes)
    FSB_G4_LAUNCH(2)
    FSB_G4_LAUNCH(3)
    FSB_G4_LAUNCH(4)
#undef FSB_G4_LAUNCH
    fsb_host::set_error("fsb_spmm_csr: gather4 tile of %d lanes", 1 << lpn_log2);
    return FSB_ERR_INVALID;
}

int* gather_error_word();  // fsb_spmm_gather.cu: the device error word

// FSB_ALGO_SEQ with FSB_PLAN_TMA_GATHER.  Strict: FSB_ERR_UNSUPPORTED when
// the operands do not admit the gather4 form (float32 / float16 / bfloat16
// values with float accumulators, 16-byte aligned B and C rows, n_cols and
// n_dense below 2^31).
template <class V, class A, class O, class I, class P>
int launch_g4(const fsb_csr* Am, const V* val, const I* col, const P* ptr, const I* rmap, const V* B, int64_t ldb,
              int64_t n_dense, O* C, int64_t ldc, const fsb_plan* plan, void* workspace, int64_t workspace_bytes,
              cudaStream_t st) {
    constexpr bool kTypeOk = (std::is_same<V, float>::value || std::is_same<V, __half>::value ||
                              std::is_same<V, __nv_bfloat16>::value) &&
                             !is_comp_acc<A>::value;
    if constexpr (!kTypeOk) {
        fsb_host::set_error("fsb_spmm_csr: the TMA gather form takes float32 / float16 / bfloat16 values with "
                            "float accumulators");
        return FSB_ERR_UNSUPPORTED;
    } else {
        constexpr int VW = 16 / (int)sizeof(V);
        const int64_t n_units = plan->n_units;
        if (plan->items_per_unit < 1 || plan->items_per_unit > kMaxItemsPerUnit ||
            n_units != ceil_div(Am->n_rows + Am->nnz, plan->items_per_unit) || !plan->unit_coords ||
            plan->row_cap > 0) {
            fsb_host::set_error("fsb_spmm_csr: seq plan does not match the matrix");
            return FSB_ERR_INVALID;
        }
        constexpr size_t kOV = sizeof(O) * VW;  // bytes of a lane's C vector
        const bool aligned = ((uintptr_t)B) % 16 == 0 && (ldb * (int64_t)sizeof(V)) % 16 == 0 &&
                             n_dense % VW == 0 && ((uintptr_t)C) % (kOV < 16 ? kOV : 16) == 0 && ldc % VW == 0;
        if (!aligned || Am->n_cols >= 0x7fffffffLL || n_dense >= 0x7fffffffLL) {
            fsb_host::set_error("fsb_spmm_csr: the TMA gather form needs 16-byte aligned B / C rows, n_dense a "
                                "multiple of %d and n_cols below 2^31",
                                VW);
            return FSB_ERR_UNSUPPORTED;
        }
        // Column tile: 256-byte rows where n_dense allows, else 128 or 64.
        const int64_t target = plan->n_tile > 0 ? plan->n_tile : n_dense;
        int lpn_log2 = 2;
        while ((int64_t)(VW << lpn_log2) < target && lpn_log2 < 4) ++lpn_log2;
        const int tw = VW << lpn_log2;
        const int64_t need = merge_scratch_bytes(n_units, n_dense, (int)sizeof(A));
        if (!workspace || workspace_bytes < need) {
            fsb_host::set_error("fsb_spmm_csr: workspace %lld bytes < %lld", (long long)workspace_bytes,
                                (long long)need);
            return FSB_ERR_WORKSPACE;
        }
        const int64_t col_tiles = ceil_div(n_dense, (int64_t)tw);
        const int64_t blocks = ceil_div(n_units, (int64_t)kG4Warps);
        if (col_tiles > 65535 || blocks > 0x7fffffffLL) {
            fsb_host::set_error("fsb_spmm_csr: gather4 grid too large");
            return FSB_ERR_LIMIT;
        }
        int* err = gather_error_word();
        if (!err) {
            fsb_host::set_error("fsb_spmm_csr: cannot resolve the device error word");
            return FSB_ERR_LAUNCH;
        }
        CUtensorMap map;
        if (!encode_g4_map(&map, Am->value_dtype, B, Am->n_cols, ldb, n_dense, tw)) {
            fsb_host::set_error("fsb_spmm_csr: no tensor map can be encoded for B");
            return FSB_ERR_UNSUPPORTED;
        }
        MergeScratch ms = merge_scratch_carve(workspace, n_units, n_dense, (int)sizeof(A));
        A* cv = static_cast<A*>(ms.carry_val);
        A* hv = static_cast<A*>(ms.head_val);
        const int64_t grid = plan->grid_blocks > 0 && plan->grid_blocks < blocks ? plan->grid_blocks : blocks;
        dim3 g((unsigned)grid, (unsigned)col_tiles);
        const int rbytes = tw * (int)sizeof(V);
        const size_t smem = rbytes == 64 ? g4_smem_bytes<64>() : rbytes == 128 ? g4_smem_bytes<128>()
                                                                                : g4_smem_bytes<256>();
        int rc = launch_g4_vw<V, A, O, I, P, VW>(lpn_log2, g, smem, st, map, val, col, ptr, rmap, C, ldc, Am->n_rows,
                                                 n_dense, plan->unit_coords, n_units, ms.carry_row, cv, hv, err);
        if (rc) return rc;
        rc = fsb_host::check_launch("k_spmm_g4");
        if (rc) return rc;
        k_spmm_merge_fixup<A, O, I, P><<<(unsigned)blocks, kSpmmThreads, 0, st>>>(
            ms.carry_row, static_cast<const A*>(ms.carry_val), static_cast<const A*>(ms.head_val), n_units, n_dense,
            ptr, rmap, C, ldc);
        return fsb_host::check_launch("k_spmm_merge_fixup");
    }
}

}  // namespace fsb
