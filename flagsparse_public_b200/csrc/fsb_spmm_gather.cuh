// fsb_spmm_gather.cuh -- the gather SpMM kernel template and its launcher
// (instantiated per value type in fsb_spmm_gather_*.cu).
// SpMM with B rows gathered by the Tensor Memory
// Accelerator into shared memory (FSB_ALGO_GATHER).
//
// Work split as in k_spmm_flat: one warp per (merge-path unit, column tile),
// NPAR = 32 / LPN nonzeros per warp step, rows flushed when the nonzero stream
// passes their end, split rows finished through carries.  The difference is
// where the B rows wait: each warp owns a ring of kGatherStages stages in
// shared memory, a stage holding the tile-wide B rows of R consecutive
// nonzeros.  R lanes issue one cp.async.bulk copy each (global -> shared,
// completion counted in bytes on the stage's mbarrier), so the bytes in flight
// do not occupy registers: while the warp accumulates stage b, stages
// b + 1 .. b + kGatherStages - 1 are being filled.
//
// Every mbarrier wait is bounded (1 s): on expiry the kernel records
// FSB_ERR_TIMEOUT in the device error word it is given, waits (bounded again)
// for the copies it still has in flight, and returns (fsb_device_error reads
// the word).
//
// Requirements (checked on the host): B base, B row stride and column-tile
// starts 16-byte aligned, tile byte widths multiples of 16 bytes.
#pragma once
#include <type_traits>

#include "fsb_spmm_common.cuh"

namespace fsb {

constexpr int kGatherStages = 4;
constexpr int kGatherRows = 8;  // nonzeros (B rows) per stage when NPAR <= 8
constexpr unsigned long long kWaitLimitNs = 1000000000ull;  // 1 s per wait
constexpr uint32_t kSuspendHintNs = 20000u;                   // sleep up to 20 us per try
constexpr int kBarBytes = (kSpmmThreads / 32) * kGatherStages * 8;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// try_wait with a suspend-time hint: a waiting warp sleeps until the phase
// completes (or the hint expires) instead of spinning on issue slots.
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(kSuspendHintNs)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait for the phase with the given parity; false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity,
                                          unsigned long long limit_ns = kWaitLimitNs) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer_ns() - t0 > limit_ns) return false;
    }
}
// Lane-vector shared-memory load (4, 8 or 16 bytes).
template <class V, int VW>
__device__ __forceinline__ vec_t<V, VW> ld_shared_vec(const unsigned char* p) {
    using R = typename raw_type<sizeof(V) * VW>::T;
    const R r = *reinterpret_cast<const R*>(p);
    vec_t<V, VW> out;
    memcpy(&out, &r, sizeof(R));
    return out;
}
// Bulk copy global -> shared, completion counted on the mbarrier, with an L2
// cache policy (B rows are kept resident: evict_last).
__device__ __forceinline__ void bulk_copy_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar,
                                              uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
            dst),
        "l"(src), "r"(bytes), "r"(bar), "l"(policy)
        : "memory");
}
__device__ __forceinline__ void fence_mbarrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

template <class V, class A, class O, class I, class P, int VW, int LPN_LOG2, bool ADDR32>
__global__ void __launch_bounds__(kSpmmThreads)
k_spmm_gather(const V* __restrict__ val, const I* __restrict__ col, const P* __restrict__ ptr,
              const I* __restrict__ row_map, const V* __restrict__ B, int64_t ldb, O* __restrict__ C, int64_t ldc,
              int64_t n_rows, int64_t n_dense, const int64_t* __restrict__ coords, int64_t n_units,
              int64_t comp_threshold, int64_t* __restrict__ carry_row, A* __restrict__ carry_val,
              A* __restrict__ head_val, int* __restrict__ err_word) {
    constexpr int LPN = 1 << LPN_LOG2;
    constexpr int NPAR = 32 >> LPN_LOG2;                      // nonzeros per warp step
    constexpr int U = NPAR >= kGatherRows ? 1 : kGatherRows / NPAR;  // steps per stage
    constexpr int R = U * NPAR;                               // B rows per stage (divides 32)
    constexpr int SLOT = LPN * VW * (int)sizeof(V);           // one tile-wide B row
    constexpr int STAGE = R * SLOT;
    constexpr int kNoEnd = 0x7fffffff;
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int64_t unit = (int64_t)blockIdx.x * (kSpmmThreads / 32) + warp;
    if (unit >= n_units) return;  // whole warp
    const unsigned full = 0xffffffffu;
    const int sub = lane >> LPN_LOG2;
    const int cl = lane & (LPN - 1);
    const int64_t tile_c = (int64_t)blockIdx.y * (LPN * VW);
    const int64_t c0 = tile_c + (int64_t)cl * VW;
    const bool col_ok = c0 < n_dense;
    const int64_t tile_cols = (n_dense - tile_c) < (int64_t)(LPN * VW) ? (n_dense - tile_c) : (int64_t)(LPN * VW);
    const uint32_t row_bytes = (uint32_t)(tile_cols * (int64_t)sizeof(V));
    const V* Bt = B + tile_c;
    const uint64_t keep_b = policy_evict_last();

    uint64_t* bars = reinterpret_cast<uint64_t*>(smem) + warp * kGatherStages;
    unsigned char* ring = smem + kBarBytes + (size_t)warp * kGatherStages * STAGE;
    if (lane == 0) {
#pragma unroll
        for (int s = 0; s < kGatherStages; ++s) mbar_init(smem_u32(bars + s), 1);
        fence_mbarrier_init();
    }
    __syncwarp();

    const int64_t r0 = coords[2 * unit], k0 = coords[2 * unit + 1];
    const int64_t r1 = coords[2 * unit + 2], k1 = coords[2 * unit + 3];
    const int64_t last_row = r1 < n_rows ? r1 : r1 - 1;
    const int nk = (int)(k1 - k0);  // unit nonzeros (host keeps units far below 2^31)
    const int n_batches = (nk + R - 1) / R;

    // Row ends relative to k0 (a row ending past the unit reads as kNoEnd).
    auto load_ends = [&](int64_t rbase) -> int {
        const int64_t r = rbase + lane;
        if (r > last_row) return kNoEnd;
        const int64_t e = idx(ptr[r + 1]) - k0;
        return e > (int64_t)kNoEnd ? kNoEnd : (int)e;
    };
    int64_t rb = r0;
    int e_win = load_ends(rb);
    int64_t row = r0;
    int64_t row_start = (r0 < n_rows) ? idx(ptr[r0]) : k0;  // global start of the current row
    const bool continued = (r0 < n_rows) && (k0 > row_start);
    int row_end = __shfl_sync(full, e_win, 0);
    // Compensated accumulation (FSB_ACC_COMP) only on rows longer than
    // comp_threshold nonzeros; shorter rows add plainly into the f32 part.
    auto row_is_long = [&]() -> bool {
        if constexpr (!is_comp_acc<A>::value) return false;
        if (row > last_row) return false;
        const int64_t len = (row_end == kNoEnd ? idx(ptr[row + 1]) : k0 + row_end) - row_start;
        return len > comp_threshold;
    };
    bool long_row = row_is_long();

    // Value window (consumer) and column-index window (producer), 32 entries
    // each plus the prefetched next 32, aligned on k0.
    int vb = 0, pb = 0;
    V v_cur = vzero<V>(), v_nxt = vzero<V>();
    I p_cur = 0, p_nxt = 0;
    if (lane < nk) { v_cur = ld_stream1(val + k0 + lane); p_cur = ld_stream1(col + k0 + lane); }
    if (32 + lane < nk) { v_nxt = ld_stream1(val + k0 + 32 + lane); p_nxt = ld_stream1(col + k0 + 32 + lane); }

    auto issue = [&](int b) {
        if (b >= n_batches) return;
        const int kp = b * R;
        if (kp - pb >= 32) {
            pb += 32;
            p_cur = p_nxt;
            p_nxt = (pb + 32 + lane < nk) ? ld_stream1(col + k0 + pb + 32 + lane) : I(0);
        }
        const int n_b = nk - kp < R ? nk - kp : R;
        const int slot = b % kGatherStages;
        // one bulk copy per B row, issued by lane j for row slot j
        const I cj = shfl_idx(full, p_cur, (kp - pb + lane) & 31, 32);
        const uint32_t bar = smem_u32(bars + slot);
        __syncwarp();
        if (lane == 0) mbar_arrive_expect_tx(bar, (uint32_t)n_b * row_bytes);
        __syncwarp();
        if (lane < n_b) {
            const V* src = ADDR32 ? Bt + (int32_t)((int32_t)cj * (int32_t)ldb) : Bt + idx(cj) * ldb;
            fence_proxy_async_smem();
            bulk_copy_g2s(smem_u32(ring + slot * STAGE + lane * SLOT), src, row_bytes, bar, keep_b);
        }
    };

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
    auto reduce = [&]() {
#pragma unroll
        for (int w = 0; w < VW; ++w) acc[w] = segment_reduce(full, acc[w], LPN, 32);
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
        // next row
        ++row;
        row_start = k0 + row_end;
        if (row <= last_row && row - rb >= 32) {
            rb += 32;
            e_win = load_ends(rb);
        }
        row_end = row <= last_row ? __shfl_sync(full, e_win, (int)(row - rb)) : kNoEnd;
        long_row = row_is_long();
    };
    // Step whose NPAR nonzeros [step, step + NPAR) reach the current row end:
    // each sub-group adds its product to the row it belongs to.
    auto boundary = [&](int step, int step_last, V a, const vec_t<V, VW>& b, bool live) {
        const int my = step + sub;
        bool done = !live;
        while (step_last >= row_end) {
            if (!done && my < row_end) {
                fma_vec(a, b);
                done = true;
            }
            flush();
        }
        if (!done) fma_vec(a, b);
    };

    for (int s = 0; s < kGatherStages - 1; ++s) issue(s);

    bool failed = false;
    int b = 0;
    for (; b < n_batches; ++b) {
        issue(b + kGatherStages - 1);
        const int slot = b % kGatherStages;
        if (!mbar_wait(smem_u32(bars + slot), (uint32_t)((b / kGatherStages) & 1))) {
            failed = true;
            break;
        }
        const int kc = b * R;
        if (kc - vb >= 32) {
            vb += 32;
            v_cur = v_nxt;
            v_nxt = (vb + 32 + lane < nk) ? ld_stream1(val + k0 + vb + 32 + lane) : vzero<V>();
        }
        const unsigned char* st = ring + slot * STAGE + sub * SLOT + cl * VW * (int)sizeof(V);
        if (kc + R <= nk) {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int step = kc + u * NPAR;
                const V a = shfl_idx(full, v_cur, (step - vb + sub) & 31, 32);
                vec_t<V, VW> bv;
                if (col_ok) bv = ld_shared_vec<V, VW>(st + u * NPAR * SLOT);
                else
#pragma unroll
                    for (int w = 0; w < VW; ++w) bv.v[w] = vzero<V>();
                if (step + NPAR - 1 >= row_end) boundary(step, step + NPAR - 1, a, bv, true);
                else fma_vec(a, bv);
            }
        } else {
            for (int u = 0; u < U; ++u) {
                const int step = kc + u * NPAR;
                if (step >= nk) break;
                const bool live = step + sub < nk;
                const V a = shfl_idx(full, v_cur, (step - vb + sub) & 31, 32);
                vec_t<V, VW> bv;
                if (live && col_ok) bv = ld_shared_vec<V, VW>(st + u * NPAR * SLOT);
                else
#pragma unroll
                    for (int w = 0; w < VW; ++w) bv.v[w] = vzero<V>();
                const int step_last = (step + NPAR < nk ? step + NPAR : nk) - 1;
                if (step_last >= row_end) boundary(step, step_last, a, bv, live);
                else if (live) fma_vec(a, bv);
            }
        }
    }
    if (failed) {
        if (lane == 0) atomicExch(err_word, FSB_ERR_TIMEOUT);
        // drain the copies still in flight (bounded) before the ring is released
        for (int d = b; d < b + kGatherStages && d < n_batches; ++d)
            mbar_wait(smem_u32(bars + d % kGatherStages), (uint32_t)((d / kGatherStages) & 1));
        if (blockIdx.y == 0 && lane == 0) carry_row[unit] = -1;
        return;
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
    if (blockIdx.y == 0 && lane == 0) carry_row[unit] = open ? r1 : -1;
}

template <class V, class A, class O, class I, class P>
int launch_gather(const fsb_csr* Am, const V* val, const I* col, const P* ptr, const I* rmap, const V* B, int64_t ldb,
                  int64_t n_dense, O* C, int64_t ldc, const fsb_plan* plan, void* workspace, int64_t workspace_bytes,
                  cudaStream_t st, int* err_word) {
    constexpr int kMaxBytes = (int)(sizeof(V) > sizeof(O) ? sizeof(V) : sizeof(O));
    constexpr int VW = 16 / kMaxBytes >= 1 ? 16 / kMaxBytes : 1;
    const int64_t n_units = plan->n_units;
    if (plan->items_per_unit < 1 || plan->items_per_unit > kMaxItemsPerUnit || n_units != ceil_div(Am->n_rows + Am->nnz, plan->items_per_unit) ||
        !plan->unit_coords || plan->row_cap > 0) {
        fsb_host::set_error("fsb_spmm_csr: gather plan does not match the matrix");
        return FSB_ERR_INVALID;
    }
    const int64_t target = plan->n_tile > 0 ? plan->n_tile : n_dense;
    int lpn_log2 = 0;
    while ((1LL << lpn_log2) * VW < target && lpn_log2 < 5) ++lpn_log2;
    // bulk copies: 16-byte aligned sources, destinations and sizes
    const int64_t tile_bytes = (int64_t)(VW << lpn_log2) * (int64_t)sizeof(V);
    const bool multi_tile = n_dense > (int64_t)(VW << lpn_log2);
    const bool aligned = aligned16(B) && (ldb * (int64_t)sizeof(V)) % 16 == 0 &&
                         (n_dense * (int64_t)sizeof(V)) % 16 == 0 && (!multi_tile || tile_bytes % 16 == 0) &&
                         ((uintptr_t)C) % (VW * sizeof(O)) == 0 && ldc % VW == 0 && n_dense % VW == 0;
    if (!aligned) {
        fsb_host::set_error("fsb_spmm_csr: the gather algorithm needs 16-byte aligned B rows and C rows");
        return FSB_ERR_UNSUPPORTED;
    }
    const int64_t need = merge_scratch_bytes(n_units, n_dense, (int)sizeof(A));
    if (!workspace || workspace_bytes < need) {
        fsb_host::set_error("fsb_spmm_csr: workspace %lld bytes < %lld", (long long)workspace_bytes, (long long)need);
        return FSB_ERR_WORKSPACE;
    }
    if (lpn_log2 < 3) {
        fsb_host::set_error("fsb_spmm_csr: the gather algorithm needs column tiles of at least 8 lanes");
        return FSB_ERR_UNSUPPORTED;
    }
    const int LPN = 1 << lpn_log2, NPAR = 32 >> lpn_log2;
    const int U = NPAR >= kGatherRows ? 1 : kGatherRows / NPAR;
    const int stage_bytes = U * NPAR * LPN * VW * (int)sizeof(V);
    const size_t smem = (size_t)kBarBytes + (size_t)(kSpmmThreads / 32) * kGatherStages * stage_bytes;
    const int64_t col_tiles = ceil_div(n_dense, (int64_t)LPN * VW);
    const int64_t blocks = ceil_div(n_units, kSpmmThreads / 32);
    if (col_tiles > 65535 || blocks > 0x7fffffffLL || smem > 200 * 1024) {
        fsb_host::set_error("fsb_spmm_csr: gather grid or ring too large");
        return FSB_ERR_LIMIT;
    }
    const bool addr32 = (Am->n_cols * ldb + n_dense) < 0x7fffffffLL;
    auto pick = [&]() {
        using K = void (*)(const V*, const I*, const P*, const I*, const V*, int64_t, O*, int64_t, int64_t, int64_t,
                           const int64_t*, int64_t, int64_t, int64_t*, A*, A*, int*);
        K k = nullptr;
#define FSB_PICK(L) \
    if (lpn_log2 == L) k = addr32 ? k_spmm_gather<V, A, O, I, P, VW, L, true> : k_spmm_gather<V, A, O, I, P, VW, L, false>;
        FSB_PICK(3)
        FSB_PICK(4)
        FSB_PICK(5)
#undef FSB_PICK
        return k;
    };
    auto kern = pick();
    if (smem > 48 * 1024) {  // per device and function; cheap to repeat
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) {
            fsb_host::set_error("cudaFuncSetAttribute: %s", cudaGetErrorString(e));
            return FSB_ERR_LAUNCH;
        }
    }
    MergeScratch ms = merge_scratch_carve(workspace, n_units, n_dense, (int)sizeof(A));
    dim3 g((unsigned)blocks, (unsigned)col_tiles);
    const int64_t thr = plan->comp_threshold > 0 ? plan->comp_threshold : 0;
    kern<<<g, kSpmmThreads, smem, st>>>(val, col, ptr, rmap, B, ldb, C, ldc, Am->n_rows, n_dense, plan->unit_coords,
                                        n_units, thr, ms.carry_row, static_cast<A*>(ms.carry_val),
                                        static_cast<A*>(ms.head_val), err_word);
    int rc = fsb_host::check_launch("k_spmm_gather");
    if (rc) return rc;
    k_spmm_merge_fixup<A, O, I, P><<<(unsigned)blocks, kSpmmThreads, 0, st>>>(
        ms.carry_row, static_cast<const A*>(ms.carry_val), static_cast<const A*>(ms.head_val), n_units, n_dense, ptr,
        rmap, C, ldc);
    return fsb_host::check_launch("k_spmm_merge_fixup");
}

// Launch for value type VSel only (each fsb_spmm_gather_*.cu instantiates one).
template <class VSel>
int gather_dispatch_for(const fsb_csr* A, const void* B, int64_t ldb, int64_t n_dense, void* C, int64_t ldc,
                        int out_dtype, int acc_mode, const fsb_plan* plan, void* workspace, int64_t workspace_bytes,
                        cudaStream_t st, int* err_word) {
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
                    return launch_gather<V, Ac, O, I, P>(
                        A, static_cast<const V*>(A->values), static_cast<const I*>(A->col_idx),
                        static_cast<const P*>(A->row_ptr), static_cast<const I*>(A->row_map),
                        static_cast<const V*>(B), ldb, n_dense, static_cast<O*>(C), ldc, plan, workspace,
                        workspace_bytes, st, err_word);
                });
            });
        }
    });
}

#define FSB_GATHER_DECL(NAME)                                                                                    \
    int NAME(const fsb_csr* A, const void* B, int64_t ldb, int64_t n_dense, void* C, int64_t ldc, int out_dtype, \
             int acc_mode, const fsb_plan* plan, void* workspace, int64_t workspace_bytes, cudaStream_t st,         \
             int* err_word)
FSB_GATHER_DECL(gather_dispatch_f16);
FSB_GATHER_DECL(gather_dispatch_bf16);
FSB_GATHER_DECL(gather_dispatch_f32);
FSB_GATHER_DECL(gather_dispatch_f64);
FSB_GATHER_DECL(gather_dispatch_c32);
FSB_GATHER_DECL(gather_dispatch_c64);
FSB_GATHER_DECL(gather_dispatch_c128);

}  // namespace fsb
