// fsb_bsr_tc.cu -- block-sparse (BSR, 16 x 16 blocks) SpMM on the 5th-generation
// tensor cores: tcgen05.mma with the accumulator in tensor memory.
//
// Where a sparse matrix is made of dense 16 x 16 blocks, each stored block is
// a real dense contraction and belongs on the tensor cores.  One CTA (four
// warps) owns one block row r and one 128-column tile of the dense operand;
// it computes the transposed tile
//
//     D[m][n] = sum over blocks (r, j):  sum_k  B[16 j + k][c0 + m] * A_rj[n][k]
//
// i.e. D (128 x 16, fp32, in TMEM: lane m, column n) = C[16 r + n][c0 + m],
// one tcgen05.mma.kind::f16 of shape M = 128, N = 16, K = 16 per stored block:
//   * the A operand is the B slice (16 rows x 128 columns), MN-major: row-major
//     B needs no transpose, only re-tiling into 8 x 8 core matrices;
//   * the B operand is the 16 x 16 block, K-major (its rows are contiguous).
// Both operands are staged by the CTA's threads into two alternating
// shared-memory stages (SWIZZLE_NONE canonical layouts); one thread issues the
// MMA and commits it to the stage's mbarrier, which frees the stage for the
// block after next.  At the end each warp reads its 32 TMEM lanes
// (tcgen05.ld 32x32b.x16) and stores 16 rows of C, coalesced along columns.
//
// Two stagings of the B slices:
//   * k_bsr_spmm_tma (default): the Tensor Memory Accelerator loads each
//     slice as two 64-column x 16-row boxes of a 2-D tensor map over B
//     (128-byte swizzle; SWIZZLE_128B MN-major operand) and each block as one
//     box of a 5-D tensor map over the block array that lands in the K-major
//     core-matrix order, into a 4-stage ring.  Persistent and warp
//     specialised: one lane loads and issues MMAs across the CTA's block rows,
//     two TMEM accumulators alternate between rows, four epilogue warps drain
//     one row while the next accumulates;
//   * k_bsr_spmm_tc: the CTA's threads copy the slice with 16-byte loads into
//     two alternating stages (SWIZZLE_NONE MN-major operand).
//
// TMEM: 32 columns per CTA (two 16-column accumulators in the persistent
// kernel); at most 16 CTAs are resident per SM, so allocations never exceed
// the SM's 512 columns and never wait.
// Every mbarrier wait is bounded (1 s, globaltimer); on expiry the kernel
// records FSB_ERR_TIMEOUT in the device error word (fsb_device_error), waits
// (bounded) for the MMA it issued, frees its TMEM and returns.
#include <type_traits>

#include "fsb_tma.cuh"

namespace fsb {

int* gather_error_word();  // fsb_spmm_gather.cu: the device error word

namespace bsr {

constexpr int kThreads = 128;
constexpr int kM = 128;                         // dense columns per tile (MMA M)
constexpr int kAStageBytes = kM * 16 * 2;       // 16 B rows x 128 columns, 16-bit
constexpr int kBStageBytes = 16 * 16 * 2;       // one 16 x 16 block
constexpr int kTmemCols = 32;                   // allocation unit (16 used)

// Instruction descriptor, kind::f16: D f32 (bits 4-5 = 1), A and B 16-bit
// (bits 7-9, 10-12: 0 = f16, 1 = bf16), A MN-major (bit 15), B K-major
// (bit 16 = 0), N >> 3 at bits 17-22, M >> 4 at bits 24-28.
template <bool BF16>
__host__ __device__ constexpr uint32_t instr_desc() {
    return (1u << 4) | ((BF16 ? 1u : 0u) << 7) | ((BF16 ? 1u : 0u) << 10) | (1u << 15) | ((16u >> 3) << 17) |
           ((uint32_t)(kM >> 4) << 24);
}

// Shared-memory matrix descriptor, SWIZZLE_NONE: start address, leading
// (K-direction) and stride (M/N-direction) byte offsets between 8 x 16-byte
// core matrices, each >> 4; version 1 (bits 46-47); layout 0 (bits 61-63).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

using tma::mbar_wait;
using tma::smem_u32;

template <class T>
__device__ __forceinline__ uint4 ld_vec16(const T* p) {
    return __ldg(reinterpret_cast<const uint4*>(p));
}

template <class V, class I, class P>
__global__ void __launch_bounds__(kThreads)
k_bsr_spmm_tc(const V* __restrict__ blocks, const I* __restrict__ bcol, const P* __restrict__ bptr,
              int64_t n_rows, int64_t n_cols, const V* __restrict__ B, int64_t ldb, int64_t n_dense,
              float* __restrict__ C, int64_t ldc, int* __restrict__ err) {
    constexpr bool kBf16 = std::is_same<V, __nv_bfloat16>::value;
    __shared__ __align__(1024) unsigned char sa[2][kAStageBytes];
    __shared__ __align__(128) unsigned char sb[2][kBStageBytes];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t tmem_base_slot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t r = blockIdx.x;
    const int64_t c0 = (int64_t)blockIdx.y * kM;
    const int cols = (int)((n_dense - c0) < kM ? (n_dense - c0) : kM);  // valid columns of the tile (multiple of 8)
    const int64_t b0 = idx(bptr[r]), b1 = idx(bptr[r + 1]);
    const int nb = (int)(b1 - b0);

    // zero both A stages once: columns past the tile's end stay zero
    for (int i = tid; i < 2 * kAStageBytes / 16; i += kThreads)
        reinterpret_cast<uint4*>(&sa[0][0])[i] = make_uint4(0, 0, 0, 0);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_slot;
    constexpr uint32_t idesc = instr_desc<kBf16>();

    bool failed = false;
    for (int b = 0; b < nb; ++b) {
        const int s = b & 1;
        if (b >= 2) {
            // stage s is free once the MMA of block b - 2 completed; the
            // outcome is made uniform across the CTA before anyone breaks
            const bool ok = mbar_wait(smem_u32(&bars[s]), (uint32_t)(((b >> 1) - 1) & 1));
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
        }
        const int64_t jb = idx(bcol[b0 + b]);
        // A stage (MN-major): element (m, k) at (m % 8) * 2 + k0 * 16 +
        // (m / 8) * 128 + k1 * (kM / 8) * 128, k = 8 k1 + k0.  Thread chunks:
        // 16-byte runs of 8 columns of one B row; a warp covers whole core
        // matrices (k0 fastest), so its stores are conflict-free.
#pragma unroll
        for (int it = 0; it < (16 * (kM / 8)) / kThreads; ++it) {
            const int L = tid + it * kThreads;
            const int k0 = L & 7, clo = (L >> 3) & 3, rest = L >> 5;
            const int chunk = (rest % (kM / 32)) * 4 + clo;  // 8-column group 0 .. kM/8-1
            const int k1 = rest / (kM / 32);
            const int k = 8 * k1 + k0;
            const int64_t brow = jb * 16 + k;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (chunk * 8 < cols && brow >= 0 && brow < n_cols) v = ld_vec16(B + brow * ldb + c0 + chunk * 8);
            *reinterpret_cast<uint4*>(&sa[s][(chunk * 128) + k0 * 16 + k1 * (kM / 8) * 128]) = v;
        }
        // B stage (K-major block): element (n, k) at (n % 8) * 16 + (k % 8) * 2
        // + (n / 8) * 256 + (k / 8) * 128; 32 chunks of 8 values
        if (tid < 32) {
            const int n = tid >> 1, kc = tid & 1;
            const uint4 v = ld_vec16(blocks + (b0 + b) * 256 + n * 16 + kc * 8);
            *reinterpret_cast<uint4*>(&sb[s][(n & 7) * 16 + (n >> 3) * 256 + kc * 128]) = v;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // A: LBO = K-direction core stride (kM / 8 cores of 128 B), SBO = 128 B
            const uint64_t adesc = smem_desc(smem_u32(&sa[s][0]), (kM / 8) * 128, 128);
            // B: LBO = K-direction core stride 128 B, SBO = N-direction 256 B
            const uint64_t bdesc = smem_desc(smem_u32(&sb[s][0]), 128, 256);
            const uint32_t accumulate = b > 0 ? 1u : 0u;
            const uint32_t zero = 0;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(zero), "r"(zero), "r"(zero), "r"(zero)
                : "memory");
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&bars[s]))
                         : "memory");
        }
    }
    // the last MMA (all earlier ones complete before it)
    if (nb > 0 && !failed) {
        const int last = nb - 1;
        const bool ok = mbar_wait(smem_u32(&bars[last & 1]), (uint32_t)((last >> 1) & 1));
        failed = __syncthreads_or(!ok) != 0;
    }
    if (failed) {
        if (tid == 0) atomicExch(err, FSB_ERR_TIMEOUT);
        // drain (bounded) whatever this CTA committed before freeing TMEM
        for (int b = nb > 2 ? nb - 2 : 0; b < nb; ++b) mbar_wait(smem_u32(&bars[b & 1]), (uint32_t)((b >> 1) & 1));
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        uint32_t d[16];
        if (nb > 0) {
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15}, [%16];"
                : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
                  "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]),
                  "=r"(d[15])
                : "r"(taddr)
                : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        } else {
#pragma unroll
            for (int n = 0; n < 16; ++n) d[n] = 0u;  // empty block row: zeros
        }
        const int m = warp * 32 + lane;
        if (m < cols) {
#pragma unroll
            for (int n = 0; n < 16; ++n) {
                const int64_t row = r * 16 + n;
                if (row < n_rows) __stcs(C + row * ldc + c0 + m, __uint_as_float(d[n]));
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

constexpr int kTmaStages = 4;
constexpr int kTmaBoxCols = 64;                      // 128 bytes of 16-bit values
constexpr int kTmaBoxBytes = kTmaBoxCols * 16 * 2;  // 2 KB per box, 2 boxes per slice

// Descriptor of a SWIZZLE_128B MN-major operand (layout type 2): 64-column x
// 8-row atoms of 1 KB; LBO = byte stride between 64-column groups, SBO =
// byte stride between 8-row K groups.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return smem_desc(addr, lbo, sbo) | (2ull << 61);
}

// L2 policies of the persistent kernel: B slices are re-read by every block
// row that names their block column (keep them), blocks and C pass once.
__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar,
                                            uint64_t pol) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1, {%2, "
        "%3}], [%4], %5;" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar), "l"(pol)
        : "memory");
}

__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap* map, int c4, uint32_t bar,
                                            uint64_t pol) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1, {%2, "
        "%3, %4, %5, %6}], [%7], %8;" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(0), "r"(0), "r"(0), "r"(c4), "r"(bar), "l"(pol)
        : "memory");
}

// C store that bypasses L1 and enters L2 as evict-first.
__device__ __forceinline__ void st_evict_first(float* p, float v, uint64_t pol) {
    asm volatile("st.global.L1::no_allocate.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(pol) : "memory");
}

// Persistent, warp-specialised pipeline.  Each CTA takes block rows
// blockIdx.x, blockIdx.x + gridDim.x, ... of one 128-column tile:
//   * warp 4, one lane: TMA loads of each stored block's B slice (two 64 x 16
//     boxes of bmap) and of the 16 x 16 block itself (one box of amap, a 5-D
//     view of the block array whose box lands in the K-major core-matrix
//     order) into an S-stage ring, up to S blocks ahead and across block-row
//     boundaries; the MMA once a stage is full and its commit to the stage's
//     empty barrier; after a row's last MMA a commit to the row's
//     accumulator barrier.  Rows alternate between two 16-column TMEM
//     accumulators, so the next row's MMAs run while the previous row drains;
//   * warps 0-3 (the four TMEM lane quarters): wait for a row's accumulator,
//     read it (tcgen05.ld 32x32b, two 8-column halves), release it through
//     the accumulator-empty barrier and store the 16 C rows.
// Every wait is bounded; on expiry the waiting thread records
// FSB_ERR_TIMEOUT, raises the CTA's fail flag (the other roles stop at their
// next wait), and the MMA lane waits (bounded) for its copies and MMAs in
// flight before the CTA frees its TMEM.
constexpr int kPersistWarps = 5;
constexpr int kPersistThreads = 32 * kPersistWarps;
constexpr int kPersistCtasPerSm = 8;

// Bounded wait that also gives up when another role raised the fail flag.
__device__ __forceinline__ bool mbar_wait_or_fail(uint32_t bar, uint32_t parity, volatile int* fail) {
    if (tma::mbar_test(bar, parity)) return true;
    const unsigned long long t0 = tma::now_ns();
    while (!tma::mbar_test(bar, parity)) {
        if (*fail) return false;
        if (tma::now_ns() - t0 > tma::kWaitNs) return false;
    }
    return true;
}

template <class V, class I, class P>
__global__ void __launch_bounds__(kPersistThreads)
k_bsr_spmm_tma(const __grid_constant__ CUtensorMap bmap, const __grid_constant__ CUtensorMap amap,
               const I* __restrict__ bcol, const P* __restrict__ bptr, int64_t n_rows, int64_t n_block_rows,
               int64_t n_dense, float* __restrict__ C, int64_t ldc, int* __restrict__ err) {
    constexpr bool kBf16 = std::is_same<V, __nv_bfloat16>::value;
    constexpr int S = kTmaStages;
    constexpr uint32_t kStageTx = 2 * kTmaBoxBytes + kBStageBytes;
    __shared__ __align__(1024) unsigned char sa[S][2 * kTmaBoxBytes];
    __shared__ __align__(128) unsigned char sb[S][kBStageBytes];
    __shared__ __align__(8) uint64_t full[S], empty[S], acc_full[2], acc_empty[2];
    __shared__ uint32_t tmem_base_slot;
    __shared__ volatile int fail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t c0 = (int64_t)blockIdx.y * kM;
    const int cols = (int)((n_dense - c0) < kM ? (n_dense - c0) : kM);
    const int64_t stride = gridDim.x;

    if (tid == 0) {
        for (int i = 0; i < S; ++i) {
            tma::mbar_init(smem_u32(&full[i]), 1);
            tma::mbar_init(smem_u32(&empty[i]), 1);
        }
        for (int i = 0; i < 2; ++i) {
            tma::mbar_init(smem_u32(&acc_full[i]), 1);
            tma::mbar_init(smem_u32(&acc_empty[i]), 4);  // one arrival per epilogue warp
        }
        tma::mbar_init_fence();
        fail = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_slot;
    constexpr uint32_t idesc = instr_desc<kBf16>();

    if (warp == 4) {
        if (lane == 0) {
            // issue cursor: block ib of row ir (ie = the row's end), issued blocks so far
            int64_t ir = blockIdx.x, ib = 0, ie = 0;
            if (ir < n_block_rows) {
                ib = idx(bptr[ir]);
                ie = idx(bptr[ir + 1]);
            }
            uint32_t issued = 0, g = 0;
            bool ok = true;
            const uint64_t keep_b = policy_evict_last(), pass_once = policy_evict_first();
            auto issue_more = [&](uint32_t upto) {  // blocks [issued, upto] of this CTA, as far as they exist
                while (ok && issued <= upto) {
                    while (ib >= ie && ir < n_block_rows) {
                        ir += stride;
                        if (ir < n_block_rows) {
                            ib = idx(bptr[ir]);
                            ie = idx(bptr[ir + 1]);
                        }
                    }
                    if (ir >= n_block_rows) return;
                    const uint32_t s = issued % S;
                    if (issued >= (uint32_t)S && !mbar_wait_or_fail(smem_u32(&empty[s]), ((issued / S) - 1) & 1u, &fail)) {
                        ok = false;
                        return;
                    }
                    const uint32_t bar = smem_u32(&full[s]);
                    tma::mbar_arrive_expect_tx(bar, kStageTx);
                    const int y = (int)(idx(bcol[ib]) * 16);
                    tma_load_2d(smem_u32(&sa[s][0]), &bmap, (int)c0, y, bar, keep_b);
                    tma_load_2d(smem_u32(&sa[s][kTmaBoxBytes]), &bmap, (int)c0 + kTmaBoxCols, y, bar, keep_b);
                    tma_load_5d(smem_u32(&sb[s][0]), &amap, (int)ib, bar, pass_once);
                    ++issued;
                    ++ib;
                }
            };
            int64_t k = 0;
            for (int64_t r = blockIdx.x; ok && r < n_block_rows; r += stride, ++k) {
                const int nb = (int)(idx(bptr[r + 1]) - idx(bptr[r]));
                const uint32_t buf = (uint32_t)(k & 1);
                if (k >= 2 && !mbar_wait_or_fail(smem_u32(&acc_empty[buf]), (uint32_t)(((k >> 1) - 1) & 1), &fail)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                for (int j = 0; j < nb; ++j) {
                    issue_more(g + S - 1);
                    if (!ok || !mbar_wait_or_fail(smem_u32(&full[g % S]), (g / S) & 1u, &fail)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t s = g % S;
                    // A: two 64-column groups 2 KB apart (LBO), 8-row groups 1 KB apart (SBO)
                    const uint64_t adesc = smem_desc_sw128(smem_u32(&sa[s][0]), kTmaBoxBytes, 1024);
                    const uint64_t bdesc = smem_desc(smem_u32(&sb[s][0]), 128, 256);
                    const uint32_t accumulate = j > 0 ? 1u : 0u;
                    const uint32_t zero = 0;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                            tmem + buf * 16u),
                        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(zero), "r"(zero), "r"(zero), "r"(zero)
                        : "memory");
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     smem_u32(&empty[s]))
                                 : "memory");
                    ++g;
                }
                if (!ok) break;
                // the row's accumulator is final once every MMA issued so far completed
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&acc_full[buf]))
                             : "memory");
            }
            if (!ok) {
                fail = 1;
                atomicExch(err, FSB_ERR_TIMEOUT);
                // drain (bounded): the copies issued and the MMAs committed
                for (uint32_t q = g; q < issued; ++q) tma::mbar_wait(smem_u32(&full[q % S]), (q / S) & 1u);
                if (g > 0) tma::mbar_wait(smem_u32(&empty[(g - 1) % S]), ((g - 1) / S) & 1u);
            }
        }
        __syncwarp();
    } else {
        // epilogue warps: TMEM lane quarter `warp` = dense columns c0 + 32 warp + lane
        const uint64_t c_pol = policy_evict_first();
        int64_t k = 0;
        for (int64_t r = blockIdx.x; r < n_block_rows; r += stride, ++k) {
            const uint32_t buf = (uint32_t)(k & 1);
            // warp-uniform outcome: the TMEM loads below are warp-collective
            const bool ready = __all_sync(0xffffffffu, mbar_wait_or_fail(smem_u32(&acc_full[buf]),
                                                                         (uint32_t)((k >> 1) & 1), &fail));
            if (!ready) {
                if (lane == 0) atomicExch(err, FSB_ERR_TIMEOUT);
                fail = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const bool any = idx(bptr[r + 1]) > idx(bptr[r]);
            uint32_t d[16];
            if (any) {
                const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + buf * 16u;
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                    : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7])
                    : "r"(taddr)
                    : "memory");
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                    : "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]),
                      "=r"(d[15])
                    : "r"(taddr + 8u)
                    : "memory");
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            } else {
#pragma unroll
                for (int n = 0; n < 16; ++n) d[n] = 0u;  // empty block row: zeros
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[buf])) : "memory");
            const int m = warp * 32 + lane;
            if (m < cols) {
#pragma unroll
                for (int n = 0; n < 16; ++n) {
                    const int64_t row = r * 16 + n;
                    if (row < n_rows) st_evict_first(C + row * ldc + c0 + m, __uint_as_float(d[n]), c_pol);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

// 2-D tensor map over B (columns innermost): 64 x 16 boxes, 128-byte swizzle,
// zero fill outside the matrix.  False when it cannot be encoded.
static bool encode_b_map(CUtensorMap* map, int value_dtype, const void* B, int64_t n_cols, int64_t ldb,
                         int64_t n_dense) {
    auto fn = tma::encode_fn();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)n_dense, (cuuint64_t)n_cols};
    const cuuint64_t strides[1] = {(cuuint64_t)ldb * 2};
    const cuuint32_t box[2] = {(cuuint32_t)kTmaBoxCols, 16};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult rc = fn(map, value_dtype == FSB_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16,
                           2, const_cast<void*>(B), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return rc == CUDA_SUCCESS;
}

// 5-D tensor map over the block array: (8 values, 8 rows, 2 halves of a
// row, 2 groups of 8 rows, block) with byte strides 32, 16, 256, 512; a box
// {8, 8, 2, 2, 1} lands as element (n, k) at (n % 8) * 16 + (k % 8) * 2 +
// (k / 8) * 128 + (n / 8) * 256, the K-major core-matrix order of a block.
static bool encode_block_map(CUtensorMap* map, int value_dtype, const void* blocks, int64_t n_blocks) {
    auto fn = tma::encode_fn();
    if (!fn || n_blocks < 1 || n_blocks >= 0x7fffffffLL) return false;
    const cuuint64_t dims[5] = {8, 8, 2, 2, (cuuint64_t)n_blocks};
    const cuuint64_t strides[4] = {32, 16, 256, 512};
    const cuuint32_t box[5] = {8, 8, 2, 2, 1};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    const CUresult rc = fn(map, value_dtype == FSB_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16,
                           5, const_cast<void*>(blocks), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return rc == CUDA_SUCCESS;
}

}  // namespace bsr
}  // namespace fsb

extern "C" int fsb_bsr_spmm_tc(const void* block_values, int value_dtype, const void* block_col, int index_dtype,
                               const void* block_row_ptr, int ptr_dtype, int64_t n_rows, int64_t n_cols,
                               int64_t n_blocks, const void* B, int64_t ldb, int64_t n_dense, float* C, int64_t ldc,
                               int staging, void* stream) {
    if (value_dtype != FSB_BF16 && value_dtype != FSB_F16) {
        fsb_host::set_error("fsb_bsr_spmm_tc: values and B must be bfloat16 or float16");
        return FSB_ERR_UNSUPPORTED;
    }
    if (n_rows < 0 || n_cols < 0 || n_blocks < 0 || n_dense < 0 || ldb < n_dense || ldc < n_dense) {
        fsb_host::set_error("fsb_bsr_spmm_tc: bad sizes");
        return FSB_ERR_INVALID;
    }
    if (n_rows == 0 || n_dense == 0) return FSB_OK;
    if (!block_row_ptr || !C || !B) {
        fsb_host::set_error("fsb_bsr_spmm_tc: null pointer");
        return FSB_ERR_INVALID;
    }
    // 16-byte row slices of B and 16-byte block rows
    if (((uintptr_t)B) % 16 || ldb % 8 || n_dense % 8 || (block_values && ((uintptr_t)block_values) % 16)) {
        fsb_host::set_error("fsb_bsr_spmm_tc: B must be 16-byte aligned with ldb and n_dense multiples of 8");
        return FSB_ERR_UNSUPPORTED;
    }
    const int64_t n_block_rows = fsb::ceil_div(n_rows, (int64_t)16);
    const int64_t tiles = fsb::ceil_div(n_dense, (int64_t)fsb::bsr::kM);
    if (n_block_rows > 0x7fffffffLL || tiles > 65535) {
        fsb_host::set_error("fsb_bsr_spmm_tc: grid too large");
        return FSB_ERR_LIMIT;
    }
    int* err = fsb::gather_error_word();
    if (!err) {
        fsb_host::set_error("fsb_bsr_spmm_tc: cannot resolve the device error word");
        return FSB_ERR_LAUNCH;
    }
    if (staging != FSB_BSR_STAGE_TMA && staging != FSB_BSR_STAGE_THREADS) {
        fsb_host::set_error("fsb_bsr_spmm_tc: staging must be FSB_BSR_STAGE_TMA or FSB_BSR_STAGE_THREADS");
        return FSB_ERR_INVALID;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    dim3 g((unsigned)n_block_rows, (unsigned)tiles);
    CUtensorMap bmap, amap;
    if (staging == FSB_BSR_STAGE_TMA) {
        if (n_cols >= 0x7fffffffLL || n_dense >= 0x7fffffffLL ||
            !fsb::bsr::encode_b_map(&bmap, value_dtype, B, n_cols, ldb, n_dense) ||
            (n_blocks > 0 && !fsb::bsr::encode_block_map(&amap, value_dtype, block_values, n_blocks))) {
            fsb_host::set_error("fsb_bsr_spmm_tc: no tensor map can be encoded for B or the blocks "
                                "(use FSB_BSR_STAGE_THREADS)");
            return FSB_ERR_UNSUPPORTED;
        }
        if (n_blocks == 0) amap = bmap;  // never read: no block row holds a block
        return fsb::dispatch_idx(index_dtype, [&](auto ti) -> int {
            using I = typename decltype(ti)::type;
            return fsb::dispatch_idx(ptr_dtype, [&](auto tp) -> int {
                using P = typename decltype(tp)::type;
                // persistent grid: kPersistCtasPerSm CTAs per SM and column tile
                int dev = 0, sms = 148;
                if (cudaGetDevice(&dev) == cudaSuccess)
                    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
                const int64_t cap = (int64_t)sms * fsb::bsr::kPersistCtasPerSm;
                dim3 gp((unsigned)(n_block_rows < cap ? n_block_rows : cap), (unsigned)tiles);
                if (value_dtype == FSB_BF16)
                    fsb::bsr::k_bsr_spmm_tma<__nv_bfloat16, I, P><<<gp, fsb::bsr::kPersistThreads, 0, st>>>(
                        bmap, amap, static_cast<const I*>(block_col), static_cast<const P*>(block_row_ptr), n_rows,
                        n_block_rows, n_dense, C, ldc, err);
                else
                    fsb::bsr::k_bsr_spmm_tma<__half, I, P><<<gp, fsb::bsr::kPersistThreads, 0, st>>>(
                        bmap, amap, static_cast<const I*>(block_col), static_cast<const P*>(block_row_ptr), n_rows,
                        n_block_rows, n_dense, C, ldc, err);
                return fsb_host::check_launch("k_bsr_spmm_tma");
            });
        });
    }
    return fsb::dispatch_idx(index_dtype, [&](auto ti) -> int {
        using I = typename decltype(ti)::type;
        return fsb::dispatch_idx(ptr_dtype, [&](auto tp) -> int {
            using P = typename decltype(tp)::type;
            if (value_dtype == FSB_BF16)
                fsb::bsr::k_bsr_spmm_tc<__nv_bfloat16, I, P><<<g, fsb::bsr::kThreads, 0, st>>>(
                    static_cast<const __nv_bfloat16*>(block_values), static_cast<const I*>(block_col),
                    static_cast<const P*>(block_row_ptr), n_rows, n_cols, static_cast<const __nv_bfloat16*>(B), ldb,
                    n_dense, C, ldc, err);
            else
                fsb::bsr::k_bsr_spmm_tc<__half, I, P><<<g, fsb::bsr::kThreads, 0, st>>>(
                    static_cast<const __half*>(block_values), static_cast<const I*>(block_col),
                    static_cast<const P*>(block_row_ptr), n_rows, n_cols, static_cast<const __half*>(B), ldb, n_dense,
                    C, ldc, err);
            return fsb_host::check_launch("k_bsr_spmm_tc");
        });
    });
}
