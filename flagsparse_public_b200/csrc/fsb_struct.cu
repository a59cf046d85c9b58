// fsb_struct.cu -- the structured form of the precision SpMV / SpMM: runs of
// consecutive columns and long rows.
//
// Matrices such as a band plus a few long rows hold most of their nonzeros
// either in runs of consecutive columns (the band) or in a few rows with many
// scattered columns.  The structured form keeps the caller's CSR arrays as
// they are and adds, once per matrix (fsb_struct_rows, fsb_struct_tiles and
// the host-side grouping of the long rows):
//   * per row: the row's longest run of consecutive columns (first column,
//     offset inside the row, length), or length -1 for a long row;
//   * per tile of 128 consecutive rows: the first column and the width
//     (a multiple of 16, at most 256) of the column span holding the tile's
//     runs; a run that does not fit is dropped (its row is then all scattered);
//   * the long rows: their indices, chunks of chunk_nnz nonzeros for the SpMM
//     and, for the SpMV, their nonzeros regrouped by blocks of xblock columns
//     of x with 16-bit offsets inside the block.
// Run values are read without their column indices; only the scattered
// nonzeros read an index.
//
// Kernels (values f16 / bf16, float32 accumulation and result; long rows
// accumulate compensated: exact products, per-batch sums folded by TwoSum):
//   * k_struct_spmv_tile: one CTA per tile, the tile's x window in shared
//     memory, a warp per row;
//   * k_struct_spmv_long + k_struct_spmv_fold: one CTA per (x block, slice of
//     the long rows) with the block of x in shared memory; a warp per (block,
//     row) segment gathers x from shared memory; partials folded in block
//     order;
//   * k_struct_spmm_band: tcgen05 -- the tile's runs as a dense 128 x span
//     operand (K-major, zeros outside each run) times the span's B rows
//     (MN-major), float32 accumulators in tensor memory; the epilogue adds
//     each row's scattered nonzeros and stores the row;
//   * k_struct_spmm_long + k_struct_spmm_fold: a warp per chunk of a long
//     row, the B rows of the next batch in flight while the current batch is
//     summed; partials folded in chunk order.
#include <algorithm>
#include <type_traits>

#include "fsb_tma.cuh"

namespace fsb {

int* gather_error_word();  // fsb_spmm_gather.cu: the device error word

namespace strc {

constexpr int kTileRows = 128;
constexpr int kSpanMax = 256;
constexpr int kThreads = 128;

using tma::mbar_wait;
using tma::smem_u32;

template <class V>
__device__ __forceinline__ unsigned short bits16(V v) {
    unsigned short u;
    memcpy(&u, &v, 2);
    return u;
}

// ------------------------------------------------------------ prepare ----
// One warp per row: the longest run of consecutive columns (the first one on
// ties) of rows with at most long_min nonzeros; runs shorter than min_run
// count as none.  Longer rows are marked long (run_len -1).
template <class I, class P>
__global__ void k_struct_rows(const I* __restrict__ col, const P* __restrict__ ptr, int64_t n_rows, int64_t long_min,
                              int min_run, int32_t* __restrict__ run_col, int32_t* __restrict__ run_off,
                              int32_t* __restrict__ run_len) {
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < n_rows; r += warps) {
        const int64_t s = idx(ptr[r]), e = idx(ptr[r + 1]);
        const int64_t len = e - s;
        if (len > long_min) {
            if (lane == 0) {
                run_col[r] = 0;
                run_off[r] = 0;
                run_len[r] = -1;
            }
            continue;
        }
        int best_len = 0, best_start = 0, cur_start = 0, cur_len = 0;
        long long prev = -2;
        for (int64_t base = 0; base < len; base += 32) {
            const int64_t k = base + lane;
            const bool valid = k < len;
            const long long c = valid ? (long long)idx(col[s + k]) : 0;
            long long pc = __shfl_up_sync(full, c, 1);
            if (lane == 0) pc = prev;
            const bool brk = valid && (k == 0 || c != pc + 1);
            unsigned bm = __ballot_sync(full, brk);
            const int n_valid = (int)((len - base) < 32 ? (len - base) : 32);
            int p = 0;
            while (bm) {  // runs break at the set bits
                const int b = __ffs(bm) - 1;
                bm &= bm - 1;
                cur_len += b - p;
                if (cur_len > best_len) {
                    best_len = cur_len;
                    best_start = cur_start;
                }
                cur_start = (int)base + b;
                cur_len = 0;
                p = b;
            }
            cur_len += n_valid - p;
            prev = __shfl_sync(full, c, n_valid - 1);
        }
        if (cur_len > best_len) {
            best_len = cur_len;
            best_start = cur_start;
        }
        if (lane == 0) {
            const bool keep = best_len >= min_run && best_len > 0;
            run_col[r] = keep ? (int32_t)idx(col[s + best_start]) : 0;
            run_off[r] = keep ? best_start : 0;
            run_len[r] = keep ? best_len : 0;
        }
    }
}

// One warp per tile of kTileRows rows: the tile's span starts at its
// smallest run column; runs ending more than kSpanMax columns after it are
// dropped (their rows become all scattered); the width is rounded up to 16.
__global__ void k_struct_tiles(int64_t n_rows, const int32_t* __restrict__ run_col, int32_t* __restrict__ run_off,
                               int32_t* __restrict__ run_len, int64_t* __restrict__ tile_base,
                               int32_t* __restrict__ tile_span, int64_t n_tiles) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int64_t t = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (t >= n_tiles) return;
    const int64_t r0 = t * kTileRows;
    long long lo = 0x7fffffffffffffffLL;
#pragma unroll
    for (int j = 0; j < kTileRows / 32; ++j) {
        const int64_t r = r0 + lane + 32 * j;
        if (r < n_rows && run_len[r] > 0) lo = min(lo, (long long)run_col[r]);
    }
    for (int o = 16; o; o >>= 1) lo = min(lo, __shfl_xor_sync(full, lo, o));
    long long hi = lo;
#pragma unroll
    for (int j = 0; j < kTileRows / 32; ++j) {
        const int64_t r = r0 + lane + 32 * j;
        if (r < n_rows && run_len[r] > 0) {
            const long long end = (long long)run_col[r] + run_len[r];
            if (end - lo > kSpanMax) {
                run_len[r] = 0;
                run_off[r] = 0;
            } else {
                hi = max(hi, end);
            }
        }
    }
    for (int o = 16; o; o >>= 1) hi = max(hi, __shfl_xor_sync(full, hi, o));
    if (lane == 0) {
        const bool any = lo != 0x7fffffffffffffffLL;
        tile_base[t] = any ? (int64_t)lo : 0;
        tile_span[t] = any ? (int32_t)((hi - lo + 15) / 16 * 16) : 0;
    }
}

// ---------------------------------------------------------------- SpMV ----
// One CTA per tile of 128 rows, the tile's x window in shared memory, one
// thread per row.  A row's run values are read as the 16-byte aligned chunks
// covering them (each element multiplied where it falls inside the run), so a
// warp's load instruction brings 8 values of each of its 32 rows; scattered
// nonzeros four at a time (their loads issued together).
template <class V, class I, class P>
__global__ void __launch_bounds__(kThreads)
k_struct_spmv_tile(const V* __restrict__ val, const I* __restrict__ col, const P* __restrict__ ptr, int64_t n_rows,
                   int64_t n_cols, const int32_t* __restrict__ run_col, const int32_t* __restrict__ run_off,
                   const int32_t* __restrict__ run_len, const int64_t* __restrict__ tile_base,
                   const int32_t* __restrict__ tile_span, const V* __restrict__ x, float* __restrict__ y) {
    __shared__ float xs[kSpanMax];
    constexpr int kVec = 16 / (int)sizeof(V);
    const int tid = threadIdx.x;
    const int64_t t = blockIdx.x;
    const int64_t kbase = tile_base[t];
    const int span = tile_span[t];
    const int64_t r = t * kTileRows + tid;
    const bool live = r < n_rows;
    const int rl = live ? run_len[r] : -1;
    int64_t s = 0, e = 0;
    int ro = 0, kc = 0;
    if (rl >= 0) {
        s = idx(ptr[r]);
        e = idx(ptr[r + 1]);
        if (rl > 0) {
            ro = run_off[r];
            kc = (int)(run_col[r] - kbase);
        }
    }
    for (int i = tid; i < span; i += kThreads) {
        const int64_t c = kbase + i;
        xs[i] = c < n_cols ? to_f32(ld_ro1(x + c)) : 0.f;
    }
    __syncthreads();
    if (rl < 0) return;  // past the matrix, or a long row (written by the long-row kernels)
    float acc = 0.f;
    if (rl > 0) {
        // the 16-byte aligned chunks holding the run: run element q is element
        // q + lead of the chunk sequence starting at cbase (an aligned chunk
        // holding a valid element lies inside one page, so the loads are safe
        // whatever the values array's alignment)
        const uintptr_t a0 = reinterpret_cast<uintptr_t>(val + s + ro);
        const V* cbase = reinterpret_cast<const V*>(a0 & ~(uintptr_t)15);
        const int lead = (int)((a0 & 15u) / sizeof(V));
        const int n_ch = (lead + rl + kVec - 1) / kVec;
        for (int ci = 0; ci < n_ch; ci += 2) {
            const vec_t<V, kVec> w0 = ld_ro<V, kVec>(cbase + ci * kVec);
            vec_t<V, kVec> w1;
            if (ci + 1 < n_ch) w1 = ld_ro<V, kVec>(cbase + (ci + 1) * kVec);
#pragma unroll
            for (int u = 0; u < kVec; ++u) {
                const int q = ci * kVec + u - lead;
                if (q >= 0 && q < rl) acc = fmaf(to_f32(w0.v[u]), xs[kc + q], acc);
            }
            if (ci + 1 < n_ch) {
#pragma unroll
                for (int u = 0; u < kVec; ++u) {
                    const int q = (ci + 1) * kVec + u - lead;
                    if (q >= 0 && q < rl) acc = fmaf(to_f32(w1.v[u]), xs[kc + q], acc);
                }
            }
        }
    }
    const int64_t n_sc = (e - s) - rl;
    for (int64_t q0 = 0; q0 < n_sc; q0 += 4) {
        int64_t k[4];
        I c[4];
        V a[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t q = q0 + u;
            k[u] = q < n_sc ? (q < ro ? s + q : s + q + rl) : -1;
            if (k[u] >= 0) {
                c[u] = ld_stream1(col + k[u]);
                a[u] = ld_stream1(val + k[u]);
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k[u] >= 0) acc = fmaf(to_f32(a[u]), to_f32(ld_ro1(x + idx(c[u]))), acc);
    }
    y[r] = acc;
}

// Blocks of x in shared memory, one warp per (block, long row) segment.  The
// segment is read as the 16-byte aligned chunks covering it (8 offsets and 8
// values per lane and load; elements outside the segment are skipped); the
// products of 16-bit values are exact in float32, so each chunk's products
// are summed plainly and the chunk sum enters the lane's (s, c) accumulator
// by TwoSum.
template <class V>
__global__ void __launch_bounds__(1024, 1)
k_struct_spmv_long(const int64_t* __restrict__ seg_ptr, const V* __restrict__ seg_val,
                   const uint16_t* __restrict__ seg_off, int64_t n_long, int32_t xblock, const V* __restrict__ x,
                   int64_t n_cols, comp_t* __restrict__ partial) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* xs = reinterpret_cast<V*>(smem_raw);
    const unsigned full = 0xffffffffu;
    const int64_t b = blockIdx.x;
    const int64_t c0 = b * (int64_t)xblock;
    const int nx = (int)((n_cols - c0) < xblock ? (n_cols - c0) : xblock);
    constexpr int kVec = 16 / (int)sizeof(V);
    static_assert(kVec == 8, "16-bit values");
    if ((reinterpret_cast<uintptr_t>(x) & 15u) == 0 && (c0 % kVec) == 0) {
        const int nv = nx / kVec;
        for (int i = threadIdx.x; i < nv; i += blockDim.x)
            reinterpret_cast<uint4*>(xs)[i] = __ldg(reinterpret_cast<const uint4*>(x + c0) + i);
        for (int i = nv * kVec + threadIdx.x; i < nx; i += blockDim.x) xs[i] = x[c0 + i];
    } else {
        for (int i = threadIdx.x; i < nx; i += blockDim.x) xs[i] = x[c0 + i];
    }
    __syncthreads();
    const int64_t per = ceil_div(n_long, (int64_t)gridDim.y);
    const int64_t l0 = (int64_t)blockIdx.y * per;
    const int64_t l1 = (l0 + per) < n_long ? (l0 + per) : n_long;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int64_t l = l0 + warp; l < l1; l += nw) {
        const int64_t s = seg_ptr[b * n_long + l], e = seg_ptr[b * n_long + l + 1];
        comp_t acc{0.f, 0.f};
        if (e > s) {
            // aligned chunks: element p of the arrays sits in chunk p / 8 of
            // both (the offset and value arrays are 16-byte aligned here)
            const int64_t cf = s / kVec, cl = (e - 1) / kVec;
            for (int64_t c = cf + lane; c <= cl; c += 32) {
                const vec_t<uint16_t, kVec> o = ld_stream<uint16_t, kVec>(seg_off + c * kVec);
                const vec_t<V, kVec> v = ld_stream<V, kVec>(seg_val + c * kVec);
                float blk = 0.f;
#pragma unroll
                for (int u = 0; u < kVec; ++u) {
                    const int64_t p = c * kVec + u;
                    if (p >= s && p < e) blk = fmaf(to_f32(v.v[u]), to_f32(xs[o.v[u]]), blk);
                }
                acc = comp_add_value(acc, blk, 0.f);
            }
        }
        for (int o = 16; o; o >>= 1) acc = acc_add(acc, shfl_xor(full, acc, o, 32));
        if (lane == 0) partial[b * n_long + l] = acc;
    }
}

// One thread per long row: the blocks' partials in block order.
__global__ void k_struct_spmv_fold(const comp_t* __restrict__ partial, int64_t n_long, int64_t n_xblocks,
                                   const int32_t* __restrict__ long_rows, float* __restrict__ y) {
    const int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n_long) return;
    comp_t s = partial[l];
    for (int64_t b = 1; b < n_xblocks; ++b) s = acc_add(s, partial[b * n_long + l]);
    y[long_rows[l]] = s.s + s.c;
}

// ---------------------------------------------------------------- SpMM ----
// Long rows, one warp per chunk (x column tile of 32 in blockIdx.y): 4 lanes
// per nonzero with 8 columns (16 bytes) each, 8 nonzeros per step, batches
// of 32 nonzeros; the B rows of batch i + 1 are loaded while batch i is
// summed.  Products of 16-bit values are exact in float32: a batch's products
// are summed plainly per lane and folded into the (s, c) accumulator by
// TwoSum.
template <class V, class I, class P>
__global__ void __launch_bounds__(kThreads, 4)
k_struct_spmm_long(const V* __restrict__ val, const I* __restrict__ col, const P* __restrict__ ptr,
                   const int32_t* __restrict__ long_rows, const int32_t* __restrict__ chunk_row,
                   const int64_t* __restrict__ chunk_ptr, int32_t chunk_nnz, int64_t n_chunks,
                   const V* __restrict__ B, int64_t ldb, int64_t n_dense, comp_t* __restrict__ partial) {
    constexpr int VW = 8, LPN = 4, NPAR = 8, U = 4;
    using BV = vec_t<V, VW>;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, sub = lane / LPN;
    const int64_t c0 = (int64_t)blockIdx.y * 32 + (lane % LPN) * VW;
    const bool col_ok = c0 < n_dense;
    const V* Bl = B + (col_ok ? c0 : 0);
    const uint64_t keep_b = policy_evict_last();
    const int64_t warps = (int64_t)gridDim.x * (kThreads / 32);
    for (int64_t ch = (int64_t)blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5); ch < n_chunks; ch += warps) {
        const int l = chunk_row[ch];
        const int64_t row = long_rows[l];
        const int64_t rs = idx(ptr[row]), re = idx(ptr[row + 1]);
        const int64_t k0 = rs + (ch - chunk_ptr[l]) * (int64_t)chunk_nnz;
        const int64_t k1 = (k0 + chunk_nnz) < re ? (k0 + chunk_nnz) : re;
        const int nb = (int)((k1 - k0 + 31) / 32);
        comp_t acc[VW];
#pragma unroll
        for (int w = 0; w < VW; ++w) acc[w] = comp_t{0.f, 0.f};
        auto load_win = [&](int bi, V& v, I& c) {
            const int64_t k = k0 + (int64_t)bi * 32 + lane;
            if (bi < nb && k < k1) {
                v = ld_stream1(val + k);
                c = ld_stream1(col + k);
            } else {
                v = vzero<V>();
                c = 0;
            }
        };
        auto load_b = [&](I cw, BV (&bv)[U]) {
#pragma unroll
            for (int u = 0; u < U; ++u) bv[u] = ld_keep<V, VW>(Bl + idx(shfl_idx(full, cw, u * NPAR + sub, 32)) * ldb, keep_b);
        };
        // batch bi: its values (lane l holds nonzero 32 bi + l) and B rows;
        // nonzeros past the chunk's end take no part (a zero value times a
        // non-finite B entry would not be zero)
        auto consume = [&](int bi, V vw, const BV (&bv)[U]) {
            const int cnt = (int)((k1 - k0) - (int64_t)bi * 32);
            float blk[VW];
#pragma unroll
            for (int w = 0; w < VW; ++w) blk[w] = 0.f;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const float a = to_f32(shfl_idx(full, vw, u * NPAR + sub, 32));
                if (u * NPAR + sub < cnt) {
#pragma unroll
                    for (int w = 0; w < VW; ++w) blk[w] = fmaf(a, to_f32(bv[u].v[w]), blk[w]);
                }
            }
#pragma unroll
            for (int w = 0; w < VW; ++w) acc[w] = comp_add_value(acc[w], blk[w], 0.f);
        };
        // Two batches per iteration.  At the top: (va, ca) = batch bi with its
        // B rows ba in flight, (vb, cb) = the window of batch bi + 1.
        V va, vb, vn, vm;
        I ca, cb, cn, cm;
        BV ba[U], bb[U];
        load_win(0, va, ca);
        load_win(1, vb, cb);
        load_b(ca, ba);
        for (int bi = 0; bi < nb; bi += 2) {
            if (bi + 1 < nb) load_b(cb, bb);  // batch bi + 1's B rows out before batch bi is summed
            load_win(bi + 2, vn, cn);
            consume(bi, va, ba);
            if (bi + 1 >= nb) break;
            if (bi + 2 < nb) load_b(cn, ba);  // batch bi + 2's B rows out before batch bi + 1 is summed
            load_win(bi + 3, vm, cm);
            consume(bi + 1, vb, bb);
            va = vn;
            ca = cn;
            vb = vm;
            cb = cm;
        }
#pragma unroll
        for (int w = 0; w < VW; ++w) acc[w] = segment_reduce(full, acc[w], LPN, 32);
        if (sub == 0 && col_ok) {
            comp_t* dst = partial + ch * n_dense + c0;
#pragma unroll
            for (int w = 0; w < VW; ++w) dst[w] = acc[w];
        }
    }
}

// One warp per (long row, 32-column tile): the chunks' partials in chunk order.
__global__ void k_struct_spmm_fold(const comp_t* __restrict__ partial, const int64_t* __restrict__ chunk_ptr,
                                   const int32_t* __restrict__ long_rows, int64_t n_long, int64_t n_dense,
                                   float* __restrict__ C, int64_t ldc) {
    const int64_t l = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (l >= n_long) return;
    const int64_t c = (int64_t)blockIdx.y * 32 + (threadIdx.x & 31);
    if (c >= n_dense) return;
    const int64_t a = chunk_ptr[l], z = chunk_ptr[l + 1];
    comp_t s = partial[a * n_dense + c];
    for (int64_t ch = a + 1; ch < z; ++ch) s = acc_add(s, partial[ch * n_dense + c]);
    C[(int64_t)long_rows[l] * ldc + c] = s.s + s.c;
}

// Long rows in tiles: the long rows in groups of kLtRows, the columns in
// blocks of kLtCols.  A prepared record stream holds, per (group, column
// block) segment, the group's nonzeros in that block ordered by row, each as
// one 32-bit record (16-bit value bits | column inside the block << 16),
// padded to 16 bytes, with the segment's per-row record starts (kLtRsEntries
// 16-bit entries).  One CTA of 1024 threads per (group, column range), two
// shared-memory stages: a block's B rows (contiguous), row starts and records
// arrive by bulk copies (completion on the stage's mbarrier, bounded waits).
// Each warp walks the blocks on its own, multiplying out of shared memory:
// LPN = N / 8 lanes per row, 8 columns (16 bytes) per lane, each row's
// products of a block summed plainly (exact products) and folded into its
// (s, c) accumulator by TwoSum.  A warp done with a block counts itself out
// of the stage; the last one refills the stage with the block two ahead, so
// no CTA-wide barrier separates blocks.  Each CTA stores one compensated
// partial per row; k_struct_spmm_lfold adds them in column-range order.
constexpr int kLtRows = 512;
constexpr int kLtCols = 1024;
constexpr int kLtRsEntries = 520;  // kLtRows + 1 starts, padded to 16 bytes
constexpr int kLtThreads = 1024;

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// Float32 pairs in one 64-bit register (low word: the first element).
__device__ __forceinline__ uint64_t lt_fma2(uint64_t a, uint64_t b, uint64_t c) {
    uint64_t d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ uint64_t lt_splat(float a) {
    const uint64_t u = __float_as_uint(a);
    return u | (u << 32);
}
// A 16-bit value held in the low bits of a record, as float32.
template <class V> __device__ __forceinline__ float lt_value(uint32_t bits);
template <> __device__ __forceinline__ float lt_value<__nv_bfloat16>(uint32_t bits) {
    return __uint_as_float(bits << 16);
}
template <> __device__ __forceinline__ float lt_value<__half>(uint32_t bits) {
    return __half2float(__ushort_as_half((unsigned short)bits));
}
// Two 16-bit values of a 32-bit word (the first in the low half) as a float32 pair.
template <class V> __device__ __forceinline__ uint64_t lt_widen2(uint32_t w);
template <> __device__ __forceinline__ uint64_t lt_widen2<__nv_bfloat16>(uint32_t w) {
    return (uint64_t)(w << 16) | ((uint64_t)(w & 0xffff0000u) << 32);
}
template <> __device__ __forceinline__ uint64_t lt_widen2<__half>(uint32_t w) {
    const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w));
    return (uint64_t)__float_as_uint(f.x) | ((uint64_t)__float_as_uint(f.y) << 32);
}

template <class V, int N>
__global__ void __launch_bounds__(kLtThreads, 1)
k_struct_spmm_ltile(const uint32_t* __restrict__ rec, const int64_t* __restrict__ seg_start,
                    const int32_t* __restrict__ seg_len, const uint16_t* __restrict__ row_start, int64_t n_long,
                    int64_t nbj, int32_t rec_cap, const V* __restrict__ B, int64_t n_cols,
                    comp_t* __restrict__ partial, int* __restrict__ err) {
    static_assert(N == 16 || N == 32, "tiled long rows: N of 16 or 32");
    constexpr int VW = 8, LPN = N / 8, NSUB = 32 / LPN;
    constexpr int RPS = kLtRows / (32 * NSUB);  // rows per sub-group
    constexpr int kBBytes = kLtCols * N * 2;
    constexpr int kRsBytes = kLtRsEntries * 2;
    extern __shared__ __align__(128) unsigned char sm[];
    __shared__ __align__(8) uint64_t full[2];
    __shared__ int done[2];    // warps finished with the block in each stage
    __shared__ int issued_s;   // blocks whose copies were issued
    constexpr int kWarps = kLtThreads / 32;
    const int stage_bytes = kBBytes + kRsBytes + rec_cap * 4;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int sub = lane / LPN, lig = lane % LPN;
    const int64_t g = blockIdx.x;
    const int64_t q = blockIdx.y, nq = gridDim.y;
    const int64_t j_lo = q * nbj / nq, j_hi = (q + 1) * nbj / nq;
    auto issue = [&](int64_t j, int st) {
        const int64_t key = g * nbj + j;
        const int64_t rows_b = (n_cols - j * kLtCols) < kLtCols ? (n_cols - j * kLtCols) : kLtCols;
        const uint32_t b_bytes = (uint32_t)(rows_b * N * 2);
        const uint32_t r_bytes = (uint32_t)seg_len[key] * 4u;
        unsigned char* base = sm + (size_t)st * stage_bytes;
        const uint32_t bar = smem_u32(&full[st]);
        tma::mbar_arrive_expect_tx(bar, b_bytes + kRsBytes + r_bytes);
        bulk_g2s(smem_u32(base), B + j * kLtCols * N, b_bytes, bar);
        bulk_g2s(smem_u32(base + kBBytes), row_start + key * kLtRsEntries, kRsBytes, bar);
        if (r_bytes) bulk_g2s(smem_u32(base + kBBytes + kRsBytes), rec + seg_start[key], r_bytes, bar);
    };
    if (tid == 0) {
        tma::mbar_init(smem_u32(&full[0]), 1);
        tma::mbar_init(smem_u32(&full[1]), 1);
        tma::mbar_init_fence();
        done[0] = done[1] = 0;
        int n = 0;
        if (j_lo < j_hi) issue(j_lo, 0), ++n;
        if (j_lo + 1 < j_hi) issue(j_lo + 1, 1), ++n;
        issued_s = n;
    }
    __syncthreads();
    comp_t acc[RPS][VW];
#pragma unroll
    for (int i = 0; i < RPS; ++i)
#pragma unroll
        for (int w = 0; w < VW; ++w) acc[i][w] = comp_t{0.f, 0.f};
    const int rig0 = (warp * NSUB + sub) * RPS;
    bool ok = true;
    // Each warp walks the blocks on its own: it waits for the block's copies,
    // multiplies it, and releases the stage; the last warp to release a stage
    // refills it with the block two ahead.  No CTA-wide barrier per block, so
    // a warp with fewer records in a block runs ahead into the next one.
    for (int64_t j = j_lo; j < j_hi; ++j) {
        const int st = (int)((j - j_lo) & 1);
        const uint32_t phase = (uint32_t)(((j - j_lo) >> 1) & 1);
        ok = __all_sync(0xffffffffu, mbar_wait(smem_u32(&full[st]), phase)) != 0;
        if (!ok) break;
        const unsigned char* base = sm + (size_t)st * stage_bytes;
        const V* Bs = reinterpret_cast<const V*>(base);
        const uint16_t* rs = reinterpret_cast<const uint16_t*>(base + kBBytes);
        const uint32_t* rc = reinterpret_cast<const uint32_t*>(base + kBBytes + kRsBytes);
        // one record: the B row slice as a single 16-byte shared load (the
        // slice is 16-byte aligned: row * N * 2 + lig * 16 bytes), widened to
        // float32 pairs, times the value, added by paired FMAs into blk (blk[h]
        // holds columns 2h, 2h + 1 of the lane's slice)
        uint64_t blk[VW / 2];
        auto step = [&](uint32_t rr) {
            const uint4 q4 = *reinterpret_cast<const uint4*>(Bs + (rr >> 16) * N + lig * VW);
            const uint64_t a2 = lt_splat(lt_value<V>(rr & 0xffffu));
            blk[0] = lt_fma2(a2, lt_widen2<V>(q4.x), blk[0]);
            blk[1] = lt_fma2(a2, lt_widen2<V>(q4.y), blk[1]);
            blk[2] = lt_fma2(a2, lt_widen2<V>(q4.z), blk[2]);
            blk[3] = lt_fma2(a2, lt_widen2<V>(q4.w), blk[3]);
        };
        // a row's block sum (plain float32, exact products) enters its (s, c)
        // accumulator by TwoSum
        auto fold = [&](comp_t (&a)[VW]) {
#pragma unroll
            for (int h = 0; h < VW / 2; ++h) {
                a[2 * h] = comp_add_value(a[2 * h], __uint_as_float((uint32_t)blk[h]), 0.f);
                a[2 * h + 1] = comp_add_value(a[2 * h + 1], __uint_as_float((uint32_t)(blk[h] >> 32)), 0.f);
                blk[h] = 0;
            }
        };
#pragma unroll
        for (int h = 0; h < VW / 2; ++h) blk[h] = 0;
#pragma unroll
        for (int i = 0; i < RPS; ++i) {
            const int rig = rig0 + i;
            const int lo = rs[rig], hi = rs[rig + 1];
            int k = lo;
            for (; k + 1 < hi; k += 2) {  // two independent records in flight
                const uint32_t r0 = rc[k], r1 = rc[k + 1];
                step(r0);
                step(r1);
            }
            if (k < hi) step(rc[k]);
            if (hi > lo) fold(acc[i]);
        }
        // release the stage: the warp's shared-memory reads come before its
        // arrival; the last warp to arrive refills the stage with block j + 2
        __syncwarp();
        if (lane == 0) {
            __threadfence_block();
            const int old = atomicAdd(&done[st], 1);
            if (old == kWarps - 1) {
                atomicExch(&done[st], 0);
                __threadfence_block();
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                if (j + 2 < j_hi) {
                    issue(j + 2, st);
                    atomicAdd(&issued_s, 1);
                }
            }
        }
    }
    if (__syncthreads_or(!ok)) {
        if (tid == 0) {
            atomicExch(err, FSB_ERR_TIMEOUT);
            // drain (bounded) every issued copy before the CTA exits: block
            // j_lo + d completes phase (d >> 1) & 1 of stage d & 1
            const int n = issued_s;
            for (int d = (n > 2 ? n - 2 : 0); d < n; ++d) mbar_wait(smem_u32(&full[d & 1]), (uint32_t)((d >> 1) & 1));
        }
        return;
    }
#pragma unroll
    for (int i = 0; i < RPS; ++i) {
        const int64_t l = g * kLtRows + rig0 + i;
        if (l < n_long) {
            comp_t* dst = partial + (q * n_long + l) * N + lig * VW;
#pragma unroll
            for (int w = 0; w < VW; ++w) dst[w] = acc[i][w];
        }
    }
}

// One warp per long row: the column ranges' partials in range order.
template <int N>
__global__ void k_struct_spmm_lfold(const comp_t* __restrict__ partial, int64_t nq, int64_t n_long,
                                    const int32_t* __restrict__ long_rows, float* __restrict__ C, int64_t ldc) {
    const int64_t l = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int c = threadIdx.x & 31;
    if (l >= n_long || c >= N) return;
    comp_t s = partial[l * N + c];
    for (int64_t q = 1; q < nq; ++q) s = acc_add(s, partial[(q * n_long + l) * N + c]);
    C[(int64_t)long_rows[l] * ldc + c] = s.s + s.c;
}

// Shared-memory matrix descriptor, SWIZZLE_NONE (layout 0): start address,
// leading (K-direction) and stride (M/N-direction) byte offsets between 8 x
// 16-byte core matrices, each >> 4; descriptor version 1 (bit 46).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: D float32 (bits 4-5 = 1), A and B f16 (0)
// or bf16 (1) (bits 7-9, 10-12), A K-major (bit 15 = 0), B MN-major (bit 16 =
// 1), N >> 3 at bits 17-22, M >> 4 at bits 24-28 (M = 128).
template <bool BF16, int N>
__host__ __device__ constexpr uint32_t band_idesc() {
    return (1u << 4) | ((BF16 ? 1u : 0u) << 7) | ((BF16 ? 1u : 0u) << 10) | (1u << 16) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(128 >> 4) << 24);
}

template <int X>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, uint32_t* d);
template <>
__device__ __forceinline__ void tmem_ld<8>(uint32_t taddr, uint32_t* d) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7])
                 : "r"(taddr)
                 : "memory");
}
template <>
__device__ __forceinline__ void tmem_ld<16>(uint32_t taddr, uint32_t* d) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]), "=r"(d[8]),
          "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15])
        : "r"(taddr)
        : "memory");
}

// Band tiles on the tensor cores.  One CTA of 256 threads per tile of 128
// rows; threads t and t + 128 share row t % 128 (its descriptors and
// scattered nonzeros), each owning half of the row's N columns in the
// epilogue: warp w reads TMEM lane quarter w % 4, columns (w / 4) * N / 2 on.
//   A (dynamic shared memory, K-major SWIZZLE_NONE core matrices): element
//     (m, k) at (m / 8) * sbo_a + (k / 8) * 128 + (m % 8) * 16 + (k % 8) * 2,
//     sbo_a = span / 8 * 128; row m holds its run at k = run_col - base, zeros
//     elsewhere.  The row's two threads read its run as the 16-byte aligned
//     chunks holding it (even / odd chunks, all in flight together) and store
//     the run's elements one by one.
//   B (MN-major core matrices, after A): element (k, n) at (k / 8) * lbo_b +
//     (n / 8) * 128 + (k % 8) * 16 + (n % 8) * 2, lbo_b = N / 8 * 128; the
//     span's B rows with 16-byte loads, four per thread in flight.
// The first kPrefetch scattered nonzeros of each row: indices with the run,
// the thread's half B rows while the MMAs run.  span / 16 MMAs of 128 x N x 16
// are issued by one thread and committed to an mbarrier (bounded wait).  Long
// rows are left to the long-row kernels.
constexpr int kBandThreads = 256;

template <class V, class I, class P, int N>
__global__ void __launch_bounds__(kBandThreads)
k_struct_spmm_band(const V* __restrict__ val, const I* __restrict__ col, const P* __restrict__ ptr, int64_t n_rows,
                   int64_t n_cols, const int32_t* __restrict__ run_col, const int32_t* __restrict__ run_off,
                   const int32_t* __restrict__ run_len, const int64_t* __restrict__ tile_base,
                   const int32_t* __restrict__ tile_span, const V* __restrict__ B, int64_t ldb,
                   float* __restrict__ C, int64_t ldc, int* __restrict__ err) {
    static_assert(N == 16 || N == 32 || N == 64, "band tiles: N of 16, 32 or 64");
    constexpr bool kBf16 = std::is_same<V, __nv_bfloat16>::value;
    constexpr int kTmemCols = N <= 32 ? 32 : 64;
    constexpr uint32_t kLboB = (N / 8) * 128;
    constexpr int kCh = N / 8;    // 16-byte chunks per B row
    constexpr int kHalf = N / 2;  // columns per thread in the epilogue
    constexpr int kHCh = kCh / 2;
    constexpr int kVec = 8;       // 16-bit values per 16-byte chunk
    constexpr int kRunChunks = 5;
    constexpr int kPrefetch = N <= 32 ? 4 : 2;
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_slot;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int row_t = tid & (kTileRows - 1), half = tid >> 7;
    const int64_t t = blockIdx.x, r0 = t * kTileRows;
    // descriptors of this thread's row and of the tile
    const int64_t kbase = tile_base[t];
    const int span = tile_span[t];
    const int64_t r = r0 + row_t;
    const int rl = r < n_rows ? run_len[r] : -1;
    int64_t s = 0, e = 0;
    int ro = 0, kc = 0;
    if (rl >= 0) {
        s = idx(ptr[r]);
        e = idx(ptr[r + 1]);
        if (rl > 0) {
            ro = run_off[r];
            kc = (int)(run_col[r] - kbase);
        }
    }
    const int rn = rl > 0 ? rl : 0;
    const int64_t n_sc = rl >= 0 ? (e - s) - rn : 0;
    // the first scattered nonzeros: indices and values now, B rows later
    I cp[kPrefetch];
    V vp[kPrefetch];
#pragma unroll
    for (int u = 0; u < kPrefetch; ++u) {
        cp[u] = 0;
        vp[u] = vzero<V>();
        if (u < n_sc) {
            const int64_t k = u < ro ? s + u : s + u + rn;
            cp[u] = ld_stream1(col + k);
            vp[u] = ld_stream1(val + k);
        }
    }
    const uint32_t sbo_a = (uint32_t)(span / 8) * 128;
    unsigned char* sa = sm;
    unsigned char* sb = sm + (size_t)kTileRows * span * 2;

    if (tid == 0) {
        tma::mbar_init(smem_u32(&bar), 1);
        tma::mbar_init_fence();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    for (int i = tid; i < kTileRows * span * 2 / 16; i += kBandThreads)
        reinterpret_cast<uint4*>(sa)[i] = make_uint4(0, 0, 0, 0);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;

    if (span > 0) {
        // the span's B rows -> B, four 16-byte loads in flight per thread
        const int n_q = span * kCh;
        for (int i0 = tid; i0 < n_q; i0 += 4 * kBandThreads) {
            uint4 q[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int i = i0 + u * kBandThreads;
                q[u] = make_uint4(0, 0, 0, 0);
                if (i < n_q) {
                    const int64_t br = kbase + i / kCh;
                    if (br < n_cols) q[u] = __ldg(reinterpret_cast<const uint4*>(B + br * ldb + (i % kCh) * 8));
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int i = i0 + u * kBandThreads;
                if (i < n_q) {
                    const int k = i / kCh, ch = i % kCh;
                    *reinterpret_cast<uint4*>(sb + (k >> 3) * kLboB + ch * 128 + (k & 7) * 16) = q[u];
                }
            }
        }
        // the row's run -> row row_t of A: the aligned chunks holding it
        // (even chunks by the first thread, odd by the second; an aligned
        // chunk holding a valid element lies inside one page)
        if (rn > 0) {
            const uintptr_t a0 = reinterpret_cast<uintptr_t>(val + s + ro);
            const V* cbase = reinterpret_cast<const V*>(a0 & ~(uintptr_t)15);
            const int lead = (int)((a0 & 15u) / sizeof(V));
            const int n_ch = (lead + rn + kVec - 1) / kVec;
            const uint32_t row_off = (uint32_t)(row_t >> 3) * sbo_a + (uint32_t)(row_t & 7) * 16;
            for (int c0 = half; c0 < n_ch; c0 += 2 * kRunChunks) {
                vec_t<V, kVec> w[kRunChunks];
#pragma unroll
                for (int u = 0; u < kRunChunks; ++u)
                    if (c0 + 2 * u < n_ch) w[u] = ld_stream<V, kVec>(cbase + (c0 + 2 * u) * kVec);
#pragma unroll
                for (int u = 0; u < kRunChunks; ++u) {
                    if (c0 + 2 * u < n_ch) {
#pragma unroll
                        for (int z = 0; z < kVec; ++z) {
                            const int q = (c0 + 2 * u) * kVec + z - lead;
                            if (q >= 0 && q < rn) {
                                const int k = kc + q;
                                *reinterpret_cast<V*>(sa + row_off + (uint32_t)(k >> 3) * 128 + (uint32_t)(k & 7) * 2) =
                                    w[u].v[z];
                            }
                        }
                    }
                }
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (span > 0 && tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        constexpr uint32_t idesc = band_idesc<kBf16, N>();
        for (int st = 0; st < span / 16; ++st) {
            const uint64_t adesc = sdesc(smem_u32(sa) + (uint32_t)st * 256, 128, sbo_a);
            const uint64_t bdesc = sdesc(smem_u32(sb) + (uint32_t)st * 2 * kLboB, kLboB, 128);
            const uint32_t accumulate = st > 0 ? 1u : 0u;
            const uint32_t zero = 0;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(zero), "r"(zero), "r"(zero), "r"(zero)
                : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&bar))
                     : "memory");
    }
    // this thread's half of the prefetched scattered B rows while the MMAs run
    uint4 qp[kPrefetch][kHCh];
#pragma unroll
    for (int u = 0; u < kPrefetch; ++u)
#pragma unroll
        for (int ch = 0; ch < kHCh; ++ch)
            qp[u][ch] = u < n_sc ? __ldg(reinterpret_cast<const uint4*>(B + idx(cp[u]) * ldb + half * kHalf + ch * 8))
                                 : make_uint4(0, 0, 0, 0);
    bool ok = true;
    if (span > 0) {
        ok = __syncthreads_and(mbar_wait(smem_u32(&bar), 0)) != 0;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (!ok && tid == 0) atomicExch(err, FSB_ERR_TIMEOUT);
    }
    float acc[kHalf];
    if (span > 0 && ok) {
        uint32_t d[kHalf];
#pragma unroll
        for (int q = 0; q < kHalf / 8; ++q)
            tmem_ld<8>(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(half * kHalf + q * 8), d + q * 8);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int n = 0; n < kHalf; ++n) acc[n] = __uint_as_float(d[n]);
    } else {
#pragma unroll
        for (int n = 0; n < kHalf; ++n) acc[n] = 0.f;
    }
    if (ok && rl >= 0) {
        auto fma_row = [&](float a, const uint4 (&q)[kHCh]) {
#pragma unroll
            for (int ch = 0; ch < kHCh; ++ch) {
                V b8[8];
                memcpy(b8, &q[ch], 16);
#pragma unroll
                for (int i = 0; i < 8; ++i) acc[ch * 8 + i] = fmaf(a, to_f32(b8[i]), acc[ch * 8 + i]);
            }
        };
#pragma unroll
        for (int u = 0; u < kPrefetch; ++u)
            if (u < n_sc) fma_row(to_f32(vp[u]), qp[u]);
        for (int64_t q = kPrefetch; q < n_sc; q += 2) {  // the rest, two in flight
            const int64_t ka = q < ro ? s + q : s + q + rn;
            const bool two = q + 1 < n_sc;
            const int64_t kb = two ? ((q + 1) < ro ? s + q + 1 : s + q + 1 + rn) : ka;
            const V* ba = B + idx(ld_stream1(col + ka)) * ldb + half * kHalf;
            const V* bb = B + idx(ld_stream1(col + kb)) * ldb + half * kHalf;
            uint4 qa[kHCh], qb[kHCh];
#pragma unroll
            for (int ch = 0; ch < kHCh; ++ch) {
                qa[ch] = __ldg(reinterpret_cast<const uint4*>(ba + ch * 8));
                qb[ch] = __ldg(reinterpret_cast<const uint4*>(bb + ch * 8));
            }
            fma_row(to_f32(ld_stream1(val + ka)), qa);
            if (two) fma_row(to_f32(ld_stream1(val + kb)), qb);
        }
        float* dst = C + r * ldc + half * kHalf;
#pragma unroll
        for (int n = 0; n < kHalf; n += 4)
            __stcs(reinterpret_cast<float4*>(dst + n), make_float4(acc[n], acc[n + 1], acc[n + 2], acc[n + 3]));
    }
    if (!ok) {
        // drain (bounded) the MMAs issued before freeing tensor memory
        mbar_wait(smem_u32(&bar), 0);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

inline int64_t band_smem_bytes(int span, int n) { return (int64_t)span * (kTileRows * 2 + 2 * n); }

}  // namespace strc
}  // namespace fsb

using namespace fsb;
using namespace fsb::strc;

namespace {

// Validation shared by the entry points.
int check_struct(const fsb_csr* A, const fsb_struct* S, const char* who) {
    if (!A || !S || !A->row_ptr || (A->nnz > 0 && (!A->values || !A->col_idx))) {
        fsb_host::set_error("%s: null matrix or structure", who);
        return FSB_ERR_INVALID;
    }
    if (A->row_map) {
        fsb_host::set_error("%s: row maps are not supported", who);
        return FSB_ERR_INVALID;
    }
    if (A->n_rows > 0 && (!S->run_col || !S->run_off || !S->run_len || !S->tile_base || !S->tile_span)) {
        fsb_host::set_error("%s: missing row or tile descriptors", who);
        return FSB_ERR_INVALID;
    }
    if (S->n_long < 0 || (S->n_long > 0 && !S->long_rows)) {
        fsb_host::set_error("%s: bad long-row list", who);
        return FSB_ERR_INVALID;
    }
    if (A->n_cols >= 0x7fffffffLL || A->n_rows >= 0x7fffffffLL) {
        fsb_host::set_error("%s: the structured form needs fewer than 2^31 rows and columns", who);
        return FSB_ERR_LIMIT;
    }
    if (A->value_dtype != FSB_F16 && A->value_dtype != FSB_BF16) {
        fsb_host::set_error("%s: float16 / bfloat16 values only", who);
        return FSB_ERR_UNSUPPORTED;
    }
    return FSB_OK;
}

// The tiled long-row kernel runs when the structure carries its record
// stream in the compiled tile shape (lt_rows 512, lt_cols 1024), the dense
// width is 16 or 32, B rows are contiguous (ldb == n_dense) and two stages fit
// in shared memory.
int64_t lt_stage_bytes(const fsb_struct* S, int64_t n_dense) {
    return (int64_t)kLtCols * n_dense * 2 + kLtRsEntries * 2 + (int64_t)S->lt_rec_cap * 4;
}
bool lt_usable(const fsb_struct* S, int64_t n_dense, int64_t ldb) {
    return S->lt_rows == kLtRows && S->lt_cols == kLtCols && S->lt_rec && S->lt_seg_start && S->lt_seg_len &&
           S->lt_row_start && S->lt_groups > 0 && S->lt_col_blocks > 0 && S->lt_rec_cap >= 0 &&
           S->lt_rec_cap % 4 == 0 && (n_dense == 16 || n_dense == 32) && ldb == n_dense &&
           2 * lt_stage_bytes(S, n_dense) <= 227 * 1024 - 2048;
}
// Column ranges per row group: about one CTA per SM in all.
int64_t lt_ranges(const fsb_struct* S) {
    const int64_t q = 148 / (S->lt_groups > 0 ? S->lt_groups : 1);
    return q < 1 ? 1 : (q > S->lt_col_blocks ? S->lt_col_blocks : q);
}

template <class F>
int dispatch_half(int vdt, F&& f) {
    if (vdt == FSB_F16) return f(tag<__half>{});
    return f(tag<__nv_bfloat16>{});
}

}  // namespace

extern "C" int fsb_struct_rows(const fsb_csr* A, int64_t long_min, int32_t min_run, int32_t* run_col,
                               int32_t* run_off, int32_t* run_len, void* stream) {
    if (!A || !A->row_ptr || (A->nnz > 0 && !A->col_idx) || (A->n_rows > 0 && (!run_col || !run_off || !run_len)) ||
        long_min < 0 || min_run < 1) {
        fsb_host::set_error("fsb_struct_rows: bad arguments");
        return FSB_ERR_INVALID;
    }
    if (A->n_rows == 0) return FSB_OK;
    if (A->n_cols >= 0x7fffffffLL) {
        fsb_host::set_error("fsb_struct_rows: columns must fit in 31 bits");
        return FSB_ERR_LIMIT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return dispatch_idx(A->index_dtype, [&](auto ti) -> int {
        using I = typename decltype(ti)::type;
        return dispatch_idx(A->ptr_dtype, [&](auto tp) -> int {
            using P = typename decltype(tp)::type;
            const int64_t blocks = std::min<int64_t>(ceil_div(A->n_rows, 8), 148 * 16);
            k_struct_rows<I, P><<<(unsigned)blocks, 256, 0, st>>>(
                static_cast<const I*>(A->col_idx), static_cast<const P*>(A->row_ptr), A->n_rows, long_min, min_run,
                run_col, run_off, run_len);
            return fsb_host::check_launch("k_struct_rows");
        });
    });
}

extern "C" int fsb_struct_tiles(int64_t n_rows, const int32_t* run_col, int32_t* run_off, int32_t* run_len,
                                int64_t* tile_base, int32_t* tile_span, void* stream) {
    if (n_rows < 0 || (n_rows > 0 && (!run_col || !run_off || !run_len || !tile_base || !tile_span))) {
        fsb_host::set_error("fsb_struct_tiles: bad arguments");
        return FSB_ERR_INVALID;
    }
    if (n_rows == 0) return FSB_OK;
    const int64_t n_tiles = ceil_div(n_rows, (int64_t)kTileRows);
    k_struct_tiles<<<(unsigned)ceil_div(n_tiles, 8), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        n_rows, run_col, run_off, run_len, tile_base, tile_span, n_tiles);
    return fsb_host::check_launch("k_struct_tiles");
}

extern "C" int64_t fsb_struct_workspace_bytes(int is_spmm, const fsb_struct* S, int64_t n_dense) {
    if (!S) return -1;
    if (is_spmm) {
        int64_t b = S->n_chunks * n_dense * (int64_t)sizeof(comp_t);
        if (S->lt_groups > 0) {
            const int64_t lt = lt_ranges(S) * S->n_long * n_dense * (int64_t)sizeof(comp_t);
            b = b > lt ? b : lt;
        }
        return align_up(b, 256);
    }
    return align_up(S->n_xblocks * S->n_long * (int64_t)sizeof(comp_t), 256);
}

extern "C" int fsb_struct_spmv(const fsb_csr* A, const fsb_struct* S, const void* x, float* y, void* workspace,
                               int64_t workspace_bytes, void* stream) {
    int rc = check_struct(A, S, "fsb_struct_spmv");
    if (rc) return rc;
    if (A->n_rows == 0) return FSB_OK;
    if (!y || (A->nnz > 0 && !x)) {
        fsb_host::set_error("fsb_struct_spmv: null x or y");
        return FSB_ERR_INVALID;
    }
    if (S->n_long > 0) {
        if (!S->seg_ptr || !S->seg_off || !S->seg_val || !aligned16(S->seg_off) || !aligned16(S->seg_val) ||
            S->xblock < 8 || S->xblock > 65536 ||
            S->n_xblocks != ceil_div(A->n_cols, (int64_t)S->xblock) || S->n_xblocks > 65535) {
            fsb_host::set_error("fsb_struct_spmv: bad x-block grouping of the long rows");
            return FSB_ERR_INVALID;
        }
        const int64_t need = fsb_struct_workspace_bytes(0, S, 1);
        if (!workspace || workspace_bytes < need) {
            fsb_host::set_error("fsb_struct_spmv: workspace %lld bytes < %lld", (long long)workspace_bytes,
                                (long long)need);
            return FSB_ERR_WORKSPACE;
        }
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return dispatch_half(A->value_dtype, [&](auto tv) -> int {
        using V = typename decltype(tv)::type;
        return dispatch_idx(A->index_dtype, [&](auto ti) -> int {
            using I = typename decltype(ti)::type;
            return dispatch_idx(A->ptr_dtype, [&](auto tp) -> int {
                using P = typename decltype(tp)::type;
                const int64_t n_tiles = ceil_div(A->n_rows, (int64_t)kTileRows);
                k_struct_spmv_tile<V, I, P><<<(unsigned)n_tiles, kThreads, 0, st>>>(
                    static_cast<const V*>(A->values), static_cast<const I*>(A->col_idx),
                    static_cast<const P*>(A->row_ptr), A->n_rows, A->n_cols, S->run_col, S->run_off, S->run_len,
                    S->tile_base, S->tile_span, static_cast<const V*>(x), y);
                int rc2 = fsb_host::check_launch("k_struct_spmv_tile");
                if (rc2 || S->n_long == 0) return rc2;
                const int smem = S->xblock * (int)sizeof(V);
                if (smem > 48 * 1024)
                    cudaFuncSetAttribute(k_struct_spmv_long<V>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
                comp_t* partial = static_cast<comp_t*>(workspace);
                // one wave: about one CTA per SM (128 KB of x each)
                const int64_t slices = std::max<int64_t>(1, std::min<int64_t>(148 / S->n_xblocks, S->n_long));
                dim3 g((unsigned)S->n_xblocks, (unsigned)slices);
                k_struct_spmv_long<V><<<g, 1024, smem, st>>>(S->seg_ptr, static_cast<const V*>(S->seg_val),
                                                             S->seg_off, S->n_long, S->xblock,
                                                             static_cast<const V*>(x), A->n_cols, partial);
                rc2 = fsb_host::check_launch("k_struct_spmv_long");
                if (rc2) return rc2;
                k_struct_spmv_fold<<<(unsigned)ceil_div(S->n_long, 256), 256, 0, st>>>(partial, S->n_long,
                                                                                      S->n_xblocks, S->long_rows, y);
                return fsb_host::check_launch("k_struct_spmv_fold");
            });
        });
    });
}

extern "C" int fsb_struct_spmm(const fsb_csr* A, const fsb_struct* S, const void* B, int64_t ldb, int64_t n_dense,
                               float* C, int64_t ldc, void* workspace, int64_t workspace_bytes, void* stream) {
    int rc = check_struct(A, S, "fsb_struct_spmm");
    if (rc) return rc;
    if (A->n_rows == 0 || n_dense == 0) return FSB_OK;
    if (n_dense != 16 && n_dense != 32 && n_dense != 64) {
        fsb_host::set_error("fsb_struct_spmm: n_dense must be 16, 32 or 64 (got %lld)", (long long)n_dense);
        return FSB_ERR_UNSUPPORTED;
    }
    if (!C || !B || !aligned16(B) || !aligned16(C) || ldb % 8 != 0 || ldc % 4 != 0 || ldb < n_dense ||
        ldc < n_dense) {
        fsb_host::set_error("fsb_struct_spmm: B and C must be 16-byte aligned with ldb %% 8 == 0, ldc %% 4 == 0");
        return FSB_ERR_INVALID;
    }
    if (S->max_span < 0 || S->max_span > kSpanMax || S->max_span % 16) {
        fsb_host::set_error("fsb_struct_spmm: max_span %d must be a multiple of 16 in [0, %d]", S->max_span,
                            kSpanMax);
        return FSB_ERR_INVALID;
    }
    if (S->n_long > 0) {
        if (!S->chunk_row || !S->chunk_ptr || S->chunk_nnz < 32 || S->n_chunks < S->n_long) {
            fsb_host::set_error("fsb_struct_spmm: bad long-row chunks");
            return FSB_ERR_INVALID;
        }
        const int64_t need = fsb_struct_workspace_bytes(1, S, n_dense);
        if (!workspace || workspace_bytes < need) {
            fsb_host::set_error("fsb_struct_spmm: workspace %lld bytes < %lld", (long long)workspace_bytes,
                                (long long)need);
            return FSB_ERR_WORKSPACE;
        }
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int* err = gather_error_word();
    return dispatch_half(A->value_dtype, [&](auto tv) -> int {
        using V = typename decltype(tv)::type;
        return dispatch_idx(A->index_dtype, [&](auto ti) -> int {
            using I = typename decltype(ti)::type;
            return dispatch_idx(A->ptr_dtype, [&](auto tp) -> int {
                using P = typename decltype(tp)::type;
                const V* val = static_cast<const V*>(A->values);
                const I* col = static_cast<const I*>(A->col_idx);
                const P* ptr = static_cast<const P*>(A->row_ptr);
                const V* Bv = static_cast<const V*>(B);
                const int64_t n_tiles = ceil_div(A->n_rows, (int64_t)kTileRows);
                const int smem = (int)band_smem_bytes(S->max_span, (int)n_dense);
                auto band = [&](auto kern) -> int {
                    if (smem > 48 * 1024)
                        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
                    kern<<<(unsigned)n_tiles, kBandThreads, smem, st>>>(val, col, ptr, A->n_rows, A->n_cols, S->run_col,
                                                                    S->run_off, S->run_len, S->tile_base,
                                                                    S->tile_span, Bv, ldb, C, ldc, err);
                    return fsb_host::check_launch("k_struct_spmm_band");
                };
                int rc2 = n_dense == 16   ? band(k_struct_spmm_band<V, I, P, 16>)
                          : n_dense == 32 ? band(k_struct_spmm_band<V, I, P, 32>)
                                          : band(k_struct_spmm_band<V, I, P, 64>);
                if (rc2 || S->n_long == 0) return rc2;
                comp_t* partial = static_cast<comp_t*>(workspace);
                if (lt_usable(S, n_dense, ldb)) {
                    const int64_t nq = lt_ranges(S);
                    const int smem_lt = (int)(2 * lt_stage_bytes(S, n_dense));
                    auto tiled = [&](auto kern, auto fold) -> int {
                        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_lt);
                        kern<<<dim3((unsigned)S->lt_groups, (unsigned)nq), kLtThreads, smem_lt, st>>>(
                            S->lt_rec, S->lt_seg_start, S->lt_seg_len, S->lt_row_start, S->n_long, S->lt_col_blocks,
                            S->lt_rec_cap, Bv, A->n_cols, partial, err);
                        int rc3 = fsb_host::check_launch("k_struct_spmm_ltile");
                        if (rc3) return rc3;
                        fold<<<(unsigned)ceil_div(S->n_long, (int64_t)8), 256, 0, st>>>(partial, nq, S->n_long,
                                                                                       S->long_rows, C, ldc);
                        return fsb_host::check_launch("k_struct_spmm_lfold");
                    };
                    return n_dense == 16 ? tiled(k_struct_spmm_ltile<V, 16>, k_struct_spmm_lfold<16>)
                                         : tiled(k_struct_spmm_ltile<V, 32>, k_struct_spmm_lfold<32>);
                }
                const int64_t col_tiles = ceil_div(n_dense, (int64_t)32);
                const int64_t blocks = std::min<int64_t>(ceil_div(S->n_chunks, (int64_t)(kThreads / 32)), 148 * 24);
                k_struct_spmm_long<V, I, P><<<dim3((unsigned)blocks, (unsigned)col_tiles), kThreads, 0, st>>>(
                    val, col, ptr, S->long_rows, S->chunk_row, S->chunk_ptr, S->chunk_nnz, S->n_chunks, Bv, ldb,
                    n_dense, partial);
                rc2 = fsb_host::check_launch("k_struct_spmm_long");
                if (rc2) return rc2;
                k_struct_spmm_fold<<<dim3((unsigned)ceil_div(S->n_long, (int64_t)8), (unsigned)col_tiles), 256, 0,
                                     st>>>(partial, S->chunk_ptr, S->long_rows, S->n_long, n_dense, C, ldc);
                return fsb_host::check_launch("k_struct_spmm_fold");
            });
        });
    });
}
