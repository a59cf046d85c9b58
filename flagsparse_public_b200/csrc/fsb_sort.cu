// fsb_sort.cu -- the integer prepare steps on the device: a stable LSD radix
// sort of integer keys returning the permutation (the stable argsorts of
// FlagSparse's prepare functions: the column sort of _transpose_csr_for_spmv,
// spmv_csr.py:456-494; the (row, col) key sorts of coo_to_csr_for_spmv,
// spmv_csr.py:885-909, _sort_coo_lex_inplace, spmv_coo.py:297-309 and
// spmm_coo.py:21-32), and the starts of equal-key runs of sorted keys
// (_seg_starts_from_sorted_rows, spmv_coo.py:312-327, spmm_coo.py:121-132).
//
// Radix sort: 8-bit digits, least significant first, one pass per digit of
// the caller's key width (key_bits).  A pass is three kernels over tiles of
// kTile keys:
//   * k_sort_upsweep: per-tile digit histogram (warp-aggregated shared-memory
//     counts), stored digit-major: hist[digit][tile];
//   * k_scan_rows: one CTA per digit scans its row of tile counts in place
//     (exclusive) and records the digit's total;
//   * k_sort_downsweep: each tile scans the 256 totals for the digit starts,
//     then ranks its keys in rounds of 256 (one per thread, in key order):
//     __match_any_sync groups the warp's equal digits, per-warp digit counts
//     in shared memory are prefixed over the warps by the thread that owns
//     the digit; the tile is staged in shared memory in digit order and
//     written out in order, key and permutation entry to digit start + tile
//     prefix + rank.  Ranks follow key order inside the tile and tiles
//     follow each other, so every pass is stable and the result equals a
//     stable sort (torch.sort(stable=True)) bit for bit.
// The permutation travels as 32-bit indices between passes and is written as
// int64 by the last pass.  Keys of the full signed width are ordered through
// their top bit flipped.  HBM bound: a pass reads the keys twice and the
// permutation once and writes both.
#include <algorithm>

#include "fsb_dispatch.cuh"

namespace fsb {
namespace sort {

constexpr int kThreads = 256;
constexpr int kBins = 256;
constexpr int kRounds = 16;
constexpr int kTile = kThreads * kRounds;  // keys per tile
constexpr int kWarps = kThreads / 32;

// Inclusive scan of one value per thread over the CTA; *total receives the
// CTA sum.  sums: kWarps shared words.  Contains __syncthreads.
__device__ __forceinline__ uint32_t block_scan(uint32_t v, uint32_t* sums, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) sums[warp] = v;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kWarps ? sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < kWarps; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < kWarps) sums[lane] = w;
    }
    __syncthreads();
    const uint32_t add = warp > 0 ? sums[warp - 1] : 0u;
    *total = sums[kWarps - 1];
    __syncthreads();
    return v + add;
}

template <class K>
__device__ __forceinline__ int digit_of(K k, int shift, uint32_t mask) {
    return (int)((uint32_t)(k >> shift) & mask);
}

template <class K>
__global__ void __launch_bounds__(kThreads)
k_sort_upsweep(const K* __restrict__ keys, int64_t n, K flip, int shift, uint32_t mask, uint32_t* __restrict__ hist,
               int64_t n_tiles) {
    __shared__ uint32_t h[kBins];
    const int lane = threadIdx.x & 31;
    h[threadIdx.x] = 0u;
    __syncthreads();
    const int64_t t0 = (int64_t)blockIdx.x * kTile;
#pragma unroll 4
    for (int r = 0; r < kRounds; ++r) {
        const int64_t i = t0 + (int64_t)r * kThreads + threadIdx.x;
        const int d = i < n ? digit_of<K>(keys[i] ^ flip, shift, mask) : kBins;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        if (d < kBins && (peers & ((1u << lane) - 1u)) == 0u) atomicAdd(&h[d], (uint32_t)__popc(peers));
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * n_tiles + blockIdx.x] = h[threadIdx.x];
}

// One CTA per row: rows[b * len .. b * len + len) scanned in place
// (exclusive); totals[b] = the row's sum.
__global__ void __launch_bounds__(kThreads)
k_scan_rows(uint32_t* __restrict__ rows, int64_t len, uint32_t* __restrict__ totals) {
    __shared__ uint32_t sums[kWarps];
    uint32_t* row = rows + (int64_t)blockIdx.x * len;
    uint32_t carry = 0;
    for (int64_t c0 = 0; c0 < len; c0 += (int64_t)kThreads * 4) {
        uint32_t v[4], s = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t i = c0 + (int64_t)threadIdx.x * 4 + j;
            v[j] = i < len ? row[i] : 0u;
            s += v[j];
        }
        uint32_t total;
        uint32_t ex = carry + block_scan(s, sums, &total) - s;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t i = c0 + (int64_t)threadIdx.x * 4 + j;
            if (i < len) row[i] = ex;
            ex += v[j];
        }
        carry += total;
    }
    if (threadIdx.x == 0) totals[blockIdx.x] = carry;
}

// PIn: permutation entries read (nullptr: the identity); POut: written.
// The tile's keys are ranked in registers (rank among the tile's keys of
// the same digit), staged in shared memory in digit order, and written from
// there in order, so each digit's run of the tile leaves as consecutive
// stores.
template <class K, class PIn, class POut>
__global__ void __launch_bounds__(kThreads)
k_sort_downsweep(const K* __restrict__ keys_in, K in_flip, const PIn* __restrict__ perm_in, K* __restrict__ keys_out,
                 K out_flip, POut* __restrict__ perm_out, int64_t n, int shift, uint32_t mask,
                 const uint32_t* __restrict__ hist, const uint32_t* __restrict__ totals, int64_t n_tiles) {
    __shared__ uint32_t gbase[kBins];  // output position of the tile's first key of each digit
    __shared__ uint32_t lbase[kBins];  // its position in the staged tile
    __shared__ uint32_t wcnt[2][kWarps][kBins];
    __shared__ uint32_t sums[kWarps];
    extern __shared__ __align__(16) unsigned char staged[];  // downsweep_smem<K>() bytes
    K* skey = reinterpret_cast<K*>(staged);
    uint32_t* sidx = reinterpret_cast<uint32_t*>(staged + kTile * sizeof(K));
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int64_t t0 = (int64_t)blockIdx.x * kTile;
    const int n_here = (int)((n - t0) < kTile ? (n - t0) : kTile);
    K k[kRounds];
    uint32_t src[kRounds];
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
        const int64_t i = t0 + (int64_t)r * kThreads + tid;
        k[r] = 0;
        src[r] = 0;
        if (i < n) {
            k[r] = keys_in[i] ^ in_flip;
            src[r] = perm_in ? (uint32_t)perm_in[i] : (uint32_t)i;
        }
    }
    {
        const uint32_t tot = totals[tid];
        uint32_t all;
        const uint32_t start = block_scan(tot, sums, &all) - tot;
        gbase[tid] = start + hist[(int64_t)tid * n_tiles + blockIdx.x];
    }
    uint32_t run = 0;  // keys of digit tid ranked so far in this tile
    uint32_t rank[kRounds];
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
        uint32_t(*cnt)[kBins] = wcnt[r & 1];
        const bool ok = r * kThreads + tid < n_here;
        const int d = ok ? digit_of<K>(k[r], shift, mask) : kBins;  // lanes past the end: no real digit
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const uint32_t lrank = (uint32_t)__popc(peers & ((1u << lane) - 1u));
#pragma unroll
        for (int w = 0; w < kWarps; ++w) cnt[w][tid] = 0u;
        __syncthreads();
        if (ok && lrank == 0u) cnt[warp][d] = (uint32_t)__popc(peers);
        __syncthreads();
        // the owner of digit tid: exclusive prefix over the warps for these 256 keys
        uint32_t acc = run;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t c = cnt[w][tid];
            cnt[w][tid] = acc;
            acc += c;
        }
        run = acc;
        __syncthreads();
        rank[r] = ok ? cnt[warp][d] + lrank : 0u;
    }
    {
        uint32_t all;
        lbase[tid] = block_scan(run, sums, &all) - run;  // digit starts inside the tile
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRounds; ++r) {
        if (r * kThreads + tid < n_here) {
            const uint32_t p = lbase[digit_of<K>(k[r], shift, mask)] + rank[r];
            skey[p] = k[r];
            sidx[p] = src[r];
        }
    }
    __syncthreads();
    for (int j = tid; j < n_here; j += kThreads) {
        const K kk = skey[j];
        const int d = digit_of<K>(kk, shift, mask);
        const uint32_t pos = gbase[d] + ((uint32_t)j - lbase[d]);
        if (keys_out) keys_out[pos] = kk ^ out_flip;
        perm_out[pos] = (POut)sidx[j];
    }
}

template <class K>
__global__ void __launch_bounds__(kThreads)
k_run_count(const K* __restrict__ keys, int64_t n, uint32_t* __restrict__ counts) {
    __shared__ uint32_t sums[kWarps];
    const int64_t t0 = (int64_t)blockIdx.x * kTile;
    uint32_t c = 0;
    for (int r = 0; r < kRounds; ++r) {
        const int64_t i = t0 + (int64_t)r * kThreads + threadIdx.x;
        if (i < n && (i == 0 || keys[i] != keys[i - 1])) ++c;
    }
    uint32_t total;
    block_scan(c, sums, &total);
    if (threadIdx.x == 0) counts[blockIdx.x] = total;
}

// starts[j] = position of the j-th run (in key order), starts[runs] = n,
// *count = runs + 1.  offs: exclusive prefix of the per-tile run counts.
template <class K, class O>
__global__ void __launch_bounds__(kThreads)
k_run_write(const K* __restrict__ keys, int64_t n, const uint32_t* __restrict__ offs,
            const uint32_t* __restrict__ total, int64_t n_tiles, O* __restrict__ starts, int64_t* __restrict__ count) {
    __shared__ uint32_t sums[kWarps];
    const int64_t t0 = (int64_t)blockIdx.x * kTile;
    uint32_t pos = offs[blockIdx.x];
    for (int r = 0; r < kRounds; ++r) {
        const int64_t i = t0 + (int64_t)r * kThreads + threadIdx.x;
        const uint32_t f = (i < n && (i == 0 || keys[i] != keys[i - 1])) ? 1u : 0u;
        uint32_t round_total;
        const uint32_t incl = block_scan(f, sums, &round_total);
        if (f) starts[pos + incl - 1u] = (O)i;
        pos += round_total;
    }
    if (blockIdx.x == n_tiles - 1 && threadIdx.x == 0) {
        starts[*total] = (O)n;
        *count = (int64_t)*total + 1;
    }
}

// Duplicate merge of sorted COO entries (torch's coalesce, which FlagSparse
// calls in _coalesce_coo_entries, spmm_coo.py:35-51): one thread per run of
// equal keys sums its values in sorted (= original, the sort is stable)
// order, starting from zero in the accumulation type -- float for half types
// and float32, double for float64, float / double pairs for complex -- and
// rounds once to the value type.  Fewer than two entries are copied as they
// are.  The run count is read on the device, so nothing returns to the host.
template <class V> struct CoalesceAcc;
template <> struct CoalesceAcc<float> {
    using A = float;
    static __device__ __forceinline__ A zero() { return 0.f; }
    static __device__ __forceinline__ A add(A a, float v) { return __fadd_rn(a, v); }
    static __device__ __forceinline__ float out(A a) { return a; }
};
template <> struct CoalesceAcc<double> {
    using A = double;
    static __device__ __forceinline__ A zero() { return 0.0; }
    static __device__ __forceinline__ A add(A a, double v) { return __dadd_rn(a, v); }
    static __device__ __forceinline__ double out(A a) { return a; }
};
template <> struct CoalesceAcc<__half> {
    using A = float;
    static __device__ __forceinline__ A zero() { return 0.f; }
    static __device__ __forceinline__ A add(A a, __half v) { return __fadd_rn(a, __half2float(v)); }
    static __device__ __forceinline__ __half out(A a) { return __float2half_rn(a); }
};
template <> struct CoalesceAcc<__nv_bfloat16> {
    using A = float;
    static __device__ __forceinline__ A zero() { return 0.f; }
    static __device__ __forceinline__ A add(A a, __nv_bfloat16 v) { return __fadd_rn(a, __bfloat162float(v)); }
    static __device__ __forceinline__ __nv_bfloat16 out(A a) { return __float2bfloat16_rn(a); }
};
template <> struct CoalesceAcc<c64_t> {
    using A = c64_t;
    static __device__ __forceinline__ A zero() { return c64_t{0.f, 0.f}; }
    static __device__ __forceinline__ A add(A a, c64_t v) { return c64_t{__fadd_rn(a.re, v.re), __fadd_rn(a.im, v.im)}; }
    static __device__ __forceinline__ c64_t out(A a) { return a; }
};
template <> struct CoalesceAcc<c128_t> {
    using A = c128_t;
    static __device__ __forceinline__ A zero() { return c128_t{0.0, 0.0}; }
    static __device__ __forceinline__ A add(A a, c128_t v) {
        return c128_t{__dadd_rn(a.re, v.re), __dadd_rn(a.im, v.im)};
    }
    static __device__ __forceinline__ c128_t out(A a) { return a; }
};
template <> struct CoalesceAcc<c32_t> {
    using A = c64_t;
    static __device__ __forceinline__ A zero() { return c64_t{0.f, 0.f}; }
    static __device__ __forceinline__ A add(A a, c32_t v) {
        return c64_t{__fadd_rn(a.re, __half2float(v.re)), __fadd_rn(a.im, __half2float(v.im))};
    }
    static __device__ __forceinline__ c32_t out(A a) { return c32_t{__float2half_rn(a.re), __float2half_rn(a.im)}; }
};

template <class V, class K, class O>
__global__ void __launch_bounds__(kThreads)
k_coo_segment_sum(const K* __restrict__ keys, const O* __restrict__ starts, const int64_t* __restrict__ count,
                  const int64_t* __restrict__ order, const V* __restrict__ vals, int64_t n, K* __restrict__ out_keys,
                  V* __restrict__ out_vals) {
    using C = CoalesceAcc<V>;
    const int64_t runs = *count - 1;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < runs; j += stride) {
        const int64_t s = (int64_t)starts[j], e = (int64_t)starts[j + 1];
        out_keys[j] = keys[s];
        if (n < 2) {
            out_vals[j] = vals[order[s]];
            continue;
        }
        typename C::A acc = C::zero();
        for (int64_t k = s; k < e; ++k) acc = C::add(acc, vals[order[k]]);
        out_vals[j] = C::out(acc);
    }
}

// Dynamic shared memory of k_sort_downsweep: the staged keys and permutation.
template <class K>
constexpr int downsweep_smem() {
    return kTile * ((int)sizeof(K) + 4);
}

inline int64_t align256(int64_t b) { return (b + 255) & ~(int64_t)255; }

struct SortLayout {
    int64_t n_tiles = 0, passes = 0, hist = 0, totals = 0, keys_a = 0, perm_a = 0, keys_b = 0, perm_b = 0, bytes = 0;
};

inline SortLayout sort_layout(int64_t n, int key_size, int key_bits) {
    SortLayout L;
    L.n_tiles = ceil_div(n, (int64_t)kTile);
    L.passes = (key_bits + 7) / 8;
    int64_t o = 0;
    L.hist = o;
    o += align256((int64_t)kBins * L.n_tiles * 4);
    L.totals = o;
    o += align256((int64_t)kBins * 4);
    const int64_t bufs = L.passes - 1 < 2 ? L.passes - 1 : 2;
    if (bufs >= 1) {
        L.keys_a = o;
        o += align256(n * key_size);
        L.perm_a = o;
        o += align256(n * 4);
    }
    if (bufs >= 2) {
        L.keys_b = o;
        o += align256(n * key_size);
        L.perm_b = o;
        o += align256(n * 4);
    }
    L.bytes = o;
    return L;
}

template <class K>
int run_sort(const K* keys, int64_t n, int key_bits, bool signed_full, K* keys_out, int64_t* order_out, char* ws,
             const SortLayout& L, cudaStream_t st) {
    const K flip = signed_full ? (K)((K)1 << (8 * sizeof(K) - 1)) : (K)0;
    uint32_t* hist = reinterpret_cast<uint32_t*>(ws + L.hist);
    uint32_t* totals = reinterpret_cast<uint32_t*>(ws + L.totals);
    K* kb[2] = {reinterpret_cast<K*>(ws + L.keys_a), reinterpret_cast<K*>(ws + L.keys_b)};
    uint32_t* pb[2] = {reinterpret_cast<uint32_t*>(ws + L.perm_a), reinterpret_cast<uint32_t*>(ws + L.perm_b)};
    const unsigned grid = (unsigned)L.n_tiles;
    for (int p = 0; p < L.passes; ++p) {
        const int shift = 8 * p;
        const int bits = key_bits - shift < 8 ? key_bits - shift : 8;
        const uint32_t mask = (1u << bits) - 1u;
        const bool first = p == 0, last = p == L.passes - 1;
        const K* kin = first ? keys : kb[(p - 1) & 1];
        const K fin = first ? flip : (K)0;  // intermediate keys are stored flipped
        const uint32_t* pin = first ? nullptr : pb[(p - 1) & 1];
        k_sort_upsweep<K><<<grid, kThreads, 0, st>>>(kin, n, fin, shift, mask, hist, L.n_tiles);
        k_scan_rows<<<kBins, kThreads, 0, st>>>(hist, L.n_tiles, totals);
        constexpr int dyn = downsweep_smem<K>();
        if (last) {
            auto kern = k_sort_downsweep<K, uint32_t, int64_t>;
            if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) != cudaSuccess) {
                fsb_host::set_error("fsb_stable_sort: cannot reserve %d bytes of shared memory", dyn);
                return FSB_ERR_LAUNCH;
            }
            kern<<<grid, kThreads, dyn, st>>>(kin, fin, pin, keys_out, flip, order_out, n, shift, mask, hist, totals,
                                              L.n_tiles);
        } else {
            auto kern = k_sort_downsweep<K, uint32_t, uint32_t>;
            if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) != cudaSuccess) {
                fsb_host::set_error("fsb_stable_sort: cannot reserve %d bytes of shared memory", dyn);
                return FSB_ERR_LAUNCH;
            }
            kern<<<grid, kThreads, dyn, st>>>(kin, fin, pin, kb[p & 1], (K)0, pb[p & 1], n, shift, mask, hist,
                                              totals, L.n_tiles);
        }
        const int rc = fsb_host::check_launch("k_sort_downsweep");
        if (rc) return rc;
    }
    return FSB_OK;
}

}  // namespace sort
}  // namespace fsb

using namespace fsb;

static int sort_args(int64_t n, int key_dtype, int key_bits, const char* who) {
    if (key_dtype != FSB_I32 && key_dtype != FSB_I64) {
        fsb_host::set_error("%s: keys must be int32 or int64", who);
        return FSB_ERR_UNSUPPORTED;
    }
    const int width = key_dtype == FSB_I32 ? 32 : 64;
    if (n < 0 || key_bits < 1 || key_bits > width) {
        fsb_host::set_error("%s: bad size or key_bits", who);
        return FSB_ERR_INVALID;
    }
    if (n > 0x7fffffffLL) {
        fsb_host::set_error("%s: %lld keys exceed the 2^31 - 1 limit", who, (long long)n);
        return FSB_ERR_LIMIT;
    }
    return FSB_OK;
}

extern "C" int64_t fsb_sort_workspace_bytes(int64_t n, int key_dtype, int key_bits) {
    if (sort_args(n, key_dtype, key_bits, "fsb_sort_workspace_bytes") != FSB_OK) return -1;
    return sort::sort_layout(n, key_dtype == FSB_I32 ? 4 : 8, key_bits).bytes;
}

extern "C" int fsb_stable_sort(const void* keys, int key_dtype, int64_t n, int key_bits, void* keys_out,
                               int64_t* order_out, void* workspace, int64_t workspace_bytes, void* stream) {
    int rc = sort_args(n, key_dtype, key_bits, "fsb_stable_sort");
    if (rc) return rc;
    if (n == 0) return FSB_OK;
    if (!keys || !order_out) {
        fsb_host::set_error("fsb_stable_sort: null pointer");
        return FSB_ERR_INVALID;
    }
    const int width = key_dtype == FSB_I32 ? 32 : 64;
    const sort::SortLayout L = sort::sort_layout(n, width / 8, key_bits);
    if (!workspace || workspace_bytes < L.bytes) {
        fsb_host::set_error("fsb_stable_sort: workspace %lld bytes < %lld", (long long)workspace_bytes,
                            (long long)L.bytes);
        return FSB_ERR_WORKSPACE;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* ws = static_cast<char*>(workspace);
    const bool signed_full = key_bits == width;
    if (width == 32)
        return sort::run_sort<uint32_t>(static_cast<const uint32_t*>(keys), n, key_bits, signed_full,
                                        static_cast<uint32_t*>(keys_out), order_out, ws, L, st);
    return sort::run_sort<uint64_t>(static_cast<const uint64_t*>(keys), n, key_bits, signed_full,
                                    static_cast<uint64_t*>(keys_out), order_out, ws, L, st);
}

extern "C" int64_t fsb_run_starts_workspace_bytes(int64_t n) {
    if (n < 0) return -1;
    return sort::align256(ceil_div(n, (int64_t)sort::kTile) * 4) + 256;
}

extern "C" int fsb_run_starts(const void* sorted_keys, int key_dtype, int64_t n, void* starts, int starts_dtype,
                              int64_t* count, void* workspace, int64_t workspace_bytes, void* stream) {
    int rc = sort_args(n, key_dtype, key_dtype == FSB_I32 ? 32 : 64, "fsb_run_starts");
    if (rc) return rc;
    if (starts_dtype != FSB_I32 && starts_dtype != FSB_I64) {
        fsb_host::set_error("fsb_run_starts: starts must be int32 or int64");
        return FSB_ERR_UNSUPPORTED;
    }
    if (n == 0) return FSB_OK;
    if (!sorted_keys || !starts || !count) {
        fsb_host::set_error("fsb_run_starts: null pointer");
        return FSB_ERR_INVALID;
    }
    const int64_t need = fsb_run_starts_workspace_bytes(n);
    if (!workspace || workspace_bytes < need) {
        fsb_host::set_error("fsb_run_starts: workspace %lld bytes < %lld", (long long)workspace_bytes,
                            (long long)need);
        return FSB_ERR_WORKSPACE;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t n_tiles = ceil_div(n, (int64_t)sort::kTile);
    uint32_t* counts = static_cast<uint32_t*>(workspace);
    uint32_t* total = reinterpret_cast<uint32_t*>(static_cast<char*>(workspace) + sort::align256(n_tiles * 4));
    auto go = [&](auto tk, auto to) -> int {
        using K = typename decltype(tk)::type;
        using O = typename decltype(to)::type;
        const K* keys = static_cast<const K*>(sorted_keys);
        sort::k_run_count<K><<<(unsigned)n_tiles, sort::kThreads, 0, st>>>(keys, n, counts);
        sort::k_scan_rows<<<1, sort::kThreads, 0, st>>>(counts, n_tiles, total);
        sort::k_run_write<K, O><<<(unsigned)n_tiles, sort::kThreads, 0, st>>>(keys, n, counts, total, n_tiles,
                                                                              static_cast<O*>(starts), count);
        return fsb_host::check_launch("k_run_write");
    };
    if (key_dtype == FSB_I32) {
        if (starts_dtype == FSB_I32) return go(tag<int32_t>{}, tag<int32_t>{});
        return go(tag<int32_t>{}, tag<int64_t>{});
    }
    if (starts_dtype == FSB_I32) return go(tag<int64_t>{}, tag<int32_t>{});
    return go(tag<int64_t>{}, tag<int64_t>{});
}

extern "C" int fsb_coo_coalesce(const void* sorted_keys, int key_dtype, const int64_t* order, const void* values,
                                int value_dtype, int64_t n, const void* starts, int starts_dtype, const int64_t* count,
                                void* out_keys, void* out_values, void* stream) {
    if (n < 0 || (key_dtype != FSB_I32 && key_dtype != FSB_I64) ||
        (starts_dtype != FSB_I32 && starts_dtype != FSB_I64)) {
        fsb_host::set_error("fsb_coo_coalesce: bad sizes or index dtypes");
        return FSB_ERR_INVALID;
    }
    if (n == 0) return FSB_OK;
    if (!sorted_keys || !order || !values || !starts || !count || !out_keys || !out_values) {
        fsb_host::set_error("fsb_coo_coalesce: null pointer");
        return FSB_ERR_INVALID;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t blocks = std::min<int64_t>(ceil_div(n, (int64_t)sort::kThreads), 148 * 16);
    auto go = [&](auto tv) -> int {
        using V = typename decltype(tv)::type;
        auto go2 = [&](auto tk, auto to) -> int {
            using K = typename decltype(tk)::type;
            using O = typename decltype(to)::type;
            sort::k_coo_segment_sum<V, K, O><<<(unsigned)blocks, sort::kThreads, 0, st>>>(
                static_cast<const K*>(sorted_keys), static_cast<const O*>(starts), count, order,
                static_cast<const V*>(values), n, static_cast<K*>(out_keys), static_cast<V*>(out_values));
            return fsb_host::check_launch("k_coo_segment_sum");
        };
        if (key_dtype == FSB_I32) {
            return starts_dtype == FSB_I32 ? go2(tag<int32_t>{}, tag<int32_t>{}) : go2(tag<int32_t>{}, tag<int64_t>{});
        }
        return starts_dtype == FSB_I32 ? go2(tag<int64_t>{}, tag<int32_t>{}) : go2(tag<int64_t>{}, tag<int64_t>{});
    };
    switch (value_dtype) {
    case FSB_F16: return go(tag<__half>{});
    case FSB_BF16: return go(tag<__nv_bfloat16>{});
    case FSB_F32: return go(tag<float>{});
    case FSB_F64: return go(tag<double>{});
    case FSB_C64: return go(tag<c64_t>{});
    case FSB_C128: return go(tag<c128_t>{});
    case FSB_C32: return go(tag<c32_t>{});
    default:
        fsb_host::set_error("fsb_coo_coalesce: unsupported value dtype %d", value_dtype);
        return FSB_ERR_UNSUPPORTED;
    }
}
