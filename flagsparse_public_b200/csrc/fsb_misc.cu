// fsb_misc.cu -- merge-path partition, COO atomic kernels, workspace sizing and
// error reporting of the C ABI.
#include <stdarg.h>
#include <stdio.h>

#include "fsb_partition.cuh"

namespace fsb_host {
static thread_local char g_last_error[512] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

int check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return FSB_ERR_LAUNCH;
    }
    return FSB_OK;
}
}  // namespace fsb_host

namespace fsb {

template <class V, class A, class I>
__global__ void k_spmv_coo_atomic(const V* __restrict__ val, const I* __restrict__ row, const I* __restrict__ col,
                                  int64_t nnz, const V* __restrict__ x, A* __restrict__ y) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nnz) return;
    const A p = Acc<V, A>::fma(ld_stream1(val + k), ld_ro1(x + idx(ld_stream1(col + k))), Acc<V, A>::zero());
    atomic_accumulate(y + idx(ld_stream1(row + k)), p);
}

template <class V, class A, class I>
__global__ void k_spmm_coo_atomic(const V* __restrict__ val, const I* __restrict__ row, const I* __restrict__ col,
                                  int64_t nnz, const V* __restrict__ B, int64_t ldb, int64_t n_dense,
                                  A* __restrict__ C, int64_t ldc) {
    // One warp per nonzero, lanes over dense columns.
    const int64_t k = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (k >= nnz) return;
    const V a = ld_stream1(val + k);
    const int64_t r = idx(ld_stream1(row + k)), c = idx(ld_stream1(col + k));
    for (int64_t n = lane; n < n_dense; n += 32) {
        const A p = Acc<V, A>::fma(a, ld_ro1(B + c * ldb + n), Acc<V, A>::zero());
        atomic_accumulate(C + r * ldc + n, p);
    }
}

// Structural check of a CSR matrix: row lengths from adjacent row offsets
// and column indices in grid-stride loops, each CTA's six figures reduced in
// shared memory and written to its slot of part[]; one CTA then folds the
// slots into out[].  No memset or copy-engine work, and out[] may be pinned
// host memory, so the check does not queue behind host<->device copies.
constexpr int kCheckThreads = 256;
constexpr int64_t kCheckMaxBlocks = 148 * 8;

__device__ __forceinline__ unsigned long long check_fold(int f, unsigned long long a, unsigned long long b) {
    return (f == 2 || f == 3) ? (a > b ? a : b) : a + b;  // slots 2, 3 are maxima
}

template <class P, class I>
__global__ void __launch_bounds__(kCheckThreads) k_csr_check_part(const P* __restrict__ ptr, int64_t n_rows,
                                                                   const I* __restrict__ col, int64_t nnz,
                                                                   unsigned long long* __restrict__ part) {
    // slot f of a CTA: rows of negative length, negative columns, largest
    // column, longest row, sum of squared lengths, empty rows
    unsigned long long v[6] = {0, 0, 0, 0, 0, 0};
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (int64_t r = t0; r < n_rows; r += stride) {
        const int64_t len = idx(ptr[r + 1]) - idx(ptr[r]);
        if (len < 0) {
            ++v[0];
        } else {
            const unsigned long long u = (unsigned long long)len;
            v[3] = u > v[3] ? u : v[3];
            v[4] += u * u;
            v[5] += (len == 0);
        }
    }
    for (int64_t k = t0; k < nnz; k += stride) {
        const int64_t c = idx(col[k]);
        if (c < 0) ++v[1];
        else v[2] = (unsigned long long)c > v[2] ? (unsigned long long)c : v[2];
    }
    __shared__ unsigned long long red[6][kCheckThreads / 32];
#pragma unroll
    for (int f = 0; f < 6; ++f)
        for (int o = 16; o > 0; o >>= 1) v[f] = check_fold(f, v[f], __shfl_xor_sync(0xffffffffu, v[f], o));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
#pragma unroll
        for (int f = 0; f < 6; ++f) red[f][warp] = v[f];
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int f = threadIdx.x;
        unsigned long long a = red[f][0];
        for (int w = 1; w < kCheckThreads / 32; ++w) a = check_fold(f, a, red[f][w]);
        part[(int64_t)blockIdx.x * 6 + f] = a;
    }
}

template <class P>
__global__ void __launch_bounds__(kCheckThreads) k_csr_check_final(const P* __restrict__ ptr, int64_t n_rows,
                                                                    const unsigned long long* __restrict__ part,
                                                                    int n_parts, int64_t* out) {
    __shared__ unsigned long long red[6][kCheckThreads / 32];
    unsigned long long v[6] = {0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < n_parts; b += blockDim.x)
#pragma unroll
        for (int f = 0; f < 6; ++f) v[f] = check_fold(f, v[f], part[(int64_t)b * 6 + f]);
#pragma unroll
    for (int f = 0; f < 6; ++f)
        for (int o = 16; o > 0; o >>= 1) v[f] = check_fold(f, v[f], __shfl_xor_sync(0xffffffffu, v[f], o));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
#pragma unroll
        for (int f = 0; f < 6; ++f) red[f][warp] = v[f];
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int f = threadIdx.x;
        unsigned long long a = red[f][0];
        for (int w = 1; w < kCheckThreads / 32; ++w) a = check_fold(f, a, red[f][w]);
        out[2 + f] = (int64_t)a;
    } else if (threadIdx.x == 32) {
        out[0] = idx(ptr[0]);
        out[1] = idx(ptr[n_rows]);
    }
}

static int64_t check_blocks(int64_t n_rows, int64_t nnz) {
    const int64_t work = n_rows > nnz ? n_rows : nnz;
    const int64_t b = ceil_div(work, (int64_t)kCheckThreads * 8);
    return b < 1 ? 1 : (b > kCheckMaxBlocks ? kCheckMaxBlocks : b);
}

}  // namespace fsb

using namespace fsb;

extern "C" int fsb_abi_version(void) { return FSB_ABI_VERSION; }

extern "C" const char* fsb_status_string(int status) {
    switch (status) {
    case FSB_OK: return "ok";
    case FSB_ERR_INVALID: return "invalid argument";
    case FSB_ERR_UNSUPPORTED: return "unsupported dtype or mode";
    case FSB_ERR_LAUNCH: return "kernel launch failed";
    case FSB_ERR_WORKSPACE: return "workspace too small";
    case FSB_ERR_TIMEOUT: return "device wait timed out";
    case FSB_ERR_LIMIT: return "size exceeds entry-point limit";
    default: return "unknown status";
    }
}

extern "C" const char* fsb_last_error(void) { return fsb_host::g_last_error; }

extern "C" int64_t fsb_workspace_bytes(int is_spmm, const fsb_csr* A, int64_t n_dense, int acc_mode, int out_dtype,
                                       const fsb_plan* plan) {
    (void)out_dtype;
    if (!A || !plan) return 0;
    if (plan->algo != FSB_ALGO_MERGE && plan->algo != FSB_ALGO_FLAT && plan->algo != FSB_ALGO_GATHER &&
        plan->algo != FSB_ALGO_SEQ)
        return 0;
    const int ab = acc_size(A->value_dtype, acc_mode);
    if (ab == 0) return 0;
    return merge_scratch_bytes(plan->n_units, is_spmm ? n_dense : 1, ab);
}

extern "C" int fsb_merge_partition(const void* row_ptr, int ptr_dtype, int64_t n_rows, int64_t nnz,
                                   int32_t items_per_unit, int64_t snap_threshold, int64_t* unit_coords,
                                   int64_t n_units, void* stream) {
    if (!row_ptr || !unit_coords || items_per_unit < 1 || n_rows < 0 || nnz < 0) {
        fsb_host::set_error("fsb_merge_partition: bad arguments");
        return FSB_ERR_INVALID;
    }
    if (n_units != ceil_div(n_rows + nnz, items_per_unit)) {
        fsb_host::set_error("fsb_merge_partition: n_units must be ceil((n_rows + nnz) / items_per_unit)");
        return FSB_ERR_INVALID;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return dispatch_idx(ptr_dtype, [&](auto tp) -> int {
        using P = typename decltype(tp)::type;
        const int64_t threads = n_units + 1;
        k_merge_partition<P><<<(unsigned)ceil_div(threads, 256), 256, 0, st>>>(
            static_cast<const P*>(row_ptr), n_rows, nnz, items_per_unit, snap_threshold, unit_coords, n_units);
        return fsb_host::check_launch("k_merge_partition");
    });
}

extern "C" int fsb_merge_runs(const void* row_ptr, int ptr_dtype, int64_t n_rows, const int64_t* unit_coords,
                              int64_t n_units, int64_t* unit_runs, void* stream) {
    if (!row_ptr || !unit_coords || !unit_runs || n_rows < 0 || n_units < 0) {
        fsb_host::set_error("fsb_merge_runs: bad arguments");
        return FSB_ERR_INVALID;
    }
    if (n_units == 0) return FSB_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return dispatch_idx(ptr_dtype, [&](auto tp) -> int {
        using P = typename decltype(tp)::type;
        k_merge_runs<P><<<(unsigned)ceil_div(n_units, 256), 256, 0, st>>>(static_cast<const P*>(row_ptr), n_rows,
                                                                         unit_coords, n_units, unit_runs);
        return fsb_host::check_launch("k_merge_runs");
    });
}

extern "C" int64_t fsb_csr_check_workspace_bytes(int64_t n_rows, int64_t nnz) {
    if (n_rows < 0 || nnz < 0) return 0;
    return check_blocks(n_rows, nnz) * 6 * (int64_t)sizeof(unsigned long long);
}

extern "C" int fsb_csr_check(const void* row_ptr, int ptr_dtype, int64_t n_rows, const void* col_idx, int index_dtype,
                             int64_t nnz, int64_t* out, void* workspace, int64_t workspace_bytes, void* stream) {
    if (!row_ptr || !out || n_rows < 0 || nnz < 0 || (nnz > 0 && !col_idx)) {
        fsb_host::set_error("fsb_csr_check: bad arguments");
        return FSB_ERR_INVALID;
    }
    const int64_t blocks = check_blocks(n_rows, nnz);
    if (!workspace || workspace_bytes < blocks * 6 * (int64_t)sizeof(unsigned long long)) {
        fsb_host::set_error("fsb_csr_check: workspace %lld bytes < %lld", (long long)workspace_bytes,
                            (long long)(blocks * 6 * (int64_t)sizeof(unsigned long long)));
        return FSB_ERR_WORKSPACE;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned long long* part = static_cast<unsigned long long*>(workspace);
    return dispatch_idx(ptr_dtype, [&](auto tp) -> int {
        using P = typename decltype(tp)::type;
        int rc = dispatch_idx(nnz > 0 ? index_dtype : FSB_I32, [&](auto ti) -> int {
            using I = typename decltype(ti)::type;
            k_csr_check_part<P, I><<<(unsigned)blocks, kCheckThreads, 0, st>>>(
                static_cast<const P*>(row_ptr), n_rows, static_cast<const I*>(col_idx), nnz, part);
            return fsb_host::check_launch("k_csr_check_part");
        });
        if (rc) return rc;
        k_csr_check_final<P><<<1, kCheckThreads, 0, st>>>(static_cast<const P*>(row_ptr), n_rows, part,
                                                          (int)blocks, out);
        return fsb_host::check_launch("k_csr_check_final");
    });
}

// Value/accumulator pairs of the atomic routes: the accumulator buffer is the
// value type or its wide type.
template <class F>
static int dispatch_atomic(int vdt, int adt, F&& f) {
    if (vdt == FSB_F32 && adt == FSB_F32) return f(tag<float>{}, tag<float>{});
    if (vdt == FSB_F32 && adt == FSB_F64) return f(tag<float>{}, tag<double>{});
    if (vdt == FSB_F64 && adt == FSB_F64) return f(tag<double>{}, tag<double>{});
    if (vdt == FSB_C64 && adt == FSB_C64) return f(tag<c64_t>{}, tag<c64_t>{});
    if (vdt == FSB_C64 && adt == FSB_C128) return f(tag<c64_t>{}, tag<c128_t>{});
    if (vdt == FSB_C128 && adt == FSB_C128) return f(tag<c128_t>{}, tag<c128_t>{});
    if (vdt == FSB_C32 && adt == FSB_C64) return f(tag<c32_t>{}, tag<c64_t>{});
    if (vdt == FSB_F16 && adt == FSB_F32) return f(tag<__half>{}, tag<float>{});
    if (vdt == FSB_BF16 && adt == FSB_F32) return f(tag<__nv_bfloat16>{}, tag<float>{});
    fsb_host::set_error("atomic route: unsupported value/accumulator pair (%d, %d)", vdt, adt);
    return FSB_ERR_UNSUPPORTED;
}

extern "C" int fsb_spmv_coo_atomic(const void* values, const void* row, const void* col, int value_dtype,
                                   int index_dtype, int64_t nnz, const void* x, void* y, int acc_dtype,
                                   void* stream) {
    if (nnz < 0) return FSB_ERR_INVALID;
    if (nnz == 0) return FSB_OK;
    if (!values || !row || !col || !x || !y) {
        fsb_host::set_error("fsb_spmv_coo_atomic: null pointer");
        return FSB_ERR_INVALID;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return dispatch_atomic(value_dtype, acc_dtype, [&](auto tv, auto ta) -> int {
        using V = typename decltype(tv)::type;
        using Ac = typename decltype(ta)::type;
        return dispatch_idx(index_dtype, [&](auto ti) -> int {
            using I = typename decltype(ti)::type;
            k_spmv_coo_atomic<V, Ac, I><<<(unsigned)ceil_div(nnz, 256), 256, 0, st>>>(
                static_cast<const V*>(values), static_cast<const I*>(row), static_cast<const I*>(col), nnz,
                static_cast<const V*>(x), static_cast<Ac*>(y));
            return fsb_host::check_launch("k_spmv_coo_atomic");
        });
    });
}

extern "C" int fsb_spmm_coo_atomic(const void* values, const void* row, const void* col, int value_dtype,
                                   int index_dtype, int64_t nnz, const void* B, int64_t ldb, int64_t n_dense,
                                   void* C, int64_t ldc, int acc_dtype, void* stream) {
    if (nnz < 0 || n_dense < 0) return FSB_ERR_INVALID;
    if (nnz == 0 || n_dense == 0) return FSB_OK;
    if (!values || !row || !col || !B || !C) {
        fsb_host::set_error("fsb_spmm_coo_atomic: null pointer");
        return FSB_ERR_INVALID;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return dispatch_atomic(value_dtype, acc_dtype, [&](auto tv, auto ta) -> int {
        using V = typename decltype(tv)::type;
        using Ac = typename decltype(ta)::type;
        return dispatch_idx(index_dtype, [&](auto ti) -> int {
            using I = typename decltype(ti)::type;
            const int64_t blocks = ceil_div(nnz, 256 / 32);
            if (blocks > 0x7fffffffLL) return FSB_ERR_LIMIT;
            k_spmm_coo_atomic<V, Ac, I><<<(unsigned)blocks, 256, 0, st>>>(
                static_cast<const V*>(values), static_cast<const I*>(row), static_cast<const I*>(col), nnz,
                static_cast<const V*>(B), ldb, n_dense, static_cast<Ac*>(C), ldc);
            return fsb_host::check_launch("k_spmm_coo_atomic");
        });
    });
}

namespace fsb {
// offsets[b] = number of keys < b, for b in [0, n_bins]: a lower-bound search
// of each bin boundary in the sorted keys (thread per boundary).
template <class K>
__global__ void k_sorted_keys_to_offsets(const K* __restrict__ keys, int64_t n, int64_t n_bins,
                                         int64_t* __restrict__ offsets) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b > n_bins) return;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = lo + ((hi - lo) >> 1);
        if (idx(keys[mid]) < b) lo = mid + 1;
        else hi = mid;
    }
    offsets[b] = lo;
}
}  // namespace fsb

extern "C" int fsb_sorted_keys_to_offsets(const void* keys, int key_dtype, int64_t n, int64_t n_bins,
                                          int64_t* offsets, void* stream) {
    if (n < 0 || n_bins < 0 || !offsets || (n > 0 && !keys)) {
        fsb_host::set_error("fsb_sorted_keys_to_offsets: bad arguments");
        return FSB_ERR_INVALID;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return fsb::dispatch_idx(key_dtype, [&](auto tk) -> int {
        using K = typename decltype(tk)::type;
        const int64_t threads = n_bins + 1;
        fsb::k_sorted_keys_to_offsets<K><<<(unsigned)fsb::ceil_div(threads, (int64_t)256), 256, 0, st>>>(
            static_cast<const K*>(keys), n, n_bins, offsets);
        return fsb_host::check_launch("k_sorted_keys_to_offsets");
    });
}
