// fsb_diag.cu -- diagnostic CSR SpMM forms: fixed-order accumulation in a
// chosen arithmetic, for numerical diagnosis rather than speed.
//
// FlagSparse ships "stable" and "candidate" SpMM paths next to its opt path
// for its diagnose scripts (spmm_csr.py:922-1249 stable kernels, :1363-1454
// stable runners, :1501-1634 candidate short-row kernels, :1998-2086 the
// entry points).  Their arithmetic, per output element and in nonzero order:
//   FSB_DIAG_NATIVE     acc = fma(a, b, acc) in the value precision
//   FSB_DIAG_WIDE       acc = fma(a, b, acc) in float64, stored in the value
//                       type (the stable path: float64 accumulation,
//                       float32 store)
//   FSB_DIAG_KAHAN      Kahan's compensated sum in the value precision:
//                       y = fma(a, b, -comp); t = acc + y;
//                       comp = (t - acc) - y; acc = t
//   FSB_DIAG_KAHAN_WIDE the same in float64 (the candidate short-row kernels)
// Rows of at most short_max nonzeros use mode_short, longer rows mode_long.
//
// Layout: one warp per row, one dense column per lane (column tiles of 32 on
// the grid's y axis), the row's nonzeros walked in order so every element is
// the exact sequential recurrence above -- bit-reproducible, and equal to a
// scalar CPU restatement with the same operations.  Every add, subtract and
// fused multiply-add is an explicitly rounded intrinsic, so the compiler
// cannot contract or reorder them.
#include "fsb_partition.cuh"

namespace fsb {

constexpr int kDiagWarps = 8;

template <class T> struct DiagOps;
template <> struct DiagOps<float> {
    static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
};
template <> struct DiagOps<double> {
    static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
};

// One row's dot product with dense column n in accumulator type T.
template <class T, class V, class I>
__device__ __forceinline__ T diag_dot(const V* __restrict__ val, const I* __restrict__ col, int64_t s, int64_t e,
                                      const V* __restrict__ B, int64_t ldb, int64_t n, bool kahan) {
    using O = DiagOps<T>;
    T acc = T(0), comp = T(0);
    for (int64_t k = s; k < e; ++k) {
        const T a = (T)val[k];
        const T b = (T)B[idx(col[k]) * ldb + n];
        if (kahan) {
            const T y = O::fma(a, b, -comp);
            const T t = O::add(acc, y);
            comp = O::sub(O::sub(t, acc), y);
            acc = t;
        } else {
            acc = O::fma(a, b, acc);
        }
    }
    return acc;
}

template <class V, class I, class P>
__global__ void __launch_bounds__(kDiagWarps * 32)
k_spmm_diag(const V* __restrict__ val, const I* __restrict__ col, const P* __restrict__ ptr, int64_t n_rows,
            const V* __restrict__ B, int64_t ldb, int64_t n_dense, V* __restrict__ C, int64_t ldc, int mode_short,
            int mode_long, int64_t short_max) {
    const int64_t row = (int64_t)blockIdx.x * kDiagWarps + (threadIdx.x >> 5);
    const int64_t n = (int64_t)blockIdx.y * 32 + (threadIdx.x & 31);
    if (row >= n_rows || n >= n_dense) return;
    const int64_t s = idx(ptr[row]), e = idx(ptr[row + 1]);
    const int mode = (e - s) <= short_max ? mode_short : mode_long;
    const bool kahan = mode == FSB_DIAG_KAHAN || mode == FSB_DIAG_KAHAN_WIDE;
    V out;
    if (mode == FSB_DIAG_WIDE || mode == FSB_DIAG_KAHAN_WIDE) {
        out = (V)diag_dot<double, V, I>(val, col, s, e, B, ldb, n, kahan);
    } else {
        out = diag_dot<V, V, I>(val, col, s, e, B, ldb, n, kahan);
    }
    C[row * ldc + n] = out;
}

}  // namespace fsb

using namespace fsb;

extern "C" int fsb_spmm_csr_diag(const fsb_csr* A, const void* B, int64_t ldb, int64_t n_dense, void* C, int64_t ldc,
                                 int mode_short, int mode_long, int64_t short_max, void* stream) {
    if (!A || n_dense < 0 || A->n_rows < 0 || A->nnz < 0) {
        fsb_host::set_error("fsb_spmm_csr_diag: bad arguments");
        return FSB_ERR_INVALID;
    }
    for (int m : {mode_short, mode_long}) {
        if (m < FSB_DIAG_NATIVE || m > FSB_DIAG_KAHAN_WIDE) {
            fsb_host::set_error("fsb_spmm_csr_diag: unknown mode %d", m);
            return FSB_ERR_INVALID;
        }
    }
    if (A->value_dtype != FSB_F32 && A->value_dtype != FSB_F64) {
        fsb_host::set_error("fsb_spmm_csr_diag: float32 / float64 values only");
        return FSB_ERR_UNSUPPORTED;
    }
    if (A->n_rows == 0 || n_dense == 0) return FSB_OK;
    if (!A->row_ptr || !C || (A->nnz > 0 && (!A->values || !A->col_idx || !B)) || ldb < n_dense || ldc < n_dense) {
        fsb_host::set_error("fsb_spmm_csr_diag: null pointer or stride below n_dense");
        return FSB_ERR_INVALID;
    }
    const int64_t gx = ceil_div(A->n_rows, (int64_t)kDiagWarps), gy = ceil_div(n_dense, (int64_t)32);
    if (gx > 0x7fffffffLL || gy > 65535) {
        fsb_host::set_error("fsb_spmm_csr_diag: grid too large");
        return FSB_ERR_LIMIT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    auto run = [&](auto tv) -> int {
        using V = typename decltype(tv)::type;
        return dispatch_idx(A->index_dtype, [&](auto ti) -> int {
            using I = typename decltype(ti)::type;
            return dispatch_idx(A->ptr_dtype, [&](auto tp) -> int {
                using P = typename decltype(tp)::type;
                k_spmm_diag<V, I, P><<<dim3((unsigned)gx, (unsigned)gy), kDiagWarps * 32, 0, st>>>(
                    static_cast<const V*>(A->values), static_cast<const I*>(A->col_idx),
                    static_cast<const P*>(A->row_ptr), A->n_rows, static_cast<const V*>(B), ldb, n_dense,
                    static_cast<V*>(C), ldc, mode_short, mode_long, short_max);
                return fsb_host::check_launch("k_spmm_diag");
            });
        });
    };
    return A->value_dtype == FSB_F32 ? run(tag<float>{}) : run(tag<double>{});
}
