// fsb_sddmm.cu -- sampled dense-dense matrix multiplication on a CSR pattern:
//     out[p] = alpha * dot(x[row(p)], y[col(p)]) + beta * data[p]
// for every stored position p (FlagSparse's flagsparse_sddmm_csr,
// sddmm_csr.py:350-422, kernel _sddmm_csr_real_kernel :108-152).
//
// A sub-group of LPN lanes computes one dot product, each lane covering VW
// consecutive elements of K per step (16-byte vectors where x and y allow);
// a warp takes NPAR = 32 / LPN positions per step and kSddmmU steps per
// batch, whose x / y loads are all issued before the multiply-adds use them
// (the y rows are random gathers, latency bound).  The dot product is reduced
// inside its sub-group (log2 LPN xor-shuffles).  float32 accumulates in
// float32, float64 in float64, as FlagSparse's baseline kernel does.
#include "fsb_dispatch.cuh"

namespace fsb {

constexpr int kSddmmThreads = 256;
constexpr int kSddmmU = 4;

// 4 resident CTAs of 256 threads per SM (64 registers): the random y-row
// gathers are latency bound, so resident warps beat unspilled registers
// (measured: 80 registers / 3 CTAs 0.239 ms, 64 / 4 0.188 ms, 51 / 5
// 0.197 ms on the power-law pattern at K = 64).
template <class V, class A, class I, int VW, int LPN_LOG2>
__global__ void __launch_bounds__(kSddmmThreads, 4)
k_sddmm(const I* __restrict__ col, const int32_t* __restrict__ row_ids, int64_t nnz, const V* __restrict__ x,
        int64_t ldx, const V* __restrict__ y, int64_t ldy, int64_t k, const V* __restrict__ data,
        V* __restrict__ out, A alpha, A beta) {
    constexpr int LPN = 1 << LPN_LOG2;
    constexpr int NPAR = 32 >> LPN_LOG2;
    constexpr int STEP = NPAR * kSddmmU;  // positions per warp batch
    const int lane = threadIdx.x & 31;
    const int sub = lane >> LPN_LOG2, cl = lane & (LPN - 1);
    const int64_t warp = ((int64_t)blockIdx.x * kSddmmThreads + threadIdx.x) >> 5;
    const int64_t n_warps = ((int64_t)gridDim.x * kSddmmThreads) >> 5;
    for (int64_t base = warp * STEP; base < nnz; base += n_warps * STEP) {
        int64_t p[kSddmmU], r[kSddmmU], c[kSddmmU];
        A acc[kSddmmU];
#pragma unroll
        for (int u = 0; u < kSddmmU; ++u) {
            p[u] = base + u * NPAR + sub;
            const bool ok = p[u] < nnz;
            r[u] = ok ? (int64_t)row_ids[p[u]] : 0;
            c[u] = ok ? idx(col[p[u]]) : 0;
            acc[u] = A(0);
        }
        for (int64_t kk = (int64_t)cl * VW; kk < k; kk += (int64_t)LPN * VW) {
            vec_t<V, VW> xv[kSddmmU], yv[kSddmmU];
#pragma unroll
            for (int u = 0; u < kSddmmU; ++u) {
                if (p[u] < nnz) {
                    xv[u] = ld_ro<V, VW>(x + r[u] * ldx + kk);
                    yv[u] = ld_ro<V, VW>(y + c[u] * ldy + kk);
                } else {
#pragma unroll
                    for (int w = 0; w < VW; ++w) xv[u].v[w] = yv[u].v[w] = V(0);
                }
            }
#pragma unroll
            for (int u = 0; u < kSddmmU; ++u)
#pragma unroll
                for (int w = 0; w < VW; ++w) acc[u] = fma((A)xv[u].v[w], (A)yv[u].v[w], acc[u]);
        }
#pragma unroll
        for (int u = 0; u < kSddmmU; ++u) {
#pragma unroll
            for (int o = LPN / 2; o > 0; o >>= 1) acc[u] += __shfl_xor_sync(0xffffffffu, acc[u], o, LPN);
            if (cl == 0 && p[u] < nnz) {
                A v = alpha * acc[u];
                if (data) v += (A)data[p[u]] * beta;
                out[p[u]] = (V)v;
            }
        }
    }
}

template <class V, class A, class I, int VW>
int launch_sddmm_vw(int lpn_log2, const I* col, const int32_t* rows, int64_t nnz, const V* x, int64_t ldx, const V* y,
                    int64_t ldy, int64_t k, const V* data, V* out, A alpha, A beta, cudaStream_t st) {
    const int npar = 32 >> lpn_log2;
    const int64_t warps = ceil_div(nnz, (int64_t)npar * kSddmmU);
    int64_t blocks = ceil_div(warps, (int64_t)(kSddmmThreads / 32));
    if (blocks > 148 * 64) blocks = 148 * 64;  // grid-stride beyond ~64 waves of CTAs
#define FSB_SDDMM(L)                                                                                           \
    case L:                                                                                                    \
        k_sddmm<V, A, I, VW, L><<<(unsigned)blocks, kSddmmThreads, 0, st>>>(col, rows, nnz, x, ldx, y, ldy, k, \
                                                                             data, out, alpha, beta);          \
        break;
    switch (lpn_log2) {
        FSB_SDDMM(0)
        FSB_SDDMM(1)
        FSB_SDDMM(2)
        FSB_SDDMM(3)
        FSB_SDDMM(4)
        FSB_SDDMM(5)
        default:
            fsb_host::set_error("fsb_sddmm_csr: bad lane count");
            return FSB_ERR_INVALID;
    }
#undef FSB_SDDMM
    return fsb_host::check_launch("k_sddmm");
}

}  // namespace fsb

extern "C" int fsb_sddmm_csr(const void* col_idx, int index_dtype, const int32_t* row_ids, int64_t nnz, int64_t n_rows,
                             int64_t n_cols, const void* x, int64_t ldx, const void* y, int64_t ldy, int64_t k,
                             const void* data, void* out, int value_dtype, double alpha, double beta, void* stream) {
    if (nnz < 0 || k < 0 || n_rows < 0 || n_cols < 0 || ldx < k || ldy < k) {
        fsb_host::set_error("fsb_sddmm_csr: bad sizes");
        return FSB_ERR_INVALID;
    }
    if (nnz == 0) return FSB_OK;
    if (!col_idx || !row_ids || !out || (k > 0 && (!x || !y))) {
        fsb_host::set_error("fsb_sddmm_csr: null pointer");
        return FSB_ERR_INVALID;
    }
    if (value_dtype != FSB_F32 && value_dtype != FSB_F64) {
        fsb_host::set_error("fsb_sddmm_csr: values must be float32 or float64");
        return FSB_ERR_UNSUPPORTED;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return fsb::dispatch_idx(index_dtype, [&](auto ti) -> int {
        using I = typename decltype(ti)::type;
        auto run = [&](auto tv) -> int {
            using V = typename decltype(tv)::type;
            using A = V;
            constexpr int kVW = 16 / (int)sizeof(V);
            const V* xv = static_cast<const V*>(x);
            const V* yv = static_cast<const V*>(y);
            const bool vec = k % kVW == 0 && ldx % kVW == 0 && ldy % kVW == 0 && ((uintptr_t)xv) % 16 == 0 &&
                             ((uintptr_t)yv) % 16 == 0;
            const int vw = vec ? kVW : 1;
            int lpn_log2 = 0;
            while ((int64_t)(vw << lpn_log2) < k && lpn_log2 < 5) ++lpn_log2;
            const I* col = static_cast<const I*>(col_idx);
            const V* d = static_cast<const V*>(data);
            V* o = static_cast<V*>(out);
            if (vec)
                return fsb::launch_sddmm_vw<V, A, I, kVW>(lpn_log2, col, row_ids, nnz, xv, ldx, yv, ldy, k, d, o,
                                                          (A)alpha, (A)beta, st);
            return fsb::launch_sddmm_vw<V, A, I, 1>(lpn_log2, col, row_ids, nnz, xv, ldx, yv, ldy, k, d, o, (A)alpha,
                                                    (A)beta, st);
        };
        if (value_dtype == FSB_F32) return run(fsb::tag<float>{});
        return run(fsb::tag<double>{});
    });
}
