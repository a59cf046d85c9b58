// fsb_spmm_common.cuh -- pieces shared by the SpMM kernel files: C-row stores,
// accumulator reset and the merge-path carry fix-up.
#pragma once
#include "fsb_dispatch.cuh"

namespace fsb {

constexpr int kSpmmThreads = 128;

template <class O, class A, int VW>
__device__ __forceinline__ void store_row(O* __restrict__ C, int64_t ldc, int64_t out_row, int64_t c0,
                                          const A (&acc)[VW]) {
    if constexpr (VW > 1 && sizeof(O) * VW == 32) {
        // two 16-byte halves
        constexpr int H = VW / 2;
        vec_t<O, H> lo, hi;
#pragma unroll
        for (int w = 0; w < H; ++w) {
            lo.v[w] = Out<O, A>::cvt(acc[w]);
            hi.v[w] = Out<O, A>::cvt(acc[H + w]);
        }
        st_stream<O, H>(C + out_row * ldc + c0, lo);
        st_stream<O, H>(C + out_row * ldc + c0 + H, hi);
    } else if constexpr (VW > 1 && (sizeof(O) * VW == 16 || sizeof(O) * VW == 8 || sizeof(O) * VW == 4)) {
        vec_t<O, VW> o;
#pragma unroll
        for (int w = 0; w < VW; ++w) o.v[w] = Out<O, A>::cvt(acc[w]);
        st_stream<O, VW>(C + out_row * ldc + c0, o);
    } else {
#pragma unroll
        for (int w = 0; w < VW; ++w) C[out_row * ldc + c0 + w] = Out<O, A>::cvt(acc[w]);
    }
}

template <class A> struct is_comp_acc { static constexpr bool value = false; };
template <> struct is_comp_acc<comp_t> { static constexpr bool value = true; };

template <class A, int VW>
__device__ __forceinline__ void zero_acc(A (&acc)[VW]) {
#pragma unroll
    for (int w = 0; w < VW; ++w) acc[w] = A{};
}

// One warp per unit: the first unit of each run carrying the same open row
// folds the run's carries (unit order) and the ending unit's head partial.
template <class A, class O, class I, class P>
__global__ void __launch_bounds__(kSpmmThreads)
k_spmm_merge_fixup(const int64_t* __restrict__ carry_row, const A* __restrict__ carry_val,
                   const A* __restrict__ head_val, int64_t n_units, int64_t n_dense, const P* __restrict__ ptr,
                   const I* __restrict__ row_map, O* __restrict__ C, int64_t ldc) {
    const int64_t t = (int64_t)blockIdx.x * (kSpmmThreads / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (t >= n_units) return;
    const int64_t r = carry_row[t];
    if (r < 0) return;
    if (t > 0 && carry_row[t - 1] == r) return;
    // end of the run of units carrying row r: 32 entries per step, first
    // mismatch by ballot (a long row spans many units)
    int64_t u_end = t + 1;
    while (true) {
        const int64_t u = u_end + lane;
        const bool same = u < n_units && carry_row[u] == r;
        const unsigned stop = __ballot_sync(0xffffffffu, !same);
        if (stop) {
            u_end += __ffs(stop) - 1;
            break;
        }
        u_end += 32;
    }
    const int64_t out_row = row_map ? idx(row_map[idx(ptr[r])]) : r;
    for (int64_t c = lane; c < n_dense; c += 32) {
        // loads four carries ahead, adds in unit order (deterministic)
        A sum = carry_val[t * n_dense + c];
        int64_t u = t + 1;
        for (; u + 4 <= u_end; u += 4) {
            const A a0 = carry_val[u * n_dense + c], a1 = carry_val[(u + 1) * n_dense + c];
            const A a2 = carry_val[(u + 2) * n_dense + c], a3 = carry_val[(u + 3) * n_dense + c];
            sum = acc_add(acc_add(acc_add(acc_add(sum, a0), a1), a2), a3);
        }
        for (; u < u_end; ++u) sum = acc_add(sum, carry_val[u * n_dense + c]);
        if (u_end < n_units) sum = acc_add(sum, head_val[u_end * n_dense + c]);
        C[out_row * ldc + c] = Out<O, A>::cvt(sum);
    }
}


// FSB_ALGO_GATHER launch (fsb_spmm_gather.cu), dtype dispatch included.
int spmm_gather_dispatch(const fsb_csr* A, const void* B, int64_t ldb, int64_t n_dense, void* C, int64_t ldc,
                         int out_dtype, int acc_mode, const fsb_plan* plan, void* workspace, int64_t workspace_bytes,
                         cudaStream_t st);

}  // namespace fsb
