// fsb_partition.cuh -- merge-path partition kernel (used by the partition
// entry point and by the allocation-free SpMV entry point).
#pragma once
#include "fsb_dispatch.cuh"

namespace fsb {

// One thread per unit boundary u: the merge-path coordinate of diagonal
// d = u * items, i.e. (i row ends, j nonzeros) with i + j = d, row end r
// ordered before nonzero k iff row_ptr[r + 1] <= k.
template <class P>
__global__ void k_merge_partition(const P* __restrict__ ptr, int64_t n_rows, int64_t nnz, int64_t items,
                                  int64_t snap, int64_t* __restrict__ coords, int64_t n_units) {
    const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u > n_units) return;
    const int64_t total = n_rows + nnz;
    int64_t d = u * items;
    if (d > total) d = total;
    int64_t lo = d - nnz > 0 ? d - nnz : 0;
    int64_t hi = d < n_rows ? d : n_rows;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (idx(ptr[mid + 1]) <= d - mid - 1) lo = mid + 1; else hi = mid;
    }
    const int64_t i = lo;
    int64_t j = d - lo;
    if (snap > 0 && i < n_rows && u > 0 && u < n_units) {
        const int64_t rs = idx(ptr[i]), re = idx(ptr[i + 1]);
        if (j > rs && re - rs < snap) j = rs;
    }
    coords[2 * u] = i;
    coords[2 * u + 1] = j;
}

}  // namespace fsb
