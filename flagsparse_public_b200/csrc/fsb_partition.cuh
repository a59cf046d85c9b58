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

// One thread per unit u: the run of units holding the row that is open at
// u's end.  Unit u ends at (r, k) = coords[u + 1]; the row is open when
// k > max(row_ptr[r], k0(u)) (part of r lies in u).  The run's first unit is
// the smallest v whose end coordinate is past (r, row_ptr[r]) in the
// lexicographic order of the (monotone) coordinates; its last unit is the
// one holding r's end, the smallest v whose end row is past r.
template <class P>
__global__ void k_merge_runs(const P* __restrict__ ptr, int64_t n_rows, const int64_t* __restrict__ coords,
                             int64_t n_units, int64_t* __restrict__ runs) {
    const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n_units) return;
    const int64_t r = coords[2 * u + 2], k1 = coords[2 * u + 3], k0 = coords[2 * u + 1];
    int64_t first = -1, last = -1;
    if (r < n_rows) {
        const int64_t s = idx(ptr[r]);
        if (k1 > (s > k0 ? s : k0)) {
            int64_t lo = 0, hi = u;  // first: smallest v in [0, u] with end > (r, s)
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                const int64_t er = coords[2 * mid + 2], ek = coords[2 * mid + 3];
                if (er > r || (er == r && ek > s)) hi = mid; else lo = mid + 1;
            }
            first = lo;
            lo = u + 1;
            hi = n_units - 1;  // last: smallest v in [u + 1, n_units - 1] with end row > r
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                if (coords[2 * mid + 2] > r) hi = mid; else lo = mid + 1;
            }
            last = lo;
        }
    }
    runs[2 * u] = first;
    runs[2 * u + 1] = last;
}

}  // namespace fsb
