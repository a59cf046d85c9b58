// fsb_spmv.cu -- CSR SpMV on sm_100a: y = A x.
//
// Two kernel families, chosen per matrix by the host plan:
//   * k_spmv_rows  : a group of 2^k lanes per row (k = 0..5; 32 lanes is
//                    warp-per-row), 128-bit streaming loads of values and column
//                    indices on the aligned body of each row, read-only cached
//                    gathers of x, xor-butterfly reduction inside the group.
//   * k_spmv_merge : merge-path tiles over the (row ends + nonzeros) path
//                    (Merrill & Garland, SC'16): every CTA gets the same number
//                    of path items whatever the row-length skew.  Products are
//                    staged in shared memory, each thread walks its stretch of
//                    the path, a warp-shuffle segmented scan carries partial
//                    rows across threads, and rows that cross tile boundaries
//                    are finished by k_spmv_merge_fixup from per-tile carries.
//
// FlagSparse computes the same products in _spmv_csr_real_kernel
// (spmv_csr.py:158-184), _spmv_csr_complex_kernel (:187-219), the CSR-vector
// bucket kernels (:225-343) and the COO row-run kernels (spmv_coo.py:131-226).
#include <cstring>
#include <cmath>
#include <mutex>

#include "fsb_partition.cuh"

namespace fsb {

constexpr int kRowsThreads = 256;
constexpr int kMergeThreads = 128;
constexpr int kMergeMaxItemsPerThread = 8;
constexpr int kMergeMaxTile = kMergeThreads * kMergeMaxItemsPerThread;
// FSB_PLAN_OVERLAP_LAUNCH applies to grids of at most one wave at four
// resident CTAs per SM (a waiting successor then takes no slot a later wave
// of this kernel would need)
constexpr int64_t kOverlapMaxBlocks = 148 * 4;

// Partial sum of row nonzeros [s, e) handled by `lane` of a T-lane group.
// VEC-wide aligned body, scalar head and tail.
template <class V, class A, class I>
__device__ __forceinline__ A row_partial(const V* __restrict__ val, const I* __restrict__ col,
                                         const V* __restrict__ x, int64_t s, int64_t e,
                                         int lane, int T, bool vec_ok) {
    constexpr int VV = VecWidth<V>::value;
    constexpr int VI = VecWidth<I>::value;
    constexpr int VEC = VV < VI ? VV : VI;
    A acc = Acc<V, A>::zero();
    if (VEC > 1 && vec_ok) {
        int64_t a0 = (s + VEC - 1) & ~(int64_t)(VEC - 1);
        if (a0 > e) a0 = e;
        int64_t a1 = e & ~(int64_t)(VEC - 1);
        if (a1 < a0) a1 = a0;
        for (int64_t k = s + lane; k < a0; k += T)
            acc = Acc<V, A>::fma(ld_stream1(val + k), ld_ro1(x + idx(ld_stream1(col + k))), acc);
#pragma unroll 2
        for (int64_t kb = a0 + (int64_t)lane * VEC; kb < a1; kb += (int64_t)T * VEC) {
            vec_t<V, VEC> vv = ld_stream<V, VEC>(val + kb);
            vec_t<I, VEC> cc = ld_stream<I, VEC>(col + kb);
            V xv[VEC];
#pragma unroll
            for (int j = 0; j < VEC; ++j) xv[j] = ld_ro1(x + idx(cc.v[j]));
#pragma unroll
            for (int j = 0; j < VEC; ++j) acc = Acc<V, A>::fma(vv.v[j], xv[j], acc);
        }
        for (int64_t k = a1 + lane; k < e; k += T)
            acc = Acc<V, A>::fma(ld_stream1(val + k), ld_ro1(x + idx(ld_stream1(col + k))), acc);
    } else {
#pragma unroll 4
        for (int64_t k = s + lane; k < e; k += T)
            acc = Acc<V, A>::fma(ld_stream1(val + k), ld_ro1(x + idx(ld_stream1(col + k))), acc);
    }
    return acc;
}

template <class A> struct is_comp { static constexpr bool value = false; };
template <> struct is_comp<comp_t> { static constexpr bool value = true; };

template <class V, class A, class O, class I, class P>
__global__ void __launch_bounds__(kRowsThreads)
k_spmv_rows(const V* __restrict__ val, const I* __restrict__ col, const P* __restrict__ ptr,
            const I* __restrict__ row_map, const V* __restrict__ x, O* __restrict__ y,
            int64_t n_rows, int64_t row_cap, int64_t comp_threshold, int lanes_log2, int vec_ok, int overlap) {
    // programmatic dependent launch: wait until the previous kernel on the
    // stream has completed and its writes are visible -- nothing is read
    // before -- and let the next launch start once this CTA's rows are done
    if (overlap) asm volatile("griddepcontrol.wait;" ::: "memory");
    const int T = 1 << lanes_log2;
    const int wl = threadIdx.x & 31;
    const int lane = wl & (T - 1);
    const unsigned mask = segment_mask(wl, T);
    const int64_t stride = ((int64_t)gridDim.x * blockDim.x) >> lanes_log2;
    for (int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> lanes_log2; row < n_rows;
         row += stride) {
        const int64_t s = idx(ptr[row]);
        int64_t e = idx(ptr[row + 1]);
        if (row_cap > 0 && e - s > row_cap) e = s + row_cap;
        A acc;
        if constexpr (is_comp<A>::value) {
            if (e - s > comp_threshold) {
                acc = row_partial<V, comp_t, I>(val, col, x, s, e, lane, T, vec_ok);
            } else {
                acc = comp_t{row_partial<V, float, I>(val, col, x, s, e, lane, T, vec_ok), 0.f};
            }
        } else {
            acc = row_partial<V, A, I>(val, col, x, s, e, lane, T, vec_ok);
        }
        acc = segment_reduce(mask, acc, 1, T);
        if (lane == 0) {
            const int64_t out_row = row_map ? idx(row_map[s]) : row;
            y[out_row] = Out<O, A>::cvt(acc);
        }
    }
    if (overlap) asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ---------------------------------------------------------- merge path ----
// unit_coords[2u], [2u+1] = (rows ended, nonzeros consumed) at the start of tile u.
// Scratch per tile: carry_row (row still open at the tile end, -1 if none),
// carry_val (its partial), head_val (partial of the tile's first finished row
// when that row began in an earlier tile).
template <class V, class A, class O, class I, class P>
__global__ void __launch_bounds__(kMergeThreads)
k_spmv_merge(const V* __restrict__ val, const I* __restrict__ col, const P* __restrict__ ptr,
             const I* __restrict__ row_map, const V* __restrict__ x, O* __restrict__ y,
             int64_t n_rows, const int64_t* __restrict__ coords, int items_per_thread,
             int64_t* __restrict__ carry_row, A* __restrict__ carry_val, A* __restrict__ head_val) {
    __shared__ A s_prod[kMergeMaxTile];
    __shared__ int s_end[kMergeMaxTile];
    __shared__ A s_wv[kMergeThreads / 32];
    __shared__ int s_wf[kMergeThreads / 32];

    const int64_t tile = blockIdx.x;
    const int64_t r0 = coords[2 * tile], k0 = coords[2 * tile + 1];
    const int64_t r1 = coords[2 * tile + 2], k1 = coords[2 * tile + 3];
    const int rows_tile = (int)(r1 - r0);  // row ends inside the tile
    const int nnz_tile = (int)(k1 - k0);
    const int items = rows_tile + nnz_tile;
    const int tid = threadIdx.x;
    // Coordinates that do not come from an unsnapped partition with this tile
    // size would overrun the shared-memory staging: leave such a tile alone
    // (uniform across the block, before any barrier).
    if (r1 < r0 || k1 < k0 || (r1 - r0) + (k1 - k0) > (int64_t)kMergeThreads * items_per_thread) return;

    for (int j = tid; j < nnz_tile; j += kMergeThreads) {
        const int64_t k = k0 + j;
        s_prod[j] = Acc<V, A>::fma(ld_stream1(val + k), ld_ro1(x + idx(ld_stream1(col + k))), Acc<V, A>::zero());
    }
    for (int i = tid; i < rows_tile; i += kMergeThreads) s_end[i] = (int)(idx(ptr[r0 + i + 1]) - k0);
    __syncthreads();

    // This thread's stretch of the tile-local path: [d0, d1).
    const int d0 = min(tid * items_per_thread, items);
    const int d1 = min(d0 + items_per_thread, items);
    int lo = max(0, d0 - nnz_tile), hi = min(d0, rows_tile);
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (s_end[mid] <= d0 - mid - 1) lo = mid + 1; else hi = mid;
    }
    int i = lo, j = d0 - lo;

    const bool continued = (r0 < n_rows) && (k0 > idx(ptr[r0]));
    A run = Acc<V, A>::zero(), first = Acc<V, A>::zero();
    int first_i = -1;
    bool head = false;
    for (int d = d0; d < d1; ++d) {
        if (i < rows_tile && s_end[i] <= j) {
            if (!head) {
                head = true;
                first = run;
                first_i = i;
            } else {
                const int64_t r = r0 + i;
                const int64_t out_row = row_map ? idx(row_map[idx(ptr[r])]) : r;
                y[out_row] = Out<O, A>::cvt(run);
            }
            run = Acc<V, A>::zero();
            ++i;
        } else {
            run = acc_add(run, s_prod[j]);
            ++j;
        }
    }

    // Segmented inclusive scan of (head, run) across the block:
    // (f1, v1) . (f2, v2) = (f1 | f2, f2 ? v2 : v1 + v2).
    const int wl = tid & 31, warp = tid >> 5;
    bool f = head;
    A v = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const A vu = shfl_up(0xffffffffu, v, o);
        const int fu = __shfl_up_sync(0xffffffffu, (int)f, o);
        if (wl >= o) {
            if (!f) v = acc_add(vu, v);
            f = f || fu;
        }
    }
    if (wl == 31) {
        s_wv[warp] = v;
        s_wf[warp] = (int)f;
    }
    __syncthreads();
    A pv = Acc<V, A>::zero();
    for (int w = 0; w < warp; ++w) pv = s_wf[w] ? s_wv[w] : acc_add(pv, s_wv[w]);
    const A incl = f ? v : acc_add(pv, v);
    A excl = shfl_up(0xffffffffu, incl, 1);
    if (wl == 0) excl = pv;

    if (head) {
        const A total = acc_add(excl, first);
        if (first_i == 0 && continued) {
            head_val[tile] = total;
        } else {
            const int64_t r = r0 + first_i;
            const int64_t out_row = row_map ? idx(row_map[idx(ptr[r])]) : r;
            y[out_row] = Out<O, A>::cvt(total);
        }
    }
    if (tid == kMergeThreads - 1) {
        const bool open = (r1 < n_rows) && (k1 > idx(ptr[r1]));
        carry_row[tile] = open ? r1 : -1;
        if (open) carry_val[tile] = incl;
    }
}

// One thread per tile: the first tile of each run of tiles carrying the same
// open row sums the run's carries in tile order, adds the partial held by the
// tile where the row ends and writes the row once.
template <class A, class O, class I, class P>
__global__ void k_spmv_merge_fixup(const int64_t* __restrict__ carry_row, const A* __restrict__ carry_val,
                                   const A* __restrict__ head_val, int64_t n_tiles, const P* __restrict__ ptr,
                                   const I* __restrict__ row_map, O* __restrict__ y) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tiles) return;
    const int64_t r = carry_row[t];
    if (r < 0) return;
    if (t > 0 && carry_row[t - 1] == r) return;
    A sum = carry_val[t];
    int64_t u = t + 1;
    while (u < n_tiles && carry_row[u] == r) {
        sum = acc_add(sum, carry_val[u]);
        ++u;
    }
    if (u < n_tiles) sum = acc_add(sum, head_val[u]);
    const int64_t out_row = row_map ? idx(row_map[idx(ptr[r])]) : r;
    y[out_row] = Out<O, A>::cvt(sum);
}

}  // namespace fsb

using namespace fsb;

extern "C" int fsb_spmv_csr(const fsb_csr* A, const void* x, void* y, int out_dtype, int acc_mode,
                            const fsb_plan* plan, void* workspace, int64_t workspace_bytes, void* stream) {
    if (!A || !plan) {
        fsb_host::set_error("fsb_spmv_csr: null matrix or plan");
        return FSB_ERR_INVALID;
    }
    if (A->n_rows < 0 || A->nnz < 0) {
        fsb_host::set_error("fsb_spmv_csr: negative size");
        return FSB_ERR_INVALID;
    }
    if (A->n_rows == 0) return FSB_OK;
    if (!A->row_ptr || !y || (A->nnz > 0 && (!A->values || !A->col_idx || !x))) {
        fsb_host::set_error("fsb_spmv_csr: null data pointer");
        return FSB_ERR_INVALID;
    }
    if (A->row_map && A->row_map_dtype != A->index_dtype) {
        fsb_host::set_error("fsb_spmv_csr: row_map dtype must equal index dtype");
        return FSB_ERR_INVALID;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int vdt = A->value_dtype;
    return dispatch_vao(vdt, acc_mode, out_dtype, [&](auto tv, auto ta, auto to) -> int {
        using V = typename decltype(tv)::type;
        using Ac = typename decltype(ta)::type;
        using O = typename decltype(to)::type;
        return dispatch_idx(A->index_dtype, [&](auto ti) -> int {
            using I = typename decltype(ti)::type;
            return dispatch_idx(A->ptr_dtype, [&](auto tp) -> int {
                using P = typename decltype(tp)::type;
                const V* val = static_cast<const V*>(A->values);
                const I* col = static_cast<const I*>(A->col_idx);
                const P* ptr = static_cast<const P*>(A->row_ptr);
                const I* rmap = static_cast<const I*>(A->row_map);
                const V* xv = static_cast<const V*>(x);
                O* yv = static_cast<O*>(y);
                if (plan->algo == FSB_ALGO_ROWS) {
                    int lanes = plan->lanes;
                    if (lanes < 1 || lanes > 32 || (lanes & (lanes - 1))) {
                        fsb_host::set_error("fsb_spmv_csr: lanes=%d is not a power of two in [1, 32]", lanes);
                        return FSB_ERR_INVALID;
                    }
                    int lg = 0;
                    while ((1 << lg) < lanes) ++lg;
                    const int vec_ok = aligned16(val) && aligned16(col);
                    const int64_t rows_per_block = kRowsThreads / lanes;
                    int64_t grid = ceil_div(A->n_rows, rows_per_block);
                    if (plan->grid_blocks > 0 && grid > plan->grid_blocks) grid = plan->grid_blocks;
                    if (grid > 0x7fffffffLL) grid = 0x7fffffffLL;
                    const int64_t thr = plan->comp_threshold > 0 ? plan->comp_threshold : 0;
                    const int overlap = (plan->flags & FSB_PLAN_OVERLAP_LAUNCH) && grid <= kOverlapMaxBlocks;
                    if (!overlap) {
                        k_spmv_rows<V, Ac, O, I, P><<<(unsigned)grid, kRowsThreads, 0, st>>>(
                            val, col, ptr, rmap, xv, yv, A->n_rows, plan->row_cap, thr, lg, vec_ok, 0);
                        return fsb_host::check_launch("k_spmv_rows");
                    }
                    cudaLaunchConfig_t cfg = {};
                    cfg.gridDim = dim3((unsigned)grid);
                    cfg.blockDim = dim3(kRowsThreads);
                    cfg.stream = st;
                    cudaLaunchAttribute attr[1];
                    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
                    attr[0].val.programmaticStreamSerializationAllowed = 1;
                    cfg.attrs = attr;
                    cfg.numAttrs = 1;
                    const int64_t nr = A->n_rows, rc_cap = plan->row_cap;
                    const cudaError_t e = cudaLaunchKernelEx(&cfg, k_spmv_rows<V, Ac, O, I, P>, val, col, ptr, rmap,
                                                             xv, yv, nr, rc_cap, thr, lg, vec_ok, 1);
                    if (e != cudaSuccess) {
                        fsb_host::set_error("k_spmv_rows (overlapped launch): %s", cudaGetErrorString(e));
                        return FSB_ERR_LAUNCH;
                    }
                    return fsb_host::check_launch("k_spmv_rows");
                }
                if (plan->algo != FSB_ALGO_MERGE) {
                    fsb_host::set_error("fsb_spmv_csr: unknown algo %d", plan->algo);
                    return FSB_ERR_INVALID;
                }
                const int ipt = plan->items_per_unit / kMergeThreads;
                if (plan->items_per_unit % kMergeThreads || ipt < 1 || ipt > kMergeMaxItemsPerThread) {
                    fsb_host::set_error("fsb_spmv_csr: items_per_unit=%d must be %d x [1, %d]", plan->items_per_unit,
                                        kMergeThreads, kMergeMaxItemsPerThread);
                    return FSB_ERR_INVALID;
                }
                const int64_t n_units = plan->n_units;
                if (n_units != ceil_div(A->n_rows + A->nnz, plan->items_per_unit) || !plan->unit_coords) {
                    fsb_host::set_error("fsb_spmv_csr: merge plan does not match the matrix");
                    return FSB_ERR_INVALID;
                }
                if (plan->row_cap > 0) {
                    fsb_host::set_error("fsb_spmv_csr: row_cap needs the rows algorithm");
                    return FSB_ERR_INVALID;
                }
                const int64_t need = merge_scratch_bytes(n_units, 1, (int)sizeof(Ac));
                if (!workspace || workspace_bytes < need) {
                    fsb_host::set_error("fsb_spmv_csr: workspace %lld bytes < %lld", (long long)workspace_bytes,
                                        (long long)need);
                    return FSB_ERR_WORKSPACE;
                }
                MergeScratch ms = merge_scratch_carve(workspace, n_units, 1, (int)sizeof(Ac));
                if (n_units > 0x7fffffffLL) {
                    fsb_host::set_error("fsb_spmv_csr: too many merge tiles");
                    return FSB_ERR_LIMIT;
                }
                k_spmv_merge<V, Ac, O, I, P><<<(unsigned)n_units, kMergeThreads, 0, st>>>(
                    val, col, ptr, rmap, xv, yv, A->n_rows, plan->unit_coords, ipt, ms.carry_row,
                    static_cast<Ac*>(ms.carry_val), static_cast<Ac*>(ms.head_val));
                int rc = fsb_host::check_launch("k_spmv_merge");
                if (rc) return rc;
                k_spmv_merge_fixup<Ac, O, I, P><<<(unsigned)ceil_div(n_units, 256), 256, 0, st>>>(
                    ms.carry_row, static_cast<const Ac*>(ms.carry_val), static_cast<const Ac*>(ms.head_val),
                    n_units, ptr, rmap, yv);
                return fsb_host::check_launch("k_spmv_merge_fixup");
            });
        });
    });
}

// ------------------------------------------------------ one-shot SpMV ----
// fsb_spmv_csr_checked: structural check, one device->host read of its
// figures, the heuristic plan from them, the product -- one host call.

namespace {
int64_t check_bytes(const fsb_csr* A) { return align_up(fsb_csr_check_workspace_bytes(A->n_rows, A->nnz), 256); }

// Row-group width / merge-path choice from the check's figures: merge path
// for skewed rows that are short on average, else 2 * mean / (16-byte vector
// elements) lanes rounded to a power of two in [2, 32] (ties to even).
void checked_plan(const fsb_csr* A, const int64_t* fig, fsb_plan* plan) {
    memset(plan, 0, sizeof(*plan));
    const int esz = elem_size(A->value_dtype);
    const int vec = esz >= 16 ? 1 : 16 / esz;
    const double mean = A->n_rows ? (double)A->nnz / (double)A->n_rows : 0.0;
    const bool skewed = (double)fig[5] > 8.0 * (mean > 1.0 ? mean : 1.0) + 256.0;
    if (A->n_rows > 0 && skewed && mean < 32.0) {
        plan->algo = FSB_ALGO_MERGE;
        plan->items_per_unit = kMergeThreads * (esz <= 4 ? 8 : 4);
        plan->n_units = ceil_div(A->n_rows + A->nnz, plan->items_per_unit);
        return;
    }
    double v = A->n_rows ? 2.0 * mean / vec : 32.0;
    if (v < 1.0) v = 1.0;
    int lanes = 1 << (int)std::nearbyint(std::log2(v));
    plan->algo = FSB_ALGO_ROWS;
    plan->lanes = lanes < 2 ? 2 : (lanes > 32 ? 32 : lanes);
    plan->flags = FSB_PLAN_OVERLAP_LAUNCH;
}

int64_t checked_merge_bytes(const fsb_csr* A, int acc_mode, int out_dtype) {
    fsb_plan mp;
    memset(&mp, 0, sizeof(mp));
    mp.algo = FSB_ALGO_MERGE;
    mp.items_per_unit = kMergeThreads * (elem_size(A->value_dtype) <= 4 ? 8 : 4);
    mp.n_units = ceil_div(A->n_rows + A->nnz, mp.items_per_unit);
    const int64_t coords = align_up((mp.n_units + 1) * 2 * (int64_t)sizeof(int64_t), 256);
    return coords + fsb_workspace_bytes(0, A, 1, acc_mode, out_dtype, &mp);
}
}  // namespace

extern "C" int64_t fsb_spmv_csr_checked_workspace_bytes(const fsb_csr* A, int acc_mode, int out_dtype) {
    if (!A || A->n_rows < 0 || A->nnz < 0) return 0;
    return check_bytes(A) + checked_merge_bytes(A, acc_mode, out_dtype);
}

extern "C" int fsb_spmv_csr_checked(const fsb_csr* A, const void* x, void* y, int out_dtype, int acc_mode,
                                    void* workspace, int64_t workspace_bytes, int64_t* figures, fsb_plan* plan_out,
                                    void* stream) {
    if (!A || !figures || A->n_rows < 0 || A->nnz < 0) {
        fsb_host::set_error("fsb_spmv_csr_checked: bad arguments");
        return FSB_ERR_INVALID;
    }
    const int64_t need = fsb_spmv_csr_checked_workspace_bytes(A, acc_mode, out_dtype);
    if (!workspace || workspace_bytes < need) {
        fsb_host::set_error("fsb_spmv_csr_checked: workspace %lld bytes < %lld", (long long)workspace_bytes,
                            (long long)need);
        return FSB_ERR_WORKSPACE;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the check's kernels write the figures straight into a pinned buffer of
    // this host thread: no copy-engine work to queue behind uploads
    static thread_local int64_t* staged = nullptr;
    if (!staged && cudaHostAlloc(reinterpret_cast<void**>(&staged), 8 * sizeof(int64_t),
                                 cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) {
        staged = nullptr;
        return fsb_host::check_launch("fsb_spmv_csr_checked: pinned figure buffer");
    }
    const int64_t cb = check_bytes(A);
    int rc = fsb_csr_check(A->row_ptr, A->ptr_dtype, A->n_rows, A->col_idx, A->index_dtype, A->nnz, staged,
                           workspace, cb, stream);
    if (rc) return rc;
    if (cudaStreamSynchronize(st) != cudaSuccess) return fsb_host::check_launch("fsb_spmv_csr_checked: check");
    memcpy(figures, staged, 8 * sizeof(int64_t));
    if (figures[0] != 0 || figures[1] != A->nnz || figures[2] != 0 ||
        (A->nnz > 0 && (figures[3] != 0 || figures[4] >= A->n_cols))) {
        fsb_host::set_error("fsb_spmv_csr_checked: malformed CSR structure (figures returned)");
        return FSB_ERR_INVALID;
    }
    fsb_plan plan;
    checked_plan(A, figures, &plan);
    if (plan_out) *plan_out = plan;
    if (A->n_rows == 0) return FSB_OK;
    char* rest = static_cast<char*>(workspace) + cb;
    int64_t rest_bytes = workspace_bytes - cb;
    if (plan.algo == FSB_ALGO_MERGE) {
        int64_t* coords = reinterpret_cast<int64_t*>(rest);
        const int64_t cb = align_up((plan.n_units + 1) * 2 * (int64_t)sizeof(int64_t), 256);
        rc = fsb_merge_partition(A->row_ptr, A->ptr_dtype, A->n_rows, A->nnz, plan.items_per_unit, 0, coords,
                                 plan.n_units, stream);
        if (rc) return rc;
        plan.unit_coords = coords;
        rest += cb;
        rest_bytes -= cb;
    }
    return fsb_spmv_csr(A, x, y, out_dtype, acc_mode, &plan, rest, rest_bytes, stream);
}

// --------------------------------------------------- allocation-free SpMV ----
// fsb_spmv_csr_noalloc: the merge-path SpMV for callers that cannot allocate
// device memory -- a C program or plug-in that receives device pointers from
// a host framework owning all device memory, or a latency-critical loop in
// which cudaMalloc's implicit device-wide synchronisation is not acceptable.
// The caller still passes the matrix, x and y; the scratch this algorithm
// needs (merge-path tile coordinates and per-tile carries) lives in the
// file-scope device array below, of a fixed size, held by every GPU that loads
// this library until the process exits.
//
// Limit: at most kNoAllocMaxTiles merge-path tiles, i.e.
// n_rows + nnz <= kNoAllocMaxTiles * items_per_unit (16384 tiles: 16.7 M path
// items at 1024 items per tile); larger matrices are rejected with
// FSB_ERR_LIMIT.  Every call on a device shares the one array: two calls whose
// kernels overlap on the GPU (for example on two streams) race on it, so
// callers must order such calls.  Nothing in the array has to start at zero:
// each call writes the coordinates and every tile's carry slot before they
// are read.  The first call in a CUDA context (the device's primary context,
// or a host framework's own context current on the calling thread) resolves
// the array's device address in that context (cudaGetSymbolAddress) and
// caches it per context; that first call should come before any stream
// capture.
constexpr int64_t kNoAllocMaxTiles = 16384;
constexpr int64_t kNoAllocCoordBytes = ((kNoAllocMaxTiles + 1) * 2 * 8 + 255) / 256 * 256;
constexpr int64_t kNoAllocBytes = kNoAllocCoordBytes + (kNoAllocMaxTiles * 8 + 255) / 256 * 256 +
                                  2 * ((kNoAllocMaxTiles * 16 + 255) / 256 * 256);
static __device__ __align__(256) unsigned char g_spmv_noalloc_scratch[kNoAllocBytes];

namespace {
// The array's device address belongs to the CUDA context that was current
// when it was resolved: a plug-in may run inside its host framework's own
// driver context rather than the device's primary context.  Addresses are
// therefore cached per context (cuCtxGetCurrent, reached through the
// runtime's driver entry-point query), not per device ordinal.
using CtxGetCurrentFn = int (*)(void**);
constexpr int kMaxContexts = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_ctx[kMaxContexts] = {};
void* g_noalloc_ptr[kMaxContexts] = {};
int g_noalloc_used = 0;

CtxGetCurrentFn ctx_get_current() {
    static std::once_flag once;
    static CtxGetCurrentFn fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(p);
    });
    return fn;
}

// Device address of the scratch array in the current context (resolved on
// the first call made in that context).
int noalloc_scratch(void** out) {
    CtxGetCurrentFn get_ctx = ctx_get_current();
    if (!get_ctx) {
        fsb_host::set_error("fsb_spmv_csr_noalloc: cuCtxGetCurrent is not available");
        return FSB_ERR_LAUNCH;
    }
    void* ctx = nullptr;
    if (get_ctx(&ctx) != 0) ctx = nullptr;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (ctx) {
        for (int i = 0; i < g_noalloc_used; ++i) {
            if (g_noalloc_ctx[i] == ctx) {
                *out = g_noalloc_ptr[i];
                return FSB_OK;
            }
        }
    }
    // First call in this context (or no context current yet: the runtime
    // then makes the current device's primary context current here).
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_spmv_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        fsb_host::set_error("fsb_spmv_csr_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        return FSB_ERR_LAUNCH;
    }
    if (!ctx && (get_ctx(&ctx) != 0 || !ctx)) {
        fsb_host::set_error("fsb_spmv_csr_noalloc: no current CUDA context");
        return FSB_ERR_LAUNCH;
    }
    if (g_noalloc_used < kMaxContexts) {
        g_noalloc_ctx[g_noalloc_used] = ctx;
        g_noalloc_ptr[g_noalloc_used] = p;
        ++g_noalloc_used;
    }
    *out = p;
    return FSB_OK;
}
}  // namespace

extern "C" int fsb_spmv_csr_noalloc(const fsb_csr* A, const void* x, void* y, int out_dtype, int acc_mode,
                                    int32_t items_per_unit, void* stream) {
    if (!A) {
        fsb_host::set_error("fsb_spmv_csr_noalloc: null matrix");
        return FSB_ERR_INVALID;
    }
    if (A->n_rows < 0 || A->nnz < 0) {
        fsb_host::set_error("fsb_spmv_csr_noalloc: negative size");
        return FSB_ERR_INVALID;
    }
    if (items_per_unit % kMergeThreads || items_per_unit < kMergeThreads || items_per_unit > kMergeMaxTile) {
        fsb_host::set_error("fsb_spmv_csr_noalloc: items_per_unit=%d must be %d x [1, %d]", items_per_unit,
                            kMergeThreads, kMergeMaxItemsPerThread);
        return FSB_ERR_INVALID;
    }
    if (A->n_rows == 0) return FSB_OK;
    const int64_t n_tiles = ceil_div(A->n_rows + A->nnz, items_per_unit);
    if (n_tiles > kNoAllocMaxTiles) {
        fsb_host::set_error("fsb_spmv_csr_noalloc: %lld tiles exceed the fixed scratch of %lld tiles "
                            "(n_rows + nnz must be <= %lld at items_per_unit=%d)",
                            (long long)n_tiles, (long long)kNoAllocMaxTiles,
                            (long long)(kNoAllocMaxTiles * items_per_unit), items_per_unit);
        return FSB_ERR_LIMIT;
    }
    if (!A->row_ptr || !y || (A->nnz > 0 && (!A->values || !A->col_idx || !x))) {
        fsb_host::set_error("fsb_spmv_csr_noalloc: null data pointer");
        return FSB_ERR_INVALID;
    }
    if (A->row_map && A->row_map_dtype != A->index_dtype) {
        fsb_host::set_error("fsb_spmv_csr_noalloc: row_map dtype must equal index dtype");
        return FSB_ERR_INVALID;
    }
    void* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    int64_t* coords = static_cast<int64_t*>(scratch);
    void* carries = static_cast<unsigned char*>(scratch) + kNoAllocCoordBytes;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return dispatch_vao(A->value_dtype, acc_mode, out_dtype, [&](auto tv, auto ta, auto to) -> int {
        using V = typename decltype(tv)::type;
        using Ac = typename decltype(ta)::type;
        using O = typename decltype(to)::type;
        return dispatch_idx(A->index_dtype, [&](auto ti) -> int {
            using I = typename decltype(ti)::type;
            return dispatch_idx(A->ptr_dtype, [&](auto tp) -> int {
                using P = typename decltype(tp)::type;
                const P* ptr = static_cast<const P*>(A->row_ptr);
                k_merge_partition<P><<<(unsigned)ceil_div(n_tiles + 1, 256), 256, 0, st>>>(
                    ptr, A->n_rows, A->nnz, items_per_unit, 0, coords, n_tiles);
                int rc2 = fsb_host::check_launch("k_merge_partition (noalloc)");
                if (rc2) return rc2;
                MergeScratch ms = merge_scratch_carve(carries, n_tiles, 1, (int)sizeof(Ac));
                O* yv = static_cast<O*>(y);
                const I* rmap = static_cast<const I*>(A->row_map);
                k_spmv_merge<V, Ac, O, I, P><<<(unsigned)n_tiles, kMergeThreads, 0, st>>>(
                    static_cast<const V*>(A->values), static_cast<const I*>(A->col_idx), ptr, rmap,
                    static_cast<const V*>(x), yv, A->n_rows, coords, items_per_unit / kMergeThreads, ms.carry_row,
                    static_cast<Ac*>(ms.carry_val), static_cast<Ac*>(ms.head_val));
                rc2 = fsb_host::check_launch("k_spmv_merge (noalloc)");
                if (rc2) return rc2;
                k_spmv_merge_fixup<Ac, O, I, P><<<(unsigned)ceil_div(n_tiles, 256), 256, 0, st>>>(
                    ms.carry_row, static_cast<const Ac*>(ms.carry_val), static_cast<const Ac*>(ms.head_val),
                    n_tiles, ptr, rmap, yv);
                return fsb_host::check_launch("k_spmv_merge_fixup (noalloc)");
            });
        });
    });
}
