// fsb_probe.cu -- the gather floor of an SpMM: how fast this GPU can deliver
// the B rows one CSR product must read, with nothing else done.
//
// A merge-path SpMM over a matrix with scattered columns gathers one B-row
// slice per nonzero; with B resident in L2 these gathers, not HBM bandwidth,
// set its speed limit.  k_gather_floor reads the same column-index stream and
// gathers the same B rows (full 16-byte lane vectors, L2 evict-last like the
// product kernels), adds them into per-lane sums and writes one float per
// thread: no row bookkeeping, no multiply by the values, no C rows.  Its time
// on a matrix is the floor the product kernels are measured against.
//
// Warps take chunks of NPAR * U consecutive nonzeros (NPAR = 32 / LPN
// sub-groups, U gathers per lane), a persistent grid striding over the chunks;
// the next chunk's column indices are loaded while the current chunk's rows
// are in flight.  Variants trade gathers per lane against resident warps.
#include "fsb_dispatch.cuh"

namespace fsb {

template <int LPN_LOG2, int U, int MINB>
__global__ void __launch_bounds__(128, MINB)
k_gather_floor(const int32_t* __restrict__ col, int64_t nnz, const float* __restrict__ B, int64_t ldb,
               float* __restrict__ out) {
    constexpr int NPAR = 32 >> LPN_LOG2;
    constexpr int CH = NPAR * U;  // nonzeros per chunk
    const int lane = threadIdx.x & 31;
    const int sub = lane >> LPN_LOG2;
    const int gl = lane & ((1 << LPN_LOG2) - 1);
    const int64_t warp = (int64_t)blockIdx.x * 4 + (threadIdx.x >> 5);
    const int64_t stride = (int64_t)gridDim.x * 4 * CH;
    const float* Bl = B + gl * 4;
    const uint64_t pol = policy_evict_last();
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
    int64_t base = warp * CH;
    int cn[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int64_t i = base + u * NPAR + sub;
        cn[u] = i < nnz ? __ldcs(col + i) : -1;
    }
    while (base < nnz) {
        int cc[U];
#pragma unroll
        for (int u = 0; u < U; ++u) cc[u] = cn[u];
        base += stride;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t i = base + u * NPAR + sub;
            cn[u] = i < nnz ? __ldcs(col + i) : -1;
        }
        vec_t<float, 4> v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (cc[u] >= 0) {
                v[u] = ld_keep<float, 4>(Bl + (int64_t)cc[u] * ldb, pol);
            } else {
                v[u].v[0] = v[u].v[1] = v[u].v[2] = v[u].v[3] = 0.f;
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            s0 += v[u].v[0];
            s1 += v[u].v[1];
            s2 += v[u].v[2];
            s3 += v[u].v[3];
        }
    }
    out[(int64_t)blockIdx.x * 128 + threadIdx.x] = (s0 + s1) + (s2 + s3);
}

namespace {

template <int LPN_LOG2, int U, int MINB>
int launch_floor(const int32_t* col, int64_t nnz, const float* B, int64_t ldb, float* out, int64_t out_len,
                 int sms, cudaStream_t st) {
    const int64_t grid = (int64_t)sms * MINB;
    if (out_len < grid * 128) {
        fsb_host::set_error("fsb_gather_floor: out holds %lld floats, %lld needed", (long long)out_len,
                            (long long)(grid * 128));
        return FSB_ERR_INVALID;
    }
    k_gather_floor<LPN_LOG2, U, MINB><<<(unsigned)grid, 128, 0, st>>>(col, nnz, B, ldb, out);
    return fsb_host::check_launch("k_gather_floor");
}

template <int LPN_LOG2>
int floor_variant(int variant, const int32_t* col, int64_t nnz, const float* B, int64_t ldb, float* out,
                  int64_t out_len, int sms, cudaStream_t st) {
    switch (variant) {
        case 0: return launch_floor<LPN_LOG2, 4, 16>(col, nnz, B, ldb, out, out_len, sms, st);
        case 1: return launch_floor<LPN_LOG2, 8, 8>(col, nnz, B, ldb, out, out_len, sms, st);
        case 2: return launch_floor<LPN_LOG2, 16, 4>(col, nnz, B, ldb, out, out_len, sms, st);
        case 3: return launch_floor<LPN_LOG2, 6, 12>(col, nnz, B, ldb, out, out_len, sms, st);
        default: break;
    }
    fsb_host::set_error("fsb_gather_floor: variant %d not in [0, %d)", variant, FSB_GATHER_FLOOR_VARIANTS);
    return FSB_ERR_INVALID;
}

}  // namespace
}  // namespace fsb

extern "C" int fsb_gather_floor(const int32_t* col_idx, int64_t nnz, const float* B, int64_t ldb, int64_t n_dense,
                                float* out, int64_t out_len, int variant, void* stream) {
    using namespace fsb;
    if (nnz < 0 || (nnz > 0 && (!col_idx || !B)) || !out) {
        fsb_host::set_error("fsb_gather_floor: null pointer or negative size");
        return FSB_ERR_INVALID;
    }
    if ((n_dense != 32 && n_dense != 64 && n_dense != 128) || ldb < n_dense || ldb % 4 ||
        reinterpret_cast<uintptr_t>(B) % 16) {
        fsb_host::set_error("fsb_gather_floor: n_dense must be 32, 64 or 128 with 16-byte aligned B rows");
        return FSB_ERR_UNSUPPORTED;
    }
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                  cudaSuccess) {
        fsb_host::set_error("fsb_gather_floor: cannot read the SM count");
        return FSB_ERR_LAUNCH;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n_dense == 32) return floor_variant<3>(variant, col_idx, nnz, B, ldb, out, out_len, sms, st);
    if (n_dense == 64) return floor_variant<4>(variant, col_idx, nnz, B, ldb, out, out_len, sms, st);
    return floor_variant<5>(variant, col_idx, nnz, B, ldb, out, out_len, sms, st);
}
