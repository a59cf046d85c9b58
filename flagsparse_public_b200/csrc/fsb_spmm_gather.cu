// fsb_spmm_gather.cu -- entry of the gather SpMM (FSB_ALGO_GATHER): value-type
// dispatch to the per-type instantiation files, the device error word of the
// bounded waits, and the wait self-test.
#include <mutex>

#include "fsb_spmm_gather.cuh"

namespace fsb {

__device__ int g_gather_error = 0;

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_err_mutex;
int* g_err_ptr[kMaxDevices] = {};
}  // namespace

// Device address of the error word for the current device (resolved once).
int* gather_error_word() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lock(g_err_mutex);
    if (!g_err_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_gather_error) != cudaSuccess) return nullptr;
        g_err_ptr[dev] = static_cast<int*>(p);
    }
    return g_err_ptr[dev];
}

int spmm_gather_dispatch(const fsb_csr* A, const void* B, int64_t ldb, int64_t n_dense, void* C, int64_t ldc,
                         int out_dtype, int acc_mode, const fsb_plan* plan, void* workspace, int64_t workspace_bytes,
                         cudaStream_t st) {
    int* err = gather_error_word();
    if (!err) {
        fsb_host::set_error("fsb_spmm_csr: cannot resolve the device error word");
        return FSB_ERR_LAUNCH;
    }
    switch (A->value_dtype) {
    case FSB_F16: return gather_dispatch_f16(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st, err);
    case FSB_BF16: return gather_dispatch_bf16(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st, err);
    case FSB_F32: return gather_dispatch_f32(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st, err);
    case FSB_F64: return gather_dispatch_f64(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st, err);
    case FSB_C32: return gather_dispatch_c32(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st, err);
    case FSB_C64: return gather_dispatch_c64(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st, err);
    case FSB_C128: return gather_dispatch_c128(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st, err);
    default:
        fsb_host::set_error("fsb_spmm_csr: value dtype code %d", A->value_dtype);
        return FSB_ERR_UNSUPPORTED;
    }
}

}  // namespace fsb

namespace fsb {
// Waits on an mbarrier that nothing arrives on; the bounded wait must give
// up after limit_ns and record FSB_ERR_TIMEOUT.
__global__ void k_selftest_wait_timeout(unsigned long long limit_ns) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(smem_u32(&bar), 1);
        fence_mbarrier_init();
    }
    __syncwarp();
    if (!mbar_wait(smem_u32(&bar), 0, limit_ns) && threadIdx.x == 0) atomicExch(&g_gather_error, FSB_ERR_TIMEOUT);
}
}  // namespace fsb

extern "C" int fsb_selftest_wait_timeout(int64_t limit_ns, void* stream) {
    if (limit_ns <= 0 || limit_ns > 2000000000LL) {
        fsb_host::set_error("fsb_selftest_wait_timeout: limit must be in (0, 2 s]");
        return FSB_ERR_INVALID;
    }
    fsb::k_selftest_wait_timeout<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>((unsigned long long)limit_ns);
    return fsb_host::check_launch("k_selftest_wait_timeout");
}

extern "C" int fsb_device_error(int* status_out, int reset) {
    int v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, fsb::g_gather_error, sizeof(int));
    if (e != cudaSuccess) {
        fsb_host::set_error("fsb_device_error: %s", cudaGetErrorString(e));
        return FSB_ERR_LAUNCH;
    }
    if (status_out) *status_out = v;
    if (reset) {
        const int zero = 0;
        e = cudaMemcpyToSymbol(fsb::g_gather_error, &zero, sizeof(int));
        if (e != cudaSuccess) {
            fsb_host::set_error("fsb_device_error: %s", cudaGetErrorString(e));
            return FSB_ERR_LAUNCH;
        }
    }
    return FSB_OK;
}
