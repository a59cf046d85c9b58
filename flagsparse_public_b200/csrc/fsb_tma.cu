// fsb_tma.cu -- host side of the TMA-staged kernels: the driver's tensor-map
// encoder (resolved once through the runtime) and the tensor map of the
// gather4 SpMM.
#include <mutex>

#include "fsb_tma.cuh"

namespace fsb {
namespace tma {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

}  // namespace tma

bool encode_g4_map(CUtensorMap* map, int value_dtype, const void* B, int64_t n_rows_b, int64_t ldb, int64_t n_dense,
                   int tw) {
    auto fn = tma::encode_fn();
    if (!fn || n_rows_b < 1 || n_dense < 1 || tw < 1 || tw > 256) return false;
    CUtensorMapDataType dt;
    int es;
    switch (value_dtype) {
        case FSB_F32: dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT32; es = 4; break;
        case FSB_F16: dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT16; es = 2; break;
        case FSB_BF16: dt = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16; es = 2; break;
        default: return false;
    }
    if ((tw * es) % 16 != 0) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)n_dense, (cuuint64_t)n_rows_b};
    const cuuint64_t strides[1] = {(cuuint64_t)(ldb * es)};
    const cuuint32_t box[2] = {(cuuint32_t)tw, 1};  // gather4 boxes are one row high
    const cuuint32_t estr[2] = {1, 1};
    const CUresult rc = fn(map, dt, 2, const_cast<void*>(B), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return rc == CUDA_SUCCESS;
}

}  // namespace fsb
