// fsb_tma.cuh -- shared-memory mbarrier and Tensor Memory Accelerator helpers
// of the kernels that stage operands with cp.async.bulk.tensor (the BSR
// tensor-core kernel and the gather4 SpMM).
//
// Every wait is bounded: mbar_wait gives up after kWaitNs of globaltimer and
// returns false, the caller records FSB_ERR_TIMEOUT in the device error word
// and drains its copies in flight before returning.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

#include "fsb_dispatch.cuh"

namespace fsb {
namespace tma {

constexpr unsigned long long kWaitNs = 1000000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// One arrival that also expects tx bytes of asynchronous copies.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t tx) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(tx) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(20000u)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase of the given parity; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    if (mbar_test(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    while (!mbar_test(bar, parity))
        if (now_ns() - t0 > kWaitNs) return false;
    return true;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (resolved
// once; nullptr when the driver does not provide it).  fsb_tma.cu.
PFN_cuTensorMapEncodeTiled_v12000 encode_fn();

}  // namespace tma

// 2-D tensor map over B (columns innermost) with one-row boxes of tw columns,
// no swizzle, zero fill outside the matrix: the map tile::gather4 reads.
// False when it cannot be encoded.  fsb_tma.cu.
bool encode_g4_map(CUtensorMap* map, int value_dtype, const void* B, int64_t n_rows_b, int64_t ldb, int64_t n_dense,
                   int tw);

}  // namespace fsb
