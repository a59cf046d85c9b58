// Gather SpMM instantiations for __nv_bfloat16 values (see fsb_spmm_gather.cuh).
#include "fsb_spmm_gather.cuh"

namespace fsb {
FSB_GATHER_DECL(gather_dispatch_bf16) {
    return gather_dispatch_for<__nv_bfloat16>(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes,
                                     st, err_word);
}
}  // namespace fsb
