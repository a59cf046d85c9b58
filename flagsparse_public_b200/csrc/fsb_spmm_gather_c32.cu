// Gather SpMM instantiations for c32_t (complex32) values (see fsb_spmm_gather.cuh).
#include "fsb_spmm_gather.cuh"

namespace fsb {
FSB_GATHER_DECL(gather_dispatch_c32) {
    return gather_dispatch_for<c32_t>(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes,
                                     st, err_word);
}
}  // namespace fsb
