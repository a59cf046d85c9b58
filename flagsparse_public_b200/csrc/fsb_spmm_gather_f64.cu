// Gather SpMM instantiations for double values (see fsb_spmm_gather.cuh).
#include "fsb_spmm_gather.cuh"

namespace fsb {
FSB_GATHER_DECL(gather_dispatch_f64) {
    return gather_dispatch_for<double>(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes,
                                     st, err_word);
}
}  // namespace fsb
