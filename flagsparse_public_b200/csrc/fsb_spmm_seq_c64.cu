// Sequential-nonzero SpMM instantiations for c64_t values (see fsb_spmm_seq.cuh).
#include "fsb_spmm_seq.cuh"

namespace fsb {
FSB_SEQ_DECL(seq_dispatch_c64) {
    return seq_dispatch_for<c64_t>(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st);
}
}  // namespace fsb
