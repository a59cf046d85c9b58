// Sequential-nonzero SpMM instantiations for c32_t (complex32) values (see fsb_spmm_seq.cuh).
#include "fsb_spmm_seq.cuh"

namespace fsb {
FSB_SEQ_DECL(seq_dispatch_c32) {
    return seq_dispatch_for<c32_t>(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st);
}
}  // namespace fsb
