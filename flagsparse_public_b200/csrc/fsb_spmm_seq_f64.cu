// Sequential-nonzero SpMM instantiations for double values (see fsb_spmm_seq.cuh).
#include "fsb_spmm_seq.cuh"

namespace fsb {
FSB_SEQ_DECL(seq_dispatch_f64) {
    return seq_dispatch_for<double>(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st);
}
}  // namespace fsb
