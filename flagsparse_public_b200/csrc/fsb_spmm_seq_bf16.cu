// Sequential-nonzero SpMM instantiations for __nv_bfloat16 values (see fsb_spmm_seq.cuh).
#include "fsb_spmm_seq.cuh"

namespace fsb {
FSB_SEQ_DECL(seq_dispatch_bf16) {
    return seq_dispatch_for<__nv_bfloat16>(A, B, ldb, n_dense, C, ldc, out_dtype, acc_mode, plan, workspace, workspace_bytes, st);
}
}  // namespace fsb
