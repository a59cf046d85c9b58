"""SpMV / SpMM operators with FlagSparse's ``sparse_operations`` interface.

Re-exports the hot-path names of FlagSparse ``sparse_operations/__init__.py``
(:29-54): CSR/COO SpMV, CSR SpMM (ALG1, opt, opt-alg2) and COO SpMM, and the
benchmark entry points of that path.
"""

from .spmv_csr import (
    PreparedCsrSpmv,
    flagsparse_spmv_coo_tocsr,
    flagsparse_spmv_csr,
    prepare_spmv_coo_tocsr,
    prepare_spmv_csr,
)
from .spmv_coo import PreparedCoo, flagsparse_spmv_coo, prepare_spmv_coo
from .spmm_csr import PreparedCsrSpmmOpt, flagsparse_spmm_csr, flagsparse_spmm_csr_opt, prepare_spmm_csr_opt
from .spmm_csr_opt_alg2 import PreparedCsrSpmmOptAlg2, flagsparse_spmm_csr_opt_alg2, prepare_spmm_csr_opt_alg2
from .spmm_coo import flagsparse_spmm_coo
from .benchmarks import (
    benchmark_sddmm_case,
    benchmark_spmm_case,
    benchmark_spmm_opt_alg2_case,
    benchmark_spmm_opt_case,
    benchmark_spmv_case,
)

__all__ = [
    "benchmark_sddmm_case",
    "benchmark_spmm_case",
    "benchmark_spmm_opt_alg2_case",
    "benchmark_spmm_opt_case",
    "benchmark_spmv_case",
    "PreparedCoo",
    "PreparedCsrSpmv",
    "PreparedCsrSpmmOpt",
    "PreparedCsrSpmmOptAlg2",
    "flagsparse_spmm_coo",
    "flagsparse_spmm_csr",
    "flagsparse_spmm_csr_opt",
    "flagsparse_spmm_csr_opt_alg2",
    "flagsparse_spmv_coo",
    "flagsparse_spmv_coo_tocsr",
    "flagsparse_spmv_csr",
    "prepare_spmm_csr_opt",
    "prepare_spmm_csr_opt_alg2",
    "prepare_spmv_coo",
    "prepare_spmv_coo_tocsr",
    "prepare_spmv_csr",
]
