"""flagsparse_public_b200: FlagSparse's CSR/COO SpMV and SpMM on B200 (sm_100a).

The operator API is FlagSparse's (``flagsparse_spmv_csr``, ``prepare_spmv_csr``,
``flagsparse_spmm_csr(_opt)(_alg2)``, ``flagsparse_spmv_coo(_tocsr)``,
``flagsparse_spmm_coo`` and their ``Prepared*`` caches); the products run in
hand-written CUDA kernels for sm_100a behind the C ABI declared in
``include/flagsparse_b200.h`` (``libflagsparse_b200.so``, loaded with ctypes).

To use it where code imports ``flagsparse``::

    import sys, flagsparse_public_b200
    sys.modules["flagsparse"] = flagsparse_public_b200
    sys.modules["flagsparse.sparse_operations"] = flagsparse_public_b200.sparse_operations
"""

__version__ = "1.0.0"

_EXPORTS = {
    "PreparedCoo": "spmv_coo",
    "PreparedCsrSpmv": "spmv_csr",
    "PreparedCsrSpmmOpt": "spmm_csr",
    "PreparedCsrSpmmOptAlg2": "spmm_csr_opt_alg2",
    "prepare_spmv_csr": "spmv_csr",
    "prepare_spmm_csr_opt": "spmm_csr",
    "prepare_spmm_csr_opt_alg2": "spmm_csr_opt_alg2",
    "prepare_spmv_coo": "spmv_coo",
    "prepare_spmv_coo_tocsr": "spmv_csr",
    "flagsparse_spmv_csr": "spmv_csr",
    "flagsparse_spmv_coo": "spmv_coo",
    "flagsparse_spmv_coo_tocsr": "spmv_csr",
    "flagsparse_spmm_csr": "spmm_csr",
    "flagsparse_spmm_csr_opt": "spmm_csr",
    "flagsparse_spmm_csr_opt_alg2": "spmm_csr_opt_alg2",
    "flagsparse_spmm_coo": "spmm_coo",
    "SDDMMPrepared": "sddmm_csr",
    "prepare_sddmm_csr": "sddmm_csr",
    "flagsparse_sddmm_csr": "sddmm_csr",
    "PreparedCsrMixed": "precision",
    "prepare_csr_mixed": "precision",
    "flagsparse_spmv_csr_mixed": "precision",
    "flagsparse_spmm_csr_mixed": "precision",
    "benchmark_spmv_case": "benchmarks",
    "benchmark_spmm_case": "benchmarks",
    "benchmark_spmm_opt_case": "benchmarks",
    "benchmark_spmm_opt_alg2_case": "benchmarks",
    "benchmark_sddmm_case": "benchmarks",
}

__all__ = sorted(_EXPORTS)


def __getattr__(name):
    if name in _EXPORTS:
        import importlib

        mod = importlib.import_module(f".sparse_operations.{_EXPORTS[name]}", __name__)
        return getattr(mod, name)
    if name == "sparse_operations":
        import importlib

        return importlib.import_module(".sparse_operations", __name__)
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")


def __dir__():
    return sorted(list(globals()) + __all__)
