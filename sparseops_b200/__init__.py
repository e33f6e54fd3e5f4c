"""SparseOps hot path on B200 (sm_100a): hand-written CUDA kernels behind a C ABI.

Host API mirrors the reference's SpOps.h names (SpOps_csr, csr_to_*, ...);
see spops.py.  The native library is libsparseops_b200.so in this directory.
"""
from ._lib import SpOpsError, lib  # noqa: F401
from .spops import (Batch, CSR_Matrix, Context, DeviceCSR, SpMM_csr, SpOps_csr, default_context,  # noqa: F401
                    spmv_host_async, spmv_host_wait)
from .formats import (BSR_Matrix, COO_Matrix, CSR5_Matrix, SpOps_csr5, csr_to_csr5, DIA_Matrix, ELL_Matrix, S_ELL_Matrix, SELL_C_R_Matrix,  # noqa: F401
                      SELL_C_Sigma_Matrix, SpOps_bsr, SpOps_coo, SpOps_dia, SpOps_ell, SpOps_sell, SpOps_sell_c_R,
                      SpOps_sell_c_sigma, SpOps_auto, convert_to, coo_to_csr, csr_to_bsr, matrix_features, matrix_tile_features, select_format, csr_to_coo, csr_to_dia, csr_to_ell, csr_to_sell,
                      csr_to_sell_c_R, csr_to_sell_c_sigma, read_coo_matrix, read_csr_matrix, csr_reorder_rows)

__all__ = ["read_coo_matrix", "read_csr_matrix", "csr_reorder_rows", "SpOpsError", "lib", "Batch", "SpMM_csr", "CSR_Matrix", "Context", "SpOps_csr", "default_context", "COO_Matrix",
           "ELL_Matrix", "S_ELL_Matrix", "SELL_C_Sigma_Matrix", "SELL_C_R_Matrix", "DIA_Matrix", "BSR_Matrix",
           "csr_to_coo", "csr_to_ell", "csr_to_sell", "csr_to_sell_c_sigma", "csr_to_sell_c_R", "csr_to_dia",
           "csr_to_bsr", "SpOps_coo", "SpOps_ell", "SpOps_sell", "SpOps_sell_c_sigma", "SpOps_sell_c_R",
           "SpOps_dia", "SpOps_bsr", "CSR5_Matrix", "csr_to_csr5", "SpOps_csr5", "coo_to_csr", "DeviceCSR",
           "matrix_features", "matrix_tile_features", "select_format", "convert_to", "SpOps_auto", "spmv_host_async",
           "spmv_host_wait"]
