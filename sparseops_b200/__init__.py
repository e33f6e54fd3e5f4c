"""SparseOps hot path on B200 (sm_100a): hand-written CUDA kernels behind a C ABI.

Host API mirrors the reference's SpOps.h names (SpOps_csr, csr_to_*, ...);
see spops.py.  The native library is libsparseops_b200.so in this directory.
"""
from ._lib import SpOpsError, lib  # noqa: F401
from .spops import CSR_Matrix, Context, SpOps_csr, default_context  # noqa: F401

__all__ = ["SpOpsError", "lib", "CSR_Matrix", "Context", "SpOps_csr", "default_context"]
