"""ctypes binding of libsparseops_b200.so (the C ABI in include/sparseops_b200.h).

The product path has no fallback: if the shared library is missing or does
not load, every entry point raises.  Build it with
``python -m sparseops_b200.build`` (``__graft_entry__.build()``).
"""
from __future__ import annotations

import atexit
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsparseops_b200.so")

i64, i32, u64, dbl, vp = C.c_int64, C.c_int32, C.c_uint64, C.c_double, C.c_void_p


class SpOpsError(RuntimeError):
    """A C ABI call returned a status other than SPOPS_OK."""

    def __init__(self, status: int, func: str, msg: str):
        self.status = status
        super().__init__(f"{func} -> {STATUS_NAMES.get(status, status)}: {msg}")


STATUS_NAMES = {0: "SPOPS_OK", 1: "SPOPS_ERR_INVALID", 2: "SPOPS_ERR_UNSUPPORTED", 3: "SPOPS_ERR_ALLOC",
                4: "SPOPS_ERR_CUDA", 5: "SPOPS_ERR_TOO_LARGE", 6: "SPOPS_ERR_TIMEOUT"}

INDEX = {"i32": 0, "i64": 1}
VALUE = {"f32": 0, "f64": 1}
FORMATS = {"csr": 0, "coo": 1, "ell": 2, "sell": 3, "sell_c_sigma": 4, "sell_c_R": 5, "dia": 6, "bsr": 7,
           "csr5": 8}


class MatrixInfo(C.Structure):
    _fields_ = [("rows", i64), ("cols", i64), ("nnz", i64), ("format", i32), ("index_type", i32),
                ("value_type", i32), ("layout", i32), ("sigma", i64), ("chunk", i64), ("alignment", i64),
                ("extra", i64 * 8)]


class SpgemmStats(C.Structure):
    _fields_ = [("flops", i64), ("clusters", i64), ("dense_clusters", i64), ("pairs", i64),
                ("cluster_columns", i64), ("c_cluster_columns", i64), ("minhash_ms", dbl), ("lsh_ms", dbl),
                ("hc_ms", dbl), ("cluster_ms", dbl), ("symbolic_ms", dbl), ("numeric_ms", dbl), ("to_csr_ms", dbl)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class FormatParams(C.Structure):
    _fields_ = [("sigma", i64), ("chunk", i64), ("alignment", i64), ("max_diags", i64), ("block_rows", i64),
                ("block_cols", i64), ("layout", i32), ("reserved", i32)]


FEATURE_NAMES = ("rows", "cols", "nnz", "nnz_lower", "nnz_upper", "nnz_diagonal", "ndiags", "min_nnz_row",
                 "max_nnz_row", "min_nnz_col", "max_nnz_col", "nnz_ratio", "diag_close_ratio", "pattern_symm",
                 "value_symm", "nz_row_ratio", "ave_nnz_row", "var_nnz_row", "std_nnz_row", "p_ratio_row",
                 "gini_row", "nz_col_ratio", "ave_nnz_col", "var_nnz_col", "std_nnz_col", "p_ratio_col",
                 "gini_col", "diagonal_dominant_ratio", "max_value_offdiag", "max_value_diagonal",
                 "row_variability", "col_variability")


class Features(C.Structure):
    _fields_ = [(n, i64) for n in FEATURE_NAMES[:11]] + [(n, C.c_double) for n in FEATURE_NAMES[11:]]

    def as_dict(self):
        return {n: getattr(self, n) for n in FEATURE_NAMES}


TILE_FEATURE_NAMES = ("num_blocks", "rows_per_block", "rows_mod", "cols_per_block", "cols_mod", "min_nnz_tile",
                      "max_nnz_tile", "min_nnz_rb", "max_nnz_rb", "min_nnz_cb", "max_nnz_cb", "nz_ratio_tiles",
                      "ave_nnz_tile", "var_nnz_tile", "std_nnz_tile", "p_ratio_tiles", "gini_tiles", "nz_ratio_rb",
                      "ave_nnz_rb", "var_nnz_rb", "std_nnz_rb", "p_ratio_rb", "gini_rb", "nz_ratio_cb",
                      "ave_nnz_cb", "var_nnz_cb", "std_nnz_cb", "p_ratio_cb", "gini_cb", "uniq_r", "uniq_c",
                      "pot_reuse_r", "pot_reuse_c", "distance_per_row")


class TileFeatures(C.Structure):
    _fields_ = [(n, i64) for n in TILE_FEATURE_NAMES[:11]] + [(n, C.c_double) for n in TILE_FEATURE_NAMES[11:]]

    def as_dict(self):
        return {n: getattr(self, n) for n in TILE_FEATURE_NAMES}


# spops_tile_maps_t: (name, per tile?, integer?)
TILE_MAP_FIELDS = (("tile_nnz", True, True), ("tile_rows", True, True), ("tile_cols", True, True),
                   ("tile_max_row_nnz", True, True), ("tile_ave_row_nnz", True, False),
                   ("tile_std_row_nnz", True, False), ("rb_nnz", False, True), ("rb_max_row_nnz", False, True),
                   ("rb_ave_row_nnz", False, False), ("rb_std_row_nnz", False, False), ("cb_nnz", False, True),
                   ("cb_max_col_nnz", False, True), ("cb_ave_col_nnz", False, False),
                   ("cb_std_col_nnz", False, False))


class TileMaps(C.Structure):
    _fields_ = [(n, vp) for n, _, _ in TILE_MAP_FIELDS]


# name -> argtypes (restype is spops_status_t unless listed in _RESTYPE)
_SIGS = {
    "spops_create": [vp, C.c_int, vp],
    "spops_destroy": [vp],
    "spops_set_stream": [vp, vp],
    "spops_synchronize": [vp],
    "spops_check_device": [vp, vp],
    "spops_set_option": [vp, C.c_char_p, i64],
    "spops_csr_create": [vp, vp, i64, i64, i64, vp, vp, vp, C.c_int, C.c_int, C.c_int],
    "spops_coo_to_csr": [vp, vp, C.c_int32, C.POINTER(vp)],
    "spops_csr_reorder_rows": [vp, vp, vp, C.POINTER(vp)],
    "spops_vlcluster_create": [vp, C.POINTER(vp), i64, i64, i64, i64, i64, vp, vp, vp, vp, vp, C.c_int, C.c_int,
                               C.c_int],
    "spops_csr_to_vlength_cluster": [vp, vp, vp, i64, C.POINTER(vp)],
    "spops_vlength_cluster_to_csr": [vp, vp, C.POINTER(vp)],
    "spops_spgemm_vlength": [vp, vp, vp, C.c_int32, C.c_double, C.POINTER(vp), vp],
    "spops_matrix_features": [vp, vp, vp],
    "spops_matrix_tile_features": [vp, vp, i64, vp, vp],
    "spops_select_format": [vp, vp, i32, C.POINTER(C.c_int), vp, C.POINTER(C.c_double)],
    "spops_matrix_destroy": [vp],
    "spops_matrix_info": [vp, vp],
    "spops_matrix_touch": [vp],
    "spops_matrix_analyse": [vp, vp],
    "spops_matrix_device_bytes": [vp, vp],
    "spops_coo_create": [vp, vp, i64, i64, i64, vp, vp, vp, C.c_int, C.c_int, C.c_int],
    "spops_convert": [vp, vp, C.c_int, vp, vp],
    "spops_padded_create": [vp, vp, C.c_int, i64, i64, i64, i64, i64, i64, C.c_int, vp, vp, i64, vp, vp, i64,
                            C.c_int, C.c_int, C.c_int],
    "spops_dia_create": [vp, vp, i64, i64, i64, i64, i64, vp, vp, C.c_int, C.c_int],
    "spops_bsr_create": [vp, vp, i64, i64, i64, i64, i64, i64, vp, vp, vp, C.c_int, C.c_int, C.c_int],
    "spops_matrix_array": [vp, C.c_int, vp, vp, vp],
    "spops_matrix_download": [vp, vp, C.c_int, vp, i64],
    "spops_csr_set_values": [vp, vp],
    "spops_csr_upload_values": [vp, vp, vp],
    "spops_pairs_cluster": [vp, vp, vp, i64, vp, vp, vp],
    "spops_pairs_create": [vp, vp, vp, vp, i64, i32, vp],
    "spops_select_format_from_features": [vp, vp, vp],
    "spops_spmv_t": [vp, dbl, vp, vp, dbl, vp],
    "spops_sddmm": [vp, dbl, vp, vp, vp, vp],
    "spops_spmm": [vp, dbl, vp, vp, i64, i64, dbl, vp, i64],
    "spops_batch_create": [vp, vp, i64, vp, i64],
    "spops_batch_destroy": [vp],
    "spops_batch_set_vectors": [vp, vp, vp, vp, vp],
    "spops_batch_tune": [vp, vp, i32],
    "spops_batch_run": [vp, vp, dbl, dbl],
    "spops_batch_capture": [vp, vp, dbl, dbl],
    "spops_batch_info": [vp, vp, vp, vp],
    "spops_minhash": [vp, vp, i32, u64, vp],
    "spops_minhash_host": [vp, vp, i32, u64, vp],
    "spops_lsh_pairs": [vp, vp, i32, i32, u64, i32, vp],
    "spops_lsh_pairs_from_signatures": [vp, vp, i64, i32, i32, i32, vp],
    "spops_pairs_count": [vp, vp],
    "spops_pairs_arrays": [vp, vp, vp, vp],
    "spops_pairs_download": [vp, vp, vp, vp],
    "spops_pairs_destroy": [vp],
    "spops_hierarchical_clustering": [vp, vp, i64, vp, vp, vp, i64, i64, vp, vp, vp],
    "spops_spgemm_clustered": [vp, vp, vp, vp, vp, i64, i32, dbl, vp, vp],
    "spops_spgemm_rowwise": [vp, vp, vp, i32, i32, vp, vp],
    "spops_mtx_read_coo": [vp, C.c_char_p, C.c_int, C.c_int, vp],
    "spops_mtx_parse_coo": [vp, C.c_char_p, i64, C.c_int, C.c_int, vp],
    "spops_mtx_read_csr": [vp, C.c_char_p, C.c_int, C.c_int, i32, vp],
    "spops_mtx_parse_csr": [vp, C.c_char_p, i64, C.c_int, C.c_int, i32, vp],
    "spops_spgemm_topk": [vp, vp, i64, vp],
    "spops_spgemm_lsh": [vp, vp, vp, i32, i32, u64, i64, i32, dbl, vp, vp],
    "spops_csr_spmv_noalloc": [i64, i64, i64, vp, vp, vp, C.c_int, C.c_int, dbl, vp, dbl, vp, vp],
    "spops_spmv": [vp, dbl, vp, vp, dbl, vp],
    "spops_spmv_host": [vp, dbl, vp, vp, dbl, vp],
    "spops_spmv_host_async": [vp, dbl, vp, vp, dbl, vp],
    "spops_spmv_host_wait": [vp],
}
_RESTYPE = {"spops_last_error": C.c_char_p, "spops_status_string": C.c_char_p, "spops_abi_version": C.c_int}

_L = None
_SHUTDOWN = False


def _mark_shutdown() -> None:
    global _SHUTDOWN
    _SHUTDOWN = True


# Handles still alive when the interpreter exits are not destroyed one by one:
# the process exit releases their device memory, and the CUDA runtime may be
# torn down before the last finalisers run.
atexit.register(_mark_shutdown)


def release(name: str, handle, owner_ctx=None) -> None:
    """Destroy a handle with `name` (spops_*_destroy) unless the interpreter is
    exiting or its owning context was closed first (its stream and device
    binding are gone with it)."""
    if _SHUTDOWN or _L is None or not handle:
        return
    if owner_ctx is not None and not getattr(owner_ctx, "handle", None):
        return
    getattr(_L, name)(handle)


def lib() -> C.CDLL:
    """Load the library once; raise if it is missing (no fallback path)."""
    global _L
    if _L is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m sparseops_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, argt in _SIGS.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.argtypes = argt
            f.restype = C.c_int
        for name, rt in _RESTYPE.items():
            getattr(L, name).restype = rt
        _L = L
    return _L


def call(name: str, *args) -> None:
    """Call a C ABI function and raise SpOpsError on a non-OK status."""
    L = lib()
    st = getattr(L, name)(*args)
    if st != 0:
        msg = L.spops_last_error()
        raise SpOpsError(st, name, msg.decode() if msg else "")


def exported_symbols() -> list[str]:
    return list(_SIGS) + list(_RESTYPE)
