"""The reference's storage formats and their SpMV entry points.

Every class mirrors one struct of the reference's include/sparse_format.h and
every function one template of include/SpOps.h:

    csr_to_sell_c_sigma / SpOps_sell_c_sigma   SELL_C_Sigma_Matrix
    csr_to_sell_c_R     / SpOps_sell_c_R       SELL_C_R_Matrix
    csr_to_sell         / SpOps_sell           S_ELL_Matrix
    csr_to_ell          / SpOps_ell            ELL_Matrix
    csr_to_dia          / SpOps_dia            DIA_Matrix
    csr_to_bsr          / SpOps_bsr            BSR_Matrix
    csr_to_coo          / SpOps_coo            COO_Matrix

Conversions run on the device (spops_convert).  The result lives in device
memory; the reference's host arrays (reorder, chunk_len, per-chunk
col_index / values, diag_offsets, ...) are downloaded on first access.
Objects can also be built from host arrays laid out as the reference builds
them (``from_arrays``), e.g. to run a struct produced by the reference itself.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import FormatParams, call, i64, vp
from .spops import (CSR_Matrix, Matrix_Features, _Handle, _is_cuda_tensor, _itype, _ptr, _spmv, _vtype,
                    default_context)

# reference defaults (include/general_config.h, include/plat_config.h as shipped)
SELL_SIGMA = 16384
CHUNK_SIZE = 4
MAX_DIAG_NUM = 10240
BSR_BlockDimRow = 16
SIMD_WIDTH = 256
RowMajor, ColMajor = 0, 1

_ARR = dict(row=0, col=1, val=2, reorder=3, chunk_len=4, chunk_off=5, row_len=6, diag_offsets=7,
            block_row_ptr=8, block_col=9, tile_ptr=10, tile_desc=11)
_NP = {(4, "i"): np.int32, (8, "i"): np.int64, (4, "f"): np.float32, (8, "f"): np.float64}


def _default_align(values) -> int:
    return SIMD_WIDTH // 8 // np.dtype(str(values.dtype).replace("torch.", "")).itemsize


class _Converted(Matrix_Features):
    """A format held on the device; host arrays fetched lazily."""

    _fmt: str = ""

    def _download(self, name: str, kind: str):
        h = self._h
        p, n, eb = vp(), C.c_int64(), C.c_int32()
        call("spops_matrix_array", h.handle, _ARR[name], C.byref(p), C.byref(n), C.byref(eb))
        out = np.empty(n.value, _NP[(eb.value, kind)])
        if n.value:
            call("spops_matrix_download", h.ctx.handle, h.handle, _ARR[name], out.ctypes.data_as(vp), n)
        return out

    def device(self, ctx=None) -> _Handle:
        if self._h is None:
            self._create(ctx or default_context())
        return self._h

    def _info(self):
        return self.device().info()


def _convert(csr: CSR_Matrix, fmt: str, **params) -> _Handle:
    h = csr.device()
    p = FormatParams()
    for k, v in params.items():
        setattr(p, k, int(v))
    out = vp()
    call("spops_convert", h.ctx.handle, h.handle, _lib.FORMATS[fmt], C.byref(p), C.byref(out))
    return _Handle(h.ctx, out, (h,))


class _Padded(_Converted):
    """Shared behaviour of SELL-C-sigma, SELL-C-R, S-ELL and ELL."""

    def __init__(self):
        super().__init__()
        self._cache = {}

    def _arr(self, name, kind="i"):
        if name not in self._cache:
            self._cache[name] = self._download(name, kind)
        return self._cache[name]

    def _chunks(self, name, kind):
        flat = self._arr(name, kind)
        off = self._arr("chunk_off", "i")
        return [flat[off[c]:off[c + 1]] for c in range(len(off) - 1)]

    @property
    def col_index(self):  # list of per-chunk arrays, -1 marks padding
        return self._chunks("col", "i")

    @property
    def values(self):
        return self._chunks("val", "f")

    @property
    def stored_elements(self) -> int:
        return int(self._arr("chunk_off", "i")[-1])

    def _from_arrays_create(self, ctx, fmt, C_, sigma, align, layout, reorder, chunk_len, col, val):
        h = vp()
        on_dev = _is_cuda_tensor(val)
        call("spops_padded_create", ctx.handle, C.byref(h), _lib.FORMATS[fmt], i64(self.num_rows),
             i64(self.num_cols), i64(self.num_nnzs), i64(C_), i64(sigma), i64(align), int(layout), _ptr(reorder),
             _ptr(chunk_len), i64(len(chunk_len)), _ptr(col), _ptr(val), i64(len(col)), _itype(col), _vtype(val),
             0 if on_dev else 1)
        self._h = _Handle(ctx, h, (reorder, chunk_len, col, val) if on_dev else ())


class SELL_C_Sigma_Matrix(_Padded):
    """SELL-C-sigma (include/sparse_format.h:221-250)."""

    _fmt = "sell_c_sigma"

    @property
    def reorder(self):
        return self._arr("reorder")

    @property
    def chunk_len(self):
        return self._arr("chunk_len")

    @property
    def sliceNum(self):
        return (self.num_rows + self.sliceWidth_Sigma - 1) // self.sliceWidth_Sigma

    @property
    def chunk_num_per_slice(self):
        return self.sliceWidth_Sigma // self.chunkWidth_C

    @property
    def chunkNum(self):
        return self.sliceNum * self.chunk_num_per_slice

    @property
    def validchunkNum(self):
        return (self.num_rows + self.chunkWidth_C - 1) // self.chunkWidth_C

    @classmethod
    def from_arrays(cls, num_rows, num_cols, num_nnzs, sigma, C_, alignment, reorder, chunk_len, col_flat,
                    val_flat, layout=RowMajor, ctx=None):
        """Wrap reference-layout arrays (chunks concatenated) on the device."""
        m = cls()
        m.num_rows, m.num_cols, m.num_nnzs = int(num_rows), int(num_cols), int(num_nnzs)
        m.sliceWidth_Sigma, m.chunkWidth_C, m.alignment = int(sigma), int(C_), int(alignment)
        m._from_arrays_create(ctx or default_context(), cls._fmt, C_, sigma, alignment, layout, reorder, chunk_len,
                              col_flat, val_flat)
        return m


class SELL_C_R_Matrix(_Padded):
    """SELL-C-R: SELL-C-sigma with one global sort (include/sparse_format.h:253-276)."""

    _fmt = "sell_c_R"

    @property
    def reorder(self):
        return self._arr("reorder")

    @property
    def chunk_len(self):
        return self._arr("chunk_len")

    @property
    def validchunkNum(self):
        return (self.num_rows + self.chunkWidth_C - 1) // self.chunkWidth_C


class S_ELL_Matrix(_Padded):
    """Sliced ELL (include/sparse_format.h:190-218); chunks of C consecutive rows."""

    _fmt = "sell"

    @property
    def row_width(self):
        return self._arr("chunk_len")

    @property
    def chunk_num(self):
        return (self.num_rows + self.sliceWidth - 1) // self.sliceWidth


class ELL_Matrix(_Padded):
    """ELLPACK (include/sparse_format.h:170-188); ld = RowMajor or ColMajor."""

    _fmt = "ell"

    @property
    def col_index(self):  # one [num_rows * max_row_width] array, as the reference stores it
        return self._arr("col", "i")

    @property
    def values(self):
        return self._arr("val", "f")

    @property
    def max_row_width(self):
        return int(self._info().extra[0])

    @property
    def min_row_width(self):
        return int(self._info().extra[1])


class DIA_Matrix(_Converted):
    """Diagonal storage (include/sparse_format.h:172-184)."""

    _fmt = "dia"

    @property
    def diag_offsets(self):
        return self._download("diag_offsets", "i")

    @property
    def diag_data(self):
        return self._download("val", "f")

    @property
    def complete_ndiags(self):
        return int(self._info().extra[0])

    @property
    def stride(self):
        return int(self._info().extra[1])


class BSR_Matrix(_Converted):
    """Block CSR, blocks row-major (include/sparse_format.h:110-127)."""

    _fmt = "bsr"

    @property
    def row_ptr(self):
        return self._download("block_row_ptr", "i")

    @property
    def block_colindex(self):
        return self._download("block_col", "i")

    @property
    def block_data(self):
        return self._download("val", "f")

    @property
    def nnzb(self):
        return int(self._info().extra[2])

    @property
    def mb(self):
        return int(self._info().extra[0])

    @property
    def nb(self):
        return int(self._info().extra[1])


class COO_Matrix(_Converted):
    """Triplets (include/sparse_format.h:72-81); rows need not be sorted."""

    _fmt = "coo"

    def __init__(self, num_rows=0, num_cols=0, row_index=None, col_index=None, values=None):
        super().__init__()
        self.num_rows, self.num_cols = int(num_rows), int(num_cols)
        self._arrays = (row_index, col_index, values)
        self.num_nnzs = 0 if col_index is None else int(len(col_index))

    def _create(self, ctx):
        r, c, v = self._arrays
        on_dev = _is_cuda_tensor(v)
        h = vp()
        call("spops_coo_create", ctx.handle, C.byref(h), i64(self.num_rows), i64(self.num_cols),
             i64(self.num_nnzs), _ptr(r), _ptr(c), _ptr(v), _itype(c), _vtype(v), 0 if on_dev else 1)
        self._h = _Handle(ctx, h, self._arrays if on_dev else ())

    @property
    def row_index(self):
        return self._download("row", "i")

    @property
    def col_index(self):
        return self._download("col", "i")

    @property
    def values(self):
        return self._download("val", "f")


class CSR5_Matrix(_Converted):
    """CSR5 (include/sparse_format.h:137-166) with device tiles of omega = 32
    lanes x sigma = 16 entries; tile_ptr / tile_desc follow that tiling."""

    _fmt = "csr5"
    sigma = 16
    omega = 32

    @property
    def _p(self):
        return int(self._info().extra[0])

    @property
    def tile_ptr(self):
        return self._download("tile_ptr", "i").view(np.uint32)

    @property
    def tile_desc(self):
        return self._download("tile_desc", "i").view(np.uint32)


def _wrap(cls, csr: CSR_Matrix, h: _Handle, **fields):
    m = cls()
    m.num_rows, m.num_cols, m.num_nnzs = csr.num_rows, csr.num_cols, csr.num_nnzs
    m.kernel_flag = csr.kernel_flag
    m._h = h
    for k, v in fields.items():
        setattr(m, k, v)
    return m


# ------------------------------------------------------------------ conversions
def csr_to_sell_c_sigma(csr: CSR_Matrix, fp_feature=None, slicewidth: int = SELL_SIGMA,
                        chunkwidth: int = CHUNK_SIZE, alignment: int | None = None, layout: int = RowMajor):
    """include/sparse_conversion.h:344 (fp_feature is accepted and ignored)."""
    alignment = alignment or _default_align(csr.values)
    h = _convert(csr, "sell_c_sigma", sigma=slicewidth, chunk=chunkwidth, alignment=alignment, layout=layout)
    return _wrap(SELL_C_Sigma_Matrix, csr, h, sliceWidth_Sigma=slicewidth, chunkWidth_C=chunkwidth,
                 alignment=alignment)


def csr_to_sell_c_R(csr: CSR_Matrix, fp_feature=None, chunkwidth: int = CHUNK_SIZE, alignment: int | None = None,
                    layout: int = RowMajor):
    """include/sparse_conversion.h:490."""
    alignment = alignment or _default_align(csr.values)
    h = _convert(csr, "sell_c_R", chunk=chunkwidth, alignment=alignment, layout=layout)
    return _wrap(SELL_C_R_Matrix, csr, h, chunkWidth_C=chunkwidth, alignment=alignment)


def csr_to_sell(csr: CSR_Matrix, fp_feature=None, chunkwidth: int = CHUNK_SIZE, alignment: int | None = None,
                layout: int = RowMajor):
    """include/sparse_conversion.h:265."""
    alignment = alignment or _default_align(csr.values)
    h = _convert(csr, "sell", chunk=chunkwidth, alignment=alignment, layout=layout)
    return _wrap(S_ELL_Matrix, csr, h, sliceWidth=chunkwidth, alignment=alignment)


def csr_to_ell(csr: CSR_Matrix, ld: int = RowMajor):
    """include/sparse_conversion.h:194."""
    h = _convert(csr, "ell", layout=ld)
    return _wrap(ELL_Matrix, csr, h, ld=ld)


def csr_to_dia(csr: CSR_Matrix, max_diags: int = MAX_DIAG_NUM, fp_feature=None, alignment: int | None = None):
    """include/sparse_conversion.h:619 (too many diagonals raises instead of exit(1))."""
    alignment = alignment or _default_align(csr.values)
    h = _convert(csr, "dia", max_diags=max_diags, alignment=alignment)
    return _wrap(DIA_Matrix, csr, h)


def csr_to_bsr(csr: CSR_Matrix, blockDimRow: int = BSR_BlockDimRow, blockDimCol: int | None = None):
    """include/sparse_conversion.h:776."""
    blockDimCol = blockDimCol or _default_align(csr.values)
    h = _convert(csr, "bsr", block_rows=blockDimRow, block_cols=blockDimCol)
    return _wrap(BSR_Matrix, csr, h, blockDim_r=blockDimRow, blockDim_c=blockDimCol,
                 blockNNZ=blockDimRow * blockDimCol)


def csr_to_csr5(csr: CSR_Matrix, fp_feature=None):
    """include/sparse_conversion.h:946 (device tiles; see CSR5_Matrix)."""
    h = _convert(csr, "csr5")
    return _wrap(CSR5_Matrix, csr, h, row_offset=csr.row_offset, col_index=csr.col_index, values=csr.values)


def matrix_features(csr: CSR_Matrix) -> dict:
    """Structure features of the matrix, on the device: the non-tile part of
    the reference's MTX::CalculateFeatures (src/sparse_features.cpp:643) as
    a dict (names of spops_features_t)."""
    h = csr.device()
    f = _lib.Features()
    call("spops_matrix_features", h.ctx.follow_torch().handle, h.handle, C.byref(f))
    return f.as_dict()


def matrix_tile_features(csr: CSR_Matrix, num_blocks: int = 256, maps: bool = False):
    """Tile features of the matrix, on the device: the tile part of the
    reference's MTX::MtxLoad / CalculateTilesFeatures and the row distance of
    CalculateTilesExtraFeatures (src/sparse_features.cpp:181-265, 484-625,
    783-846, 943-965) on a num_blocks x num_blocks grid (MAT_TILE_SIZE = 256).
    Returns a dict (names of spops_tile_features_t); with maps=True also the
    per-tile arrays (num_blocks x num_blocks) and per-block arrays as a second
    dict (names of spops_tile_maps_t)."""
    h = csr.device()
    f = _lib.TileFeatures()
    B = 256 if num_blocks <= 0 else int(num_blocks)
    arrays, m = {}, None
    if maps:
        m = _lib.TileMaps()
        for name, per_tile, integer in _lib.TILE_MAP_FIELDS:
            a = np.zeros((B, B) if per_tile else B, np.int64 if integer else np.float64)
            arrays[name] = a
            setattr(m, name, a.ctypes.data)
    call("spops_matrix_tile_features", h.ctx.follow_torch().handle, h.handle, i64(B), C.byref(f),
         C.byref(m) if m is not None else None)
    return (f.as_dict(), arrays) if maps else f.as_dict()


_FORMAT_NAMES = {v: k for k, v in _lib.FORMATS.items()}


def select_format(csr: CSR_Matrix, timed: bool = False, learned: bool = False) -> dict:
    """Storage format for SpMV with this matrix on this GPU: rules on the
    features (default), the fastest of the candidate formats measured on the
    device (timed=True), or the fitted decision tree over the features
    (learned=True).  Returns {"format", "params", "ms"}; the params are the
    spops_convert parameters (see convert_to)."""
    h = csr.device()
    fmt = C.c_int()
    p = FormatParams()
    ms = C.c_double()
    mode = 1 if timed else (2 if learned else 0)
    call("spops_select_format", h.ctx.follow_torch().handle, h.handle, C.c_int32(mode), C.byref(fmt),
         C.byref(p), C.byref(ms))
    params = {k: int(getattr(p, k)) for k, _ in FormatParams._fields_ if k != "reserved" and getattr(p, k)}
    return {"format": _FORMAT_NAMES[fmt.value], "params": params, "ms": ms.value}


def select_format_from_features(features: dict) -> dict:
    """The learned choice (select_format(learned=True)) from features already
    computed -- a dict with the names of spops_features_t -- without device
    work.  Returns {"format", "params"}."""
    f = _lib.Features()
    for k in _lib.FEATURE_NAMES:
        setattr(f, k, features[k])
    fmt = C.c_int()
    p = FormatParams()
    call("spops_select_format_from_features", C.byref(f), C.byref(fmt), C.byref(p))
    params = {k: int(getattr(p, k)) for k, _ in FormatParams._fields_ if k != "reserved" and getattr(p, k)}
    return {"format": _FORMAT_NAMES[fmt.value], "params": params}


_CONVERTED = {"sell_c_sigma": SELL_C_Sigma_Matrix, "sell_c_R": SELL_C_R_Matrix, "sell": S_ELL_Matrix,
              "ell": ELL_Matrix, "dia": DIA_Matrix, "bsr": BSR_Matrix, "csr5": CSR5_Matrix}


def convert_to(csr: CSR_Matrix, fmt: str, **params):
    """The matrix in format `fmt` with spops_convert parameters (e.g. the
    result of select_format); "csr" returns the matrix itself."""
    if fmt == "csr":
        return csr
    if fmt == "coo":
        return csr_to_coo(csr)
    return _wrap(_CONVERTED[fmt], csr, _convert(csr, fmt, **params))


def SpOps_auto(alpha, csr: CSR_Matrix, x, beta, y, timed: bool = False, learned: bool = False):
    """y = alpha*A*x + beta*y in the format select_format picks for A (rules,
    timed or learned); the choice and the converted matrix are kept on the
    CSR object."""
    key = "timed" if timed else ("learned" if learned else "rules")
    cache = getattr(csr, "_auto", None)
    if cache is None or cache[0] != key:
        choice = select_format(csr, timed, learned)
        cache = (key, choice, convert_to(csr, choice["format"], **choice["params"]))
        csr._auto = cache
    return _spmv(alpha, cache[2], x, beta, y)


def coo_to_csr(coo: COO_Matrix, compact: bool = False):
    """include/sparse_conversion.h:37 on the device: CSR with rows in order and
    file order kept within a row; compact=True also sums duplicates like
    sum_csr_duplicates (include/sparse_operation.h:21): distinct columns in
    reverse order of first appearance, exact-zero sums dropped."""
    from .spops import DeviceCSR
    h = coo.device()
    ctx = h.ctx.follow_torch()
    out = vp()
    call("spops_coo_to_csr", ctx.handle, h.handle, C.c_int32(1 if compact else 0), C.byref(out))
    return DeviceCSR(_Handle(ctx, out), coo.num_rows, coo.num_cols)


def csr_reorder_rows(csr: CSR_Matrix, row_permutation):
    """include/sparse_conversion.h:1879 on the device: row i of the result is
    row row_permutation[i] of csr; a DeviceCSR.  The permutation must hold
    every row once (SpOpsError otherwise)."""
    from .spops import DeviceCSR
    h = csr.device()
    ctx = h.ctx.follow_torch()
    it = np.int32 if int(h.info().index_type) == 0 else np.int64
    perm = np.ascontiguousarray(np.asarray(row_permutation), dtype=it)
    if len(perm) < csr.num_rows:
        raise ValueError("row_permutation size must be >= matrix rows")
    out = vp()
    call("spops_csr_reorder_rows", ctx.handle, h.handle, perm.ctypes.data_as(vp), C.byref(out))
    return DeviceCSR(_Handle(ctx, out), csr.num_rows, csr.num_cols)


def _mtx_types(index_dtype, value_dtype):
    it = 0 if np.dtype(index_dtype) == np.int32 else 1
    vt = 0 if np.dtype(value_dtype) == np.float32 else 1
    return C.c_int(it), C.c_int(vt)


def read_coo_matrix(mm_filename, index_dtype=np.int32, value_dtype=np.float64, ctx=None) -> COO_Matrix:
    """utils/sparse_io.cpp:26 with the text parsed on the device: the file's
    entries in file order (symmetric files expanded), 0-based, held by a
    device handle; host arrays on first access."""
    ctx = ctx or default_context()
    out = vp()
    call("spops_mtx_read_coo", ctx.handle, str(mm_filename).encode(), *_mtx_types(index_dtype, value_dtype),
         C.byref(out))
    h = _Handle(ctx, out)
    info = h.info()
    m = COO_Matrix()
    m.num_rows, m.num_cols, m.num_nnzs = int(info.rows), int(info.cols), int(info.nnz)
    m._h = h
    m._arrays = (None, None, None)
    return m


def read_csr_matrix(mm_filename, compact: bool = False, index_dtype=np.int32, value_dtype=np.float64, ctx=None):
    """utils/sparse_io.cpp:193 on the device: read_coo_matrix then coo_to_csr
    (compact: duplicates summed); a DeviceCSR."""
    from .spops import DeviceCSR
    ctx = ctx or default_context()
    out = vp()
    call("spops_mtx_read_csr", ctx.handle, str(mm_filename).encode(), *_mtx_types(index_dtype, value_dtype),
         C.c_int32(1 if compact else 0), C.byref(out))
    h = _Handle(ctx, out)
    info = h.info()
    return DeviceCSR(h, int(info.rows), int(info.cols))


def csr_to_coo(csr: CSR_Matrix):
    """include/sparse_conversion.h:152."""
    h = _convert(csr, "coo")
    m = _wrap(COO_Matrix, csr, h)
    m._arrays = (None, None, None)
    return m


# -------------------------------------------------------------------- SpMV
def SpOps_sell_c_sigma(alpha, A: SELL_C_Sigma_Matrix, x, beta, y):
    """src/spmv_sell_c_sigma.cpp:189."""
    return _spmv(alpha, A, x, beta, y)


def SpOps_sell_c_R(alpha, A: SELL_C_R_Matrix, x, beta, y):
    """src/spmv_sell_c_R.cpp:190."""
    return _spmv(alpha, A, x, beta, y)


def SpOps_sell(alpha, A: S_ELL_Matrix, x, beta, y):
    """src/spmv_s_ell.cpp:202."""
    return _spmv(alpha, A, x, beta, y)


def SpOps_ell(alpha, A: ELL_Matrix, x, beta, y):
    """src/spmv_ell.cpp:225."""
    return _spmv(alpha, A, x, beta, y)


def SpOps_dia(alpha, A: DIA_Matrix, x, beta, y):
    """src/spmv_dia.cpp:177."""
    return _spmv(alpha, A, x, beta, y)


def SpOps_bsr(alpha, A: BSR_Matrix, x, beta, y):
    """src/spmv_bsr.cpp:214."""
    return _spmv(alpha, A, x, beta, y)


def SpOps_csr5(alpha, A: CSR5_Matrix, x, beta, y):
    """src/spmv_csr5.cpp:439."""
    return _spmv(alpha, A, x, beta, y)


def SpOps_coo(alpha, A: COO_Matrix, x, beta, y):
    """src/spmv_coo.cpp:160."""
    return _spmv(alpha, A, x, beta, y)
