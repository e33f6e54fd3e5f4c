"""Seeded synthetic workloads (numpy, host memory).

The reference benchmarks on SuiteSparse matrices that are not available
here; each workload below is a seeded synthetic matrix with the shape, size
and value distribution of one benchmark configuration.  The generators live
in csrc/synth.cpp (libsparseops_synth.so): every row draws from its own
counter-based stream, so a workload is a pure function of its parameters.

Every CSR returned has rows with strictly increasing column indices, like a
Matrix Market file read by the reference's read_csr_matrix
(utils/sparse_io.cpp:190).
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_i64, _u64, _dbl, _vp = C.c_int64, C.c_uint64, C.c_double, C.c_void_p


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libsparseops_synth.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run __graft_entry__.build() (or python -m sparseops_b200.build)")
        _LIB = C.CDLL(path)
        _LIB.synth_laplacian_nnz.restype = _i64
    return _LIB


def _p(a):
    return a.ctypes.data_as(_vp)


def uniform(n: int, seed: int, lo: float = -1.0, hi: float = 1.0) -> np.ndarray:
    out = np.empty(n, np.float64)
    _lib().synth_uniform_f64(_i64(n), _u64(seed), _dbl(lo), _dbl(hi), _p(out))
    return out


def normal(n: int, seed: int) -> np.ndarray:
    out = np.empty(n, np.float64)
    _lib().synth_normal_f64(_i64(n), _u64(seed), _p(out))
    return out


def _rowptr(lens: np.ndarray, dtype=np.int64) -> np.ndarray:
    rp = np.zeros(len(lens) + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    return rp.astype(dtype, copy=False)


def laplacian_2d(nx: int, ny: int | None = None):
    """5-point Laplacian of an nx x ny grid: diagonal 4.0, neighbours -1.0."""
    ny = nx if ny is None else ny
    n = nx * ny
    nnz = int(_lib().synth_laplacian_nnz(_i64(nx), _i64(ny)))
    rp = np.zeros(n + 1, np.int32)
    ci = np.empty(nnz, np.int32)
    v = np.empty(nnz, np.float64)
    _lib().synth_laplacian_fill_i32(_i64(nx), _i64(ny), _p(rp), _p(ci), _p(v))
    return rp, ci, v


def powerlaw(n: int, mu: float = math.log(12.0), sigma: float = 1.2, lo: int = 1, hi: int = 20000,
             seed: int = 1, ncols: int | None = None):
    """Row lengths round(lognormal(mu, sigma)) clipped to [lo, hi]; columns
    uniform without replacement; values N(0, 1).  Index type int32."""
    ncols = n if ncols is None else ncols
    lens = np.empty(n, np.int64)
    _lib().synth_powerlaw_rowlen(_i64(n), _i64(ncols), _dbl(mu), _dbl(sigma), _i64(lo), _i64(hi), _u64(seed),
                                 _p(lens))
    rp64 = _rowptr(lens)
    nnz = int(rp64[-1])
    if nnz >= 2**31:
        raise ValueError("power-law matrix too large for int32 indices")
    ci = np.empty(nnz, np.int32)
    v = np.empty(nnz, np.float64)
    _lib().synth_powerlaw_fill_i32(_i64(n), _i64(ncols), _u64(seed), _p(rp64), _p(ci), _p(v))
    return rp64.astype(np.int32), ci, v


def banded_random(n: int, mean: float = 16.0, band: int = 64, seed: int = 3):
    """nnz/row ~ Poisson(mean) (>= 1 draw); half the draws within |i-j| <= band,
    half uniform; duplicates removed; values N(0, 1).  Index type int32."""
    lens = np.empty(n, np.int64)
    _lib().synth_banded_rowlen(_i64(n), _dbl(mean), _i64(band), _u64(seed), _p(lens))
    rp64 = _rowptr(lens)
    ci = np.empty(int(rp64[-1]), np.int32)
    v = np.empty(int(rp64[-1]), np.float64)
    _lib().synth_banded_fill_i32(_i64(n), _dbl(mean), _i64(band), _u64(seed), _p(rp64), _p(ci), _p(v))
    return rp64.astype(np.int32), ci, v


def symmetric_graph(n: int, mean_degree: float = 32.0, sigma: float = 1.0, seed: int = 4,
                    lo: float = 0.1, hi: float = 1.0):
    """Random graph with a symmetric pattern: row i proposes about
    lognormal/2 neighbours; the pattern is proposals plus their mirrors,
    deduplicated, so the mean degree is about `mean_degree`.  Values are
    U[lo, hi] per stored entry (the values are NOT symmetric).  int32 index."""
    mu = math.log(mean_degree) - 0.5 * sigma * sigma
    cnt = np.empty(n, np.int64)
    _lib().synth_graph_proposals_count(_i64(n), _dbl(mu), _dbl(sigma), _u64(seed), _p(cnt))
    off = _rowptr(cnt)
    dst = np.empty(int(off[-1]), np.int64)
    _lib().synth_graph_proposals_fill(_i64(n), _u64(seed), _p(off), _p(dst))
    src = np.repeat(np.arange(n, dtype=np.int64), cnt)
    key = np.concatenate([src * n + dst, dst * n + src])
    key = np.unique(key)
    rows = key // n
    cols = (key % n).astype(np.int32)
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=rp[1:])
    v = np.empty(len(cols), np.float64)
    _lib().synth_row_uniform_values(_i64(n), _u64(seed), _p(rp), _dbl(lo), _dbl(hi), _p(v))
    return rp.astype(np.int32), cols, v


def planted_communities(n: int, ncols: int | None = None, ncomm: int = 2048, mean: float = 20.0,
                        sigma: float = 0.8, p_in: float = 0.85, seed: int = 5):
    """Rows pick one of `ncomm` column communities (contiguous column blocks)
    uniformly; row length lognormal with the given mean; each draw lands in
    the row's community with probability p_in, else uniform; duplicates
    removed; values N(0, 1).  Index type int64 (the reference instantiates
    its SpGEMM for int64_t only, src/spgemm.cpp:844-1010)."""
    ncols = n if ncols is None else ncols
    mu = math.log(mean) - 0.5 * sigma * sigma
    lens = np.empty(n, np.int64)
    _lib().synth_planted_rowlen(_i64(n), _i64(ncols), _i64(ncomm), _dbl(mu), _dbl(sigma), _dbl(p_in),
                                _u64(seed), _p(lens))
    rp = _rowptr(lens)
    ci = np.empty(int(rp[-1]), np.int64)
    v = np.empty(int(rp[-1]), np.float64)
    _lib().synth_planted_fill_i64(_i64(n), _i64(ncols), _i64(ncomm), _dbl(mu), _dbl(sigma), _dbl(p_in),
                                  _u64(seed), _p(rp), _p(ci), _p(v))
    return rp, ci, v


def grouped_rows(n: int, group: int = 32, width: int = 12, mean: float = 10.0, sigma: float = 0.5,
                 p_in: float = 0.995, seed: int = 8, ncols: int | None = None):
    """Rows in contiguous groups of `group`; a group draws from one block of
    `width` columns (with probability p_in, else uniformly), so rows of a
    group are near-duplicates: MinHash-LSH pairs them into multi-row
    clusters and C = A A^T has dense group x group blocks.  Row length
    lognormal with the given mean, clipped to [1, width]; duplicates removed;
    values N(0, 1).  Default ncols = n / group * width.  Index type int64.
    Returns (rp, ci, v, ncols)."""
    ncols = n // group * width if ncols is None else ncols
    mu = math.log(mean) - 0.5 * sigma * sigma
    lens = np.empty(n, np.int64)
    _lib().synth_grouped_rowlen(_i64(n), _i64(ncols), _i64(group), _i64(width), _dbl(mu), _dbl(sigma), _dbl(p_in),
                                _u64(seed), _p(lens))
    rp = _rowptr(lens)
    ci = np.empty(int(rp[-1]), np.int64)
    v = np.empty(int(rp[-1]), np.float64)
    _lib().synth_grouped_fill_i64(_i64(n), _i64(ncols), _i64(group), _i64(width), _dbl(mu), _dbl(sigma), _dbl(p_in),
                                  _u64(seed), _p(rp), _p(ci), _p(v))
    return rp, ci, v, ncols


def transpose(rp, ci, v, ncols: int):
    """Plain CSR transpose (stable by row), same index dtype as the input."""
    n = len(rp) - 1
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp.astype(np.int64)))
    order = np.lexsort((rows, ci))
    trp = np.zeros(ncols + 1, np.int64)
    np.cumsum(np.bincount(ci, minlength=ncols), out=trp[1:])
    return trp.astype(rp.dtype), rows[order].astype(ci.dtype), v[order]
