"""Device format conversions and per-format SpMV.

Layout arrays (SELL reorder / chunk_len, S-ELL row_width, DIA diag_offsets,
BSR row_ptr / block_colindex) must equal the reference's bit for bit (golden
fixtures written by the reference itself); padded col/val arrays must equal
the reference layout built from them; SpMV results must match the oracle to
1e-12 on the componentwise metric.
"""
import math

import numpy as np
import pytest

from sparseops_b200 import synth

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def _csr(rp, ci, v, ncols=None, on_device=True):
    from sparseops_b200 import CSR_Matrix
    n = len(rp) - 1
    ncols = n if ncols is None else ncols
    if on_device:
        return CSR_Matrix(n, ncols, _dev(rp), _dev(ci), _dev(v))
    return CSR_Matrix(n, ncols, rp, ci, v)


def _spmv(fn, A, x, alpha=0.8, beta=0.7, y0=None):
    import torch
    n = A.num_rows
    y0 = np.ones(n) if y0 is None else y0
    xd, yd = _dev(x), _dev(y0.copy())
    fn(alpha, A, xd, beta, yd)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


def _check(orc, rp, ci, v, x, y, alpha=0.8, beta=0.7, y0=None):
    n = len(rp) - 1
    y0 = np.ones(n) if y0 is None else y0
    yref = orc.spmv_csr(rp, ci, v, x, alpha, beta, y0)
    den = abs(alpha) * orc.absdot(rp, ci, v, x) + np.abs(beta * y0)
    err = (np.abs(y - yref) / np.maximum(den, 1e-300)).max() if n else 0.0
    assert err <= TOL, err


def _ref_layout(rp, ci, v, reorder, chunk_len, C):
    """Reference row-major padded arrays (include/sparse_conversion.h:460-484)."""
    n = len(rp) - 1
    off = np.concatenate([[0], np.cumsum(chunk_len.astype(np.int64) * C)])
    col = np.full(off[-1], -1, np.int32)
    val = np.zeros(off[-1])
    for i in range(n):
        r = reorder[i] if reorder is not None else i
        c = i // C
        base = off[c] + (i - c * C) * chunk_len[c]
        L = rp[r + 1] - rp[r]
        col[base:base + L] = ci[rp[r]:rp[r + 1]]
        val[base:base + L] = v[rp[r]:rp[r + 1]]
    return col, val


@pytest.mark.parametrize("tag,sigma,C,align", [("a", 512, 32, 8), ("b", 64, 4, 4), ("c", 16384, 4, 4)])
def test_sell_c_sigma(cuda, golden, orc, tag, sigma, C, align):
    from sparseops_b200 import SpOps_sell_c_sigma, csr_to_sell_c_sigma
    g = golden
    rp, ci, v, x = g["pl_rp"], g["pl_ci"], g["pl_v"], g["pl_x"]
    S = csr_to_sell_c_sigma(_csr(rp, ci, v), None, sigma, C, align)
    assert np.array_equal(S.reorder, g[f"scs_{tag}_reorder"])
    assert np.array_equal(S.chunk_len, g[f"scs_{tag}_chunk_len"])
    col, val = _ref_layout(rp, ci, v, S.reorder, S.chunk_len, C)
    assert np.array_equal(np.concatenate(S.col_index), col) and np.array_equal(np.concatenate(S.values), val)
    assert S.validchunkNum == len(S.chunk_len)
    _check(orc, rp, ci, v, x, _spmv(SpOps_sell_c_sigma, S, x))


def test_sell_c_sigma_col_major_and_uploaded(cuda, golden, orc):
    """Device-native column-major chunks, and a struct uploaded from host
    arrays in the reference layout, give the same SpMV."""
    from sparseops_b200 import SELL_C_Sigma_Matrix, SpOps_sell_c_sigma, csr_to_sell_c_sigma
    g = golden
    rp, ci, v, x = g["pl_rp"], g["pl_ci"], g["pl_v"], g["pl_x"]
    S = csr_to_sell_c_sigma(_csr(rp, ci, v), None, 512, 32, 8, layout=1)
    _check(orc, rp, ci, v, x, _spmv(SpOps_sell_c_sigma, S, x))
    col, val = _ref_layout(rp, ci, v, g["scs_a_reorder"], g["scs_a_chunk_len"], 32)
    U = SELL_C_Sigma_Matrix.from_arrays(len(rp) - 1, len(rp) - 1, len(ci), 512, 32, 8, g["scs_a_reorder"],
                                        g["scs_a_chunk_len"], col, val)
    _check(orc, rp, ci, v, x, _spmv(SpOps_sell_c_sigma, U, x))


def test_sell_c_R(cuda, golden, orc):
    from sparseops_b200 import SpOps_sell_c_R, csr_to_sell_c_R
    g = golden
    rp, ci, v, x = g["pl_rp"], g["pl_ci"], g["pl_v"], g["pl_x"]
    S = csr_to_sell_c_R(_csr(rp, ci, v), None, 32, 8)
    assert np.array_equal(S.reorder, g["scr_reorder"]) and np.array_equal(S.chunk_len, g["scr_chunk_len"])
    _check(orc, rp, ci, v, x, _spmv(SpOps_sell_c_R, S, x))


def test_s_ell(cuda, golden, orc):
    from sparseops_b200 import SpOps_sell, csr_to_sell
    g = golden
    rp, ci, v, x = g["pl_rp"], g["pl_ci"], g["pl_v"], g["pl_x"]
    S = csr_to_sell(_csr(rp, ci, v), None, 4, 4)
    assert np.array_equal(S.row_width, g["sell_row_width"])
    col, val = _ref_layout(rp, ci, v, None, S.row_width, 4)
    assert np.array_equal(np.concatenate(S.col_index), col)
    _check(orc, rp, ci, v, x, _spmv(SpOps_sell, S, x))


@pytest.mark.parametrize("ld", [0, 1])
def test_ell(cuda, golden, orc, ld):
    from sparseops_b200 import SpOps_ell, csr_to_ell
    g = golden
    rp, ci, v, x = g["lap_rp"], g["lap_ci"], g["lap_v"], g["lap_x"]
    E = csr_to_ell(_csr(rp, ci, v), ld)
    assert E.max_row_width == int(np.diff(rp).max())
    n, w = len(rp) - 1, E.max_row_width
    col = np.asarray(E.col_index).reshape((n, w) if ld == 0 else (w, n))
    if ld == 1:
        col = col.T
    for r in (0, 1, n // 2, n - 1):  # row r holds its entries first, then -1
        L = rp[r + 1] - rp[r]
        assert np.array_equal(col[r, :L], ci[rp[r]:rp[r + 1]]) and (col[r, L:] == -1).all()
    _check(orc, rp, ci, v, x, _spmv(SpOps_ell, E, x))


@pytest.mark.parametrize("name", ["lap", "band"])
def test_dia(cuda, golden, orc, name):
    from sparseops_b200 import SpOps_dia, csr_to_dia
    g = golden
    rp, ci, v = g[f"{name}_rp"], g[f"{name}_ci"], g[f"{name}_v"]
    x = synth.uniform(len(rp) - 1, 17)
    D = csr_to_dia(_csr(rp, ci, v), 10240, None, 4)
    assert np.array_equal(D.diag_offsets, g[f"dia_{name}_offsets"])
    assert D.stride == int(g[f"dia_{name}_stride"])
    _check(orc, rp, ci, v, x, _spmv(SpOps_dia, D, x))


def test_dia_too_many_diagonals(cuda):
    from sparseops_b200 import SpOpsError, csr_to_dia
    rp, ci, v = synth.powerlaw(3000, seed=30)
    with pytest.raises(SpOpsError) as e:
        csr_to_dia(_csr(rp, ci, v), 100)
    assert e.value.status == 5


@pytest.mark.parametrize("name,br,bc", [("lap", 16, 4), ("pl", 16, 8)])
def test_bsr(cuda, golden, orc, name, br, bc):
    from sparseops_b200 import SpOps_bsr, csr_to_bsr
    g = golden
    rp, ci, v = g[f"{name}_rp"], g[f"{name}_ci"], g[f"{name}_v"]
    x = synth.uniform(len(rp) - 1, 18)
    B = csr_to_bsr(_csr(rp, ci, v), br, bc)
    assert np.array_equal(B.row_ptr, g[f"bsr_{name}_row_ptr"]) and np.array_equal(B.block_colindex,
                                                                                  g[f"bsr_{name}_col"])
    _check(orc, rp, ci, v, x, _spmv(SpOps_bsr, B, x))


def test_coo(cuda, golden, orc):
    from sparseops_b200 import COO_Matrix, SpOps_coo, csr_to_coo
    g = golden
    rp, ci, v, x = g["pl_rp"], g["pl_ci"], g["pl_v"], g["pl_x"]
    K = csr_to_coo(_csr(rp, ci, v))
    rows = np.repeat(np.arange(len(rp) - 1, dtype=np.int32), np.diff(rp))
    assert np.array_equal(K.row_index, rows) and np.array_equal(K.col_index, ci)
    _check(orc, rp, ci, v, x, _spmv(SpOps_coo, K, x))
    # unsorted triplets from the host
    perm = np.random.default_rng(3).permutation(len(ci))
    U = COO_Matrix(len(rp) - 1, len(rp) - 1, rows[perm], ci[perm], v[perm])
    _check(orc, rp, ci, v, x, _spmv(SpOps_coo, U, x))


def test_sell_long_rows_and_empty_rows(cuda, orc):
    """Stored rows longer than one piece (2048 slots) and empty rows, both layouts."""
    from sparseops_b200 import SpOps_sell_c_sigma, csr_to_sell_c_sigma
    rng = np.random.default_rng(9)
    n, ncols = 5000, 100000
    lens = rng.integers(0, 30, n)
    lens[7], lens[1500], lens[4999] = 9000, 2049, 30000
    lens[100:700] = 0
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    ci = np.concatenate([np.sort(rng.choice(ncols, L, replace=False)) for L in lens]).astype(np.int32)
    v = rng.standard_normal(len(ci))
    x = rng.uniform(-1, 1, ncols)
    rp = rp.astype(np.int32)
    for layout in (0, 1):
        S = csr_to_sell_c_sigma(_csr(rp, ci, v, ncols), None, 512, 32, 8, layout=layout)
        _check(orc, rp, ci, v, x, _spmv(SpOps_sell_c_sigma, S, x))


@pytest.mark.parametrize("tails,order", [(0, 1), (1, 1), (0, 0)])
@pytest.mark.parametrize("sigma", [32, 512, 1 << 20])
def test_sell_col_major_windows_and_packing(cuda, orc, sigma, tails, order):
    """C = 32 column-major: chunks cut into step windows (rows longer than 128
    slots, one with more than 2048), rows of very different lengths in one
    chunk (the lane re-dealing path), empty rows, rows past the last full
    chunk, unsorted (sigma = C) and sorted slices; FP64 and FP32 values; the
    slots past a chunk's fourth-longest row read from row-contiguous tails
    (tails = 1, tail windows of up to 1024 entries) or in place (the default);
    the windows listed longest chunk first (the default) or in chunk order."""
    from sparseops_b200 import default_context
    default_context().set_option("sell_tails", tails)
    default_context().set_option("sell_order", order)
    try:
        _sell_windows_case(orc, sigma)
    finally:
        default_context().set_option("sell_tails", 0)
        default_context().set_option("sell_order", 1)


def _sell_windows_case(orc, sigma):
    from sparseops_b200 import SpOps_sell_c_sigma, csr_to_sell_c_sigma
    rng = np.random.default_rng(21)
    n, ncols = 3000 + 17, 50000
    lens = rng.integers(0, 12, n)
    lens[rng.choice(n, 40, replace=False)] = rng.integers(130, 900, 40)
    lens[5], lens[33], lens[2999] = 2500, 129, 4097
    lens[64:96] = 0
    lens[200:232] = np.arange(1, 33) * 7
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    ci = np.concatenate([np.sort(rng.choice(ncols, L, replace=False)) for L in lens]).astype(np.int32)
    v = rng.standard_normal(len(ci))
    x = rng.uniform(-1, 1, ncols)
    y0 = rng.uniform(-1, 1, n)
    rp = rp.astype(np.int32)
    S = csr_to_sell_c_sigma(_csr(rp, ci, v, ncols), None, sigma, 32, 1, layout=1)
    for _ in range(2):  # the window counters must be back at zero for the next call
        _check(orc, rp, ci, v, x, _spmv(SpOps_sell_c_sigma, S, x, 0.8, 0.7, y0), 0.8, 0.7, y0)
    v32, x32 = v.astype(np.float32), x.astype(np.float32)
    S32 = csr_to_sell_c_sigma(_csr(rp, ci, v32, ncols), None, sigma, 32, 1, layout=1)
    y = _spmv(SpOps_sell_c_sigma, S32, x32, 1.0, 0.0, np.zeros(n, np.float32))
    yref = orc.spmv_csr(rp, ci, v32.astype(np.float64), x32.astype(np.float64))
    den = orc.absdot(rp, ci, v32, x32)
    assert (np.abs(y - yref) / np.maximum(den, 1e-300)).max() <= 1e-5


def test_powerlaw_full_sell_and_ell(cuda, orc):
    """Power-law config at full size: SELL-C-sigma (C=32, sigma=512) and
    SELL-C-R match the oracle; ELL is refused (it would need ~1 TB)."""
    from sparseops_b200 import (SpOps_sell_c_R, SpOps_sell_c_sigma, SpOpsError, csr_to_ell, csr_to_sell_c_R,
                                csr_to_sell_c_sigma)
    n = 4194304
    rp, ci, v = synth.powerlaw(n, mu=math.log(12.0), sigma=1.2, lo=1, hi=20000, seed=1)
    x = synth.uniform(n, 1)
    A = _csr(rp, ci, v)
    S = csr_to_sell_c_sigma(A, None, 512, 32, 8)
    _check(orc, rp, ci, v, x, _spmv(SpOps_sell_c_sigma, S, x, 1.0, 0.0), 1.0, 0.0)
    del S
    R = csr_to_sell_c_R(A, None, 32, 8)
    _check(orc, rp, ci, v, x, _spmv(SpOps_sell_c_R, R, x, 1.0, 0.0), 1.0, 0.0)
    del R
    with pytest.raises(SpOpsError) as e:
        csr_to_ell(A)
    assert e.value.status == 5


@pytest.mark.parametrize("name", ["lap", "pl"])
def test_csr5_golden(cuda, golden, orc, name):
    from sparseops_b200 import SpOps_csr5, csr_to_csr5
    g = golden
    rp, ci, v, x = g[f"{name}_rp"], g[f"{name}_ci"], g[f"{name}_v"], g[f"{name}_x"]
    T = csr_to_csr5(_csr(rp, ci, v))
    assert T._p == (len(ci) + 511) // 512 and len(T.tile_ptr) == T._p + 1
    _check(orc, rp, ci, v, x, _spmv(SpOps_csr5, T, x))


@pytest.mark.parametrize("itype,vtype", [(np.int32, np.float64), (np.int64, np.float64), (np.int32, np.float32)])
def test_csr5_edges(cuda, orc, itype, vtype):
    """Rows spanning many tiles, rows ending exactly on lane/tile boundaries,
    runs of empty rows (also at the start and end), a partial last tile."""
    from sparseops_b200 import SpOps_csr5, csr_to_csr5
    rng = np.random.default_rng(11)
    n, ncols = 7000, 50000
    lens = rng.integers(0, 20, n)
    lens[:5] = 0
    lens[10], lens[11], lens[12] = 16, 512, 5000
    lens[3000:3100] = 0
    lens[-7:] = 0
    lens[-8] = 1001
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    ci = np.concatenate([np.sort(rng.choice(ncols, L, replace=False)) for L in lens])
    v = rng.standard_normal(len(ci))
    x = rng.uniform(-1, 1, ncols)
    T = csr_to_csr5(_csr(rp.astype(itype), ci.astype(itype), v.astype(vtype), ncols))
    y = _spmv(SpOps_csr5, T, x.astype(vtype), 0.8, 0.7, np.ones(n, vtype))
    if vtype == np.float64:
        _check(orc, rp, ci, v, x, y)
    else:
        v32, x32 = v.astype(np.float32).astype(np.float64), x.astype(np.float32).astype(np.float64)
        yref = orc.spmv_csr(rp, ci, v32, x32, 0.8, 0.7, np.ones(n))
        den = 0.8 * orc.absdot(rp, ci, v32, x32) + 0.7
        assert (np.abs(y - yref) / den).max() <= 1e-5


def test_csr5_powerlaw_full(cuda, orc):
    from sparseops_b200 import SpOps_csr5, csr_to_csr5
    n = 4194304
    rp, ci, v = synth.powerlaw(n, mu=math.log(12.0), sigma=1.2, lo=1, hi=20000, seed=1)
    x = synth.uniform(n, 1)
    T = csr_to_csr5(_csr(rp, ci, v))
    _check(orc, rp, ci, v, x, _spmv(SpOps_csr5, T, x, 1.0, 0.0), 1.0, 0.0)


@pytest.mark.parametrize("compact", [0, 1])
def test_coo_to_csr_golden_device(cuda, golden, compact):
    """Device coo_to_csr against the reference's own output, bit for bit."""
    import torch
    from sparseops_b200 import COO_Matrix, coo_to_csr
    n, nc = (int(t) for t in golden["coo_shape"])
    coo = COO_Matrix(n, nc, _dev(golden["coo_ri"]), _dev(golden["coo_ci"]), _dev(golden["coo_v"]))
    C = coo_to_csr(coo, bool(compact))
    torch.cuda.synchronize()
    rp, ci, v = C.host()
    assert np.array_equal(rp, golden[f"coo_rp{compact}"])
    assert np.array_equal(ci, golden[f"coo_csr_ci{compact}"])
    assert np.array_equal(v, golden[f"coo_csr_v{compact}"])


@pytest.mark.parametrize("itype,vtype", [(np.int32, np.float64), (np.int64, np.float32), (np.int32, np.float32)])
@pytest.mark.parametrize("compact", [False, True])
def test_coo_to_csr_vs_oracle(cuda, orc, itype, vtype, compact):
    """Random file order with duplicates, exact cancellations, empty rows, a
    long row; also an already row-sorted COO (its arrays are borrowed by the
    view, the result must still own copies) and an empty matrix."""
    import torch
    from sparseops_b200 import COO_Matrix, SpOps_csr, coo_to_csr
    rng = np.random.default_rng(5)
    n, nc, m = 5000, 3000, 120000
    ri = rng.integers(0, n, m)
    ri[:20000] = 17  # a long row with many duplicates
    ri[(ri >= 100) & (ri < 400)] = 99  # rows 100..399 empty
    ci = rng.integers(0, nc, m)
    v = (rng.integers(-4, 5, m) * 0.5).astype(vtype)
    for order in ("file", "sorted"):
        if order == "sorted":
            p = np.argsort(ri, kind="stable")
            ri, ci, v = ri[p], ci[p], v[p]
        coo = COO_Matrix(n, nc, _dev(ri.astype(itype)), _dev(ci.astype(itype)), _dev(v))
        C = coo_to_csr(coo, compact)
        rp, oc, ov = C.host()
        erp, eci, ev = orc.coo_to_csr(n, ri, ci, v, compact)
        assert np.array_equal(rp.astype(np.int64), erp) and np.array_equal(oc.astype(np.int64), eci)
        assert ov.dtype == vtype and np.array_equal(ov, ev)
        del coo  # the result owns its arrays
        x = torch.ones(nc, dtype=torch.float64 if vtype == np.float64 else torch.float32, device="cuda")
        y = torch.zeros(n, dtype=x.dtype, device="cuda")
        SpOps_csr(1.0, C, x, 0.0, y)
        torch.cuda.synchronize()
        ref = np.add.reduceat(np.concatenate([ev, [0]]).astype(np.float64), erp[:-1]) * (np.diff(erp) > 0)
        assert np.allclose(y.cpu().numpy(), ref, rtol=1e-5, atol=1e-5)
    empty = coo_to_csr(COO_Matrix(7, 3, _dev(np.zeros(0, itype)), _dev(np.zeros(0, itype)), _dev(np.zeros(0, vtype))),
                       compact)
    rp, oc, ov = empty.host()
    assert np.array_equal(rp, np.zeros(8)) and len(oc) == 0


@pytest.mark.parametrize("itype", [np.int32, np.int64])
@pytest.mark.parametrize("vtype", [np.float64, np.float32])
def test_csr_reorder_rows(cuda, itype, vtype):
    """csr_reorder_rows (include/sparse_conversion.h:1879): row i of the
    result is row perm[i] of the input, entries copied in order; empty rows
    kept; a non-permutation is refused."""
    from sparseops_b200 import SpOpsError, csr_reorder_rows
    rp, ci, v = synth.powerlaw(20000, hi=500, seed=44)
    lens = np.diff(rp)
    lens[::7] = 0  # empty rows
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(itype)
    ci = ci[:int(rp[-1])].astype(itype)
    v = v[:int(rp[-1])].astype(vtype)
    n = len(rp) - 1
    A = _csr(rp, ci, v, n)
    perm = np.random.default_rng(3).permutation(n)
    R = csr_reorder_rows(A, perm)
    rrp, rci, rv = R.host()
    exp_lens = lens[perm]
    assert np.array_equal(np.diff(rrp.astype(np.int64)), exp_lens)
    starts = rp[perm].astype(np.int64)
    idx = np.concatenate([np.arange(s, s + L) for s, L in zip(starts, exp_lens)]) if exp_lens.sum() else np.zeros(0, int)
    assert np.array_equal(rci.astype(np.int64), ci[idx].astype(np.int64))
    assert np.array_equal(rv, v[idx])
    bad = perm.copy()
    bad[5] = bad[6]  # a repeated row
    with pytest.raises(SpOpsError):
        csr_reorder_rows(A, bad)
    bad = perm.copy()
    bad[0] = n  # out of range
    with pytest.raises(SpOpsError):
        csr_reorder_rows(A, bad)
