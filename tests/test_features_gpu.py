"""Device structure features and the format selector.

Features: against the reference's own MtxLoad + CalculateFeatures (golden
fixtures) and the oracle restatement; integer features exact, the others to
1e-12 relative (the device sums in a different order).  Selector: the rules
pick DIA for a few dense diagonals and CSR otherwise; the timed mode returns
one of its candidates; SpOps_auto gives the oracle's y (1e-12)."""
import numpy as np
import pytest

from sparseops_b200 import synth

pytestmark = pytest.mark.gpu


def _csr(rp, ci, v, nc):
    import torch
    from sparseops_b200 import CSR_Matrix
    d = torch.device("cuda")
    return CSR_Matrix(len(rp) - 1, nc, torch.from_numpy(np.ascontiguousarray(rp)).to(d),
                      torch.from_numpy(np.ascontiguousarray(ci)).to(d), torch.from_numpy(np.ascontiguousarray(v)).to(d))


def _vec(f):
    from sparseops_b200._lib import FEATURE_NAMES
    return np.array([float(f[n]) for n in FEATURE_NAMES])


def _close(got, ref):
    assert np.array_equal(got[:11], ref[:11]), (got[:11], ref[:11])
    both_nan = np.isnan(got) & np.isnan(ref)
    rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)
    ok = both_nan | (rel <= 1e-12) | (got == ref)
    assert ok.all(), [(i, got[i], ref[i]) for i in np.where(~ok)[0]]


@pytest.mark.parametrize("k", [0, 1, 2])
def test_features_golden(cuda, golden, k):
    from sparseops_b200 import matrix_features
    A = _csr(golden[f"feat{k}_rp"], golden[f"feat{k}_ci"], golden[f"feat{k}_v"], int(golden[f"feat{k}_nc"]))
    _close(_vec(matrix_features(A)), golden[f"feat{k}_out"])


@pytest.mark.parametrize("case", ["powerlaw", "laplacian", "graph", "f32", "i64"])
def test_features_vs_oracle(cuda, orc, case):
    from sparseops_b200 import matrix_features
    if case == "powerlaw":
        rp, ci, v = synth.powerlaw(100000, hi=5000, seed=12)
    elif case == "laplacian":
        rp, ci, v = synth.laplacian_2d(256)
    elif case in ("graph", "f32"):
        rp, ci, v = synth.symmetric_graph(50000, 16.0, seed=6)
    else:
        rp, ci, v = synth.powerlaw(30000, hi=2000, seed=13)
        rp, ci = rp.astype(np.int64), ci.astype(np.int64)
    nc = len(rp) - 1
    vv = v.astype(np.float32) if case == "f32" else v
    got = _vec(matrix_features(_csr(rp, ci, vv, nc)))
    ref = orc.features(rp.astype(np.int64), ci.astype(np.int64), vv.astype(np.float64), nc)
    _close(got, ref)


def _partly_symmetric(n, seed):
    """Random pattern where about half the off-diagonal entries have a mirror;
    mirror values equal, equal to six decimals, of the other sign, or
    different; a diagonal entry in some rows.  Rows sorted by column."""
    rng = np.random.default_rng(seed)
    m = 8 * n
    r = rng.integers(0, n, m)
    c = rng.integers(0, n, m)
    v = rng.standard_normal(m)
    mir = rng.random(m) < 0.5
    kind = rng.integers(0, 4, m)
    mv = np.where(kind == 0, v, np.where(kind == 1, v + 1e-9, np.where(kind == 2, -v, v + 0.5)))
    d = rng.integers(0, n, n // 3)
    R = np.concatenate([r, c[mir], d])
    Cc = np.concatenate([c, r[mir], d])
    V = np.concatenate([v, mv[mir], rng.standard_normal(len(d))])
    key = R.astype(np.int64) * n + Cc
    key, first = np.unique(key, return_index=True)  # one entry per (row, col)
    R, Cc, V = key // n, key % n, V[first]
    rp = np.concatenate([[0], np.cumsum(np.bincount(R, minlength=n))]).astype(np.int32)
    return rp, Cc.astype(np.int32), V


def test_symmetry_both_paths(cuda, orc):
    """pattern_symm and value_symm by each of the three counts: ascending rows
    on a fresh handle (row by row on the CSR's own arrays), the same rows
    shuffled (sorted (row, col) keys), and ascending rows once the tile
    features have left a transpose pattern on the handle (column by column
    over it).  All three give the oracle's values exactly."""
    import torch
    from sparseops_b200 import matrix_features, matrix_tile_features
    from sparseops_b200._lib import FEATURE_NAMES
    n = 6000
    rp, ci, v = _partly_symmetric(n, seed=21)
    rng = np.random.default_rng(22)
    ci_u, v_u = ci.copy(), v.copy()
    for r in range(n):  # shuffle every row's entries: the unsorted path
        s, e = rp[r], rp[r + 1]
        p = s + rng.permutation(e - s)
        ci_u[s:e], v_u[s:e] = ci[p], v[p]
    assert any(np.any(np.diff(ci_u[rp[r]:rp[r + 1]]) < 0) for r in range(n))
    iP, iV = FEATURE_NAMES.index("pattern_symm"), FEATURE_NAMES.index("value_symm")
    A = _csr(rp, ci, v, n)
    got_s = _vec(matrix_features(A))
    got_u = _vec(matrix_features(_csr(rp, ci_u, v_u, n)))
    matrix_tile_features(A, 256)  # builds and keeps the transpose on the handle
    torch.cuda.synchronize()
    got_c = _vec(matrix_features(A))
    ref = orc.features(rp.astype(np.int64), ci.astype(np.int64), v, n)
    assert 0.2 < ref[iP] < 0.9 and 0.0 < ref[iV] < ref[iP]
    for got in (got_s, got_u, got_c):
        assert got[iP] == ref[iP] and got[iV] == ref[iV], (got[iP], got[iV], ref[iP], ref[iV])
    _close(got_s, ref)
    _close(got_c, ref)


def test_select_rules(cuda):
    from sparseops_b200 import select_format
    rp, ci, v = synth.laplacian_2d(200)
    assert select_format(_csr(rp, ci, v, len(rp) - 1))["format"] == "dia"
    rp, ci, v = synth.powerlaw(50000, hi=3000, seed=3)
    assert select_format(_csr(rp, ci, v, len(rp) - 1))["format"] == "csr"


@pytest.mark.parametrize("timed", [False, True])
def test_spops_auto(cuda, orc, timed):
    import torch
    from sparseops_b200 import SpOps_auto, select_format
    for rp, ci, v in (synth.laplacian_2d(300), synth.powerlaw(80000, hi=4000, seed=8)):
        n = len(rp) - 1
        A = _csr(rp, ci, v, n)
        choice = select_format(A, timed)
        assert choice["format"] in ("csr", "sell_c_R", "sell_c_sigma", "csr5", "dia")
        if timed:
            assert choice["ms"] > 0
        x = synth.uniform(n, 4)
        y0 = synth.uniform(n, 5)
        xd = torch.from_numpy(x).cuda()
        yd = torch.from_numpy(y0.copy()).cuda()
        SpOps_auto(0.8, A, xd, 0.7, yd, timed)
        torch.cuda.synchronize()
        ref = orc.spmv_csr(rp, ci, v, x, 0.8, 0.7, y0)
        den = 0.8 * orc.absdot(rp, ci, v, x) + np.abs(0.7 * y0)
        assert (np.abs(yd.cpu().numpy() - ref) / den).max() <= 1e-12


# ---------------------------------------------------------------- tile features
def _tile_parts(f, arrays):
    """The device result in the layout of the oracle / golden tuples."""
    from sparseops_b200._lib import TILE_FEATURE_NAMES
    sc = np.array([float(f[n]) for n in TILE_FEATURE_NAMES])
    ti = np.stack([arrays[n].ravel() for n in ("tile_nnz", "tile_rows", "tile_cols", "tile_max_row_nnz")])
    td = np.stack([arrays[n].ravel() for n in ("tile_ave_row_nnz", "tile_std_row_nnz")])
    bi = np.stack([arrays[n] for n in ("rb_nnz", "rb_max_row_nnz", "cb_nnz", "cb_max_col_nnz")])
    bd = np.stack([arrays[n] for n in ("rb_ave_row_nnz", "rb_std_row_nnz", "cb_ave_col_nnz", "cb_std_col_nnz")])
    return sc, ti, td, bi, bd


def _tile_close(got, ref):
    """Integers exact, floating-point values to 1e-12 relative, except the
    variances (and deviations) of the tile, RB and CB counts: the reference
    adds the len squared deviations one after another, so its own result is
    only known to the bound of recursive summation, (len - 1) * 2^-53 times
    the sum, which for 65,536 or 1,048,576 tiles is above 1e-12; the device
    sums in a tree.  Those three pairs are held to that bound."""
    sc_g, sc_r = np.asarray(got[0], np.float64), np.asarray(ref[0], np.float64)
    B = int(sc_r[0])
    spread = {}
    for var_i, std_i, L in ((13, 14, B * B), (19, 20, B), (25, 26, B)):
        total = sc_r[var_i] * L + 1.0  # the sum of squared deviations
        tol = max(1e-12 * abs(sc_r[var_i]), (L - 1) * 2.0 ** -53 * total / L + 1e-300)
        assert abs(sc_g[var_i] - sc_r[var_i]) <= tol, (var_i, sc_g[var_i], sc_r[var_i], tol)
        assert abs(sc_g[std_i] ** 2 - sc_r[std_i] ** 2) <= tol + 1e-12 * sc_r[std_i] ** 2, (std_i, sc_g[std_i],
                                                                                         sc_r[std_i])
        spread.update({var_i: True, std_i: True})
    keep = np.array([i not in spread for i in range(len(sc_r))])
    for g, r, name in zip((sc_g[keep],) + tuple(got[1:]), (sc_r[keep],) + tuple(ref[1:]),
                          ("sc", "ti", "td", "bi", "bd")):
        g, r = np.asarray(g).reshape(r.shape), np.asarray(r)
        if name == "sc":
            assert np.array_equal(g[:11], r[:11]), (g[:11], r[:11])
        if r.dtype == np.int64:
            assert np.array_equal(g, r), name
            continue
        rel = np.abs(g - r) / np.maximum(np.abs(r), 1e-300)
        ok = (rel <= 1e-12) | (g == r) | (np.isnan(g) & np.isnan(r))
        assert ok.all(), (name, np.argwhere(~ok)[:5].ravel(), g[~ok][:5], r[~ok][:5])


@pytest.mark.parametrize("k", [0, 1, 2, 3])
def test_tile_features_golden(cuda, golden, k):
    """Against the reference's own MtxLoad + CalculateFeatures +
    CalculateTilesExtraFeatures on its 256 x 256 grid: integers exact,
    floating-point values to 1e-12 (the device sums in another order)."""
    from sparseops_b200 import matrix_tile_features
    from test_oracle_golden import tile_case
    rp, ci, nc = tile_case(golden, k)
    f, arrays = matrix_tile_features(_csr(rp, ci, np.ones(len(ci)), nc), maps=True)
    ref = tuple(golden[f"tile{k}_{s}"] for s in ("sc", "ti", "td", "bi", "bd"))
    _tile_close(_tile_parts(f, arrays), ref)


@pytest.mark.parametrize("case,B", [("powerlaw", 256), ("laplacian", 256), ("graph", 256), ("narrow", 256),
                                    ("i64", 256), ("powerlaw", 64), ("graph", 1024), ("powerlaw", 2048)])
def test_tile_features_vs_oracle(cuda, orc, case, B):
    """Against the oracle on larger matrices, other grid sizes (64 .. 2048
    tiles per side), int64 indices and a matrix with fewer rows than tiles."""
    from sparseops_b200 import matrix_tile_features
    if case == "powerlaw":
        rp, ci, v = synth.powerlaw(60000, hi=4000, seed=22)
        nc = len(rp) - 1
    elif case == "laplacian":
        rp, ci, v = synth.laplacian_2d(300)
        nc = len(rp) - 1
    elif case == "graph":
        rp, ci, v = synth.symmetric_graph(40000, 12.0, seed=7)
        nc = len(rp) - 1
    elif case == "narrow":  # 100 rows: every row block but the first 100 is empty
        rng = np.random.default_rng(4)
        lens = rng.integers(0, 300, 100)
        rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
        ci = rng.integers(0, 70000, int(rp[-1])).astype(np.int32)
        v, nc = np.ones(len(ci)), 70000
    else:
        rp, ci, v = synth.powerlaw(30000, hi=2000, seed=13)
        rp, ci = rp.astype(np.int64), ci.astype(np.int64)
        nc = len(rp) - 1
    f, arrays = matrix_tile_features(_csr(rp, ci, v, nc), num_blocks=B, maps=True)
    _tile_close(_tile_parts(f, arrays), orc.tile_features(rp.astype(np.int64), ci.astype(np.int64), nc, B))


def test_tile_features_refusals(cuda):
    from sparseops_b200 import SpOpsError, matrix_tile_features
    rp, ci, v = synth.laplacian_2d(20)
    with pytest.raises(SpOpsError) as e:
        matrix_tile_features(_csr(rp, ci, v, len(rp) - 1), num_blocks=4096)
    assert e.value.status == 5
