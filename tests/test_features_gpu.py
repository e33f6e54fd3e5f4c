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
