"""Batched SpMV / SpMM in one persistent launch, and single-matrix SpMM.

Uneven matrices on the banded-plus-random pattern (half the draws within
bandwidth 64, half uniform, Poisson(16) per row), k in {1, 8, 32}
right-hand sides; every output against the oracle (componentwise 1e-12).
"""
import numpy as np
import pytest

from sparseops_b200 import synth

pytestmark = pytest.mark.gpu


def _mats(count, seed=0, long_row=False):
    rng = np.random.default_rng(seed)
    out = []
    for m in range(count):
        n = int(np.exp(rng.uniform(np.log(1000), np.log(20000))))
        rp, ci, v = synth.banded_random(n, 16.0, 64, seed=1000 + m)
        if long_row and m == 1:  # one dense-ish row to exercise the long-row path
            rows = [ci[rp[r]:rp[r + 1]] for r in range(n)]
            rows[3] = np.arange(0, n, 2, dtype=np.int32)
            lens = np.array([len(r) for r in rows])
            rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
            ci = np.concatenate(rows).astype(np.int32)
            v = synth.normal(len(ci), 77)
        out.append((rp, ci, v))
    return out


def _err(orc, rp, ci, v, X, Y, Yref, alpha, beta, Y0):
    absA = (np.abs(v), np.abs(X))
    den = abs(alpha) * orc.spmm_csr(rp, ci, absA[0], absA[1]) + np.abs(beta * Y0)
    return (np.abs(Y - Yref) / np.maximum(den, 1e-300)).max()


@pytest.mark.parametrize("k", [1, 8, 16, 32])
@pytest.mark.parametrize("tune", [False, True])
def test_batch_matches_oracle(cuda, orc, k, tune):
    import torch
    from sparseops_b200 import Batch, CSR_Matrix
    mats = _mats(24, seed=k, long_row=True)
    dev = torch.device("cuda")
    A = [CSR_Matrix(len(rp) - 1, len(rp) - 1, torch.from_numpy(rp).to(dev), torch.from_numpy(ci).to(dev),
                    torch.from_numpy(v).to(dev)) for rp, ci, v in mats]
    Xs = [synth.uniform((len(rp) - 1) * k, 100 + i).reshape(-1, k) for i, (rp, _, _) in enumerate(mats)]
    Y0 = [synth.uniform((len(rp) - 1) * k, 200 + i).reshape(-1, k) for i, (rp, _, _) in enumerate(mats)]
    X = [torch.from_numpy(x).to(dev) for x in Xs]
    Y = [torch.from_numpy(y.copy()).to(dev) for y in Y0]
    if k == 1:
        X = [x.reshape(-1) for x in X]
        Y = [y.reshape(-1) for y in Y]
    B = Batch(A, k=k)
    B.set_vectors(X, Y)
    if tune:
        B.tune()
        for y, y0 in zip(Y, Y0):  # the tuner wrote into Y: restore it
            y.copy_(torch.from_numpy(y0.reshape(y.shape)))
    B.run(0.8, 0.7)
    torch.cuda.synchronize()
    items, choice, kt = B.info()
    assert items > 0 and len(choice) == len(mats)
    for (rp, ci, v), x, y, y0 in zip(mats, Xs, Y, Y0):
        ref = orc.spmm_csr(rp, ci, v, x, 0.8, 0.7, y0)
        got = y.cpu().numpy().reshape(ref.shape)
        assert _err(orc, rp, ci, v, x, got, ref, 0.8, 0.7, y0) <= 1e-12


def test_band_staging_gives_the_same_bits(cuda, orc):
    """The "batch_band" option (x windows of banded CSR segments staged in
    shared memory) changes where x is read from, not the products or their
    order: the same bits as plain gathers, and within 1e-12 of the oracle."""
    import torch
    from sparseops_b200 import Batch, CSR_Matrix, default_context
    mats = _mats(20, seed=41, long_row=True)
    dev = torch.device("cuda")
    ctx = default_context()
    Xs = [synth.uniform(len(rp) - 1, 500 + i) for i, (rp, _, _) in enumerate(mats)]
    out = []
    try:
        for band in (0, 1):
            ctx.set_option("batch_band", band)
            A = [CSR_Matrix(len(rp) - 1, len(rp) - 1, torch.from_numpy(rp).to(dev), torch.from_numpy(ci).to(dev),
                            torch.from_numpy(v).to(dev)) for rp, ci, v in mats]
            X = [torch.from_numpy(x).to(dev) for x in Xs]
            Y = [torch.zeros(len(rp) - 1, dtype=torch.float64, device=dev) for rp, _, _ in mats]
            B = Batch(A, k=1)
            B.set_vectors(X, Y)
            B.run(1.0, 0.0)
            torch.cuda.synchronize()
            out.append([y.cpu().numpy() for y in Y])
    finally:
        ctx.set_option("batch_band", 0)
    for (rp, ci, v), x, y0, y1 in zip(mats, Xs, out[0], out[1]):
        assert np.array_equal(y0.view(np.uint64), y1.view(np.uint64))
        ref = orc.spmm_csr(rp, ci, v, x.reshape(-1, 1)).reshape(-1)
        den = orc.spmm_csr(rp, ci, np.abs(v), np.abs(x).reshape(-1, 1)).reshape(-1)
        assert (np.abs(y1 - ref) / np.maximum(den, 1e-300)).max() <= 1e-12


def test_graph_capture_replay(cuda, orc):
    import torch
    from sparseops_b200 import Batch, CSR_Matrix
    mats = _mats(16, seed=5)
    dev = torch.device("cuda")
    A = [CSR_Matrix(len(rp) - 1, len(rp) - 1, torch.from_numpy(rp).to(dev), torch.from_numpy(ci).to(dev),
                    torch.from_numpy(v).to(dev)) for rp, ci, v in mats]
    Xs = [synth.uniform(len(rp) - 1, 300 + i) for i, (rp, _, _) in enumerate(mats)]
    X = [torch.from_numpy(x).to(dev) for x in Xs]
    Y = [torch.zeros(len(rp) - 1, dtype=torch.float64, device=dev) for rp, _, _ in mats]
    B = Batch(A, k=1)
    B.set_vectors(X, Y)
    B.capture(1.0, 0.0)
    for y in Y:
        y.zero_()
    for _ in range(3):
        B.run(1.0, 0.0)  # graph replay
    torch.cuda.synchronize()
    for (rp, ci, v), x, y in zip(mats, Xs, Y):
        ref = orc.spmv_csr(rp, ci, v, x)
        assert (np.abs(y.cpu().numpy() - ref) / orc.absdot(rp, ci, v, x)).max() <= 1e-12


@pytest.mark.parametrize("k", [3, 8, 16, 32, 40])
def test_single_spmm(cuda, orc, k):
    import torch
    from sparseops_b200 import CSR_Matrix, SpMM_csr
    rp, ci, v = synth.powerlaw(30000, hi=3000, seed=31)
    n = len(rp) - 1
    X = synth.uniform(n * k, 9).reshape(n, k)
    Y0 = synth.uniform(n * k, 10).reshape(n, k)
    dev = torch.device("cuda")
    A = CSR_Matrix(n, n, torch.from_numpy(rp).to(dev), torch.from_numpy(ci).to(dev), torch.from_numpy(v).to(dev))
    Xd, Yd = torch.from_numpy(X).to(dev), torch.from_numpy(Y0.copy()).to(dev)
    SpMM_csr(0.8, A, Xd, 0.7, Yd)
    torch.cuda.synchronize()
    ref = orc.spmm_csr(rp, ci, v, X, 0.8, 0.7, Y0)
    assert _err(orc, rp, ci, v, X, Yd.cpu().numpy(), ref, 0.8, 0.7, Y0) <= 1e-12


@pytest.mark.parametrize("case", ["empty_rows", "int64", "f32", "wide_ld", "misaligned", "beta0_nan"])
def test_spmm8_tiles(cuda, orc, case):
    """k = 8 runs on the SpMV's tile plan (register sums per lane, 32-byte X-row
    gathers): empty rows (tiles that span them), a long row over many tiles,
    int64 indices, FP32, a row stride wider than 8, beta = 0 over NaN, and a
    misaligned X (the segment kernel then runs); every case against the
    oracle, and two runs bit-identical."""
    import torch
    from sparseops_b200 import CSR_Matrix, SpMM_csr
    rng = np.random.default_rng(41)
    n, k = 40000, 8
    lens = rng.poisson(12, n)
    lens[rng.random(n) < 0.1] = 0
    lens[7] = 5000
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    ci = rng.integers(0, n, int(rp[-1])).astype(np.int32)
    v = rng.standard_normal(len(ci))
    dt, tol = (np.float32, 1e-5) if case == "f32" else (np.float64, 1e-12)
    if case == "int64":
        rp, ci = rp.astype(np.int64), ci.astype(np.int64)
    ld = 12 if case == "wide_ld" else k
    Xfull = rng.standard_normal((n + 1, ld)).astype(dt)
    Y0 = rng.standard_normal((n, ld)).astype(dt)
    dev = torch.device("cuda")
    A = CSR_Matrix(n, n, torch.from_numpy(rp).to(dev), torch.from_numpy(ci).to(dev),
                   torch.from_numpy(v.astype(dt)).to(dev))
    Xd_full = torch.from_numpy(Xfull).to(dev)
    if case == "misaligned":  # X starts one element after a 32-byte boundary
        flat = torch.from_numpy(np.concatenate([[0.0], Xfull[:n].ravel()]).astype(dt)).to(dev)
        Xd = flat[1:].view(n, ld)
    else:
        Xd = Xd_full[:n, :k] if ld != k else Xd_full[:n]
    X = Xd.cpu().numpy()
    beta = 0.0 if case == "beta0_nan" else 0.7
    outs = []
    for _ in range(2):
        Yfull = torch.from_numpy(Y0.copy()).to(dev)
        if case == "beta0_nan":
            Yfull[:, :k] = float("nan")
        Yd = Yfull[:, :k]
        SpMM_csr(0.8, A, Xd, beta, Yd)
        torch.cuda.synchronize()
        outs.append(Yfull.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])
    Y = outs[0][:, :k].astype(np.float64)
    if ld != k:
        assert np.array_equal(outs[0][:, k:], Y0[:, k:])  # columns past k untouched
    rp32, ci32 = rp.astype(np.int32), ci.astype(np.int32)  # the oracle's SpMM takes int32 indices
    Y0k = Y0[:, :k].astype(np.float64)
    ref = orc.spmm_csr(rp32, ci32, v.astype(dt).astype(np.float64), X.astype(np.float64), 0.8, beta, Y0k)
    assert _err(orc, rp32, ci32, v.astype(dt).astype(np.float64), X.astype(np.float64), Y, ref, 0.8, beta,
                Y0k) <= tol


def test_batch_k8_tiles_mixed_and_replayed(cuda, orc):
    """k = 8: matrices whose X rows allow 32-byte gathers run as register-tile
    items (with one calibration launch for all of them); every other matrix
    has a misaligned X and stays on segment items in the same run.  Direct
    run, tuned run and graph replay all against the oracle; replays
    bit-identical."""
    import torch
    from sparseops_b200 import Batch, CSR_Matrix
    k = 8
    mats = _mats(8, seed=5, long_row=True)
    dev = torch.device("cuda")
    A = [CSR_Matrix(len(rp) - 1, len(rp) - 1, torch.from_numpy(rp).to(dev), torch.from_numpy(ci).to(dev),
                    torch.from_numpy(v).to(dev)) for rp, ci, v in mats]
    Xs, Ys, Y0s, keep = [], [], [], []
    for m, (rp, ci, v) in enumerate(mats):
        n = len(rp) - 1
        X = synth.uniform(n * k, 300 + m).reshape(n, k)
        if m % 2:  # misaligned: one element past a 32-byte boundary
            buf = torch.zeros(n * k + 1, dtype=torch.float64, device=dev)
            buf[1:] = torch.from_numpy(X.ravel()).to(dev)
            Xd = buf[1:].view(n, k)
            keep.append(buf)
        else:
            Xd = torch.from_numpy(X).to(dev)
        Xs.append(Xd)
        Y0 = synth.uniform(n * k, 400 + m).reshape(n, k)
        Y0s.append(Y0)
        Ys.append(torch.from_numpy(Y0.copy()).to(dev))
    B = Batch(A, k=k)
    B.set_vectors(Xs, Ys)
    B.run(0.8, 0.7)
    torch.cuda.synchronize()
    for (rp, ci, v), Xd, Yd, Y0 in zip(mats, Xs, Ys, Y0s):
        X = Xd.cpu().numpy()
        ref = orc.spmm_csr(rp, ci, v, X, 0.8, 0.7, Y0)
        assert _err(orc, rp, ci, v, X, Yd.cpu().numpy(), ref, 0.8, 0.7, Y0) <= 1e-12
    B.tune()
    B.capture(1.0, 0.0)
    outs = []
    for _ in range(2):
        for Yd in Ys:
            Yd.fill_(float("nan"))  # beta = 0: never read
        B.run(1.0, 0.0)  # replays the captured graph
        torch.cuda.synchronize()
        outs.append([Yd.cpu().numpy().copy() for Yd in Ys])
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a, b)
    for (rp, ci, v), Xd, Y in zip(mats, Xs, outs[0]):
        X = Xd.cpu().numpy()
        ref = orc.spmm_csr(rp, ci, v, X)
        assert _err(orc, rp, ci, v, X, Y, ref, 1.0, 0.0, np.zeros_like(Y)) <= 1e-12
