"""CSR SpMV on the device vs the oracle (and the reference's golden outputs).

Error metric (FP64): componentwise |y - y_ref| / (sum_j |a_ij x_j| + |beta*y0_i|),
bound 1e-12.  FP32 values/accumulation: bound 1e-5 on the same metric.
"""
import numpy as np
import pytest

from sparseops_b200 import synth

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 1e-5


def _run(rp, ci, v, x, alpha=1.0, beta=0.0, y0=None, ncols=None, dev="cuda"):
    import torch
    from sparseops_b200 import CSR_Matrix, SpOps_csr
    n = len(rp) - 1
    ncols = len(x) if ncols is None else ncols
    A = CSR_Matrix(n, ncols, torch.from_numpy(rp).to(dev), torch.from_numpy(ci).to(dev), torch.from_numpy(v).to(dev))
    xd = torch.from_numpy(x).to(dev)
    yd = torch.from_numpy(y0.copy()).to(dev) if y0 is not None else torch.full((n,), float("nan"), dtype=xd.dtype,
                                                                                device=dev)
    SpOps_csr(alpha, A, xd, beta, yd)
    torch.cuda.synchronize()
    return yd.cpu().numpy(), A


def _err(orc, rp, ci, v, x, y, yref, beta=0.0, y0=None, alpha=1.0):
    den = abs(alpha) * orc.absdot(rp, ci, v, x)
    if y0 is not None:
        den = den + np.abs(beta * y0)
    return (np.abs(y - yref) / np.maximum(den, 1e-300)).max() if len(y) else 0.0


@pytest.mark.parametrize("name", ["lap", "pl"])
def test_golden_reference_outputs(cuda, golden, orc, name):
    g = golden
    rp, ci, v, x, y0 = g[f"{name}_rp"], g[f"{name}_ci"], g[f"{name}_v"], g[f"{name}_x"], g[f"{name}_y0"]
    y, _ = _run(rp, ci, v, x, 0.8, 0.7, y0)
    assert _err(orc, rp, ci, v, x, y, g[f"{name}_y"], 0.7, y0) <= TOL64


def test_laplacian_512_full_config(cuda, orc):
    rp, ci, v = synth.laplacian_2d(512)
    x = synth.uniform(len(rp) - 1, 0)
    y, _ = _run(rp, ci, v, x)
    assert _err(orc, rp, ci, v, x, y, orc.spmv_csr(rp, ci, v, x)) <= TOL64


@pytest.mark.parametrize("alpha,beta", [(1.0, 0.0), (0.8, 0.7), (-2.0, 1.0), (0.0, 0.5), (1.0, -1.0)])
def test_alpha_beta(cuda, orc, alpha, beta):
    rp, ci, v = synth.powerlaw(20000, hi=5000, seed=21)
    n = len(rp) - 1
    x, y0 = synth.uniform(n, 1), synth.uniform(n, 2)
    y, _ = _run(rp, ci, v, x, alpha, beta, y0)
    yref = orc.spmv_csr(rp, ci, v, x, alpha, beta, y0)
    assert _err(orc, rp, ci, v, x, y, yref, beta, y0, alpha) <= TOL64


def test_beta_zero_ignores_nan_y(cuda, orc):
    rp, ci, v = synth.powerlaw(5000, seed=22)
    x = synth.uniform(5000, 3)
    y, _ = _run(rp, ci, v, x, 1.5, 0.0, None)  # y starts as NaN
    assert np.isfinite(y).all()
    assert _err(orc, rp, ci, v, x, y, orc.spmv_csr(rp, ci, v, x, 1.5, 0.0), alpha=1.5) <= TOL64


def test_long_rows_and_empty_rows(cuda, orc):
    """Rows longer than one chunk (multi-block path), runs of > 1024 empty rows,
    and a row exactly at the chunk boundary."""
    rng = np.random.default_rng(5)
    n, ncols = 9000, 300000
    lens = rng.integers(0, 40, n)
    lens[100] = 100000      # many chunks
    lens[101] = 2048        # exactly one chunk
    lens[102] = 2049        # just over
    lens[2000:4500] = 0     # long empty run
    lens[n - 1] = 70000     # long last row
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    ci = np.concatenate([np.sort(rng.choice(ncols, L, replace=False)) for L in lens]).astype(np.int32)
    v = rng.standard_normal(len(ci))
    x = rng.uniform(-1, 1, ncols)
    rp = rp.astype(np.int32)
    y, _ = _run(rp, ci, v, x, 0.8, 0.7, np.ones(n))
    yref = orc.spmv_csr(rp, ci, v, x, 0.8, 0.7, np.ones(n))
    assert _err(orc, rp, ci, v, x, y, yref, 0.7, np.ones(n), 0.8) <= TOL64


def test_deterministic(cuda):
    rp, ci, v = synth.powerlaw(100000, seed=23)
    x = synth.uniform(100000, 4)
    y1, A = _run(rp, ci, v, x)
    y2, _ = _run(rp, ci, v, x)
    assert np.array_equal(y1, y2)


def test_int64_indices(cuda, orc):
    rp, ci, v = synth.powerlaw(30000, seed=24)
    x = synth.uniform(30000, 5)
    y, _ = _run(rp.astype(np.int64), ci.astype(np.int64), v, x, 0.8, 0.7, np.ones(30000))
    yref = orc.spmv_csr(rp, ci, v, x, 0.8, 0.7, np.ones(30000))
    assert _err(orc, rp, ci, v, x, y, yref, 0.7, np.ones(30000)) <= TOL64


def test_float32(cuda, orc):
    rp, ci, v = synth.powerlaw(30000, seed=25)
    x = synth.uniform(30000, 6)
    v32, x32 = v.astype(np.float32), x.astype(np.float32)
    y, _ = _run(rp, ci, v32, x32)
    yref = orc.spmv_csr(rp, ci, v32, x32)
    assert _err(orc, rp, ci, v32.astype(np.float64), x32.astype(np.float64), y.astype(np.float64), yref) <= TOL32


def test_empty_matrices(cuda):
    # no rows
    y, _ = _run(np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0), np.zeros(5))
    assert y.shape == (0,)
    # rows but no entries: y = beta*y0
    n = 3000
    y, _ = _run(np.zeros(n + 1, np.int32), np.zeros(0, np.int32), np.zeros(0), np.zeros(7), 1.0, 0.5, np.ones(n))
    assert np.array_equal(y, np.full(n, 0.5))


def test_host_vectors(cuda, orc):
    """numpy x / y: the host path (spops_spmv_host) uploads x and downloads y."""
    from sparseops_b200 import CSR_Matrix, SpOps_csr
    rp, ci, v = synth.powerlaw(40000, seed=26)
    x, y0 = synth.uniform(40000, 7), synth.uniform(40000, 8)
    A = CSR_Matrix(40000, 40000, rp, ci, v)
    y = y0.copy()
    SpOps_csr(0.8, A, x, 0.7, y)
    yref = orc.spmv_csr(rp, ci, v, x, 0.8, 0.7, y0)
    assert _err(orc, rp, ci, v, x, y, yref, 0.7, y0) <= TOL64


def test_powerlaw_full_config(cuda, orc):
    """Power-law config at full size: n = 4,194,304, lognormal(ln 12, 1.2) rows."""
    import math
    n = 4194304
    rp, ci, v = synth.powerlaw(n, mu=math.log(12.0), sigma=1.2, lo=1, hi=20000, seed=1)
    x = synth.uniform(n, 1)
    y, _ = _run(rp, ci, v, x)
    assert _err(orc, rp, ci, v, x, y, orc.spmv_csr(rp, ci, v, x)) <= TOL64


def test_unaligned_borrowed_arrays(cuda, orc):
    """Arrays that start 4/8 bytes past a 16-byte boundary (views into larger
    buffers) give the right answer."""
    import torch
    from sparseops_b200 import CSR_Matrix, SpOps_csr
    rp, ci, v = synth.powerlaw(20000, seed=28)
    x = synth.uniform(20000, 10)
    d = torch.device("cuda")
    big_ci = torch.zeros(len(ci) + 1, dtype=torch.int32, device=d)
    big_ci[1:] = torch.from_numpy(ci).to(d)
    big_v = torch.zeros(len(v) + 1, dtype=torch.float64, device=d)
    big_v[1:] = torch.from_numpy(v).to(d)
    A = CSR_Matrix(20000, 20000, torch.from_numpy(rp).to(d), big_ci[1:], big_v[1:])
    xd, yd = torch.from_numpy(x).to(d), torch.zeros(20000, dtype=torch.float64, device=d)
    SpOps_csr(1.0, A, xd, 0.0, yd)
    torch.cuda.synchronize()
    y = yd.cpu().numpy()
    assert _err(orc, rp, ci, v, x, y, orc.spmv_csr(rp, ci, v, x)) <= TOL64


def test_invalid_pattern_rejected(cuda):
    """A column index outside [0, cols) is reported at analysis, never gathered."""
    import torch
    from sparseops_b200 import CSR_Matrix, SpOpsError
    rp = np.array([0, 2, 3], np.int32)
    ci = np.array([0, 5, 1], np.int32)   # 5 >= cols = 3
    v = np.ones(3)
    A = CSR_Matrix(2, 3, rp, ci, v)
    with pytest.raises(SpOpsError) as e:
        A.device()
    assert e.value.status == 1


@pytest.mark.parametrize("dtype,itype", [(np.float64, np.int32), (np.float32, np.int32), (np.float64, np.int64)])
def test_kernel_variants_identical(cuda, orc, dtype, itype):
    """Every CSR kernel (spops_set_option "csr_variant") agrees with the oracle,
    including long rows (chunk and tile combines) and empty-row runs; the
    segment-kernel shapes (2, 3, 4) give the same y bit for bit."""
    from sparseops_b200 import default_context
    rng = np.random.default_rng(11)
    n, ncols = 20000, 120000
    lens = rng.poisson(20, n)
    lens[7], lens[8], lens[9] = 30000, 256, 257
    lens[500:900] = 0
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    ci = np.concatenate([np.sort(rng.choice(ncols, L, replace=False)) for L in lens]).astype(itype)
    v = rng.standard_normal(len(ci)).astype(dtype)
    x = rng.uniform(-1, 1, ncols).astype(dtype)
    y0 = rng.uniform(-1, 1, n).astype(dtype)
    rp = rp.astype(itype)
    ctx = default_context()
    ys = []
    try:
        for var in range(11):
            ctx.set_option("csr_variant", var)
            y, _ = _run(rp, ci, v, x, 0.8, 0.7, y0)
            ys.append(y)
    finally:
        ctx.set_option("csr_variant", 0)
    yref = orc.spmv_csr(rp.astype(np.int64), ci.astype(np.int64), v.astype(np.float64), x.astype(np.float64),
                        0.8, 0.7, y0.astype(np.float64))
    tol = TOL64 if dtype == np.float64 else TOL32
    for var, y in enumerate(ys):
        assert _err(orc, rp.astype(np.int64), ci.astype(np.int64), v.astype(np.float64), x.astype(np.float64),
                    y.astype(np.float64), yref, 0.7, y0.astype(np.float64), 0.8) <= tol, var
        if var in (3, 4):
            assert np.array_equal(y, ys[2]), var


@pytest.mark.parametrize("nnz", [0, 100, 256, 512, 777, 256 * 600, 256 * 600 + 3])
def test_staged_tile_counts(cuda, orc, nnz):
    """The staged tile kernel (bulk copies into shared memory) on tile counts
    around its edges: no full tile, exactly one or two tiles, a partial last
    tile, more tiles than resident warps, with and without a partial tail."""
    rng = np.random.default_rng(nnz + 3)
    n, ncols = max(1, nnz // 7), 5000
    rows = np.sort(rng.integers(0, n, nnz))
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, rows + 1, 1)
    rp = np.cumsum(rp)
    ci = np.concatenate([np.sort(rng.choice(ncols, int(L), replace=False)) for L in np.diff(rp)]
                        + [np.zeros(0, np.int64)]).astype(np.int32)
    rp = rp.astype(np.int32)
    v = rng.standard_normal(nnz)
    x = rng.uniform(-1, 1, ncols)
    y0 = rng.uniform(-1, 1, n)
    yref = orc.spmv_csr(rp.astype(np.int64), ci.astype(np.int64), v, x, 1.5, -0.5, y0)
    ys = {}
    for var in (0, 10):
        ys[var], _ = _with_variant(var, lambda: _run(rp, ci, v, x, 1.5, -0.5, y0))
        assert _err(orc, rp.astype(np.int64), ci.astype(np.int64), v, x, ys[var], yref, -0.5, y0, 1.5) <= TOL64, var
    from sparseops_b200 import default_context
    assert default_context().check_device() == 0  # no bounded wait ran out


def _with_variant(var, fn):
    from sparseops_b200 import default_context
    ctx = default_context()
    ctx.set_option("csr_variant", var)
    try:
        return fn()
    finally:
        ctx.set_option("csr_variant", 0)


@pytest.mark.parametrize("var", [7, 8, 9])
def test_windows_wide_tiles_and_empty(cuda, orc, var):
    """Column-sorted windows: tiles whose columns span more than 65535 (full
    columns stored aside), empty rows and windows, FP64 and FP32."""
    rng = np.random.default_rng(5)
    n, ncols = 3000, 5_000_000
    lens = rng.integers(0, 4, n)
    lens[100:400] = 0
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    ci = np.concatenate([np.sort(rng.choice(ncols, L, replace=False)) for L in lens]).astype(np.int64)
    for dtype, tol in [(np.float64, TOL64), (np.float32, TOL32)]:
        v = rng.standard_normal(len(ci)).astype(dtype)
        x = rng.uniform(-1, 1, ncols).astype(dtype)
        y0 = rng.uniform(-1, 1, n).astype(dtype)
        y, _ = _with_variant(var, lambda: _run(rp, ci, v, x, 0.8, 0.7, y0))
        f = lambda a: a.astype(np.float64)
        yref = orc.spmv_csr(rp, ci, f(v), f(x), 0.8, 0.7, f(y0))
        assert _err(orc, rp, ci, f(v), f(x), f(y), yref, 0.7, f(y0), 0.8) <= tol


@pytest.mark.parametrize("var", [7, 8])
def test_windows_no_entries(cuda, var):
    rp = np.zeros(1001, np.int64)
    ci = np.zeros(0, np.int64)
    v = np.zeros(0)
    x = np.ones(50)
    y0 = np.arange(1000, dtype=np.float64)
    y, _ = _with_variant(var, lambda: _run(rp, ci, v, x, 1.0, 0.5, y0))
    assert np.array_equal(y, 0.5 * y0)
    y, _ = _with_variant(var, lambda: _run(rp, ci, v, x, 1.0, 0.0, y0))
    assert np.array_equal(y, np.zeros(1000))


def test_windows_powerlaw_and_value_updates(cuda, orc):
    """Windows on a power-law matrix large enough for many rows per window;
    new values through spops_csr_set_values and in place with touch()."""
    import torch
    from sparseops_b200 import CSR_Matrix, SpOps_csr, default_context
    from sparseops_b200._lib import call, vp
    rp, ci, v = synth.powerlaw(300000, hi=20000, seed=3)
    n = len(rp) - 1
    x = synth.uniform(n, 4)
    dev = "cuda"
    A = CSR_Matrix(n, n, torch.from_numpy(rp).to(dev), torch.from_numpy(ci).to(dev), torch.from_numpy(v).to(dev))
    xd = torch.from_numpy(x).to(dev)
    yd = torch.zeros(n, dtype=torch.float64, device=dev)
    ctx = default_context()
    ctx.set_option("csr_variant", 7)
    try:
        SpOps_csr(1.0, A, xd, 0.0, yd)
        assert _err(orc, rp, ci, v, x, yd.cpu().numpy(), orc.spmv_csr(rp, ci, v, x)) <= TOL64
        v2 = -2.0 * v + 1.0
        vd2 = torch.from_numpy(v2).to(dev)
        call("spops_csr_set_values", A.device().handle, vp(vd2.data_ptr()))
        SpOps_csr(1.0, A, xd, 0.0, yd)
        assert _err(orc, rp, ci, v2, x, yd.cpu().numpy(), orc.spmv_csr(rp, ci, v2, x)) <= TOL64
        vd2.mul_(0.5)
        A.touch()
        SpOps_csr(1.0, A, xd, 0.0, yd)
        v3 = 0.5 * v2
        assert _err(orc, rp, ci, v3, x, yd.cpu().numpy(), orc.spmv_csr(rp, ci, v3, x)) <= TOL64
    finally:
        ctx.set_option("csr_variant", 0)


@pytest.mark.parametrize("pinned", [True, False])
def test_host_path_pipelined(cuda, orc, pinned):
    """spops_spmv_host on a matrix large enough for the ranged path (rows >=
    2^20): y comes back range by range while later ranges compute; the result
    equals the device-resident SpMV bit for bit (same kernel and order)."""
    import torch
    from sparseops_b200 import CSR_Matrix, default_context
    from sparseops_b200._lib import call, dbl, vp
    rp, ci, v = synth.powerlaw(1_300_000, mu=1.5, sigma=1.0, hi=3000, seed=9)
    n = len(rp) - 1
    x = synth.uniform(n, 3)
    y0 = synth.uniform(n, 4)
    ctx = default_context()
    A = CSR_Matrix(n, n, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda())
    h = A.device(ctx)
    xd = torch.from_numpy(x).cuda()
    for alpha, beta in [(1.0, 0.0), (0.5, 0.25)]:
        yd = torch.from_numpy(y0.copy()).cuda()
        call("spops_spmv", ctx.handle, dbl(alpha), h.handle, vp(xd.data_ptr()), dbl(beta), vp(yd.data_ptr()))
        xh = torch.from_numpy(x.copy())
        yh = torch.from_numpy(y0.copy())
        if pinned:
            xh, yh = xh.pin_memory(), yh.pin_memory()
        call("spops_spmv_host", ctx.handle, dbl(alpha), h.handle, vp(xh.data_ptr()), dbl(beta), vp(yh.data_ptr()))
        torch.cuda.synchronize()
        assert torch.equal(yh, yd.cpu())
        yref = orc.spmv_csr(rp.astype(np.int64), ci.astype(np.int64), v, x, alpha, beta, y0)
        assert _err(orc, rp.astype(np.int64), ci.astype(np.int64), v, x, yh.numpy(), yref, beta, y0, alpha) <= TOL64


@pytest.mark.parametrize("rows,pinned", [(1_300_000, True), (50_000, True), (50_000, False)])
def test_host_path_queued(cuda, rows, pinned):
    """spops_spmv_host_async: six independent requests (different x, alpha,
    beta and y0, separate host buffers) queued back to back through the two
    device slots, then one wait; every y equals the device-resident SpMV of
    its own request bit for bit.  Covers the ranged path (rows >= 2^20), the
    single-range path and pageable buffers (which run each call to the end)."""
    import torch
    from sparseops_b200 import CSR_Matrix, default_context, spmv_host_async, spmv_host_wait
    from sparseops_b200._lib import call, dbl, vp
    rp, ci, v = synth.powerlaw(rows, mu=1.5, sigma=1.0, hi=3000, seed=10)
    n = len(rp) - 1
    ctx = default_context()
    A = CSR_Matrix(n, n, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda())
    h = A.device(ctx)
    reqs = [(1.0, 0.0), (0.5, 0.25), (2.0, 0.0), (-1.0, 1.0), (1.0, 0.0), (0.75, -0.5)]
    xs, y0s, yhs = [], [], []
    for i, (alpha, beta) in enumerate(reqs):
        x, y0 = synth.uniform(n, 20 + i), synth.uniform(n, 40 + i)
        xh, yh = torch.from_numpy(x.copy()), torch.from_numpy(y0.copy())
        if pinned:
            xh, yh = xh.pin_memory(), yh.pin_memory()
        xs.append(x)
        y0s.append(y0)
        yhs.append((xh, yh))
    for (alpha, beta), (xh, yh) in zip(reqs, yhs):
        spmv_host_async(alpha, A, xh, beta, yh)
    spmv_host_wait(A)
    for (alpha, beta), x, y0, (_, yh) in zip(reqs, xs, y0s, yhs):
        xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y0.copy()).cuda()
        call("spops_spmv", ctx.handle, dbl(alpha), h.handle, vp(xd.data_ptr()), dbl(beta), vp(yd.data_ptr()))
        torch.cuda.synchronize()
        assert torch.equal(yh, yd.cpu()), (alpha, beta)
    # a blocking call after queued ones waits for them first
    xh, yh = yhs[0][0], torch.zeros(n, dtype=torch.float64)
    spmv_host_async(1.0, A, yhs[1][0], 0.0, yhs[1][1])
    call("spops_spmv_host", ctx.handle, dbl(1.0), h.handle, vp(xh.data_ptr()), dbl(0.0), vp(yh.data_ptr()))
    xd, yd = torch.from_numpy(xs[0]).cuda(), torch.empty(n, dtype=torch.float64, device="cuda")
    call("spops_spmv", ctx.handle, dbl(1.0), h.handle, vp(xd.data_ptr()), dbl(0.0), vp(yd.data_ptr()))
    torch.cuda.synchronize()
    assert torch.equal(yh, yd.cpu())
