"""Differentiable SpMV: grad_x = A^T g and grad_values = SDDMM(g, x).

Checks, on the fwd+bwd configuration (random graph, symmetric pattern, mean
degree 32, values U[0.1, 1]):
  * grad_x against the oracle's transpose SpMV (pinned to the reference's
    csr_transpose + SpOps_csr through the golden fixtures), componentwise 1e-12;
  * grad_values against g_i * x_j exactly (one rounding);
  * both against central finite differences (h = 1e-6, FP64) on 1,000 random
    coordinates, |fd - grad| <= 1e-6 * scale;
  * FP32 values with FP32 accumulation against the FP64 oracle, 1e-5.
"""
import numpy as np
import pytest

from sparseops_b200 import synth

pytestmark = pytest.mark.gpu


def _pattern(rp, ci, v, dev="cuda"):
    import torch
    from sparseops_b200.autograd import SparsePattern
    n = len(rp) - 1
    vt = torch.from_numpy(v).to(dev)
    return SparsePattern(n, n, torch.from_numpy(rp).to(dev), torch.from_numpy(ci).to(dev), vt), vt


def _graph(n, seed=4):
    return synth.symmetric_graph(n, mean_degree=32.0, sigma=1.0, seed=seed)


@pytest.mark.parametrize("n", [20000, 1048576])
def test_fwd_bwd_vs_oracle(cuda, orc, n):
    import torch
    from sparseops_b200.autograd import spmv
    rp, ci, v = _graph(n)
    x, g = synth.uniform(n, 41), synth.normal(n, 42)
    P, vt = _pattern(rp, ci, v)
    vt.requires_grad_(True)
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    y = spmv(vt, xt, P)
    y.backward(torch.from_numpy(g).cuda())
    torch.cuda.synchronize()
    # forward
    yref = orc.spmv_csr(rp, ci, v, x)
    assert (np.abs(y.detach().cpu().numpy() - yref) / orc.absdot(rp, ci, v, x)).max() <= 1e-12
    # grad_x = A^T g
    gx = xt.grad.cpu().numpy()
    gx_ref = orc.spmv_t(rp, ci, v, g, n)
    den = orc.spmv_t(rp, ci, np.abs(v), np.abs(g), n)
    assert (np.abs(gx - gx_ref) / np.maximum(den, 1e-300)).max() <= 1e-12
    # grad_values = g_i x_j
    gv = vt.grad.cpu().numpy()
    assert np.array_equal(gv, orc.sddmm(rp, ci, g, x))


def test_finite_differences(cuda):
    """Central differences, h = 1e-6, FP64, on 1,000 random coordinates."""
    import torch
    from sparseops_b200.autograd import spmv
    n = 1048576
    rp, ci, v = _graph(n)
    x, g = synth.uniform(n, 43), synth.normal(n, 44)
    P, vt = _pattern(rp, ci, v)
    vt.requires_grad_(True)
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    gt = torch.from_numpy(g).cuda()
    y = spmv(vt, xt, P)
    y.backward(gt)
    gv, gx = vt.grad.detach(), xt.grad.detach()
    rng = np.random.default_rng(45)
    h = 1e-6
    rows_of = np.repeat(np.arange(n), np.diff(rp))
    cols_t = synth.transpose(rp, ci, v, n)
    with torch.no_grad():
        # values: only row i of y moves when entry k = (i, j) moves
        for k in rng.integers(0, len(ci), 500):
            i = int(rows_of[k])
            orig = float(vt[k])
            vt[k] = orig + h
            yp = float(spmv(vt, xt, P)[i])
            vt[k] = orig - h
            ym = float(spmv(vt, xt, P)[i])
            vt[k] = orig
            fd = g[i] * (yp - ym) / (2 * h)
            scale = abs(g[i]) * (abs(x[ci[k]]) + np.abs(v[rp[i]:rp[i + 1]] * x[ci[rp[i]:rp[i + 1]]]).sum())
            assert abs(fd - float(gv[k])) <= 1e-6 * scale + 1e-12
        # x: L = g . y over the rows that hold column j
        for j in rng.integers(0, n, 500):
            rows = cols_t[1][cols_t[0][j]:cols_t[0][j + 1]].astype(np.int64)
            if len(rows) == 0:
                continue
            rows_t = torch.from_numpy(rows).cuda()
            orig = float(xt[j])
            xt[j] = orig + h
            yp = spmv(vt, xt, P)[rows_t]
            xt[j] = orig - h
            ym = spmv(vt, xt, P)[rows_t]
            xt[j] = orig
            fd = float((gt[rows_t] * (yp - ym)).sum() / (2 * h))
            scale = float((np.abs(g[rows]) * np.abs(cols_t[2][cols_t[0][j]:cols_t[0][j + 1]])).sum())
            assert abs(fd - float(gx[j])) <= 1e-6 * max(scale, 1.0)


def test_float32_values(cuda, orc):
    import torch
    from sparseops_b200.autograd import spmv
    n = 200000
    rp, ci, v = _graph(n, seed=6)
    v32 = v.astype(np.float32)
    x, g = synth.uniform(n, 46).astype(np.float32), synth.normal(n, 47).astype(np.float32)
    P, vt = _pattern(rp, ci, v32)
    vt.requires_grad_(True)
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    y = spmv(vt, xt, P)
    y.backward(torch.from_numpy(g).cuda())
    gx_ref = orc.spmv_t(rp, ci, v32.astype(np.float64), g.astype(np.float64), n)
    den = orc.spmv_t(rp, ci, np.abs(v32.astype(np.float64)), np.abs(g.astype(np.float64)), n)
    assert (np.abs(xt.grad.cpu().numpy() - gx_ref) / np.maximum(den, 1e-30)).max() <= 1e-5
    yref = orc.spmv_csr(rp, ci, v32, x)
    assert (np.abs(y.detach().cpu().numpy() - yref) /
            orc.absdot(rp, ci, v32.astype(np.float64), x.astype(np.float64))).max() <= 1e-5


def test_values_update_refreshes_transpose(cuda, orc):
    """After an in-place update of the values the transpose follows them."""
    import torch
    from sparseops_b200.autograd import SparseLinear
    n = 30000
    rp, ci, v = _graph(n, seed=8)
    m = SparseLinear(n, n, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda())
    opt = torch.optim.SGD(m.parameters(), lr=1e-4)
    x = torch.from_numpy(synth.uniform(n, 48)).cuda().requires_grad_(True)
    for _ in range(3):
        opt.zero_grad()
        x.grad = None
        y = m(x)
        (y * y).sum().backward()
        opt.step()
    vals = m.values.detach().cpu().numpy()
    y = m(x)
    g = (2 * y).detach()
    x.grad = None
    y.backward(g)
    gx_ref = orc.spmv_t(rp, ci, vals, g.cpu().numpy(), n)
    den = orc.spmv_t(rp, ci, np.abs(vals), np.abs(g.cpu().numpy()), n)
    assert (np.abs(x.grad.cpu().numpy() - gx_ref) / np.maximum(den, 1e-300)).max() <= 1e-12


@pytest.mark.parametrize("itype", ["int32", "int64"])
def test_sddmm_tile_path_exact(cuda, itype):
    """SDDMM on the tile plan (default CSR variant) and on the segment plan
    (variant 2) give g_i * x_j * alpha exactly, on rows of very different
    lengths: empty rows (also inside tiles), one row of 5,000 entries, and a
    last tile cut short."""
    import torch
    from sparseops_b200 import CSR_Matrix, default_context
    from sparseops_b200._lib import call, dbl, vp
    rng = np.random.default_rng(23)
    n, ncols = 3001, 7000
    lens = rng.integers(0, 40, n)
    lens[rng.choice(n, 300, replace=False)] = 0
    lens[17] = 5000
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    ci = np.concatenate([np.sort(rng.choice(ncols, L, replace=False)) for L in lens]).astype(itype)
    rp = rp.astype(itype)
    v = rng.standard_normal(len(ci))
    x, g = rng.uniform(-1, 1, ncols), rng.standard_normal(n)
    dev = torch.device("cuda")
    A = CSR_Matrix(n, ncols, torch.from_numpy(rp).to(dev), torch.from_numpy(ci).to(dev), torch.from_numpy(v).to(dev))
    ctx = default_context()
    h = A.device(ctx)
    xd, gd = torch.from_numpy(x).to(dev), torch.from_numpy(g).to(dev)
    rows = np.repeat(np.arange(n), np.diff(rp.astype(np.int64)))
    want = (0.75 * g[rows]) * x[ci.astype(np.int64)]
    outs = []
    try:
        for variant in (0, 2):
            ctx.set_option("csr_variant", variant)
            out = torch.full((len(ci),), np.nan, dtype=torch.float64, device=dev)
            call("spops_sddmm", ctx.handle, dbl(0.75), h.handle, vp(gd.data_ptr()), vp(xd.data_ptr()),
                 vp(out.data_ptr()))
            torch.cuda.synchronize()
            outs.append(out.cpu().numpy())
    finally:
        ctx.set_option("csr_variant", 0)
    for o in outs:
        assert np.array_equal(o.view(np.uint64), want.view(np.uint64))


@pytest.mark.parametrize("itype", ["int32", "int64"])
def test_transpose_spmv_values_through_permutation(cuda, orc, itype):
    """A^T g right after a value change reads A's values through the
    transpose's permutation inside the SpMV (default CSR variant); the segment
    variant refreshes the reordered copy first.  Both agree with the oracle's
    transpose SpMV to 1e-12 on a rectangular matrix with empty rows and
    columns and one long row, before and after the values change in place."""
    import torch
    from sparseops_b200 import CSR_Matrix, default_context
    from sparseops_b200._lib import call, dbl, vp
    rng = np.random.default_rng(29)
    n, ncols = 2500, 9000
    lens = rng.integers(0, 30, n)
    lens[rng.choice(n, 200, replace=False)] = 0
    lens[5] = 4000
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    ci = np.concatenate([np.sort(rng.choice(ncols, L, replace=False)) for L in lens]).astype(np.int32)
    v = rng.standard_normal(len(ci))
    g = rng.standard_normal(n)
    dev = torch.device("cuda")
    vd = torch.from_numpy(v).to(dev)
    A = CSR_Matrix(n, ncols, torch.from_numpy(rp.astype(itype)).to(dev), torch.from_numpy(ci.astype(itype)).to(dev), vd)
    ctx = default_context()
    h = A.device(ctx)
    gd = torch.from_numpy(g).to(dev)
    rp32 = rp.astype(np.int32)
    try:
        for step in range(2):
            if step == 1:  # values changed in place: the handle is told
                vd.mul_(-1.5).add_(0.25)
                call("spops_matrix_touch", h.handle)
            vals = vd.cpu().numpy()
            want = orc.spmv_t(rp32, ci, vals, g, ncols)
            den = orc.spmv_t(rp32, ci, np.abs(vals), np.abs(g), ncols)
            for variant in (0, 2):
                ctx.set_option("csr_variant", variant)
                call("spops_matrix_touch", h.handle)
                out = torch.full((ncols,), np.nan, dtype=torch.float64, device=dev)
                call("spops_spmv_t", ctx.handle, dbl(1.0), h.handle, vp(gd.data_ptr()), dbl(0.0), vp(out.data_ptr()))
                torch.cuda.synchronize()
                err = np.abs(out.cpu().numpy() - want) / np.maximum(den, 1e-300)
                assert err.max() <= 1e-12, (step, variant, err.max())
    finally:
        ctx.set_option("csr_variant", 0)


@pytest.mark.parametrize("long_row", [4000, 40000])
def test_transpose_spmv_source_row_bands(cuda, orc, long_row):
    """A^T g through the permutation in source-row bands (context option
    "adjoint_bands"): 1, 3 and 8 bands give the oracle's alpha A^T g + beta y
    to 1e-12, with beta = 0 over a NaN-filled y and beta != 0 over y0, on a
    rectangular matrix with empty rows and columns.  With one row holding
    most entries, several of the 8 bands are empty.  Each band count gives
    the same bits on a second call (the bands are rebuilt when the count
    changes)."""
    import torch
    from sparseops_b200 import CSR_Matrix, default_context
    from sparseops_b200._lib import call, dbl, vp
    rng = np.random.default_rng(31)
    n, ncols = 2500, 9000
    lens = rng.integers(0, 30, n)
    lens[rng.choice(n, 200, replace=False)] = 0
    lens[5] = long_row
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    ci = np.concatenate([np.sort(rng.choice(ncols, L, replace=L > ncols)) for L in lens]).astype(np.int32)
    v = rng.standard_normal(len(ci))
    g = rng.standard_normal(n)
    y0 = rng.standard_normal(ncols)
    dev = torch.device("cuda")
    A = CSR_Matrix(n, ncols, torch.from_numpy(rp.astype(np.int32)).to(dev), torch.from_numpy(ci).to(dev),
                   torch.from_numpy(v).to(dev))
    ctx = default_context()
    h = A.device(ctx)
    gd = torch.from_numpy(g).to(dev)
    rp32 = rp.astype(np.int32)
    at_g = orc.spmv_t(rp32, ci, v, g, ncols)
    den = orc.spmv_t(rp32, ci, np.abs(v), np.abs(g), ncols)
    try:
        for bands in (1, 3, 8, 3):
            ctx.set_option("adjoint_bands", bands)
            for alpha, beta in ((1.0, 0.0), (0.8, 0.7)):
                outs = []
                for _ in range(2):
                    call("spops_matrix_touch", h.handle)  # values "changed": the permutation path
                    init = np.full(ncols, np.nan) if beta == 0.0 else y0
                    out = torch.from_numpy(init.copy()).to(dev)
                    call("spops_spmv_t", ctx.handle, dbl(alpha), h.handle, vp(gd.data_ptr()), dbl(beta),
                         vp(out.data_ptr()))
                    torch.cuda.synchronize()
                    outs.append(out.cpu().numpy())
                assert np.array_equal(outs[0], outs[1])
                want = alpha * at_g + beta * y0
                err = np.abs(outs[0] - want) / np.maximum(alpha * den + abs(beta) * np.abs(y0), 1e-300)
                assert err.max() <= 1e-12, (bands, alpha, beta, err.max())
    finally:
        ctx.set_option("adjoint_bands", 0)
