"""spops_csr_spmv_noalloc: the CSR SpMV entry point that allocates nothing.

It exists for callers that cannot allocate device memory when they need the
product (device memory reserved up front by a pool, plug-in or callback code
that must not call cudaMalloc, loops that cannot take an allocation's
synchronisation).  Its scratch is one fixed 4 MiB device array of the library.

The test calls it through the C ABI (ctypes, device pointers from torch) and
compares y with the handle-based entry point (spops_csr_create + spops_spmv)
and with the oracle on the same inputs, componentwise within 1e-12 for FP64
values (1e-5 for FP32 values), for two calls in a row (the second call reuses
the shared scratch left by the first).  Malformed inputs -- a column index
equal to cols, a row pointer that decreases, a row pointer whose last entry is
not nnz -- must come back as SPOPS_ERR_INVALID without touching memory outside
the arrays.  It runs last (file name) and passes alone in a fresh process as
well as after the others.
"""
import ctypes as C

import numpy as np
import pytest

from sparseops_b200 import synth

pytestmark = pytest.mark.gpu

TOL = 1e-12
TOL_F32 = 1e-5
ERR_INVALID = 1


def _noalloc(rp, ci, v, x, y, alpha, beta, ncols, stream):
    from sparseops_b200._lib import call, dbl, i64, vp
    it = 0 if rp.dtype.itemsize == 4 else 1
    vt = 0 if v.dtype.itemsize == 4 else 1
    call("spops_csr_spmv_noalloc", i64(len(rp) - 1), i64(ncols), i64(ci.numel()), vp(rp.data_ptr()),
         vp(ci.data_ptr()), vp(v.data_ptr()), C.c_int(it), C.c_int(vt), dbl(alpha), vp(x.data_ptr()), dbl(beta),
         vp(y.data_ptr()), vp(stream))


def _matrices():
    rng = np.random.default_rng(3)
    n = 6000
    lens = rng.integers(0, 30, n)
    lens[5], lens[6], lens[4000:4100], lens[-3:] = 5000, 1024, 0, 0  # long rows, empty runs, trailing empties
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    ci = np.concatenate([np.sort(rng.choice(20000, L, replace=False)) for L in lens])
    v = rng.standard_normal(len(ci))
    yield "ragged", rp.astype(np.int32), ci.astype(np.int32), v, 20000
    rp2, ci2, v2 = synth.powerlaw(200000, hi=20000, seed=40)
    yield "powerlaw", rp2, ci2, v2, 200000
    rp3, ci3, v3 = synth.laplacian_2d(128)
    yield "laplacian_i64", rp3.astype(np.int64), ci3.astype(np.int64), v3, len(rp3) - 1


def _scale(rp, ci, v, x, y0, alpha, beta):
    """Componentwise error scale |alpha| sum_j |a_ij x_j| + |beta y0_i|."""
    n = len(rp) - 1
    rows = np.repeat(np.arange(n), np.diff(rp.astype(np.int64)))
    den = abs(alpha) * np.abs(v.astype(np.float64)) * np.abs(x[ci.astype(np.int64)])
    return np.bincount(rows, weights=den, minlength=n) + abs(beta) * np.abs(y0)


@pytest.mark.parametrize("case", [m[0] for m in _matrices()])
def test_noalloc_matches_handle_path(cuda, orc, case):
    import torch
    from sparseops_b200 import CSR_Matrix, default_context
    from sparseops_b200._lib import call, dbl, vp
    name, rp, ci, v, ncols = next(m for m in _matrices() if m[0] == case)
    n = len(rp) - 1
    d = torch.device("cuda")
    rpt, cit, vt = (torch.from_numpy(a).to(d) for a in (rp, ci, v))
    x = torch.from_numpy(synth.uniform(ncols, 5)).to(d)
    y0 = torch.from_numpy(synth.uniform(n, 6)).to(d)
    # the existing entry point
    ctx = default_context(0)
    A = CSR_Matrix(n, ncols, rpt, cit, vt)
    y_ref = y0.clone()
    call("spops_spmv", ctx.handle, dbl(0.8), A.device(ctx).handle, vp(x.data_ptr()), dbl(0.7), vp(y_ref.data_ptr()))
    torch.cuda.synchronize()
    xh, y0h = x.cpu().numpy(), y0.cpu().numpy()
    scale = np.maximum(_scale(rp, ci, v, xh, y0h, 0.8, 0.7), 1e-300)
    y_orc = orc.spmv_csr(rp.astype(np.int32), ci.astype(np.int32), v, xh, 0.8, 0.7, y0h)
    assert (np.abs(y_ref.cpu().numpy() - y_orc) / scale).max() <= TOL
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # two calls in a row share the fixed scratch
        y = y0.clone()
        _noalloc(rpt, cit, vt, x, y, 0.8, 0.7, ncols, stream)
        yh = y.cpu().numpy()
        assert (np.abs(yh - y_ref.cpu().numpy()) / scale).max() <= TOL
        assert (np.abs(yh - y_orc) / scale).max() <= TOL


def test_noalloc_float32_values(cuda, orc):
    """FP32 values and vectors (sums carried in float, window sums combined in
    double) against the oracle and the handle path, two calls in a row."""
    import torch
    from sparseops_b200 import CSR_Matrix, default_context
    from sparseops_b200._lib import call, dbl, vp
    rp, ci, v = synth.powerlaw(100000, hi=20000, seed=41)
    n = len(rp) - 1
    v32 = v.astype(np.float32)
    x32 = synth.uniform(n, 7).astype(np.float32)
    y032 = synth.uniform(n, 8).astype(np.float32)
    d = torch.device("cuda")
    rpt, cit, vt, x, y0 = (torch.from_numpy(a).to(d) for a in (rp, ci, v32, x32, y032))
    y_orc = orc.spmv_csr(rp, ci, v32, x32, 1.5, -0.5, y032)
    scale = np.maximum(_scale(rp, ci, v32, x32.astype(np.float64), y032.astype(np.float64), 1.5, -0.5), 1e-300)
    ctx = default_context(0)
    A = CSR_Matrix(n, n, rpt, cit, vt)
    y_ref = y0.clone()
    call("spops_spmv", ctx.handle, dbl(1.5), A.device(ctx).handle, vp(x.data_ptr()), dbl(-0.5), vp(y_ref.data_ptr()))
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        y = y0.clone()
        _noalloc(rpt, cit, vt, x, y, 1.5, -0.5, n, stream)
        yh = y.cpu().numpy().astype(np.float64)
        assert (np.abs(yh - y_orc) / scale).max() <= TOL_F32
        assert (np.abs(yh - y_ref.cpu().numpy().astype(np.float64)) / scale).max() <= TOL_F32


def test_noalloc_column_out_of_range(cuda, orc):
    """One column index equal to cols: SPOPS_ERR_INVALID, the entry skipped,
    every row computed from the other entries."""
    import torch
    from sparseops_b200._lib import SpOpsError
    rp, ci, v = synth.powerlaw(50000, hi=5000, seed=42)
    n = len(rp) - 1
    bad = int(rp[777]) + 1 if rp[778] - rp[777] > 1 else int(rp[777])
    ci_bad = ci.copy()
    ci_bad[bad] = n
    x = synth.uniform(n, 9)
    d = torch.device("cuda")
    rpt, cit, vt, xt = (torch.from_numpy(a).to(d) for a in (rp, ci_bad, v, x))
    y = torch.zeros(n, dtype=torch.float64, device=d)
    stream = torch.cuda.current_stream().cuda_stream
    with pytest.raises(SpOpsError) as e:
        _noalloc(rpt, cit, vt, xt, y, 1.0, 0.0, n, stream)
    assert e.value.status == ERR_INVALID
    v_skip = v.copy()
    v_skip[bad] = 0.0
    y_orc = orc.spmv_csr(rp, ci, v_skip, x)  # the bad entry contributes nothing
    scale = np.maximum(_scale(rp, ci, v, x, np.zeros(n), 1.0, 0.0), 1e-300)
    assert (np.abs(y.cpu().numpy() - y_orc) / scale).max() <= TOL


@pytest.mark.parametrize("kind", ["decreasing", "last_below_nnz", "first_not_zero"])
def test_noalloc_bad_row_pointer(cuda, kind):
    """A row pointer that is not a CSR row pointer is refused on the device
    before any window is summed: SPOPS_ERR_INVALID, y untouched."""
    import torch
    from sparseops_b200._lib import SpOpsError
    rp, ci, v = synth.powerlaw(30000, hi=3000, seed=43)
    n, nnz = len(rp) - 1, len(ci)
    rp_bad = rp.copy()
    if kind == "decreasing":
        rp_bad[1000] = rp_bad[1001] + 5  # rp[1000] > rp[1001], still inside [0, nnz]
    elif kind == "last_below_nnz":
        rp_bad[n] = nnz - 5
    else:
        rp_bad[0] = 3
    x = synth.uniform(n, 10)
    d = torch.device("cuda")
    rpt, cit, vt, xt = (torch.from_numpy(a).to(d) for a in (rp_bad, ci, v, x))
    y = torch.full((n,), 7.0, dtype=torch.float64, device=d)
    stream = torch.cuda.current_stream().cuda_stream
    with pytest.raises(SpOpsError) as e:
        _noalloc(rpt, cit, vt, xt, y, 1.0, 0.0, n, stream)
    assert e.value.status == ERR_INVALID
    assert bool((y == 7.0).all())


def test_noalloc_rejects_oversize(cuda):
    """More entries than the fixed scratch covers: refused before any work."""
    from sparseops_b200._lib import SpOpsError, call, dbl, i64, vp
    with pytest.raises(SpOpsError) as e:
        call("spops_csr_spmv_noalloc", i64(10), i64(10), i64(1 << 40), vp(0), vp(0), vp(0), C.c_int(0), C.c_int(1),
             dbl(1.0), vp(0), dbl(0.0), vp(0), vp(0))
    assert e.value.status == 5
