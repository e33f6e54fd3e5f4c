"""spops_csr_spmv_noalloc: the CSR SpMV entry point that allocates nothing.

It exists for callers that cannot allocate device memory when they need the
product (device memory reserved up front by a pool, plug-in or callback code
that must not call cudaMalloc, loops that cannot take an allocation's
synchronisation).  Its scratch is one fixed 4 MiB device array of the library.

The test calls it through the C ABI (ctypes, device pointers from torch) and
compares y with the handle-based entry point (spops_csr_create + spops_spmv)
on the same inputs, componentwise within 1e-12, for two calls in a row (the
second call reuses the shared scratch left by the first).  It runs last
(file name) and passes alone in a fresh process as well as after the others.
"""
import ctypes as C

import numpy as np
import pytest

from sparseops_b200 import synth

pytestmark = pytest.mark.gpu

TOL = 1e-12


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


@pytest.mark.parametrize("case", [m[0] for m in _matrices()])
def test_noalloc_matches_handle_path(cuda, case):
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
    den = (0.8 * torch.from_numpy(np.abs(v)).to(d) * x[cit.long()].abs()).cpu().numpy()
    rows = np.repeat(np.arange(n), np.diff(rp.astype(np.int64)))
    scale = np.bincount(rows, weights=den, minlength=n) + 0.7 * np.abs(y0.cpu().numpy())
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # two calls in a row share the fixed scratch
        y = y0.clone()
        _noalloc(rpt, cit, vt, x, y, 0.8, 0.7, ncols, stream)
        err = (np.abs(y.cpu().numpy() - y_ref.cpu().numpy()) / np.maximum(scale, 1e-300)).max()
        assert err <= TOL


def test_noalloc_rejects_oversize(cuda):
    """More entries than the fixed scratch covers: refused before any work."""
    from sparseops_b200._lib import SpOpsError, call, dbl, i64, vp
    with pytest.raises(SpOpsError) as e:
        call("spops_csr_spmv_noalloc", i64(10), i64(10), i64(1 << 40), vp(0), vp(0), vp(0), C.c_int(0), C.c_int(1),
             dbl(1.0), vp(0), dbl(0.0), vp(0), vp(0))
    assert e.value.status == 5
