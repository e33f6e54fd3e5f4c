"""LeSpGEMM: MinHash-LSH row clustering and the cluster-wise SpGEMM.

Names follow the reference (include/spgemm_MinHashLSH.h, include/spgemm_utility.h,
src/spgemm.cpp):

    minhash_signatures_flat(csr, k, seed)                    device, bit-identical
    lsh_candidate_pairs_vector(csr, k, bands, seed, ...)     device, bit-identical
    hierarchical_clustering_v0_fast(rp, ci, n, pairs, cs)    host, bit-identical
    LeSpGEMM_clustered(A, B, perm, offsets, ...)             device (kernel-3 rules)
    LeSpGEMM_lsh(A, B, k, bands, seed, cluster_size, ...)    the whole pipeline
    LeSpGEMM(A, B, kernel_flag, sort_output)                 device, row-wise kernels 1-3
    HashSpGEMMTopK(A, top_k)                                 device, top-k Jaccard rows

Results of the SpGEMM are CSR matrices in A's original row order with
ascending columns (``SpGEMMResult``), kept on the device; host copies are
made on first access.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import SpgemmStats, call, dbl, i32, i64, u64, vp
from .spops import CSR_Matrix, DeviceCSR, _Handle, default_context

L2_BUDGET_DEFAULT = 67108864 * 0.75  # reference CPU_L2CACHE_SIZE (as shipped) x MIXED_L2_FRACTION


def _p(a):
    return a.ctypes.data_as(vp)


def minhash_signatures_flat(csr: CSR_Matrix, k: int = 64, seed: int = 12345) -> np.ndarray:
    """[rows x k] uint64 signatures (include/spgemm_MinHashLSH.h:119)."""
    import torch
    h = csr.device()
    ctx = h.ctx.follow_torch()
    sig = torch.empty(max(csr.num_rows, 1) * k, dtype=torch.int64, device=f"cuda:{ctx.device}")
    call("spops_minhash", ctx.handle, h.handle, i32(k), u64(seed), vp(sig.data_ptr()))
    torch.cuda.synchronize()
    return sig.cpu().numpy().view(np.uint64)[:csr.num_rows * k].reshape(csr.num_rows, k)


class CandidatePairs:
    """Sorted unique pairs (i < j) with scores, on the device."""

    def __init__(self, ctx, handle):
        self.ctx, self.handle = ctx, handle
        n = C.c_int64()
        call("spops_pairs_count", handle, C.byref(n))
        self.count = n.value

    def __del__(self):  # pragma: no cover
        try:
            _lib.release("spops_pairs_destroy", self.handle, self.ctx)
        except Exception:
            pass

    def host(self):
        i, j, s = np.empty(self.count, np.int64), np.empty(self.count, np.int64), np.empty(self.count)
        if self.count:
            call("spops_pairs_download", self.handle, _p(i), _p(j), _p(s))
        return i, j, s


def lsh_candidate_pairs_vector(csr: CSR_Matrix, k: int, num_bands: int, seed: int = 12345,
                               constrain_large_buckets: bool = True) -> CandidatePairs:
    """include/spgemm_MinHashLSH.h:777."""
    h = csr.device()
    ctx = h.ctx.follow_torch()
    out = vp()
    call("spops_lsh_pairs", ctx.handle, h.handle, i32(k), i32(num_bands), u64(seed),
         i32(1 if constrain_large_buckets else 0), C.byref(out))
    return CandidatePairs(ctx, out)


def hierarchical_clustering_v0_fast(rowptr, colids, num_rows: int, pairs, cluster_size: int):
    """include/spgemm_utility.h:742 on host arrays; pairs = (i, j, score)
    arrays sorted by (i, j) or a CandidatePairs.  Returns (permutation, offsets)."""
    if isinstance(pairs, CandidatePairs):
        pairs = pairs.host()
    pi, pj, ps = (np.ascontiguousarray(a) for a in (pairs[0].astype(np.int64), pairs[1].astype(np.int64),
                                                     pairs[2].astype(np.float64)))
    rp = np.ascontiguousarray(np.asarray(rowptr, np.int64))
    ci = np.ascontiguousarray(np.asarray(colids, np.int64))
    perm = np.empty(num_rows, np.int64)
    offs = np.empty(num_rows + 1, np.int64)
    nc = C.c_int64()
    call("spops_hierarchical_clustering", _p(rp), _p(ci), i64(num_rows), _p(pi), _p(pj), _p(ps), i64(len(pi)),
         i64(cluster_size), _p(perm), _p(offs), C.byref(nc))
    return perm, offs[:nc.value + 1]


class SpGEMMResult(DeviceCSR):
    """C = A*B as a device CSR handle; arrays downloaded on first access."""

    def __init__(self, handle: _Handle, rows: int, cols: int, itype, vtype, stats: dict):
        super().__init__(handle, rows, cols)
        self.stats = stats


def _types(A: CSR_Matrix):
    info = A.device().info()
    return info.index_type, info.value_type


def LeSpGEMM_clustered(A: CSR_Matrix, B: CSR_Matrix, permutation, offsets, sort_output: bool = False,
                       l2_budget: float = L2_BUDGET_DEFAULT) -> SpGEMMResult:
    """Cluster-wise C = A*B for a given clustering (kernel-3 rules)."""
    ha, hb = A.device(), B.device()
    ctx = ha.ctx.follow_torch()
    perm = np.ascontiguousarray(np.asarray(permutation, np.int64))
    offs = np.ascontiguousarray(np.asarray(offsets, np.int64))
    out = vp()
    st = SpgemmStats()
    call("spops_spgemm_clustered", ctx.handle, ha.handle, hb.handle, _p(perm), _p(offs), i64(len(offs) - 1),
         i32(1 if sort_output else 0), dbl(l2_budget), C.byref(out), C.byref(st))
    it, vt = _types(A)
    return SpGEMMResult(_Handle(ctx, out), A.num_rows, B.num_cols, it, vt, st.as_dict())


def LeSpGEMM_lsh(A: CSR_Matrix, B: CSR_Matrix, k: int = 64, num_bands: int = 16, seed: int = 7,
                 cluster_size: int = 8, sort_output: bool = False,
                 l2_budget: float = L2_BUDGET_DEFAULT) -> SpGEMMResult:
    """MinHash-LSH clustering of A's rows, then the cluster-wise SpGEMM
    (the reference driver's pipeline, test/test_spgemm_hc_lsh.cpp:80-300)."""
    ha, hb = A.device(), B.device()
    ctx = ha.ctx.follow_torch()
    out = vp()
    st = SpgemmStats()
    call("spops_spgemm_lsh", ctx.handle, ha.handle, hb.handle, i32(k), i32(num_bands), u64(seed), i64(cluster_size),
         i32(1 if sort_output else 0), dbl(l2_budget), C.byref(out), C.byref(st))
    it, vt = _types(A)
    return SpGEMMResult(_Handle(ctx, out), A.num_rows, B.num_cols, it, vt, st.as_dict())


def LeSpGEMM(A: CSR_Matrix, B: CSR_Matrix, kernel_flag: int = 1, sort_output: bool = False) -> SpGEMMResult:
    """Row-wise C = A*B (src/spgemm.cpp:683): every structural entry kept,
    exact zeros included; columns ascending in every row (kernels 1-3 give
    the same entries; ascending order is valid for all of them)."""
    ha, hb = A.device(), B.device()
    ctx = ha.ctx.follow_torch()
    out = vp()
    st = SpgemmStats()
    call("spops_spgemm_rowwise", ctx.handle, ha.handle, hb.handle, i32(kernel_flag), i32(1 if sort_output else 0),
         C.byref(out), C.byref(st))
    it, vt = _types(A)
    return SpGEMMResult(_Handle(ctx, out), A.num_rows, B.num_cols, it, vt, st.as_dict())


def HashSpGEMMTopK(A: CSR_Matrix, top_k: int) -> DeviceCSR:
    """For every row, the top_k most Jaccard-similar other rows of A (by
    similarity descending, then column ascending), as values
    (src/spgemm.cpp:708)."""
    ha = A.device()
    ctx = ha.ctx.follow_torch()
    out = vp()
    call("spops_spgemm_topk", ctx.handle, ha.handle, i64(top_k), C.byref(out))
    return DeviceCSR(_Handle(ctx, out), A.num_rows, A.num_rows)
