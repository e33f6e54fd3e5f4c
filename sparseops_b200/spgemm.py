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


def pairs_from_arrays(i, j, score, ctx=None) -> CandidatePairs:
    """A device pair set from host arrays (i, j, score) of equal length: a
    caller's own candidate pairs for the device clustering."""
    ctx = (ctx or default_context()).follow_torch()
    pi, pj = (np.ascontiguousarray(np.asarray(a, np.int64)) for a in (i, j))
    ps = np.ascontiguousarray(np.asarray(score, np.float64))
    if not (len(pi) == len(pj) == len(ps)):
        raise ValueError("pairs_from_arrays: i, j and score differ in length")
    out = vp()
    call("spops_pairs_create", ctx.handle, _p(pi), _p(pj), _p(ps), i64(len(pi)), i32(1), C.byref(out))
    return CandidatePairs(ctx, out)


def hierarchical_clustering_device(csr: CSR_Matrix, pairs: CandidatePairs, cluster_size: int):
    """hierarchical_clustering_v0_fast (include/spgemm_utility.h:742) on the
    device: A's device pattern and device pairs in, the same (permutation,
    offsets) as the host loop out (numpy arrays)."""
    h = csr.device()
    ctx = h.ctx.follow_torch()
    n = int(csr.num_rows)
    perm = np.empty(n, np.int64)
    offs = np.empty(n + 1, np.int64)
    nc = C.c_int64()
    call("spops_pairs_cluster", ctx.handle, h.handle, pairs.handle, i64(cluster_size), _p(perm), _p(offs),
         C.byref(nc))
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


class VLengthCluster:
    """CSR_VlengthCluster (spgemm_cluster.h:108-143) held by a device handle:
    clusters of consecutive rows, each with the union of its rows' columns and
    values[rowptr_val[i] + p * cluster_sz[i] + k] for column p and row k."""

    def __init__(self, handle: _Handle, index_dtype, value_dtype, stats=None):
        info = handle.info()
        self._h = handle
        self.csr_rows, self.cols, self.nnzc = int(info.rows), int(info.cols), int(info.nnz)
        self.rows, self.nnzv, self.max_cluster_sz = int(info.extra[0]), int(info.extra[1]), int(info.extra[2])
        self._it = np.int32 if int(index_dtype) == 0 else np.int64  # spops_index_t / spops_value_t codes
        self._vt = np.float32 if int(value_dtype) == 0 else np.float64
        self._codes = (int(index_dtype), int(value_dtype))
        self.stats = stats or {}

    def host(self) -> dict:
        """cluster_sz, rowptr, colids, rowptr_val, values as numpy arrays."""
        h = self._h
        out = {}
        for name, which, n, dt in (("cluster_sz", 12, self.rows, self._it), ("rowptr", 0, self.rows + 1, self._it),
                                   ("colids", 1, self.nnzc, self._it), ("rowptr_val", 13, self.rows + 1, self._it),
                                   ("values", 2, self.nnzv, self._vt)):
            a = np.empty(n, dt)
            if n:
                call("spops_matrix_download", h.ctx.handle, h.handle, which, vp(a.ctypes.data), i64(n))
            out[name] = a
        return out


def csr_to_vlength_cluster(csr: CSR_Matrix, offsets) -> VLengthCluster:
    """include/sparse_conversion.h:1641 on the device: cluster i is rows
    offsets[i] .. offsets[i+1]; each cluster's columns ascending."""
    h = csr.device()
    ctx = h.ctx.follow_torch()
    offs = np.ascontiguousarray(np.asarray(offsets, np.int64))
    out = vp()
    call("spops_csr_to_vlength_cluster", ctx.handle, h.handle, _p(offs), i64(len(offs) - 1), C.byref(out))
    it, vt = _types(csr)
    return VLengthCluster(_Handle(ctx, out), it, vt)


def vlength_cluster2csr(cluster: VLengthCluster) -> DeviceCSR:
    """include/sparse_conversion.h:1778 on the device: rows in cluster order,
    exact zeros dropped."""
    h = cluster._h
    out = vp()
    call("spops_vlength_cluster_to_csr", h.ctx.handle, h.handle, C.byref(out))
    return DeviceCSR(_Handle(h.ctx, out), cluster.csr_rows, cluster.cols)


def LeSpGEMM_VLength(A_cluster: VLengthCluster, B: CSR_Matrix, sort_output: bool = True, kernel_flag: int = 3,
                     l2_budget: float = L2_BUDGET_DEFAULT) -> VLengthCluster:
    """include/spgemm.h:176: C = A*B with A clustered, C in A's clusters
    (kernel-3 rules; kernel_flag is accepted for the signature's sake)."""
    ha, hb = A_cluster._h, B.device()
    ctx = ha.ctx.follow_torch()
    out = vp()
    st = SpgemmStats()
    call("spops_spgemm_vlength", ctx.handle, ha.handle, hb.handle, i32(1 if sort_output else 0), dbl(l2_budget),
         C.byref(out), C.byref(st))
    return VLengthCluster(_Handle(ctx, out), *A_cluster._codes, st.as_dict())


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
