"""The oracle: CPU restatement of the SparseOps hot path, plus the reference
library itself compiled from its sources (oracle/_ref).

TEST INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline / reference legs may import this package, and only as
the checker or as the timed CPU baseline.  The product package
(``sparseops_b200``) never imports it.

``Oracle`` wraps liboracle.so (oracle/spops_oracle.cpp, this repository's own
restatement).  ``Reference`` wraps oracle/_ref/libspops_ref_v{3,4}.so, the
reference's own OpenMP kernels behind oracle/ref_harness.cpp.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_i64 = C.c_int64
_vp = C.c_void_p
_dbl = C.c_double


def _p(a):
    return None if a is None else a.ctypes.data_as(_vp)


def build(ref: bool = True) -> None:
    """Compile liboracle.so (and oracle/_ref when the reference sources exist)."""
    target = "all" if ref else "oracle"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


def _cpu_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            flags = f.read()
        return all(x in flags for x in ("avx512f", "avx512dq", "avx512bw", "avx512vl"))
    except OSError:
        return False


class Oracle:
    """ctypes view of liboracle.so; numpy in, numpy out."""

    def __init__(self):
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        self.L = L = C.CDLL(path)
        for name in ("orc_lsh_pairs", "orc_spgemm", "orc_spgemm_rowwise", "orc_spgemm_topk"):
            getattr(L, name).restype = _vp
        for name in ("orc_pairs_count", "orc_hc", "orc_dia_offsets", "orc_bsr_structure",
                     "orc_spgemm_flop", "orc_coo_to_csr_f64", "orc_coo_to_csr_f32"):
            getattr(L, name).restype = _i64

    # ---- SpMV
    def spmv_csr(self, rp, ci, v, x, alpha=1.0, beta=0.0, y=None):
        n = len(rp) - 1
        out = np.zeros(n) if y is None else np.array(y, dtype=np.float64, copy=True)
        if v.dtype == np.float32:
            self.L.orc_spmv_csr_f32_i32(_i64(n), _p(rp), _p(ci), _p(v), _dbl(alpha), _p(x), _dbl(beta),
                                        _p(None if y is None else np.ascontiguousarray(y, np.float32)),
                                        _p(out))
        elif rp.dtype == np.int64:
            self.L.orc_spmv_csr_f64_i64(_i64(n), _p(rp), _p(ci), _p(v), _dbl(alpha), _p(x), _dbl(beta), _p(out))
        else:
            self.L.orc_spmv_csr_f64_i32(_i64(n), _p(rp), _p(ci), _p(v), _dbl(alpha), _p(x), _dbl(beta), _p(out))
        return out

    def absdot(self, rp, ci, v, x):
        n = len(rp) - 1
        out = np.zeros(n)
        if rp.dtype != np.int32 or ci.dtype != np.int32:
            if len(ci) >= 2**31 or len(x) >= 2**31:
                raise ValueError("absdot: indices beyond int32")
            rp, ci = np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(ci, np.int32)
        self.L.orc_absdot_csr_f64_i32(_i64(n), _p(rp), _p(ci), _p(np.ascontiguousarray(v, np.float64)),
                                      _p(np.ascontiguousarray(x, np.float64)), _p(out))
        return out

    def spmm_csr(self, rp, ci, v, X, alpha=1.0, beta=0.0, Y=None):
        n, k = len(rp) - 1, X.shape[1]
        out = np.zeros((n, k)) if Y is None else np.array(Y, dtype=np.float64, copy=True)
        self.L.orc_spmm_csr_f64_i32(_i64(n), _p(rp), _p(ci), _p(v), _i64(k), _dbl(alpha),
                                    _p(np.ascontiguousarray(X)), _dbl(beta), _p(out))
        return out

    # ---- layouts
    def sell_c_sigma_layout(self, rp, sigma, C_, align):
        n = len(rp) - 1
        reorder = np.zeros(n, np.int32)
        chunk_len = np.zeros((n + C_ - 1) // C_, np.int32)
        self.L.orc_sell_c_sigma_layout(_i64(n), _p(rp), _i64(sigma), _i64(C_), _i64(align), _p(reorder),
                                       _p(chunk_len))
        return reorder, chunk_len

    def sell_row_width(self, rp, C_, align):
        n = len(rp) - 1
        w = np.zeros((n + C_ - 1) // C_, np.int32)
        self.L.orc_sell_row_width(_i64(n), _p(rp), _i64(C_), _i64(align), _p(w))
        return w

    def dia_offsets(self, rp, ci, ncols, max_out=1 << 20):
        n = len(rp) - 1
        off = np.zeros(max_out, np.int64)
        nd = self.L.orc_dia_offsets(_i64(n), _i64(ncols), _p(rp), _p(ci), _i64(max_out), _p(off))
        return off[:min(nd, max_out)], nd

    def bsr_structure(self, rp, ci, ncols, br, bc):
        n = len(rp) - 1
        mb = (n + br - 1) // br
        row_ptr = np.zeros(mb + 1, np.int32)
        nnzb = self.L.orc_bsr_structure(_i64(n), _i64(ncols), _p(rp), _p(ci), _i64(br), _i64(bc), _p(row_ptr),
                                        None)
        bcol = np.zeros(max(nnzb, 1), np.int32)
        self.L.orc_bsr_structure(_i64(n), _i64(ncols), _p(rp), _p(ci), _i64(br), _i64(bc), _p(row_ptr), _p(bcol))
        return row_ptr, bcol[:nnzb]

    # ---- LeSpGEMM preprocessing
    def minhash(self, rp, ci, k, seed):
        n = len(rp) - 1
        sig = np.zeros((n, k), np.uint64)
        self.L.orc_minhash(_p(rp), _p(ci), _i64(n), C.c_int32(k), C.c_uint64(seed), _p(sig))
        return sig

    def lsh_pairs(self, sig, bands, constrain=True):
        n, k = sig.shape
        h = self.L.orc_lsh_pairs(_p(np.ascontiguousarray(sig)), _i64(n), C.c_int32(k), C.c_int32(bands),
                                 C.c_int32(1 if constrain else 0))
        m = self.L.orc_pairs_count(_vp(h))
        i, j, s = np.zeros(m, np.int64), np.zeros(m, np.int64), np.zeros(m)
        self.L.orc_pairs_copy(_vp(h), _p(i), _p(j), _p(s))
        self.L.orc_pairs_free(_vp(h))
        return i, j, s

    def hc(self, rp, ci, pi, pj, ps, cluster_size):
        n = len(rp) - 1
        perm, offs = np.zeros(n, np.int64), np.zeros(n + 1, np.int64)
        nc = self.L.orc_hc(_p(rp), _p(ci), _i64(n), _p(pi), _p(pj), _p(ps), _i64(len(pi)), _i64(cluster_size),
                           _p(perm), _p(offs))
        return perm, offs[:nc + 1]

    def spgemm(self, A, B, perm, offsets, sort_output=False, l2_budget=67108864 * 0.75):
        arp, aci, av = A
        brp, bci, bv = B[:3]
        n = len(arp) - 1
        h = self.L.orc_spgemm(_i64(n), _p(arp), _p(aci), _p(av), _i64(len(brp) - 1), _i64(0), _p(brp), _p(bci),
                              _p(bv), _p(perm), _p(offsets), _i64(len(offsets) - 1), C.c_int32(int(sort_output)),
                              _dbl(l2_budget))
        info = np.zeros(4, np.int64)
        self.L.orc_csr_info(_vp(h), _p(info))
        rp = np.zeros(n + 1, np.int64)
        ci, v, a = np.zeros(info[1], np.int64), np.zeros(info[1]), np.zeros(info[1])
        self.L.orc_csr_copy(_vp(h), _p(rp), _p(ci), _p(v), _p(a))
        self.L.orc_csr_free(_vp(h))
        return dict(rp=rp, ci=ci, v=v, absv=a, dense_clusters=int(info[2]), flops=int(info[3]))

    def _orc_csr(self, h, n):
        info = np.zeros(4, np.int64)
        self.L.orc_csr_info(_vp(h), _p(info))
        rp = np.zeros(n + 1, np.int64)
        ci, v, a = np.zeros(info[1], np.int64), np.zeros(info[1]), np.zeros(info[1])
        self.L.orc_csr_copy(_vp(h), _p(rp), _p(ci), _p(v), _p(a))
        self.L.orc_csr_free(_vp(h))
        return dict(rp=rp, ci=ci, v=v, absv=a, flops=int(info[3]))

    def spgemm_rowwise(self, A, B):
        """Row-wise C = A*B, every structural entry kept, columns ascending."""
        arp, aci, av = (np.ascontiguousarray(np.asarray(a, t)) for a, t in zip(A[:3], (np.int64, np.int64, np.float64)))
        brp, bci, bv = (np.ascontiguousarray(np.asarray(a, t)) for a, t in zip(B[:3], (np.int64, np.int64, np.float64)))
        n = len(arp) - 1
        h = self.L.orc_spgemm_rowwise(_i64(n), _p(arp), _p(aci), _p(av), _i64(len(brp) - 1), _p(brp), _p(bci),
                                      _p(bv))
        return self._orc_csr(h, n)

    def spgemm_topk(self, rp, ci, ncols, top_k, f32=False):
        """HashSpGEMMTopK's rows: (columns, Jaccard values) per row in the
        reference's order."""
        rp = np.ascontiguousarray(np.asarray(rp, np.int64))
        ci = np.ascontiguousarray(np.asarray(ci, np.int64))
        n = len(rp) - 1
        h = self.L.orc_spgemm_topk(_i64(n), _p(rp), _p(ci), _i64(ncols), _i64(top_k), C.c_int32(1 if f32 else 0))
        return self._orc_csr(h, n)

    def spgemm_flop(self, A, B):
        arp, aci = A[0], A[1]
        brp = B[0]
        return int(self.L.orc_spgemm_flop(_i64(len(arp) - 1), _p(arp), _p(aci), _i64(len(brp) - 1), _p(brp)))

    # ---- features
    def features(self, rp, ci, v, ncols):
        """The 32 feature values (spops_features_t order) of a CSR matrix."""
        out = np.zeros(32)
        self.L.orc_features(_i64(len(rp) - 1), _i64(ncols), _p(np.ascontiguousarray(rp, np.int64)),
                            _p(np.ascontiguousarray(ci, np.int64)), _p(np.ascontiguousarray(v, np.float64)),
                            _p(out))
        return out

    def tile_features(self, rp, ci, ncols, num_blocks=256):
        """(scalars[34] in spops_tile_features_t order, tile_i[4, B*B],
        tile_d[2, B*B], blk_i[4, B], blk_d[4, B]) of a CSR matrix."""
        B = int(num_blocks)
        sc, ti, td = np.zeros(34), np.zeros(4 * B * B, np.int64), np.zeros(2 * B * B)
        bi, bd = np.zeros(4 * B, np.int64), np.zeros(4 * B)
        self.L.orc_tile_features(_i64(len(rp) - 1), _i64(ncols), _p(np.ascontiguousarray(rp, np.int64)),
                                 _p(np.ascontiguousarray(ci, np.int64)), _i64(B), _p(sc), _p(ti), _p(td), _p(bi),
                                 _p(bd))
        return sc, ti.reshape(4, -1), td.reshape(2, -1), bi.reshape(4, -1), bd.reshape(4, -1)

    # ---- COO -> CSR
    def coo_to_csr(self, n, ri, ci, v, compact=False):
        """(rp, ci, v) of coo_to_csr; v's dtype (float32 / float64) is kept."""
        ri = np.ascontiguousarray(ri, np.int64)
        ci = np.ascontiguousarray(ci, np.int64)
        f32 = np.asarray(v).dtype == np.float32
        v = np.ascontiguousarray(v, np.float32 if f32 else np.float64)
        m = len(ci)
        rp, oc, ov = np.zeros(n + 1, np.int64), np.zeros(max(m, 1), np.int64), np.zeros(max(m, 1), v.dtype)
        fn = self.L.orc_coo_to_csr_f32 if f32 else self.L.orc_coo_to_csr_f64
        k = fn(_i64(n), _i64(m), _p(ri), _p(ci), _p(v), C.c_int32(1 if compact else 0), _p(rp), _p(oc), _p(ov))
        return rp, oc[:k], ov[:k]

    # ---- adjoints
    def spmv_t(self, rp, ci, v, g, ncols):
        y = np.zeros(ncols)
        self.L.orc_spmv_t_csr_f64_i32(_i64(len(rp) - 1), _i64(ncols), _p(rp), _p(ci),
                                      _p(np.ascontiguousarray(v, np.float64)), _p(g), _p(y))
        return y

    def sddmm(self, rp, ci, g, x):
        out = np.zeros(int(rp[-1]))
        self.L.orc_sddmm_csr_f64_i32(_i64(len(rp) - 1), _p(rp), _p(ci), _p(g), _p(x), _p(out))
        return out


def _ll(a):
    """int64, C-contiguous: the reference harness takes long long arrays."""
    return np.ascontiguousarray(a, np.int64)


def _f8(a):
    return np.ascontiguousarray(a, np.float64)


class Reference:
    """ctypes view of the reference library compiled from its own sources.

    Picks the AVX-512 build when the host supports it, else the AVX2 build.
    ``threads`` sets the reference's global thread count (Le_set_thread_num).
    """

    KINDS = dict(csr=1, sell_c_sigma=2, sell_c_R=3, sell=4, ell=5, dia=6, bsr=7, coo=8)

    def __init__(self, threads: int | None = None):
        v = "v4" if _cpu_has_avx512() else "v3"
        path = os.path.join(HERE, "_ref", f"libspops_ref_{v}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference library not built: {path}")
        self.path = path
        self.L = L = C.CDLL(path)
        for name in ("ref_fmt_build", "ref_lsh_pairs", "ref_spgemm_kernel3", "ref_csr_transpose", "ref_coo_to_csr",
                     "ref_spgemm_rowwise", "ref_spgemm_topk"):
            getattr(L, name).restype = _vp
        L.ref_pairs_count.restype = _i64
        L.ref_hc.restype = _i64
        L.ref_spgemm_kernel3_time.restype = _dbl
        self.set_threads(threads or os.cpu_count() or 1)

    def set_threads(self, n: int) -> None:
        self.L.ref_set_threads(C.c_int(int(n)))
        self.threads = int(n)

    def spmv_csr(self, rp, ci, v, x, alpha=1.0, beta=0.0, y=None, flag=2, out=None):
        """Reference SpOps_csr.  `out` (contiguous, v.dtype) is written in place
        when given; otherwise a new array (initialised from y) is returned."""
        n = len(rp) - 1
        if out is None:
            out = np.zeros(n, v.dtype) if y is None else np.array(y, dtype=v.dtype, copy=True)
        ncols = len(x)
        if v.dtype == np.float32:
            self.L.ref_spmv_csr_f32(C.c_int(n), C.c_int(ncols), C.c_int(len(ci)), _p(rp), _p(ci), _p(v),
                                    C.c_float(alpha), _p(x), C.c_float(beta), _p(out), C.c_int(flag))
        elif rp.dtype == np.int64:
            self.L.ref_spmv_csr_f64_i64(_i64(n), _i64(ncols), _i64(len(ci)), _p(rp), _p(ci), _p(v), _dbl(alpha),
                                        _p(x), _dbl(beta), _p(out), C.c_int(flag))
        else:
            self.L.ref_spmv_csr_f64(C.c_int(n), C.c_int(ncols), C.c_int(len(ci)), _p(rp), _p(ci), _p(v),
                                    _dbl(alpha), _p(x), _dbl(beta), _p(out), C.c_int(flag))
        return out

    # format handle: build, inspect, run, free
    def fmt_build(self, kind, rp, ci, v, ncols, p0=0, p1=0, p2=0, flag=1):
        n = len(rp) - 1
        return self.L.ref_fmt_build(C.c_int(self.KINDS[kind]), C.c_int(n), C.c_int(ncols), C.c_int(len(ci)),
                                    _p(rp), _p(ci), _p(v), _i64(p0), _i64(p1), _i64(p2), C.c_int(flag))

    def fmt_info(self, h):
        out = np.zeros(8, np.int64)
        self.L.ref_fmt_info(_vp(h), _p(out))
        return out

    def fmt_copy(self, h, a=None, b=None, c=None, d=None):
        self.L.ref_fmt_copy(_vp(h), _p(a), _p(b), _p(c), _p(d))

    def fmt_spmv(self, h, x, alpha=1.0, beta=0.0, y=None, n=None):
        out = np.zeros(n) if y is None else np.array(y, dtype=np.float64, copy=True)
        self.L.ref_fmt_spmv(_vp(h), _dbl(alpha), _p(x), _dbl(beta), _p(out))
        return out

    def fmt_free(self, h):
        self.L.ref_fmt_free(_vp(h))

    def minhash(self, rp, ci, k, seed):
        rp, ci = _ll(rp), _ll(ci)
        n = len(rp) - 1
        sig = np.zeros((n, k), np.uint64)
        self.L.ref_minhash_flat(_p(rp), _p(ci), _i64(n), C.c_int(k), C.c_uint64(seed), _p(sig))
        return sig

    def lsh_pairs(self, rp, ci, k, bands, seed, constrain=True):
        rp, ci = _ll(rp), _ll(ci)
        h = self.L.ref_lsh_pairs(_p(rp), _p(ci), _i64(len(rp) - 1), C.c_int(k), C.c_int(bands),
                                 C.c_uint64(seed), C.c_int(1 if constrain else 0))
        m = self.L.ref_pairs_count(_vp(h))
        i, j, s = np.zeros(m, np.int64), np.zeros(m, np.int64), np.zeros(m)
        self.L.ref_pairs_copy(_vp(h), _p(i), _p(j), _p(s))
        self.L.ref_pairs_free(_vp(h))
        return i, j, s

    def hc(self, rp, ci, pi, pj, ps, cluster_size):
        rp, ci, pi, pj, ps = _ll(rp), _ll(ci), _ll(pi), _ll(pj), _f8(ps)
        n = len(rp) - 1
        perm, offs = np.zeros(n, np.int64), np.zeros(n + 1, np.int64)
        nc = self.L.ref_hc(_p(rp), _p(ci), _i64(n), _p(pi), _p(pj), _p(ps), _i64(len(pi)), _i64(cluster_size),
                           _p(perm), _p(offs))
        return perm, offs[:nc + 1]

    def spgemm_kernel3(self, A, B, perm, offsets, sort_output=False, l2_fraction=-1.0):
        arp, aci, av = _ll(A[0]), _ll(A[1]), _f8(A[2])
        brp, bci, bv = _ll(B[0]), _ll(B[1]), _f8(B[2])
        perm, offsets = _ll(perm), _ll(offsets)
        n = len(arp) - 1
        bcols = int(B[3]) if len(B) > 3 else n
        h = self.L.ref_spgemm_kernel3(_i64(n), _i64(len(brp) - 1), _i64(len(aci)), _p(arp), _p(aci), _p(av),
                                      _i64(len(brp) - 1), _i64(bcols), _i64(len(bci)), _p(brp), _p(bci),
                                      _p(bv), _p(perm), _p(offsets), _i64(len(offsets) - 1),
                                      C.c_int(int(sort_output)), _dbl(l2_fraction))
        info = np.zeros(6, np.int64)
        self.L.ref_csr_info(_vp(h), _p(info))
        rp = np.zeros(info[0] + 1, np.int64)
        ci, v = np.zeros(max(info[2], 1), np.int64), np.zeros(max(info[2], 1))
        self.L.ref_csr_copy(_vp(h), _p(rp), _p(ci), _p(v))
        self.L.ref_csr_free(_vp(h))
        return dict(rp=rp, ci=ci[:info[2]], v=v[:info[2]], dense_clusters=int(info[3]), clusters=int(info[4]))

    def _ref_csr(self, h):
        info = np.zeros(6, np.int64)
        self.L.ref_csr_info(_vp(h), _p(info))
        rp = np.zeros(info[0] + 1, np.int64)
        ci, v = np.zeros(max(info[2], 1), np.int64), np.zeros(max(info[2], 1))
        self.L.ref_csr_copy(_vp(h), _p(rp), _p(ci), _p(v))
        self.L.ref_csr_free(_vp(h))
        return dict(rp=rp, ci=ci[:info[2]], v=v[:info[2]])

    def spgemm_rowwise(self, A, B, kernel_flag=1, sort_output=False):
        """The reference's LeSpGEMM<sortOutput, int64_t, double>(A, B, C, kernel_flag)."""
        arp, aci, av = _ll(A[0]), _ll(A[1]), _f8(A[2])
        brp, bci, bv = _ll(B[0]), _ll(B[1]), _f8(B[2])
        n = len(arp) - 1
        bcols = int(B[3]) if len(B) > 3 else n
        h = self.L.ref_spgemm_rowwise(_i64(n), _i64(len(brp) - 1), _i64(len(aci)), _p(arp), _p(aci), _p(av),
                                      _i64(len(brp) - 1), _i64(bcols), _i64(len(bci)), _p(brp), _p(bci), _p(bv),
                                      C.c_int(int(kernel_flag)), C.c_int(int(sort_output)))
        return self._ref_csr(h)

    def spgemm_topk(self, rp, ci, ncols, top_k, f32=False):
        """The reference's HashSpGEMMTopK<int64_t, V>(A, C, top_k)."""
        rp, ci = _ll(rp), _ll(ci)
        n = len(rp) - 1
        h = self.L.ref_spgemm_topk(_i64(n), _i64(ncols), _i64(len(ci)), _p(rp), _p(ci), _i64(top_k),
                                   C.c_int(1 if f32 else 0))
        return self._ref_csr(h)

    def read_csr(self, path, compact=False, f32=False):
        """The reference's read_csr_matrix<long long, V>(path, compact)."""
        self.L.ref_read_csr.restype = _vp
        h = self.L.ref_read_csr(str(path).encode(), C.c_int(int(compact)), C.c_int(int(f32)))
        return self._ref_csr(h)

    def spgemm_rowwise_time(self, A, B, kernel_flag=1, top_k=-1, iters=1):
        """Mean ms of the reference's LeSpGEMM<false>(A, B, C, kernel_flag), or
        of HashSpGEMMTopK(A, C, top_k) when top_k >= 0."""
        arp, aci, av = _ll(A[0]), _ll(A[1]), _f8(A[2])
        brp, bci, bv = _ll(B[0]), _ll(B[1]), _f8(B[2])
        n = len(arp) - 1
        bcols = int(B[3]) if len(B) > 3 else n
        self.L.ref_spgemm_rowwise_time.restype = C.c_double
        return float(self.L.ref_spgemm_rowwise_time(
            _i64(n), _i64(len(brp) - 1), _i64(len(aci)), _p(arp), _p(aci), _p(av), _i64(len(brp) - 1),
            _i64(bcols), _i64(len(bci)), _p(brp), _p(bci), _p(bv), C.c_int(int(kernel_flag)), _i64(top_k),
            C.c_int(int(iters))))

    def spgemm_kernel3_time(self, A, B, perm, offsets, iters=3, l2_fraction=-1.0):
        """Mean ms of the reference's LeSpGEMM_VLength kernel 3 (numeric and
        symbolic phases on the clustered A) over `iters` runs."""
        arp, aci, av = _ll(A[0]), _ll(A[1]), _f8(A[2])
        brp, bci, bv = _ll(B[0]), _ll(B[1]), _f8(B[2])
        perm, offsets = _ll(perm), _ll(offsets)
        n = len(arp) - 1
        bcols = int(B[3]) if len(B) > 3 else n
        self.L.ref_spgemm_kernel3_time.restype = C.c_double
        return float(self.L.ref_spgemm_kernel3_time(
            _i64(n), _i64(len(brp) - 1), _i64(len(aci)), _p(arp), _p(aci), _p(av), _i64(len(brp) - 1),
            _i64(bcols), _i64(len(bci)), _p(brp), _p(bci), _p(bv), _p(perm), _p(offsets), _i64(len(offsets) - 1),
            C.c_int(int(iters)), _dbl(l2_fraction)))

    def coo_to_csr(self, n, ncols, ri, ci, v, compact=False):
        """The reference's coo_to_csr<int64_t, double> (include/sparse_conversion.h:37)."""
        ri = np.ascontiguousarray(ri, np.int64)
        ci = np.ascontiguousarray(ci, np.int64)
        v = np.ascontiguousarray(v, np.float64)
        h = self.L.ref_coo_to_csr(_i64(n), _i64(ncols), _i64(len(ci)), _p(ri), _p(ci), _p(v),
                                  C.c_int(1 if compact else 0))
        info = np.zeros(6, np.int64)
        self.L.ref_csr_info(_vp(h), _p(info))
        rp = np.zeros(info[0] + 1, np.int64)
        oc, ov = np.zeros(max(info[2], 1), np.int64), np.zeros(max(info[2], 1))
        self.L.ref_csr_copy(_vp(h), _p(rp), _p(oc), _p(ov))
        self.L.ref_csr_free(_vp(h))
        return rp, oc[:info[2]], ov[:info[2]]

    def features(self, rp, ci, v, ncols):
        """The reference's MtxLoad + CalculateFeatures on the matrix written as
        a general real Matrix Market file (entries in CSR order)."""
        import tempfile
        fd, path = tempfile.mkstemp(suffix=".mtx")
        try:
            with os.fdopen(fd, "w") as f:
                n = len(rp) - 1
                f.write("%%MatrixMarket matrix coordinate real general\n")
                f.write(f"{n} {ncols} {len(ci)}\n")
                rows = np.repeat(np.arange(n), np.diff(np.asarray(rp, np.int64)))
                for r, c, x in zip(rows, ci, v):
                    f.write(f"{r + 1} {c + 1} {float(x)!r}\n")
            out = np.zeros(32)
            self.L.ref_features.restype = C.c_int
            rc = self.L.ref_features(path.encode(), _p(out))
            if rc != 0:
                raise RuntimeError(f"ref_features failed ({rc})")
            return out
        finally:
            os.remove(path)

    def tile_features(self, rp, ci, v, ncols):
        """The reference's MtxLoad + CalculateFeatures + CalculateTilesExtraFeatures
        tile features (its 256 x 256 grid) on the matrix written as a general
        real Matrix Market file; the same tuple as Oracle.tile_features."""
        import tempfile
        fd, path = tempfile.mkstemp(suffix=".mtx")
        try:
            with os.fdopen(fd, "w") as f:
                n = len(rp) - 1
                f.write("%%MatrixMarket matrix coordinate real general\n")
                f.write(f"{n} {ncols} {len(ci)}\n")
                rows = np.repeat(np.arange(n), np.diff(np.asarray(rp, np.int64)))
                for r, c, x in zip(rows, ci, v):
                    f.write(f"{r + 1} {c + 1} {float(x)!r}\n")
            B = 256
            sc, ti, td = np.zeros(34), np.zeros(4 * B * B, np.int64), np.zeros(2 * B * B)
            bi, bd = np.zeros(4 * B, np.int64), np.zeros(4 * B)
            self.L.ref_tile_features.restype = C.c_int
            rc = self.L.ref_tile_features(path.encode(), _p(sc), _p(ti), _p(td), _p(bi), _p(bd))
            if rc != 0:
                raise RuntimeError(f"ref_tile_features failed ({rc})")
            return sc, ti.reshape(4, -1), td.reshape(2, -1), bi.reshape(4, -1), bd.reshape(4, -1)
        finally:
            os.remove(path)

    def csr_transpose(self, rp, ci, v, ncols):
        """The reference's csr_transpose on int64 / FP64 copies of the arrays."""
        rp = np.ascontiguousarray(rp, np.int64)
        ci = np.ascontiguousarray(ci, np.int64)
        v = np.ascontiguousarray(v, np.float64)
        h = self.L.ref_csr_transpose(_i64(len(rp) - 1), _i64(ncols), _i64(len(ci)), _p(rp), _p(ci), _p(v))
        info = np.zeros(6, np.int64)
        self.L.ref_csr_info(_vp(h), _p(info))
        trp = np.zeros(info[0] + 1, np.int64)
        tci, tv = np.zeros(max(info[2], 1), np.int64), np.zeros(max(info[2], 1))
        self.L.ref_csr_copy(_vp(h), _p(trp), _p(tci), _p(tv))
        self.L.ref_csr_free(_vp(h))
        return trp, tci[:info[2]], tv[:info[2]]


def reference_available() -> bool:
    v = "v4" if _cpu_has_avx512() else "v3"
    return os.path.exists(os.path.join(HERE, "_ref", f"libspops_ref_{v}.so"))
