"""LeSpGEMM on the device: MinHash, LSH pairs, clustering, cluster-wise C = A*A^T.

Integer outputs (signatures, pairs, permutation, offsets, C row_ptr / col_idx)
bit-exact against the reference's golden outputs or the pinned oracle; C
values within 1e-12 of sum_k |a_ik b_kj| (componentwise).
"""
import numpy as np
import pytest

from sparseops_b200 import synth

pytestmark = pytest.mark.gpu


def _csr(rp, ci, v, ncols=None):
    import torch
    from sparseops_b200 import CSR_Matrix
    n = len(rp) - 1
    d = torch.device("cuda")
    return CSR_Matrix(n, n if ncols is None else ncols, torch.from_numpy(rp).to(d), torch.from_numpy(ci).to(d),
                      torch.from_numpy(v).to(d))


def _check_c(C, ref):
    rp, ci, v = C.host()
    assert np.array_equal(rp.astype(np.int64), ref["rp"])
    assert np.array_equal(ci.astype(np.int64), ref["ci"])
    err = np.abs(v - ref["v"]) / np.maximum(ref["absv"], 1e-300)
    assert (err.max() if len(err) else 0.0) <= 1e-12


def test_minhash_and_pairs_golden(cuda, golden):
    from sparseops_b200.spgemm import lsh_candidate_pairs_vector, minhash_signatures_flat
    g = golden
    A = _csr(g["sp_arp"], g["sp_aci"], g["sp_av"])
    assert np.array_equal(minhash_signatures_flat(A, 64, 7), g["sp_sig"])
    i, j, s = lsh_candidate_pairs_vector(A, 64, 16, 7).host()
    assert np.array_equal(i, g["sp_pi"]) and np.array_equal(j, g["sp_pj"]) and np.array_equal(s, g["sp_ps"])


def test_lsh_window_rule_golden(cuda, golden):
    from sparseops_b200.spgemm import lsh_candidate_pairs_vector
    rp = np.arange(0, 401 * 3, 3, dtype=np.int64)
    ci = np.tile(np.array([5, 17, 99], np.int64), 400)
    A = _csr(rp, ci, np.ones(len(ci)), ncols=100)
    i, j, s = lsh_candidate_pairs_vector(A, 64, 16, 7).host()
    assert np.array_equal(i, golden["big_pi"]) and np.array_equal(j, golden["big_pj"])
    assert np.array_equal(s, golden["big_ps"])


@pytest.mark.parametrize("so", [0, 1])
def test_spgemm_clustered_golden(cuda, golden, orc, so):
    from sparseops_b200.spgemm import LeSpGEMM_clustered
    g = golden
    arp, aci, av = g["sp_arp"], g["sp_aci"], g["sp_av"]
    brp, bci, bv = synth.transpose(arp, aci, av, 1024)
    C = LeSpGEMM_clustered(_csr(arp, aci, av), _csr(brp, bci, bv), g["sp_perm"], g["sp_offsets"], sort_output=bool(so))
    ref = orc.spgemm((arp, aci, av), (brp, bci, bv), g["sp_perm"], g["sp_offsets"], sort_output=bool(so))
    assert np.array_equal(C.host()[0].astype(np.int64), g[f"sp_c{so}_rp"])
    assert np.array_equal(C.host()[1].astype(np.int64), g[f"sp_c{so}_ci"])
    _check_c(C, ref)
    assert C.stats["dense_clusters"] == int(g[f"sp_c{so}_dense"])


@pytest.mark.parametrize("n,ncomm", [(16384, 64), (131072, 512)])
def test_pipeline_vs_oracle(cuda, orc, n, ncomm):
    """MinHash -> LSH -> clustering -> SpGEMM, every stage against the oracle."""
    from sparseops_b200.spgemm import (LeSpGEMM_clustered, LeSpGEMM_lsh, hierarchical_clustering_v0_fast,
                                       lsh_candidate_pairs_vector, minhash_signatures_flat)
    arp, aci, av = synth.planted_communities(n, ncomm=ncomm, mean=20.0, seed=17)
    brp, bci, bv = synth.transpose(arp, aci, av, n)
    A, B = _csr(arp, aci, av), _csr(brp, bci, bv)
    sig = minhash_signatures_flat(A, 64, 7)
    assert np.array_equal(sig, orc.minhash(arp, aci, 64, 7))
    pairs = lsh_candidate_pairs_vector(A, 64, 16, 7).host()
    opi, opj, ops = orc.lsh_pairs(sig, 16, True)
    assert np.array_equal(pairs[0], opi) and np.array_equal(pairs[1], opj) and np.array_equal(pairs[2], ops)
    perm, offs = hierarchical_clustering_v0_fast(arp, aci, n, pairs, 8)
    operm, ooffs = orc.hc(arp, aci, opi, opj, ops, 8)
    assert np.array_equal(perm, operm) and np.array_equal(offs, ooffs)
    ref = orc.spgemm((arp, aci, av), (brp, bci, bv), perm, offs)
    _check_c(LeSpGEMM_clustered(A, B, perm, offs), ref)
    C = LeSpGEMM_lsh(A, B, 64, 16, 7, 8)
    _check_c(C, ref)
    assert C.stats["flops"] == orc.spgemm_flop((arp, aci), (brp,))


def test_lsh_band_batches(cuda, orc):
    """More records than one batch of bands holds (2^24): 600,000 rows with 32
    bands of 4 hashes go in two batches; pairs, order and scores as the
    oracle's."""
    from sparseops_b200.spgemm import lsh_candidate_pairs_vector, minhash_signatures_flat
    n = 600000
    arp, aci, av = synth.planted_communities(n, ncomm=n // 256, mean=12.0, seed=23)
    A = _csr(arp, aci, av)
    sig = minhash_signatures_flat(A, 128, 11)
    pairs = lsh_candidate_pairs_vector(A, 128, 32, 11).host()
    opi, opj, ops = orc.lsh_pairs(sig, 32, True)
    assert len(opi) > 0
    assert np.array_equal(pairs[0], opi) and np.array_equal(pairs[1], opj) and np.array_equal(pairs[2], ops)


def test_int32_and_float32(cuda, orc):
    from sparseops_b200.spgemm import LeSpGEMM_lsh
    arp, aci, av = synth.planted_communities(8192, ncomm=32, mean=12.0, seed=19)
    brp, bci, bv = synth.transpose(arp, aci, av, 8192)
    C = LeSpGEMM_lsh(_csr(arp.astype(np.int32), aci.astype(np.int32), av),
                     _csr(brp.astype(np.int32), bci.astype(np.int32), bv), 64, 16, 7, 8)
    C64 = LeSpGEMM_lsh(_csr(arp, aci, av), _csr(brp, bci, bv), 64, 16, 7, 8)
    assert np.array_equal(C.host()[0], C64.host()[0]) and np.array_equal(C.host()[1], C64.host()[1])
    assert np.array_equal(C.host()[2], C64.host()[2])
    C32 = LeSpGEMM_lsh(_csr(arp, aci, av.astype(np.float32)), _csr(brp, bci, bv.astype(np.float32)), 64, 16, 7, 8)
    assert np.array_equal(C32.host()[0], C64.host()[0])
    rel = np.abs(C32.host()[2] - C64.host()[2]) / (np.abs(C64.host()[2]) + 1e-3)
    assert rel.max() < 1e-3


def test_full_config_properties(cuda):
    """Config size (524,288 rows, 2,048 communities): C = A*A^T must be
    symmetric, and C*1 = A*(A^T*1) (linearity), checked with the SpMV kernels."""
    import torch
    from sparseops_b200 import CSR_Matrix, SpOps_csr
    from sparseops_b200.spgemm import LeSpGEMM_lsh
    n = 524288
    arp, aci, av = synth.planted_communities(n, ncomm=2048, mean=20.0, seed=5)
    brp, bci, bv = synth.transpose(arp, aci, av, n)
    A, B = _csr(arp, aci, av), _csr(brp, bci, bv)
    C = LeSpGEMM_lsh(A, B, 64, 16, 7, 8)
    rp, ci, v = C.host()
    assert C.stats["flops"] > 0 and rp[-1] == len(ci)
    # symmetry on 2,000 random rows: every (i, j, v) has its (j, i, v)
    rng = np.random.default_rng(1)
    for i in rng.integers(0, n, 2000):
        for t in range(rp[i], rp[i + 1]):
            j = ci[t]
            q = rp[j] + np.searchsorted(ci[rp[j]:rp[j + 1]], i)
            assert q < rp[j + 1] and ci[q] == i
            assert abs(v[q] - v[t]) <= 1e-12 * (1 + abs(v[t]) + np.abs(v[rp[i]:rp[i + 1]]).max())
    # linearity: C*1 vs A*(B*1)
    d = torch.device("cuda")
    ones = torch.ones(n, dtype=torch.float64, device=d)
    t, y1, y2 = (torch.zeros(n, dtype=torch.float64, device=d) for _ in range(3))
    SpOps_csr(1.0, B, ones, 0.0, t)
    SpOps_csr(1.0, A, t, 0.0, y1)
    Cd = CSR_Matrix(n, n, torch.from_numpy(rp).to(d), torch.from_numpy(ci).to(d), torch.from_numpy(v).to(d))
    SpOps_csr(1.0, Cd, ones, 0.0, y2)
    torch.cuda.synchronize()
    scale = torch.zeros(n, dtype=torch.float64, device=d)
    Ad = CSR_Matrix(n, n, torch.from_numpy(arp).to(d), torch.from_numpy(aci).to(d), torch.from_numpy(np.abs(av)).to(d))
    Bd = CSR_Matrix(n, n, torch.from_numpy(brp).to(d), torch.from_numpy(bci).to(d), torch.from_numpy(np.abs(bv)).to(d))
    tt = torch.zeros(n, dtype=torch.float64, device=d)
    SpOps_csr(1.0, Bd, ones, 0.0, tt)
    SpOps_csr(1.0, Ad, tt, 0.0, scale)
    torch.cuda.synchronize()
    assert float(((y1 - y2).abs() / (scale + 1e-300)).max()) <= 1e-12


@pytest.mark.parametrize("itype", [np.int32, np.int64])
def test_rowwise_golden(cuda, golden, orc, itype):
    """Row-wise LeSpGEMM kernels 1-3 against the reference's sorted output."""
    from sparseops_b200.spgemm import LeSpGEMM
    g = golden
    arp, aci, av = g["sp_arp"], g["sp_aci"], g["sp_av"]
    brp, bci, bv = synth.transpose(arp, aci, av, 1024)
    ref = orc.spgemm_rowwise((arp, aci, av), (brp, bci, bv))
    A = _csr(arp.astype(itype), aci.astype(itype), av)
    B = _csr(brp.astype(itype), bci.astype(itype), bv)
    for kf in (1, 2, 3):
        for so in (False, True):
            C = LeSpGEMM(A, B, kf, so)
            rp, ci, v = C.host()
            assert np.array_equal(rp.astype(np.int64), g[f"rw{kf}_rp"])
            assert np.array_equal(ci.astype(np.int64), g[f"rw{kf}_ci"])
            err = np.abs(v - g[f"rw{kf}_v"]) / np.maximum(ref["absv"], 1e-300)
            assert err.max() <= 1e-12


def test_rowwise_keeps_exact_zeros(cuda, orc):
    """Products that cancel exactly stay in C as zeros (the reference keeps
    every structural entry of the symbolic phase)."""
    from sparseops_b200.spgemm import LeSpGEMM
    arp = np.array([0, 2, 3], np.int64)
    aci = np.array([0, 1, 1], np.int64)
    av = np.array([1.0, -1.0, 2.0])
    brp = np.array([0, 1, 2], np.int64)
    bci = np.array([0, 0], np.int64)
    bv = np.array([3.0, 3.0])
    rp, ci, v = LeSpGEMM(_csr(arp, aci, av), _csr(brp, bci, bv), 1, True).host()
    assert list(rp) == [0, 1, 2] and list(ci) == [0, 0] and list(v) == [0.0, 6.0]
    ref = orc.spgemm_rowwise((arp, aci, av), (brp, bci, bv))
    assert np.array_equal(ref["rp"], rp) and np.array_equal(ref["v"], v)


@pytest.mark.parametrize("f32", [0, 1])
@pytest.mark.parametrize("itype", [np.int32, np.int64])
def test_topk_golden(cuda, golden, f32, itype):
    from sparseops_b200.spgemm import HashSpGEMMTopK
    g = golden
    vt = np.float32 if f32 else np.float64
    A = _csr(g["sp_arp"].astype(itype), g["sp_aci"].astype(itype), g["sp_av"].astype(vt))
    rp, ci, v = HashSpGEMMTopK(A, 6).host()
    assert np.array_equal(rp.astype(np.int64), g[f"topk{f32}_rp"])
    assert np.array_equal(ci.astype(np.int64), g[f"topk{f32}_ci"])
    assert np.array_equal(v.astype(np.float64), g[f"topk{f32}_v"])


@pytest.mark.parametrize("k", [0, 1, 16, 32, 33, 40])
def test_topk_vs_oracle(cuda, orc, k):
    """A larger planted matrix; k = 0 keeps nothing, k <= 32 takes the warp
    selection and 33, 40 the sort, 40 exceeds many rows."""
    from sparseops_b200.spgemm import HashSpGEMMTopK
    arp, aci, av = synth.planted_communities(20000, ncomm=128, mean=14.0, seed=29)
    ref = orc.spgemm_topk(arp, aci, 20000, k)
    rp, ci, v = HashSpGEMMTopK(_csr(arp, aci, av), k).host()
    assert np.array_equal(rp.astype(np.int64), ref["rp"])
    assert np.array_equal(ci.astype(np.int64), ref["ci"])
    assert np.array_equal(v, ref["v"])


@pytest.mark.parametrize("k", [5, 16, 32])
def test_topk_ties_and_long_rows(cuda, orc, k):
    """Groups of identical rows (every pair in a group has similarity 1, so
    the ranking falls back to the column) next to rows that share single
    columns with thousands of others (long rows of the counts product, many
    candidate merges per row)."""
    from sparseops_b200.spgemm import HashSpGEMMTopK
    rng = np.random.default_rng(31)
    rows = []
    for g in range(40):  # 40 groups of 75 identical rows, 8 columns each
        pat = np.sort(rng.choice(4000, 8, replace=False))
        rows += [pat] * 75
    hub = np.sort(rng.choice(4000, 3, replace=False))
    for _ in range(500):  # rows holding one of three hub columns and 4 random ones
        rows.append(np.unique(np.concatenate([hub[rng.integers(0, 3, 1)], rng.choice(4000, 4, replace=False)])))
    order = rng.permutation(len(rows))
    rows = [rows[o] for o in order]
    n = len(rows)
    rp = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int64)
    ci = np.concatenate(rows).astype(np.int64)
    av = np.ones(len(ci))
    ref = orc.spgemm_topk(rp, ci, 4000, k)
    got_rp, got_ci, got_v = HashSpGEMMTopK(_csr(rp, ci, av, 4000), k).host()
    assert np.array_equal(got_rp.astype(np.int64), ref["rp"])
    assert np.array_equal(got_ci.astype(np.int64), ref["ci"])
    assert np.array_equal(got_v, ref["v"])


@pytest.mark.parametrize("k", [1, 16, 32])
def test_topk_every_table_size(cuda, orc, k):
    """Rows of every product count the top-k path bins by: short random rows
    (tables of 256 and 1024 slots), rows of three 3000-row hub blocks (about
    3000 products: one block's table of 16384 slots) and four rows that hold
    all three hubs (more than 8192 products: tables in global memory)."""
    from sparseops_b200.spgemm import HashSpGEMMTopK
    rng = np.random.default_rng(37)
    n, ncols = 12000, 60000
    rows = [set(rng.choice(ncols - 3, int(rng.integers(1, 9)), replace=False).tolist()) for _ in range(n)]
    for h in range(3):
        for r in range(3000 * h, 3000 * (h + 1)):
            rows[r].add(ncols - 3 + h)
    for r in (9000, 9001, 11998, 11999):
        rows[r].update({ncols - 3, ncols - 2, ncols - 1})
    rows = [np.array(sorted(r), np.int64) for r in rows]
    rp = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int64)
    ci = np.concatenate(rows)
    ref = orc.spgemm_topk(rp, ci, ncols, k)
    for itype, vtype in [(np.int64, np.float64), (np.int32, np.float32)]:
        got = HashSpGEMMTopK(_csr(rp.astype(itype), ci.astype(itype), np.ones(len(ci), vtype), ncols), k).host()
        if vtype == np.float32:
            ref = orc.spgemm_topk(rp, ci, ncols, k, f32=True)
        assert np.array_equal(got[0].astype(np.int64), ref["rp"])
        assert np.array_equal(got[1].astype(np.int64), ref["ci"])
        assert np.array_equal(got[2].astype(np.float64), ref["v"])
    from sparseops_b200 import default_context
    assert default_context().check_device() == 0


@pytest.mark.parametrize("so", [0, 1])
def test_vlength_pipeline_golden(cuda, golden, orc, so):
    """The reference driver's flow (test/test_spgemm_hc_lsh.cpp:230-300):
    csr_reorder_rows by the clustering, csr_to_vlength_cluster,
    LeSpGEMM_VLength, vlength_cluster2csr and the inverse reorder give the
    reference's C (structure bit-exact, values to 1e-12)."""
    from sparseops_b200 import csr_reorder_rows
    from sparseops_b200.spgemm import LeSpGEMM_VLength, csr_to_vlength_cluster, vlength_cluster2csr
    g = golden
    arp, aci, av = g["sp_arp"], g["sp_aci"], g["sp_av"]
    brp, bci, bv = synth.transpose(arp, aci, av, 1024)
    perm, offs = g["sp_perm"], g["sp_offsets"]
    Acl = csr_to_vlength_cluster(csr_reorder_rows(_csr(arp, aci, av), perm), offs)
    h = Acl.host()
    assert h["cluster_sz"].sum() == len(perm) and h["rowptr"][-1] == Acl.nnzc and h["rowptr_val"][-1] == Acl.nnzv
    assert Acl.max_cluster_sz == 256  # the reference starts it at 256
    Ccl = LeSpGEMM_VLength(Acl, _csr(brp, bci, bv), sort_output=bool(so))
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    C = csr_reorder_rows(vlength_cluster2csr(Ccl), inv)
    assert np.array_equal(C.host()[0].astype(np.int64), g[f"sp_c{so}_rp"])
    assert np.array_equal(C.host()[1].astype(np.int64), g[f"sp_c{so}_ci"])
    _check_c(C, orc.spgemm((arp, aci, av), (brp, bci, bv), perm, offs, sort_output=bool(so)))


@pytest.mark.parametrize("itype,vtype", [(np.int32, np.float64), (np.int64, np.float32)])
def test_vlength_cluster_layout(cuda, itype, vtype):
    """csr_to_vlength_cluster against a plain construction: each cluster's
    columns ascending, values[rowptr_val[c] + p * sz + k]; vlength_cluster2csr
    gives the CSR back (rows sorted, no explicit zeros)."""
    from sparseops_b200.spgemm import csr_to_vlength_cluster, vlength_cluster2csr
    rng = np.random.default_rng(17)
    n, nc = 3000, 900
    rows = [np.sort(rng.choice(nc, int(rng.integers(0, 12)), replace=False)) for _ in range(n)]
    rp = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(itype)
    ci = np.concatenate(rows).astype(itype)
    v = (rng.standard_normal(len(ci)) + 3.0).astype(vtype)  # no zeros
    sizes = rng.integers(1, 14, 600)
    offs = np.concatenate([[0], np.cumsum(sizes)])
    offs = offs[offs < n]
    offs = np.concatenate([offs, [n]]).astype(np.int64)
    cl = csr_to_vlength_cluster(_csr(rp, ci, v, nc), offs)
    h = cl.host()
    assert cl.rows == len(offs) - 1 and np.array_equal(h["cluster_sz"], np.diff(offs))
    p0 = 0
    for c in range(cl.rows):
        r0, r1 = offs[c], offs[c + 1]
        cols = np.unique(ci[rp[r0]:rp[r1]].astype(np.int64))
        got = h["colids"][h["rowptr"][c]:h["rowptr"][c + 1]].astype(np.int64)
        assert np.array_equal(got, cols), c
        sz = r1 - r0
        block = h["values"][h["rowptr_val"][c]:h["rowptr_val"][c + 1]].reshape(len(cols), sz)
        for k in range(sz):
            r = r0 + k
            rc, rv = ci[rp[r]:rp[r + 1]].astype(np.int64), v[rp[r]:rp[r + 1]]
            want = np.zeros(len(cols), vtype)
            want[np.searchsorted(cols, rc)] = rv
            assert np.array_equal(block[:, k], want), (c, k)
        p0 += len(cols)
    assert p0 == cl.nnzc
    back = vlength_cluster2csr(cl).host()
    assert np.array_equal(back[0].astype(np.int64), rp.astype(np.int64))
    assert np.array_equal(back[1].astype(np.int64), ci.astype(np.int64)) and np.array_equal(back[2], v)


def _vl_edge_case(rng):
    """1200 x 500 A (every 7th row empty; rows 1000.. only in columns 400..,
    which are B's empty rows) and 500 x 400 B, with positive values so that
    no product cancels; clusters: one of 300 rows, two of none, then tens."""
    n, k, m = 1200, 500, 400
    lens = rng.integers(0, 5, n)
    lens[::7] = 0
    rows = [np.sort(rng.choice(400, int(ln), replace=False)) if r < 1000 else
            np.sort(rng.choice(np.arange(400, k), int(ln), replace=False)) for r, ln in enumerate(lens)]
    arp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    aci = np.concatenate(rows).astype(np.int64)
    av = rng.uniform(0.5, 2.0, len(aci))
    blens = rng.integers(0, 6, k)
    blens[400:] = 0
    brp = np.concatenate([[0], np.cumsum(blens)]).astype(np.int64)
    bci = np.concatenate([np.sort(rng.choice(m, int(ln), replace=False)) for ln in blens]).astype(np.int64)
    bv = rng.uniform(0.5, 2.0, len(bci))
    offs = np.array([0, 300, 300, 300] + list(range(310, n, 10)) + [n], np.int64)
    return (arp, aci, av, k), (brp, bci, bv, m), offs


@pytest.mark.parametrize("so", [0, 1])
def test_vlength_edges(cuda, so):
    """Empty clusters, a cluster of 300 rows (max_cluster_sz follows it; its
    accumulator exceeds shared memory), empty rows, and clusters whose
    product is empty: vlength_cluster2csr(LeSpGEMM_VLength) equals A*B."""
    import scipy.sparse as sp
    from sparseops_b200.spgemm import LeSpGEMM_VLength, csr_to_vlength_cluster, vlength_cluster2csr
    (arp, aci, av, k), (brp, bci, bv, m), offs = _vl_edge_case(np.random.default_rng(23))
    n = len(arp) - 1
    Acl = csr_to_vlength_cluster(_csr(arp, aci, av, k), offs)
    assert Acl.rows == len(offs) - 1 and Acl.max_cluster_sz == 300
    Ccl = LeSpGEMM_VLength(Acl, _csr(brp, bci, bv, m), sort_output=bool(so))
    assert Ccl.rows == Acl.rows and Ccl.max_cluster_sz == 300 and Ccl.csr_rows == n and Ccl.cols == m
    h = Ccl.host()
    assert np.array_equal(h["cluster_sz"].astype(np.int64), np.diff(offs))
    late = np.searchsorted(offs, 1000)  # clusters of rows 1000.. have no products
    assert np.all(np.diff(h["rowptr"].astype(np.int64))[late:] == 0)
    want = (sp.csr_matrix((av, aci, arp), shape=(n, k)) @ sp.csr_matrix((bv, bci, brp), shape=(k, m))).tocsr()
    want.sort_indices()
    rp, ci, v = vlength_cluster2csr(Ccl).host()
    got = sp.csr_matrix((v, ci.astype(np.int64), rp.astype(np.int64)), shape=(n, m))
    got.sort_indices()
    assert np.array_equal(got.indptr, want.indptr) and np.array_equal(got.indices, want.indices)
    assert np.abs(got.data - want.data).max() <= 1e-12 * np.abs(want.data).max()


def test_vlength_refusals(cuda):
    """Offsets that do not run from 0 to rows or go backwards, a plain CSR
    where a clustered A is expected, and mismatched inner sizes are errors."""
    from sparseops_b200._lib import SpOpsError
    from sparseops_b200.spgemm import LeSpGEMM_VLength, VLengthCluster, csr_to_vlength_cluster
    (arp, aci, av, k), (brp, bci, bv, m), offs = _vl_edge_case(np.random.default_rng(29))
    A = _csr(arp, aci, av, k)
    for bad in ([0, 600, 1100], [1, 600, 1200], [0, 700, 600, 1200]):
        with pytest.raises(SpOpsError):
            csr_to_vlength_cluster(A, np.array(bad, np.int64))
    Acl = csr_to_vlength_cluster(A, offs)
    with pytest.raises(SpOpsError):
        LeSpGEMM_VLength(Acl, _csr(arp, aci, av, k))  # 500 columns of A against 1200 rows
    fake = VLengthCluster.__new__(VLengthCluster)
    fake._h, fake._codes = A.device(), Acl._codes
    with pytest.raises(SpOpsError):
        LeSpGEMM_VLength(fake, _csr(brp, bci, bv, m))
