"""Parity at the full sizes of the benchmark configurations, against the
reference library itself (oracle/_ref, compiled from the reference's sources)
or the oracle.

* LeSpGEMM, C = A*A^T with A 524,288 x 524,288 (2,048 planted column
  communities, 85 % of a row's entries in its community, row nnz lognormal
  mean 20, seed 5), and with A 524,288 x 196,608 in contiguous groups of 32
  rows that share a 12-column block (multi-row clusters, most of them dense
  under the reference's rule): the device MinHash signatures (64 hashes, seed 7), the LSH
  pair list (16 bands) and the clustering permutation / offsets (cluster size
  8) bit-equal to the reference's minhash_signatures_flat,
  lsh_candidate_pairs_vector and hierarchical_clustering_v0_fast on the same
  input (the clustering both by the host loop and on the device); C bit-equal in row_ptr and per-row col_idx to the reference's kernel
  3 run through its test driver's flow (csr_reorder_rows,
  csr_to_vlength_cluster, LeSpGEMM_VLength, vlength_cluster2csr, inverse
  reorder; test/test_spgemm_hc_lsh.cpp:230-300) for sortOutput false and
  true, values within 1e-12 of sum_k |a_ik b_kj| per entry.
* SELL-C-sigma (C = 32, sigma = 512) and SELL-C-R (C = 32) of the power-law
  matrix (4,194,304 rows, lognormal(ln 12, 1.2) row lengths clipped to
  [1, 20000], seed 1): reorder and chunk_len bit-equal to the reference's
  csr_to_sell_c_sigma / csr_to_sell_c_R (include/sparse_conversion.h:344-606).
* The 256-matrix batch (n log-uniform in [1e3, 2e5], Poisson(16) entries per
  row, half within bandwidth 64, seed 2024) at k = 1, 8 and 32 right-hand
  sides, autotuned and graph-captured, against the oracle's per-matrix SpMM
  (a loop of SpOps_csr in the reference), componentwise within 1e-12.
"""
import concurrent.futures as cf
import math
import os

import numpy as np
import pytest

from sparseops_b200 import synth

pytestmark = pytest.mark.gpu

N_SPGEMM = 524288


def _spgemm_workload(name):
    """(rows, A's columns, A, B = A^T) of a SpGEMM benchmark workload."""
    n = N_SPGEMM
    if name == "planted":
        arp, aci, av = synth.planted_communities(n, ncomm=2048, mean=20.0, seed=5)
        nc = n
    else:  # contiguous row groups sharing a 12-column block: multi-row and dense clusters
        arp, aci, av, nc = synth.grouped_rows(n)
    brp, bci, bv = synth.transpose(arp, aci, av, nc)
    return n, nc, (arp, aci, av), (brp, bci, bv)


@pytest.fixture(scope="module")
def full_ref():
    from oracle import Reference, reference_available
    if not reference_available():
        pytest.skip("reference library (oracle/_ref) not built")
    return Reference(threads=os.cpu_count())


def _dev_csr(rp, ci, v, ncols):
    import torch
    from sparseops_b200 import CSR_Matrix
    d = torch.device("cuda")
    return CSR_Matrix(len(rp) - 1, ncols, torch.from_numpy(rp).to(d), torch.from_numpy(ci).to(d),
                      torch.from_numpy(v).to(d))


def _rows_sorted(rp, ci, v):
    """Each row's entries in ascending column order (rows kept in place)."""
    rows = np.repeat(np.arange(len(rp) - 1, dtype=np.int64), np.diff(rp))
    order = np.lexsort((ci, rows))
    return ci[order], v[order]


@pytest.mark.parametrize("workload", ["planted", "grouped"])
def test_spgemm_full_config_vs_reference(cuda, full_ref, orc, workload):
    from sparseops_b200.spgemm import (LeSpGEMM_clustered, hierarchical_clustering_device,
                                       hierarchical_clustering_v0_fast, lsh_candidate_pairs_vector,
                                       minhash_signatures_flat)
    n, nc, (arp, aci, av), (brp, bci, bv) = _spgemm_workload(workload)
    A, B = _dev_csr(arp, aci, av, nc), _dev_csr(brp, bci, bv, n)
    # MinHash signatures, 64 hashes, seed 7
    sig = minhash_signatures_flat(A, 64, 7)
    assert np.array_equal(sig, full_ref.minhash(arp, aci, 64, 7))
    del sig
    # LSH pairs, 16 bands (pairs, their order and their scores)
    dpairs = lsh_candidate_pairs_vector(A, 64, 16, 7)
    pairs = dpairs.host()
    rpi, rpj, rps = full_ref.lsh_pairs(arp, aci, 64, 16, 7)
    assert np.array_equal(pairs[0], rpi) and np.array_equal(pairs[1], rpj) and np.array_equal(pairs[2], rps)
    # clustering, cluster size 8
    perm, offs = hierarchical_clustering_v0_fast(arp, aci, n, pairs, 8)
    rperm, roffs = full_ref.hc(arp, aci, rpi, rpj, rps, 8)
    assert np.array_equal(perm, rperm) and np.array_equal(offs, roffs)
    dperm, doffs = hierarchical_clustering_device(A, dpairs, 8)  # the pipeline's clustering, on the device
    assert np.array_equal(dperm, rperm) and np.array_equal(doffs, roffs)
    del dpairs, dperm, doffs
    # error scale sum_k |a_ik b_kj| per entry of C (rows ascending)
    scale = orc.spgemm((arp, aci, av), (brp, bci, bv), perm, offs, sort_output=True)
    for so in (0, 1):
        C = LeSpGEMM_clustered(A, B, perm, offs, sort_output=bool(so))
        crp, cci, cv = C.host()
        C_dense = C.stats["dense_clusters"]
        del C
        ref = full_ref.spgemm_kernel3((arp, aci, av), (brp, bci, bv, n), rperm, roffs, sort_output=bool(so))
        if workload == "grouped":
            assert C_dense == ref["dense_clusters"] > 0
        assert np.array_equal(crp.astype(np.int64), ref["rp"])
        rci, rv = _rows_sorted(ref["rp"], ref["ci"], ref["v"])
        del ref
        assert np.array_equal(cci.astype(np.int64), rci)
        if so == 1:  # the sorted path has the oracle's structure exactly
            assert np.array_equal(scale["ci"], rci)
            den = scale["absv"]
        else:  # sort 0 keeps every structural column: look the scale up per entry
            key_s = scale["ci"] + np.repeat(np.arange(n, dtype=np.int64), np.diff(scale["rp"])) * n
            key_c = rci + np.repeat(np.arange(n, dtype=np.int64), np.diff(crp.astype(np.int64))) * n
            pos = np.searchsorted(key_s, key_c)
            hit = (pos < len(key_s)) & (key_s[np.minimum(pos, len(key_s) - 1)] == key_c)
            den = np.where(hit, scale["absv"][np.minimum(pos, len(key_s) - 1)], np.abs(rv))
        err = np.abs(cv - rv) / np.maximum(den, 1e-300)
        assert (err.max() if len(err) else 0.0) <= 1e-12
        del crp, cci, cv, rci, rv, den, err


@pytest.mark.parametrize("kind", ["sell_c_sigma", "sell_c_R"])
def test_powerlaw_full_sell_layout_vs_reference(cuda, full_ref, kind):
    from sparseops_b200 import csr_to_sell_c_R, csr_to_sell_c_sigma
    n = 4194304
    rp, ci, v = synth.powerlaw(n, mu=math.log(12.0), sigma=1.2, lo=1, hi=20000, seed=1)
    A = _dev_csr(rp, ci, v, n)
    if kind == "sell_c_sigma":
        S = csr_to_sell_c_sigma(A, None, 512, 32, 8)
        h = full_ref.fmt_build("sell_c_sigma", rp, ci, v, n, 512, 32, 8, flag=1)
        nchunks = int(full_ref.fmt_info(h)[2])
    else:
        S = csr_to_sell_c_R(A, None, 32, 8)
        h = full_ref.fmt_build("sell_c_R", rp, ci, v, n, 0, 32, 8, flag=1)
        nchunks = int(full_ref.fmt_info(h)[0])
    reorder, chunk_len = np.zeros(n, np.int32), np.zeros(nchunks, np.int32)
    full_ref.fmt_copy(h, reorder, chunk_len, None, None)
    full_ref.fmt_free(h)
    assert len(S.chunk_len) == nchunks
    assert np.array_equal(np.asarray(S.reorder, np.int32), reorder)
    assert np.array_equal(np.asarray(S.chunk_len, np.int32), chunk_len)


def _batch_config(count=256, seed=2024):
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(1e3), np.log(2e5), count)).astype(np.int64)
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        return list(ex.map(lambda m: synth.banded_random(int(ns[m]), 16.0, 64, seed=5000 + m), range(count)))


@pytest.mark.parametrize("k", [1, 8, 32])
def test_batched_full_config_vs_oracle(cuda, orc, k):
    import torch
    from sparseops_b200 import Batch
    mats = _batch_config()
    dev = torch.device("cuda")
    A = [_dev_csr(rp, ci, v, len(rp) - 1) for rp, ci, v in mats]
    Xs = [synth.uniform((len(rp) - 1) * k, 300 + i).reshape(-1, k) for i, (rp, _, _) in enumerate(mats)]
    X = [torch.from_numpy(x).to(dev) for x in Xs]
    Y = [torch.zeros(len(rp) - 1, k, dtype=torch.float64, device=dev) for rp, _, _ in mats]
    if k == 1:
        X = [x.reshape(-1) for x in X]
        Y = [y.reshape(-1) for y in Y]
    B = Batch(A, k=k)
    B.set_vectors(X, Y)
    B.tune()
    B.capture(1.0, 0.0)
    B.run()
    torch.cuda.synchronize()
    got = [y.cpu().numpy().reshape(-1, k) for y in Y]
    del B, X, Y, A
    torch.cuda.empty_cache()

    def check(i):
        rp, ci, v = mats[i]
        ref = orc.spmm_csr(rp, ci, v, Xs[i])
        den = orc.spmm_csr(rp, ci, np.abs(v), np.abs(Xs[i]))
        return float((np.abs(got[i] - ref) / np.maximum(den, 1e-300)).max())

    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        worst = max(ex.map(check, range(len(mats))))
    assert worst <= 1e-12
