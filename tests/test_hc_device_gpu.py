"""Hierarchical clustering on the device (spops_pairs_cluster): the same
permutation and offsets as the host loop (csrc/hc.cpp) and the reference's
hierarchical_clustering_v0_fast (include/spgemm_utility.h:742-915), bit for
bit, on LSH pairs of planted-community matrices, on rows in groups that
produce long merge chains and pairs found while merging, and on random pair
lists whose scores tie often."""
import numpy as np
import pytest

from sparseops_b200 import synth

pytestmark = pytest.mark.gpu


def _csr(rp, ci, ncols):
    import torch
    from sparseops_b200 import CSR_Matrix
    d = torch.device("cuda")
    return CSR_Matrix(len(rp) - 1, ncols, torch.from_numpy(rp).to(d), torch.from_numpy(ci).to(d),
                      torch.ones(len(ci), dtype=torch.float64, device=d))


def _check(rp, ci, ncols, cluster_size, ref):
    from sparseops_b200.spgemm import (hierarchical_clustering_device, hierarchical_clustering_v0_fast,
                                       lsh_candidate_pairs_vector)
    A = _csr(rp, ci, ncols)
    pairs = lsh_candidate_pairs_vector(A, 64, 16, 7)
    n = len(rp) - 1
    hperm, hoffs = hierarchical_clustering_v0_fast(rp, ci, n, pairs, cluster_size)
    dperm, doffs = hierarchical_clustering_device(A, pairs, cluster_size)
    assert np.array_equal(dperm, hperm) and np.array_equal(doffs, hoffs)
    pi, pj, ps = pairs.host()
    rperm, roffs = ref.hc(rp, ci, pi, pj, ps, cluster_size)
    assert np.array_equal(dperm, rperm) and np.array_equal(doffs, roffs)
    return len(doffs) - 1


@pytest.mark.parametrize("n,ncomm,cs", [(16384, 64, 8), (131072, 512, 8), (131072, 512, 3)])
def test_device_hc_planted(cuda, ref, n, ncomm, cs):
    rp, ci, _ = synth.planted_communities(n, ncomm=ncomm, mean=20.0, seed=17)
    _check(rp, ci, n, cs, ref)


@pytest.mark.parametrize("group,width,cs", [(32, 12, 8), (64, 16, 8), (16, 8, 4), (128, 24, 14)])
def test_device_hc_grouped(cuda, ref, group, width, cs):
    """Near-duplicate rows in groups: many tasks competing for few clusters,
    and pairs found while merging."""
    n = 65536
    rp, ci, _, nc = synth.grouped_rows(n, group=group, width=width, seed=group + width)
    assert _check(rp, ci, nc, cs, ref) < n  # clusters did form


def test_device_hc_random_pairs(cuda, ref):
    """Random pair lists (sorted, i < j, unique) with scores from a handful of
    values, so equal scores break ties on (i, j)."""
    from sparseops_b200.spgemm import hierarchical_clustering_device, hierarchical_clustering_v0_fast, pairs_from_arrays
    rng = np.random.default_rng(5)
    for trial in range(6):
        n = int(rng.integers(50, 3000))
        rp, ci, _ = synth.planted_communities(n, ncomm=max(1, n // 40), mean=6.0, seed=100 + trial)
        m = int(rng.integers(10, 6 * n))
        a, b = rng.integers(0, n, m), rng.integers(0, n, m)
        keep = a != b
        a, b = np.minimum(a[keep], b[keep]), np.maximum(a[keep], b[keep])
        key = np.unique(a * n + b)
        pi, pj = key // n, key % n
        ps = rng.integers(0, 9, len(pi)) / 8.0
        cs = int(rng.integers(2, 10))
        hperm, hoffs = hierarchical_clustering_v0_fast(rp, ci, n, (pi, pj, ps), cs)
        rperm, roffs = ref.hc(rp, ci, pi, pj, ps, cs)
        assert np.array_equal(hperm, rperm) and np.array_equal(hoffs, roffs)
        dperm, doffs = hierarchical_clustering_device(_csr(rp, ci, n), pairs_from_arrays(pi, pj, ps), cs)
        assert np.array_equal(dperm, hperm) and np.array_equal(doffs, hoffs), trial


def test_device_hc_unsorted_pairs_take_the_host_loop(cuda):
    """A pair list that is not sorted i < j pairs gives the host loop's result."""
    from sparseops_b200.spgemm import hierarchical_clustering_device, hierarchical_clustering_v0_fast, pairs_from_arrays
    rp, ci, _ = synth.planted_communities(2000, ncomm=40, mean=6.0, seed=9)
    pi = np.array([5, 3, 7, 100], np.int64)
    pj = np.array([9, 1, 8, 50], np.int64)
    ps = np.array([0.5, 0.5, 0.25, 0.75])
    hperm, hoffs = hierarchical_clustering_v0_fast(rp, ci, 2000, (pi, pj, ps), 4)
    dperm, doffs = hierarchical_clustering_device(_csr(rp, ci, 2000), pairs_from_arrays(pi, pj, ps), 4)
    assert np.array_equal(dperm, hperm) and np.array_equal(doffs, hoffs)
