"""The product's host clustering (spops_hierarchical_clustering) against the
reference's own output (golden fixtures), bit for bit.  Runs without a GPU:
the clustering is sequential host code inside libsparseops_b200.so."""
import numpy as np

from sparseops_b200.spgemm import hierarchical_clustering_v0_fast


def test_hc_matches_reference(golden):
    g = golden
    perm, offs = hierarchical_clustering_v0_fast(g["sp_arp"], g["sp_aci"], len(g["sp_arp"]) - 1,
                                                 (g["sp_pi"], g["sp_pj"], g["sp_ps"]), 8)
    assert np.array_equal(perm, g["sp_perm"]) and np.array_equal(offs, g["sp_offsets"])


def test_hc_matches_oracle_on_dense_pairs(orc):
    """Many merges, discovered root pairs and closed clusters: random scores on
    a random pair list, product vs oracle (itself pinned to the reference)."""
    from sparseops_b200 import synth
    rp, ci, v = synth.planted_communities(3000, ncomm=40, mean=10.0, seed=21)
    rng = np.random.default_rng(4)
    i = rng.integers(0, 3000, 20000)
    j = rng.integers(0, 3000, 20000)
    keep = i < j
    key = np.unique(i[keep] * 3000 + j[keep])
    pi, pj = key // 3000, key % 3000
    ps = rng.integers(0, 65, len(pi)) / 64.0
    for cs in (2, 4, 8):
        perm, offs = hierarchical_clustering_v0_fast(rp, ci, 3000, (pi, pj, ps), cs)
        operm, ooffs = orc.hc(rp, ci, pi, pj, ps, cs)
        assert np.array_equal(perm, operm) and np.array_equal(offs, ooffs)
