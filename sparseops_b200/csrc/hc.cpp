// Hierarchical clustering of rows from LSH candidate pairs (host, sequential).
//
// Replaces hierarchical_clustering_v0_fast (reference include/spgemm_utility.h:
// 742-915).  The merge order is inherently sequential and the output
// (permutation, offsets) must be bit-identical, so it runs on the host, once
// per pattern; everything around it (signatures, pairs, scores, reordering,
// clusters, products) runs on the device.  The merge rules, restated:
//   * candidates are consumed best first: initial pairs by score descending,
//     equal scores in reverse input order (the reference pops the back of a
//     per-score bucket); pairs discovered during merging wait in a max-heap
//     ordered by (score, i, j) and are taken before the next initial pair
//     unless they compare lower;
//   * a pair of two roots merges (if both are still open): the smaller cluster
//     joins the larger (ties: j joins i), the open-cluster count drops, and a
//     cluster that reaches cluster_size closes (count drops again);
//   * a pair whose rows are not both roots looks up the two roots; if both are
//     open and differ and the root pair is neither an initial pair nor seen
//     before, it is queued with its exact Jaccard similarity;
//   * output: clusters ordered by root row, rows ascending inside each.
#include <algorithm>
#include <cstdint>
#include <queue>
#include <set>
#include <unordered_set>
#include <vector>

#include "spops_internal.h"

namespace spops {

namespace {

struct Cand {
  double s;
  int64_t i, j;
};
struct CandLess {  // the reference's comparison of (score, (i, j))
  bool operator()(const Cand& a, const Cand& b) const {
    if (a.s != b.s) return a.s < b.s;
    if (a.i != b.i) return a.i < b.i;
    return a.j < b.j;
  }
};

struct KeyHash {
  size_t operator()(uint64_t k) const {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    return (size_t)k;
  }
};

bool row_sorted_unique(const int64_t* rp, const int64_t* ci, int64_t r) {
  for (int64_t e = rp[r] + 1; e < rp[r + 1]; ++e)
    if (ci[e - 1] >= ci[e]) return false;
  return true;
}

// |row a ∩ row b| / |row a ∪ row b| over entry counts.  Rows with strictly
// increasing columns take a merge; any other pair counts row b's entries found
// in the set of row a's columns, which gives the same number on unique rows.
double jaccard_rows(const int64_t* rp, const int64_t* ci, int64_t a, int64_t b) {
  const int64_t la = rp[a + 1] - rp[a], lb = rp[b + 1] - rp[b];
  int64_t common = 0;
  if (row_sorted_unique(rp, ci, a) && row_sorted_unique(rp, ci, b)) {
    int64_t x = rp[a], y = rp[b];
    while (x < rp[a + 1] && y < rp[b + 1]) {
      if (ci[x] == ci[y]) { ++common; ++x; ++y; }
      else if (ci[x] < ci[y]) ++x;
      else ++y;
    }
  } else {  // set of row a's columns; count row b's entries found in it
    std::set<int64_t> sa(ci + rp[a], ci + rp[a + 1]);
    for (int64_t y = rp[b]; y < rp[b + 1]; ++y) common += sa.count(ci[y]);
  }
  const int64_t u = la + lb - common;
  return u == 0 ? 0.0 : (1.0 * (double)common / (double)u);
}

}  // namespace

spops_status_t hierarchical_clustering(const int64_t* rp, const int64_t* ci, int64_t n, const int64_t* pi,
                                       const int64_t* pj, const double* ps, int64_t np, int64_t cluster_size,
                                       std::vector<int64_t>& perm, std::vector<int64_t>& offsets) {
  if (n > (int64_t)INT32_MAX) return fail(SPOPS_ERR_UNSUPPORTED, "clustering: more than 2^31 rows");
  // initial candidates, best first
  std::vector<Cand> init;
  init.reserve((size_t)np);
  for (int64_t t = np - 1; t >= 0; --t) {
    int64_t a = pi[t], b = pj[t];
    if (a > b) std::swap(a, b);
    if (a == b || a < 0 || a >= n || b >= n) continue;
    init.push_back(Cand{ps[t], a, b});
  }
  std::stable_sort(init.begin(), init.end(), [](const Cand& x, const Cand& y) { return x.s > y.s; });
  // is (a, b) one of the given pairs (the list is sorted by (i, j))
  auto given = [&](int64_t a, int64_t b) {
    int64_t lo = 0, hi = np;
    while (lo < hi) {
      const int64_t mid = lo + (hi - lo) / 2;
      if (pi[mid] < a || (pi[mid] == a && pj[mid] < b)) lo = mid + 1;
      else hi = mid;
    }
    return lo < np && pi[lo] == a && pj[lo] == b;
  };

  std::vector<int64_t> parent((size_t)n), size((size_t)n, 1);
  std::vector<unsigned char> open((size_t)n, 1);
  for (int64_t i = 0; i < n; ++i) parent[i] = i;
  auto root = [&](int64_t x) {
    int64_t r = x;
    while (parent[r] != r) r = parent[r];
    while (parent[x] != r) {
      const int64_t nx = parent[x];
      parent[x] = r;
      x = nx;
    }
    return r;
  };
  std::priority_queue<Cand, std::vector<Cand>, CandLess> found;
  std::unordered_set<uint64_t, KeyHash> seen;
  seen.reserve((size_t)(np / 8 + 1024));
  auto key_of = [](int64_t a, int64_t b) { return ((uint64_t)a << 32) ^ (uint64_t)b; };

  size_t next = 0;
  int open_clusters = (int)n;  // the reference keeps an int count
  CandLess less;
  while ((next < init.size() || !found.empty()) && open_clusters > 0) {
    Cand c;
    if (found.empty()) c = init[next++];
    else if (next >= init.size()) { c = found.top(); found.pop(); }
    else if (less(found.top(), init[next])) c = init[next++];
    else { c = found.top(); found.pop(); }
    const int64_t i = c.i, j = c.j;
    if (i >= n || j >= n) continue;
    if (parent[i] == i && parent[j] == j) {
      if (!open[i] || !open[j]) continue;
      --open_clusters;
      const int64_t keep = size[i] < size[j] ? j : i, join = keep == j ? i : j;
      parent[join] = keep;
      size[keep] += size[join];
      if (size[keep] >= cluster_size) {
        open[keep] = 0;
        --open_clusters;
      }
    } else {
      const int64_t ri = root(i), rj = root(j);
      if (!open[ri] || !open[rj] || ri == rj) continue;
      const int64_t a = std::min(ri, rj), b = std::max(ri, rj);
      if (given(a, b)) continue;
      if (seen.insert(key_of(a, b)).second) found.push(Cand{jaccard_rows(rp, ci, a, b), a, b});
    }
  }
  // clusters by root, rows ascending
  std::vector<int64_t> rt((size_t)n), count((size_t)n, 0), id((size_t)n, -1);
  for (int64_t i = 0; i < n; ++i) {
    rt[i] = root(i);
    ++count[rt[i]];
  }
  offsets.assign(1, 0);
  for (int64_t r = 0; r < n; ++r)
    if (count[r] > 0) {
      id[r] = (int64_t)offsets.size() - 1;
      offsets.push_back(offsets.back() + count[r]);
    }
  perm.assign((size_t)n, 0);
  std::vector<int64_t> cur(offsets.begin(), offsets.end() - 1);
  for (int64_t i = 0; i < n; ++i) perm[cur[id[rt[i]]]++] = i;
  return SPOPS_OK;
}

}  // namespace spops
