// CPU restatement of the SparseOps hot-path algorithms (the ORACLE).
// Test infrastructure only: see spops_oracle.h.  Plain sequential code, one
// function per reference algorithm, each citing the reference file:line it
// restates.  Pinned against the reference's own outputs by the golden
// fixtures in tests/golden/ (tests/test_oracle_golden.py).
#include "spops_oracle.h"

#include <algorithm>
#include <cfloat>
#include <cstdio>
#include <numeric>
#include <string>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <queue>
#include <set>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

namespace {

template <typename I, typename V>
void spmv_rows(int64_t nr, const I* rp, const I* ci, const V* v, double alpha, const V* x, double beta,
               double* y) {
  // src/spmv_csr.cpp:74-91: sum in stored order, then alpha/beta update.
  for (int64_t r = 0; r < nr; ++r) {
    double s = 0.0;
    for (int64_t k = rp[r]; k < rp[r + 1]; ++k) s += (double)v[k] * (double)x[ci[k]];
    if (alpha == 1.0 && beta == 0.0)
      y[r] = s;
    else
      y[r] = alpha * s + beta * y[r];
  }
}

inline int64_t round_up(int64_t a, int64_t b) { return ((a + b - 1) / b) * b; }

}  // namespace

extern "C" {

void orc_spmv_csr_f64_i32(int64_t nr, const int32_t* rp, const int32_t* ci, const double* v, double alpha,
                          const double* x, double beta, double* y) {
  spmv_rows(nr, rp, ci, v, alpha, x, beta, y);
}

void orc_spmv_csr_f64_i64(int64_t nr, const int64_t* rp, const int64_t* ci, const double* v, double alpha,
                          const double* x, double beta, double* y) {
  spmv_rows(nr, rp, ci, v, alpha, x, beta, y);
}

void orc_spmv_csr_f32_i32(int64_t nr, const int32_t* rp, const int32_t* ci, const float* v, double alpha,
                          const float* x, double beta, const float* y_in, double* y) {
  for (int64_t r = 0; r < nr; ++r) y[r] = y_in ? (double)y_in[r] : 0.0;
  spmv_rows(nr, rp, ci, v, alpha, x, beta, y);
}

void orc_absdot_csr_f64_i32(int64_t nr, const int32_t* rp, const int32_t* ci, const double* v, const double* x,
                            double* out) {
  for (int64_t r = 0; r < nr; ++r) {
    double s = 0.0;
    for (int64_t k = rp[r]; k < rp[r + 1]; ++k) s += std::fabs(v[k] * x[ci[k]]);
    out[r] = s;
  }
}

void orc_spmm_csr_f64_i32(int64_t nr, const int32_t* rp, const int32_t* ci, const double* v, int64_t k,
                          double alpha, const double* X, double beta, double* Y) {
  std::vector<double> s((size_t)k);
  for (int64_t r = 0; r < nr; ++r) {
    std::fill(s.begin(), s.end(), 0.0);
    for (int64_t e = rp[r]; e < rp[r + 1]; ++e)
      for (int64_t c = 0; c < k; ++c) s[c] += v[e] * X[(int64_t)ci[e] * k + c];
    for (int64_t c = 0; c < k; ++c) Y[r * k + c] = alpha * s[c] + beta * Y[r * k + c];
  }
}

// ------------------------------------------------------------- layouts
// include/sparse_conversion.h:373-425: rows of each sigma-slice sorted by
// the pair (nnz, row) in DESCENDING order (std::greater), so equal lengths
// put the larger original row first; chunk_len = max length in the chunk of
// C sorted rows, rounded up to `align`.
void orc_sell_c_sigma_layout(int64_t nr, const int32_t* rp, int64_t sigma, int64_t C, int64_t align,
                             int32_t* reorder, int32_t* chunk_len) {
  std::vector<std::pair<int64_t, int64_t>> key((size_t)nr);
  for (int64_t i = 0; i < nr; ++i) key[i] = {rp[i + 1] - rp[i], i};
  for (int64_t s = 0; s < nr; s += sigma) {
    int64_t e = std::min(nr, s + sigma);
    std::sort(key.begin() + s, key.begin() + e, [](const std::pair<int64_t, int64_t>& a,
                                                   const std::pair<int64_t, int64_t>& b) { return a > b; });
  }
  int64_t nch = (nr + C - 1) / C;
  for (int64_t c = 0; c < nch; ++c) chunk_len[c] = 0;
  for (int64_t i = 0; i < nr; ++i) {
    reorder[i] = (int32_t)key[i].second;
    int64_t c = i / C;
    if (key[i].first > chunk_len[c]) chunk_len[c] = (int32_t)key[i].first;
  }
  for (int64_t c = 0; c < nch; ++c) chunk_len[c] = (int32_t)round_up(chunk_len[c], align);
}

// include/sparse_conversion.h:281-306: per chunk of C consecutive rows, the
// longest row rounded up to `align`.
void orc_sell_row_width(int64_t nr, const int32_t* rp, int64_t C, int64_t align, int32_t* width) {
  int64_t nch = (nr + C - 1) / C;
  for (int64_t c = 0; c < nch; ++c) width[c] = 0;
  for (int64_t i = 0; i < nr; ++i) width[i / C] = std::max<int32_t>(width[i / C], rp[i + 1] - rp[i]);
  for (int64_t c = 0; c < nch; ++c) width[c] = (int32_t)round_up(width[c], align);
}

// include/sparse_conversion.h:642-660, 743-747: diagonals numbered in the
// order their first entry is met in a row-major scan; offset = col - row.
int64_t orc_dia_offsets(int64_t nr, int64_t nc, const int32_t* rp, const int32_t* ci, int64_t max_out,
                        int64_t* offsets) {
  std::vector<int64_t> seen((size_t)(nr + nc), -1);
  int64_t nd = 0;
  for (int64_t i = 0; i < nr; ++i)
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
      int64_t m = nr - i + ci[k];
      if (seen[m] < 0) {
        seen[m] = nd;
        if (nd < max_out) offsets[nd] = (int64_t)ci[k] - i;
        ++nd;
      }
    }
  return nd;
}

// include/sparse_conversion.h:821-885: block row i lists the block columns
// that hold at least one entry, ascending.
int64_t orc_bsr_structure(int64_t nr, int64_t nc, const int32_t* rp, const int32_t* ci, int64_t br, int64_t bc,
                          int32_t* row_ptr, int32_t* block_col) {
  int64_t mb = (nr + br - 1) / br, nb = (nc + bc - 1) / bc;
  std::vector<char> mark((size_t)nb, 0);
  int64_t nnzb = 0;
  if (row_ptr) row_ptr[0] = 0;
  for (int64_t b = 0; b < mb; ++b) {
    std::fill(mark.begin(), mark.end(), 0);
    int64_t r0 = b * br, r1 = std::min(nr, r0 + br);
    for (int64_t k = rp[r0]; k < rp[r1]; ++k) mark[ci[k] / bc] = 1;
    for (int64_t j = 0; j < nb; ++j)
      if (mark[j]) {
        if (block_col) block_col[nnzb] = (int32_t)j;
        ++nnzb;
      }
    if (row_ptr) row_ptr[b + 1] = (int32_t)nnzb;
  }
  return nnzb;
}

// --------------------------------------------------------------- MinHash
// include/spgemm_MinHashLSH.h:40-43 (LCG), 134-141 (a odd, b), 147-176:
// sig[r][d] = min over the row's columns x of a_d*x + b_d (mod 2^64);
// empty rows keep UINT64_MAX.
void orc_minhash(const int64_t* rp, const int64_t* ci, int64_t n, int32_t k, uint64_t seed, uint64_t* sig) {
  std::vector<uint64_t> a((size_t)k), b((size_t)k);
  uint64_t s = seed;
  for (int d = 0; d < k; ++d) {
    s = s * 6364136223846793005ULL + 1442695040888963407ULL;
    a[d] = (s >> 1) * 2 + 1;
    s = s * 6364136223846793005ULL + 1442695040888963407ULL;
    b[d] = s;
  }
  for (int64_t r = 0; r < n; ++r) {
    uint64_t* out = sig + r * (int64_t)k;
    for (int d = 0; d < k; ++d) out[d] = ~0ULL;
    for (int64_t e = rp[r]; e < rp[r + 1]; ++e) {
      uint64_t x = (uint64_t)ci[e];
      for (int d = 0; d < k; ++d) {
        uint64_t h = a[d] * x + b[d];
        if (h < out[d]) out[d] = h;
      }
    }
  }
}

struct OrcPairs {
  std::vector<int64_t> i, j;
  std::vector<double> s;
};

// include/spgemm_MinHashLSH.h:277-283 (band hash), 450-542 (records sorted by
// (band, bucket, row); a bucket of more than 256 rows pairs each row with the
// next 16 only), 544-562 (pairs sorted, deduplicated, scored by the fraction
// of equal signature entries, 183-204).
void* orc_lsh_pairs(const uint64_t* sig, int64_t n, int32_t k, int32_t bands, int32_t constrain) {
  OrcPairs* out = new OrcPairs();
  if (n <= 0 || bands <= 0 || k <= 0 || k % bands) return out;
  const int r = k / bands;
  std::vector<std::pair<int64_t, int64_t>> pairs;
  std::vector<std::pair<uint64_t, int64_t>> rec((size_t)n);
  for (int band = 0; band < bands; ++band) {
    for (int64_t row = 0; row < n; ++row) {
      uint64_t h = 0;
      const uint64_t* bs = sig + row * (int64_t)k + band * r;
      for (int t = 0; t < r; ++t) h = h * 0x9e3779b97f4a7c15ULL + bs[t];
      rec[row] = {h, row};
    }
    std::sort(rec.begin(), rec.end());
    for (int64_t a = 0; a < n;) {
      int64_t e = a + 1;
      while (e < n && rec[e].first == rec[a].first) ++e;
      int64_t sz = e - a;
      if (sz > 1) {
        bool window = constrain && sz > 256;
        for (int64_t p = a; p < e; ++p) {
          int64_t q_end = window ? std::min(e, p + 1 + 16) : e;
          for (int64_t q = p + 1; q < q_end; ++q) pairs.push_back({rec[p].second, rec[q].second});
        }
      }
      a = e;
    }
  }
  std::sort(pairs.begin(), pairs.end());
  pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
  out->i.resize(pairs.size());
  out->j.resize(pairs.size());
  out->s.resize(pairs.size());
  for (size_t t = 0; t < pairs.size(); ++t) {
    const uint64_t* sa = sig + pairs[t].first * (int64_t)k;
    const uint64_t* sb = sig + pairs[t].second * (int64_t)k;
    int m = 0;
    for (int d = 0; d < k; ++d) m += (sa[d] == sb[d]);
    out->i[t] = pairs[t].first;
    out->j[t] = pairs[t].second;
    out->s[t] = (double)m / (double)k;
  }
  return out;
}
int64_t orc_pairs_count(void* h) { return (int64_t) static_cast<OrcPairs*>(h)->i.size(); }
void orc_pairs_copy(void* h, int64_t* i, int64_t* j, double* s) {
  OrcPairs* p = static_cast<OrcPairs*>(h);
  std::copy(p->i.begin(), p->i.end(), i);
  std::copy(p->j.begin(), p->j.end(), j);
  std::copy(p->s.begin(), p->s.end(), s);
}
void orc_pairs_free(void* h) { delete static_cast<OrcPairs*>(h); }

// ------------------------------------------------- hierarchical clustering
// include/spgemm_utility.h:361-429 (exact Jaccard), 742-915 (merge loop).
namespace {
double jaccard(const int64_t* rp, const int64_t* ci, int64_t a, int64_t b, bool sorted_unique) {
  int64_t la = rp[a + 1] - rp[a], lb = rp[b + 1] - rp[b], common = 0;
  if (sorted_unique) {
    int64_t ia = rp[a], ib = rp[b];
    while (ia < rp[a + 1] && ib < rp[b + 1]) {
      if (ci[ia] == ci[ib]) { ++common; ++ia; ++ib; }
      else if (ci[ia] < ci[ib]) ++ia;
      else ++ib;
    }
  } else {
    std::set<int64_t> sa(ci + rp[a], ci + rp[a + 1]);
    for (int64_t e = rp[b]; e < rp[b + 1]; ++e) common += sa.count(ci[e]) ? 1 : 0;
  }
  int64_t u = la + lb - common;
  return u == 0 ? 0.0 : (1.0 * common / u);
}
}  // namespace

int64_t orc_hc(const int64_t* rp, const int64_t* ci, int64_t n, const int64_t* pi, const int64_t* pj,
               const double* ps, int64_t np, int64_t cluster_size, int64_t* perm, int64_t* offsets) {
  std::vector<int64_t> parent((size_t)n), sz((size_t)n, 1);
  std::vector<char> valid((size_t)n, 1);
  for (int64_t i = 0; i < n; ++i) parent[i] = i;
  auto find = [&](int64_t x) {
    int64_t root = x;
    while (parent[root] != root) root = parent[root];
    while (parent[x] != root) { int64_t nx = parent[x]; parent[x] = root; x = nx; }
    return root;
  };
  // Initial pairs are consumed best first: score descending; within equal
  // scores the reference pops its per-score bucket from the back, i.e. in
  // reverse input order.  Walking the input backwards and stable-sorting by
  // score gives exactly that sequence.
  struct Item { double s; int64_t i, j; };
  std::vector<Item> init;
  init.reserve((size_t)np);
  for (int64_t t = np - 1; t >= 0; --t) {
    int64_t a = pi[t], b = pj[t];
    if (a > b) std::swap(a, b);
    if (a == b || a >= n || b >= n) continue;
    init.push_back({ps[t], a, b});
  }
  std::stable_sort(init.begin(), init.end(), [](const Item& x, const Item& y) { return x.s > y.s; });
  auto less = [](const Item& x, const Item& y) {  // the reference's cmp
    if (x.s != y.s) return x.s < y.s;
    if (x.i != y.i) return x.i < y.i;
    return x.j < y.j;
  };
  std::priority_queue<Item, std::vector<Item>, decltype(less)> dyn(less);
  // membership of the ORIGINAL (sorted) pair list
  auto in_initial = [&](int64_t a, int64_t b) {
    int64_t lo = 0, hi = np;
    while (lo < hi) {
      int64_t mid = (lo + hi) / 2;
      if (pi[mid] < a || (pi[mid] == a && pj[mid] < b)) lo = mid + 1; else hi = mid;
    }
    return lo < np && pi[lo] == a && pj[lo] == b;
  };
  bool sorted_unique = true;
  for (int64_t r = 0; r < n && sorted_unique; ++r)
    for (int64_t e = rp[r] + 1; e < rp[r + 1]; ++e)
      if (ci[e - 1] >= ci[e]) { sorted_unique = false; break; }
  std::set<std::pair<int64_t, int64_t>> discovered;
  size_t ip = 0;
  int nclusters = (int)n;
  while ((ip < init.size() || !dyn.empty()) && nclusters > 0) {
    Item top;
    if (dyn.empty()) top = init[ip++];
    else if (ip >= init.size()) { top = dyn.top(); dyn.pop(); }
    else if (less(dyn.top(), init[ip])) top = init[ip++];
    else { top = dyn.top(); dyn.pop(); }
    int64_t i = top.i, j = top.j;
    if (i >= n || j >= n) continue;
    if (parent[i] == i && parent[j] == j) {
      if (!valid[i] || !valid[j]) continue;
      nclusters--;
      if (sz[i] < sz[j]) {
        parent[i] = j; sz[j] += sz[i];
        if (sz[j] >= cluster_size) { valid[j] = 0; nclusters--; }
      } else {
        parent[j] = i; sz[i] += sz[j];
        if (sz[i] >= cluster_size) { valid[i] = 0; nclusters--; }
      }
    } else {
      int64_t ri = find(i), rj = find(j);
      if (!valid[ri] || !valid[rj]) continue;
      if (ri != rj) {
        int64_t a = std::min(ri, rj), b = std::max(ri, rj);
        if (!in_initial(a, b) && discovered.insert({a, b}).second)
          dyn.push({jaccard(rp, ci, a, b, sorted_unique), a, b});
      }
    }
  }
  // clusters ordered by root id, rows ascending inside (spgemm_utility.h:887-914)
  std::vector<int64_t> root((size_t)n), cnt((size_t)n, 0), cid((size_t)n, -1);
  for (int64_t i = 0; i < n; ++i) { root[i] = find(i); cnt[root[i]]++; }
  int64_t nc = 0;
  offsets[0] = 0;
  for (int64_t r = 0; r < n; ++r)
    if (cnt[r] > 0) { cid[r] = nc; offsets[nc + 1] = offsets[nc] + cnt[r]; ++nc; }
  std::vector<int64_t> cur(offsets, offsets + nc);
  for (int64_t i = 0; i < n; ++i) perm[cur[cid[root[i]]]++] = i;
  return nc;
}

// ------------------------------------------------------------- SpGEMM
struct OrcCsr {
  int64_t rows = 0, dense = 0, flops = 0;
  std::vector<int64_t> rp, ci;
  std::vector<double> v, absv;
};

// Result of the kernel-3 pipeline for C = A*B, stated per cluster of rows
// (src/spgemm_Vlength_mixed.cpp:196-434, sparse_conversion.h:1777-1862):
//  * classify (267-319): dense iff B_access + col_range*csz*8 <= L2 budget
//    and nz/col_range >= 0.15, with B_access = num_acols*nnz(B)/rows(B)*16;
//  * a column whose |values| are all < 1e-12 across the cluster's rows is
//    dropped when the cluster is dense (150-190) or output is sorted
//    (spgemm_Vlength_hash.h:107-129);
//  * cluster -> CSR keeps entries with |v| > 0 (sparse_conversion.h:1800-1806).
void* orc_spgemm(int64_t a_rows, const int64_t* arp, const int64_t* aci, const double* av, int64_t b_rows,
                 int64_t b_cols, const int64_t* brp, const int64_t* bci, const double* bv, const int64_t* perm,
                 const int64_t* offsets, int64_t nclusters, int32_t sort_output, double l2_budget) {
  OrcCsr* out = new OrcCsr();
  out->rows = a_rows;
  const double b_rowdense = (double)brp[b_rows] / (double)b_rows;
  struct Ent { int64_t col, l; double v, a; };
  std::vector<std::vector<std::pair<int64_t, std::pair<double, double>>>> rows_out((size_t)a_rows);
  std::vector<Ent> ent;
  std::vector<int64_t> acols;
  for (int64_t c = 0; c < nclusters; ++c) {
    int64_t r0 = offsets[c], r1 = offsets[c + 1], csz = r1 - r0;
    ent.clear();
    acols.clear();
    for (int64_t l = 0; l < csz; ++l) {
      int64_t r = perm[r0 + l];
      for (int64_t e = arp[r]; e < arp[r + 1]; ++e) {
        int64_t k = aci[e];
        acols.push_back(k);
        for (int64_t f = brp[k]; f < brp[k + 1]; ++f) {
          ent.push_back({bci[f], l, av[e] * bv[f], std::fabs(av[e] * bv[f])});
          out->flops += 2;
        }
      }
    }
    std::sort(acols.begin(), acols.end());
    int64_t num_acols = (int64_t)(std::unique(acols.begin(), acols.end()) - acols.begin());
    std::stable_sort(ent.begin(), ent.end(), [](const Ent& x, const Ent& y) {
      return x.col != y.col ? x.col < y.col : x.l < y.l;
    });
    // unique columns of this cluster
    int64_t nz = 0, cmin = 0, cmax = 0;
    for (size_t t = 0; t < ent.size(); ++t)
      if (t == 0 || ent[t].col != ent[t - 1].col) {
        if (nz == 0) cmin = ent[t].col;
        cmax = ent[t].col;
        ++nz;
      }
    bool dense = false;
    if (nz > 0) {
      int64_t range = cmax - cmin + 1;
      double density = (double)nz / (double)range;
      size_t b_access = (size_t)((double)num_acols * b_rowdense * (double)(sizeof(int64_t) + sizeof(double)));
      size_t dense_bytes = (size_t)range * (size_t)csz * sizeof(double);
      dense = (double)(b_access + dense_bytes) <= l2_budget && density >= 0.15;
    }
    out->dense += dense ? 1 : 0;
    bool drop_small = dense || sort_output;
    std::vector<double> val((size_t)csz), aval((size_t)csz);
    for (size_t t = 0; t < ent.size();) {
      size_t e = t;
      std::fill(val.begin(), val.end(), 0.0);
      std::fill(aval.begin(), aval.end(), 0.0);
      while (e < ent.size() && ent[e].col == ent[t].col) {
        val[ent[e].l] += ent[e].v;
        aval[ent[e].l] += ent[e].a;
        ++e;
      }
      bool all_small = true;
      for (int64_t l = 0; l < csz; ++l)
        if (std::fabs(val[l]) >= 1e-12) { all_small = false; break; }
      if (!(drop_small && all_small))
        for (int64_t l = 0; l < csz; ++l)
          if (std::fabs(val[l]) > 0.0) rows_out[perm[r0 + l]].push_back({ent[t].col, {val[l], aval[l]}});
      t = e;
    }
  }
  out->rp.assign((size_t)a_rows + 1, 0);
  for (int64_t r = 0; r < a_rows; ++r) out->rp[r + 1] = out->rp[r] + (int64_t)rows_out[r].size();
  out->ci.resize((size_t)out->rp[a_rows]);
  out->v.resize((size_t)out->rp[a_rows]);
  out->absv.resize((size_t)out->rp[a_rows]);
  for (int64_t r = 0; r < a_rows; ++r) {
    int64_t o = out->rp[r];
    for (size_t t = 0; t < rows_out[r].size(); ++t) {
      out->ci[o + t] = rows_out[r][t].first;
      out->v[o + t] = rows_out[r][t].second.first;
      out->absv[o + t] = rows_out[r][t].second.second;
    }
  }
  (void)b_cols;
  return out;
}

// Row-wise C = A*B (src/spgemm.cpp:44-235; the hash kernel's per-row loop,
// src/spgemm_hash.cpp:246-318): per row, products a_ij * b_jk added into an
// accumulator per column in (j, k) order; every structural entry is kept,
// exact zeros included; columns ascending.
void* orc_spgemm_rowwise(int64_t a_rows, const int64_t* arp, const int64_t* aci, const double* av, int64_t b_rows,
                         const int64_t* brp, const int64_t* bci, const double* bv) {
  OrcCsr* out = new OrcCsr();
  out->rows = a_rows;
  out->rp.assign((size_t)a_rows + 1, 0);
  std::map<int64_t, std::pair<double, double>> acc;
  for (int64_t i = 0; i < a_rows; ++i) {
    acc.clear();
    for (int64_t e = arp[i]; e < arp[i + 1]; ++e) {
      const int64_t j = aci[e];
      for (int64_t f = brp[j]; f < brp[j + 1]; ++f) {
        auto& a = acc[bci[f]];
        a.first += av[e] * bv[f];
        a.second += std::fabs(av[e] * bv[f]);
        out->flops += 2;
      }
    }
    for (const auto& kv : acc) {
      out->ci.push_back(kv.first);
      out->v.push_back(kv.second.first);
      out->absv.push_back(kv.second.second);
    }
    out->rp[i + 1] = (int64_t)out->ci.size();
  }
  (void)b_rows;
  return out;
}

// HashSpGEMMTopK (src/spgemm.cpp:708-842, src/spgemm_hash.cpp:168-318): the
// binary pattern of A times its transpose gives |A_i n A_j| (sums of 1 in the
// value type); per j != i, u = |A_i| + |A_j| - inter and jacc = u == 0 ? 0 :
// 1 * inter / u (value type); per row, (jacc descending, column ascending),
// the first top_k kept.  f32: the value type is float.
}  // extern "C"

template <typename V>
static void* topk_impl(int64_t n, const int64_t* arp, const int64_t* aci, int64_t ncols, int64_t top_k) {
  OrcCsr* out = new OrcCsr();
  out->rows = n;
  out->rp.assign((size_t)n + 1, 0);
  // transpose of the pattern, rows of A^T in ascending original row
  std::vector<int64_t> trp((size_t)ncols + 1, 0), tci((size_t)arp[n]);
  for (int64_t e = 0; e < arp[n]; ++e) ++trp[(size_t)aci[e] + 1];
  for (int64_t c = 0; c < ncols; ++c) trp[c + 1] += trp[c];
  {
    std::vector<int64_t> fill(trp.begin(), trp.end() - 1);
    for (int64_t i = 0; i < n; ++i)
      for (int64_t e = arp[i]; e < arp[i + 1]; ++e) tci[(size_t)fill[aci[e]]++] = i;
  }
  std::map<int64_t, V> inter;
  std::vector<std::pair<V, int64_t>> row;
  for (int64_t i = 0; i < n; ++i) {
    inter.clear();
    for (int64_t e = arp[i]; e < arp[i + 1]; ++e) {
      const int64_t c = aci[e];
      for (int64_t f = trp[c]; f < trp[c + 1]; ++f) inter[tci[f]] += (V)1 * (V)1;
    }
    row.clear();
    const int64_t li = arp[i + 1] - arp[i];
    for (const auto& kv : inter) {
      const int64_t j = kv.first;
      if (j == i) continue;
      const int64_t u = li + (arp[j + 1] - arp[j]) - (int64_t)kv.second;
      const V jacc = u == 0 ? (V)0 : (V)1 * kv.second / (V)u;
      row.push_back({jacc, j});
    }
    std::sort(row.begin(), row.end(), [](const std::pair<V, int64_t>& a, const std::pair<V, int64_t>& b) {
      return a.first != b.first ? a.first > b.first : a.second < b.second;
    });
    const size_t keep = std::min<size_t>(row.size(), (size_t)std::max<int64_t>(top_k, 0));
    for (size_t t = 0; t < keep; ++t) {
      out->ci.push_back(row[t].second);
      out->v.push_back((double)row[t].first);
      out->absv.push_back((double)row[t].first);
    }
    out->rp[i + 1] = (int64_t)out->ci.size();
  }
  return out;
}

extern "C" {

void* orc_spgemm_topk(int64_t n, const int64_t* arp, const int64_t* aci, int64_t ncols, int64_t top_k, int32_t f32) {
  return f32 ? topk_impl<float>(n, arp, aci, ncols, top_k) : topk_impl<double>(n, arp, aci, ncols, top_k);
}

void orc_csr_info(void* h, int64_t* o) {
  OrcCsr* c = static_cast<OrcCsr*>(h);
  o[0] = c->rows; o[1] = c->rp.empty() ? 0 : c->rp.back(); o[2] = c->dense; o[3] = c->flops;
}
void orc_csr_copy(void* h, int64_t* rp, int64_t* ci, double* v, double* absv) {
  OrcCsr* c = static_cast<OrcCsr*>(h);
  std::copy(c->rp.begin(), c->rp.end(), rp);
  if (ci) std::copy(c->ci.begin(), c->ci.end(), ci);
  if (v) std::copy(c->v.begin(), c->v.end(), v);
  if (absv) std::copy(c->absv.begin(), c->absv.end(), absv);
}
void orc_csr_free(void* h) { delete static_cast<OrcCsr*>(h); }

int64_t orc_spgemm_flop(int64_t a_rows, const int64_t* arp, const int64_t* aci, int64_t b_rows,
                        const int64_t* brp) {
  int64_t f = 0;
  for (int64_t i = 0; i < a_rows; ++i)
    for (int64_t e = arp[i]; e < arp[i + 1]; ++e)
      if (aci[e] < b_rows) f += brp[aci[e] + 1] - brp[aci[e]];
  return 2 * f;
}

// ------------------------------------------------------------ COO -> CSR
// coo_to_csr (include/sparse_conversion.h:37-99): rows by a stable counting
// sort (file order kept within a row); with compact, sum_csr_duplicates
// (include/sparse_operation.h:21-69): per row, the values of a column are
// added in file order from zero; the distinct columns come out in reverse
// order of first appearance; exact-zero sums are dropped.  Returns the
// output entry count (arrays sized for nnz entries, rp for n + 1).
}  // extern "C"

template <typename V>
static int64_t coo_to_csr_impl(int64_t n, int64_t nnz, const int64_t* ri, const int64_t* ci, const V* v,
                               int32_t compact, int64_t* rp, int64_t* oc, V* ov) {
  std::vector<int64_t> cnt((size_t)n + 1, 0);
  for (int64_t e = 0; e < nnz; ++e) ++cnt[(size_t)ri[e] + 1];
  for (int64_t r = 0; r < n; ++r) cnt[(size_t)r + 1] += cnt[(size_t)r];
  std::vector<int64_t> at(cnt.begin(), cnt.end() - 1);
  std::vector<int64_t> col((size_t)nnz);
  std::vector<V> val((size_t)nnz);
  for (int64_t e = 0; e < nnz; ++e) {
    const int64_t d = at[(size_t)ri[e]]++;
    col[(size_t)d] = ci[e];
    val[(size_t)d] = v[e];
  }
  if (!compact) {
    std::copy(cnt.begin(), cnt.end(), rp);
    std::copy(col.begin(), col.end(), oc);
    std::copy(val.begin(), val.end(), ov);
    return nnz;
  }
  int64_t out = 0;
  rp[0] = 0;
  for (int64_t r = 0; r < n; ++r) {
    std::vector<int64_t> order;        // distinct columns, first appearance order
    std::map<int64_t, V> sum;
    for (int64_t e = cnt[(size_t)r]; e < cnt[(size_t)r + 1]; ++e) {
      auto it = sum.find(col[(size_t)e]);
      if (it == sum.end()) {
        order.push_back(col[(size_t)e]);
        sum.emplace(col[(size_t)e], V(0) + val[(size_t)e]);
      } else {
        it->second += val[(size_t)e];
      }
    }
    for (auto k = order.rbegin(); k != order.rend(); ++k) {
      const V s = sum[*k];
      if (s != V(0)) {
        oc[out] = *k;
        ov[out] = s;
        ++out;
      }
    }
    rp[r + 1] = out;
  }
  return out;
}

extern "C" {

int64_t orc_coo_to_csr_f64(int64_t n, int64_t nnz, const int64_t* ri, const int64_t* ci, const double* v,
                           int32_t compact, int64_t* rp, int64_t* oc, double* ov) {
  return coo_to_csr_impl<double>(n, nnz, ri, ci, v, compact, rp, oc, ov);
}

int64_t orc_coo_to_csr_f32(int64_t n, int64_t nnz, const int64_t* ri, const int64_t* ci, const float* v,
                           int32_t compact, int64_t* rp, int64_t* oc, float* ov) {
  return coo_to_csr_impl<float>(n, nnz, ri, ci, v, compact, rp, oc, ov);
}

// ------------------------------------------------------------ features
// MTX::CalculateFeatures (src/sparse_features.cpp:643-775) with the counts
// MtxLoad gathers for a general real matrix (:336-478), read in CSR order.
// out: the 32 values of spops_features_t, in its order.
static void count_stats(const std::vector<int64_t>& cnt, int64_t nnz, double* nzr, int64_t* mn, int64_t* mx,
                        double* ave, double* var, double* sd, double* p, double* gini) {
  const int64_t len = (int64_t)cnt.size();
  int64_t nzc = 0, lo = 100000000, hi = 0;
  *ave = (double)nnz / (double)len;
  double v = 0.0;
  for (int64_t c : cnt) {
    lo = std::min(lo, c);
    hi = std::max(hi, c);
    if (c) ++nzc;
    const double d = (double)c - *ave;
    v += d * d;
  }
  *nzr = (double)nzc / (double)len;
  *mn = lo;
  *mx = hi;
  *var = v / (double)len;
  *sd = std::sqrt(*var);
  std::vector<int64_t> o(cnt);
  std::sort(o.begin(), o.end());
  int64_t quit = len, count = 0, step = 0;
  double pt = 0.0, q = 0.0;
  do {
    --quit;
    ++count;
    step += o[(size_t)quit];
    pt = (double)count / (double)len;
    q = (double)step / (double)nnz;
  } while (pt + q < 1.0 && quit > 0);
  *p = pt;
  std::vector<int64_t> cum(o.size());
  std::partial_sum(o.begin(), o.end(), cum.begin());
  double area = (double)(cum[0] + 0) / 2.0;
  for (size_t i = 0; i + 1 < cum.size(); ++i) area += (double)(cum[i] + cum[i + 1]) / 2.0;
  const double total = (double)nnz * (double)len / 2.0;
  *gini = (total - area) / total;
}

// Tile features: MtxLoad's tile counting (src/sparse_features.cpp:181-265
// for the per-entry counts, :484-625 for the per-tile and per-block row
// statistics), CalculateTilesFeatures (:783-846) and the distance of
// CalculateTilesExtraFeatures (:943-965), for a general matrix read in CSR
// order.  B x B tiles; the first n % B row blocks hold n / B + 1 rows.
// As in the reference, the non-empty ratios and the variances of the tile,
// row-block and column-block counts start from -1 before they are summed.
// Output layout: sc[34] in the order of spops_tile_features_t; tile_i[4 B^2]
// (nnz, rows, cols, max row nnz), tile_d[2 B^2] (ave, std row nnz), blk_i[4 B]
// (RB nnz, RB max row nnz, CB nnz, CB max col nnz), blk_d[4 B] (RB ave, RB
// std, CB ave, CB std).
void orc_tile_features(int64_t n, int64_t nc, const int64_t* rp, const int64_t* ci, int64_t B, double* sc,
                       int64_t* tile_i, double* tile_d, int64_t* blk_i, double* blk_d) {
  const int64_t qr = n / B, mr = n % B, qc = nc / B, mc = nc % B;
  const int64_t thr = mr * (qr + 1), thc = mc * (qc + 1);
  auto rbk = [&](int64_t r) { return r < thr ? r / (qr + 1) : mr + (r - thr) / qr; };
  auto cbk = [&](int64_t c) { return c < thc ? c / (qc + 1) : mc + (c - thc) / qc; };
  auto rstart = [&](int64_t b) { return b < mr ? b * (qr + 1) : thr + (b - mr) * qr; };
  auto cstart = [&](int64_t b) { return b < mc ? b * (qc + 1) : thc + (b - mc) * qc; };
  const size_t T = (size_t)(B * B);
  const int64_t nnz = n ? rp[n] : 0;
  std::vector<int64_t> tnnz(T, 0), urows(T, 0), ucols(T, 0), tmax(T, 0), rbn(B, 0), cbn(B, 0), rbmax(B, 0),
      cbmax(B, 0), ccnt((size_t)nc, 0);
  std::vector<double> tave(T, 0.0), tstd(T, 0.0), rbave(B, 0.0), rbstd(B, 0.0), cbave(B, 0.0), cbstd(B, 0.0);
  std::unordered_map<int64_t, int64_t> colblk;  // (col, row block) pairs seen: Cols_cnt > 0
  for (int64_t r = 0; r < n; ++r)
    for (int64_t k = rp[r]; k < rp[r + 1]; ++k) {
      const int64_t tr = rbk(r), tc = cbk(ci[k]);
      ++tnnz[(size_t)(tr * B + tc)];
      ++rbn[(size_t)tr];
      ++cbn[(size_t)tc];
      ++ccnt[(size_t)ci[k]];
      if (colblk[ci[k] * B + tr]++ == 0) ++ucols[(size_t)(tr * B + tc)];
    }
  for (size_t i = 0; i < T; ++i) {
    if ((int64_t)i < mr * B) tave[i] = (double)tnnz[i] / (double)(qr + 1);
    else if (qr) tave[i] = (double)tnnz[i] / (double)qr;
  }
  for (int64_t b = 0; b < B; ++b) {
    if (b < mr) rbave[(size_t)b] = (double)rbn[(size_t)b] / (double)(qr + 1);
    else if (qr) rbave[(size_t)b] = (double)rbn[(size_t)b] / (double)qr;
    if (b < mc) cbave[(size_t)b] = (double)cbn[(size_t)b] / (double)(qc + 1);
    else if (qc) cbave[(size_t)b] = (double)cbn[(size_t)b] / (double)qc;
  }
  // Rows_cnt one row at a time: tile max / sum of squared deviations, uniq rows
  std::vector<int64_t> h((size_t)B, 0);
  for (int64_t r = 0; r < n; ++r) {
    const int64_t tr = rbk(r);
    for (int64_t k = rp[r]; k < rp[r + 1]; ++k) ++h[(size_t)cbk(ci[k])];
    for (int64_t tc = 0; tc < B; ++tc) {
      const size_t t = (size_t)(tr * B + tc);
      if (h[(size_t)tc]) ++urows[t];
      tmax[t] = std::max(tmax[t], h[(size_t)tc]);
      const double d = (double)h[(size_t)tc] - tave[t];
      tstd[t] += d * d;
      h[(size_t)tc] = 0;
    }
  }
  for (size_t i = 0; i < T; ++i) {
    if ((int64_t)i < mr * B) tstd[i] = tstd[i] / (double)(qr + 1);
    else if (qr) tstd[i] = tstd[i] / (double)qr;
    tstd[i] = std::sqrt(tstd[i]);
  }
  for (int64_t b = 0; b < B; ++b) {
    const int64_t r0 = rstart(b), r1 = b < mr ? r0 + qr + 1 : r0 + qr;
    for (int64_t r = r0; r < r1 && r < n; ++r) {
      const int64_t len = rp[r + 1] - rp[r];
      rbmax[(size_t)b] = std::max(rbmax[(size_t)b], len);
      const double d = (double)len - rbave[(size_t)b];
      rbstd[(size_t)b] += d * d;
    }
    const int64_t c0 = cstart(b), c1 = b < mc ? c0 + qc + 1 : c0 + qc;
    for (int64_t c = c0; c < c1 && c < nc; ++c) {
      cbmax[(size_t)b] = std::max(cbmax[(size_t)b], ccnt[(size_t)c]);
      const double d = (double)ccnt[(size_t)c] - cbave[(size_t)b];
      cbstd[(size_t)b] += d * d;
    }
  }
  for (int64_t b = 0; b < B; ++b) {
    if (b < mr) rbstd[(size_t)b] /= (double)(qr + 1);
    else if (qr) rbstd[(size_t)b] /= (double)qr;
    rbstd[(size_t)b] = std::sqrt(rbstd[(size_t)b]);
    if (b < mc) cbstd[(size_t)b] /= (double)(qc + 1);
    else if (qc) cbstd[(size_t)b] /= (double)qc;
    cbstd[(size_t)b] = std::sqrt(cbstd[(size_t)b]);
  }
  // CalculateTilesFeatures: counts statistics with the -1 starts
  auto stats = [&](const std::vector<int64_t>& cnt, double ave, double* nzr, int64_t* mn, int64_t* mx, double* var,
                   double* sd, double* p, double* gini) {
    double z = -1.0, v = -1.0;
    int64_t lo = 100000000, hi = 0;
    for (int64_t c : cnt) {
      if (c) ++z;
      const double d = (double)c - ave;
      v += d * d;
      lo = std::min(lo, c);
      hi = std::max(hi, c);
    }
    *nzr = z / (double)cnt.size();
    *var = v / (double)cnt.size();
    *sd = std::sqrt(std::max(*var, 0.0));
    *mn = lo;
    *mx = hi;
    double nz2, ave2, var2, sd2;
    int64_t mn2, mx2;
    count_stats(cnt, nnz, &nz2, &mn2, &mx2, &ave2, &var2, &sd2, p, gini);
  };
  double f[23];
  int64_t ii[6];
  const double ave_t = (double)nnz / ((double)B * (double)B), ave_b = (double)nnz / (double)B;
  f[1] = ave_t;
  stats(tnnz, ave_t, &f[0], &ii[0], &ii[1], &f[2], &f[3], &f[4], &f[5]);
  f[7] = ave_b;
  stats(rbn, ave_b, &f[6], &ii[2], &ii[3], &f[8], &f[9], &f[10], &f[11]);
  f[13] = ave_b;
  stats(cbn, ave_b, &f[12], &ii[4], &ii[5], &f[14], &f[15], &f[16], &f[17]);
  int64_t su = 0, sc2 = 0;
  for (size_t i = 0; i < T; ++i) {
    su += urows[i];
    sc2 += ucols[i];
  }
  f[18] = (double)su / (double)nnz;
  f[19] = (double)sc2 / (double)nnz;
  f[20] = (double)su / (double)n;
  f[21] = (double)sc2 / (double)nc;
  double dist = 0.0;
  for (int64_t r = 0; r < n; ++r) {
    const int64_t len = rp[r + 1] - rp[r];
    int64_t dis = 0;
    for (int64_t k = rp[r]; k + 1 < rp[r + 1]; ++k) dis += ci[k + 1] - ci[k];
    if (len) dist += (double)dis / (double)len;
  }
  f[22] = dist / (double)n;
  const double head[11] = {(double)B, (double)qr, (double)mr, (double)qc, (double)mc, (double)ii[0],
                           (double)ii[1], (double)ii[2], (double)ii[3], (double)ii[4], (double)ii[5]};
  std::memcpy(sc, head, sizeof(head));
  std::memcpy(sc + 11, f, sizeof(f));
  for (size_t i = 0; i < T; ++i) {
    tile_i[i] = tnnz[i];
    tile_i[T + i] = urows[i];
    tile_i[2 * T + i] = ucols[i];
    tile_i[3 * T + i] = tmax[i];
    tile_d[i] = tave[i];
    tile_d[T + i] = tstd[i];
  }
  for (int64_t b = 0; b < B; ++b) {
    blk_i[b] = rbn[(size_t)b];
    blk_i[B + b] = rbmax[(size_t)b];
    blk_i[2 * B + b] = cbn[(size_t)b];
    blk_i[3 * B + b] = cbmax[(size_t)b];
    blk_d[b] = rbave[(size_t)b];
    blk_d[B + b] = rbstd[(size_t)b];
    blk_d[2 * B + b] = cbave[(size_t)b];
    blk_d[3 * B + b] = cbstd[(size_t)b];
  }
}

void orc_features(int64_t n, int64_t nc, const int64_t* rp, const int64_t* ci, const double* v, double* out) {
  std::vector<int64_t> rcnt((size_t)n, 0), ccnt((size_t)nc, 0);
  std::vector<double> dom((size_t)n, 0.0), rmax((size_t)n, 0.0), rmin((size_t)n, 0.0), cmax((size_t)nc, 0.0),
      cmin((size_t)nc, 0.0);
  std::map<int64_t, int64_t> diag;
  int64_t lower = 0, upper = 0, dg = 0;
  double maxd = -DBL_MAX, maxo = -DBL_MAX;
  const int64_t nnz = n ? rp[n] : 0;
  for (int64_t r = 0; r < n; ++r)
    for (int64_t k = rp[r]; k < rp[r + 1]; ++k) {
      const int64_t c = ci[k], d = c - r;
      const double a = std::fabs(v[k]);
      ++rcnt[(size_t)r];
      ++ccnt[(size_t)c];
      ++diag[d];
      if (d == 0) {
        ++dg;
        maxd = std::max(maxd, a);
        dom[(size_t)r] += a;
      } else {
        if (d < 0) ++lower; else ++upper;
        maxo = std::max(maxo, a);
        dom[(size_t)r] -= a;
      }
      const double l = std::log10(a);
      if (rmax[(size_t)r] < l) rmax[(size_t)r] = l;
      if (a > 0.0 && rmin[(size_t)r] > l) rmin[(size_t)r] = l;
      if (cmax[(size_t)c] < l) cmax[(size_t)c] = l;
      if (a > 0.0 && cmin[(size_t)c] > l) cmin[(size_t)c] = l;
    }
  const int64_t thr = (n + nc - 1) / 20;
  int64_t close = 0;
  for (const auto& kv : diag)
    if (std::llabs(kv.first) <= thr) close += kv.second;
  double rvar = -1.0, cvar = -1.0;
  int64_t dominant = 0;
  for (int64_t r = 0; r < n; ++r) {
    if (rmin[(size_t)r] != 0.0) rvar = std::max(rvar, rmax[(size_t)r] - rmin[(size_t)r]);
    if (dom[(size_t)r] > 0) ++dominant;
  }
  for (int64_t c = 0; c < nc; ++c)
    if (cmin[(size_t)c] != 0.0) cvar = std::max(cvar, cmax[(size_t)c] - cmin[(size_t)c]);
  double ps = 0.0, vs = 0.0;
  if (n == nc) {
    std::map<std::pair<int64_t, int64_t>, std::string> text;
    char buf[64];
    for (int64_t r = 0; r < n; ++r)
      for (int64_t k = rp[r]; k < rp[r + 1]; ++k) {
        std::snprintf(buf, sizeof(buf), "%lf", v[k]);
        text.emplace(std::make_pair(r, ci[k]), buf);
      }
    int64_t sp = 0, sv = 0;
    for (const auto& kv : text) {
      if (kv.first.first == kv.first.second) continue;
      auto it = text.find(std::make_pair(kv.first.second, kv.first.first));
      if (it != text.end()) {
        ++sp;
        if (it->second == kv.second) ++sv;
      }
    }
    ps = (double)sp / (double)(nnz - dg);
    vs = (double)sv / (double)(nnz - dg);
  }
  double rnz, rave, rv, rsd, rp_, rg, cnz, cave, cv, csd, cp_, cg;
  int64_t rmn, rmx, cmn, cmx;
  count_stats(rcnt, nnz, &rnz, &rmn, &rmx, &rave, &rv, &rsd, &rp_, &rg);
  count_stats(ccnt, nnz, &cnz, &cmn, &cmx, &cave, &cv, &csd, &cp_, &cg);
  const double vals[32] = {(double)n, (double)nc, (double)nnz, (double)lower, (double)upper, (double)dg,
                           (double)diag.size(), (double)rmn, (double)rmx, (double)cmn, (double)cmx,
                           (double)nnz / ((double)n * (double)nc), (double)close / (double)nnz, ps, vs, rnz, rave, rv,
                           rsd, rp_, rg, cnz, cave, cv, csd, cp_, cg, (double)dominant / (double)std::min(n, nc),
                           maxo, maxd, rvar, cvar};
  std::memcpy(out, vals, sizeof(vals));
}

// ------------------------------------------------------------ adjoints
void orc_spmv_t_csr_f64_i32(int64_t nr, int64_t nc, const int32_t* rp, const int32_t* ci, const double* v,
                            const double* g, double* y) {
  for (int64_t j = 0; j < nc; ++j) y[j] = 0.0;
  for (int64_t r = 0; r < nr; ++r)
    for (int64_t k = rp[r]; k < rp[r + 1]; ++k) y[ci[k]] += v[k] * g[r];
}

void orc_sddmm_csr_f64_i32(int64_t nr, const int32_t* rp, const int32_t* ci, const double* g, const double* x,
                           double* out) {
  for (int64_t r = 0; r < nr; ++r)
    for (int64_t k = rp[r]; k < rp[r + 1]; ++k) out[k] = g[r] * x[ci[k]];
}

}  // extern "C"
