// Exercises include/spops_b200/SpOps.h the way a caller of the reference's
// SpOps.h would: host structs and vectors in, host results out.  Every SpMV
// is checked against a plain CPU loop (componentwise error over |A||x|,
// 1e-12 for double, 1e-5 for float); conversions against properties of the
// reference layouts.  Prints "shim OK" and exits 0 on success.
#include "SpOps.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

static int failures = 0;
#define EXPECT(cond, msg)                                          \
  do {                                                             \
    if (!(cond)) {                                                 \
      std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, msg);     \
      ++failures;                                                  \
    }                                                              \
  } while (0)

template <typename I, typename V>
CSR_Matrix<I, V> random_csr(I n, I ncols, unsigned seed, bool banded) {
  std::mt19937_64 rng(seed);
  std::vector<I> rp(1, 0), ci;
  std::vector<V> v;
  for (I r = 0; r < n; ++r) {
    int len = (int)(rng() % 40);
    if (r % 97 == 5) len = 0;     // empty rows
    if (r == 11) len = 900;       // a long row
    std::vector<I> cols;
    for (int k = 0; k < len; ++k) {
      I c = banded ? (I)((int64_t)r + (int64_t)(rng() % 9) - 4) : (I)(rng() % (uint64_t)ncols);
      if (c >= 0 && c < ncols) cols.push_back(c);
    }
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
    for (I c : cols) {
      ci.push_back(c);
      v.push_back((V)((double)(rng() % 2001) / 1000.0 - 1.0));
    }
    rp.push_back((I)ci.size());
  }
  CSR_Matrix<I, V> A;
  std::memset(static_cast<void*>(&A), 0, sizeof(A));
  A.num_rows = n;
  A.num_cols = ncols;
  A.num_nnzs = (I)ci.size();
  A.row_offset = spops_b200::detail::host_alloc<I>((int64_t)rp.size());
  A.col_index = spops_b200::detail::host_alloc<I>((int64_t)ci.size());
  A.values = spops_b200::detail::host_alloc<V>((int64_t)v.size());
  std::copy(rp.begin(), rp.end(), A.row_offset);
  std::copy(ci.begin(), ci.end(), A.col_index);
  std::copy(v.begin(), v.end(), A.values);
  return A;
}

template <typename I, typename V>
void check_y(const char* what, const CSR_Matrix<I, V>& A, const std::vector<V>& x, const std::vector<V>& y0,
             double alpha, double beta, const std::vector<V>& y) {
  const double tol = sizeof(V) == 8 ? 1e-12 : 1e-5;
  double worst = 0;
  for (I r = 0; r < A.num_rows; ++r) {
    double s = 0, a = 0;
    for (I k = A.row_offset[r]; k < A.row_offset[r + 1]; ++k) {
      s += (double)A.values[k] * (double)x[A.col_index[k]];
      a += std::fabs((double)A.values[k] * (double)x[A.col_index[k]]);
    }
    const double ref = alpha * s + beta * (double)y0[r];
    const double den = std::fabs(alpha) * a + std::fabs(beta * (double)y0[r]);
    worst = std::max(worst, std::fabs((double)y[r] - ref) / std::max(den, 1e-300));
  }
  if (worst > tol) std::printf("  %s: error %.3e\n", what, worst);
  EXPECT(worst <= tol, what);
}

template <typename I, typename V>
void run_all() {
  const I n = 3001, nc = 2500;
  CSR_Matrix<I, V> A = random_csr<I, V>(n, nc, 7, false);
  std::vector<V> x(nc), y0(n);
  std::mt19937_64 rng(3);
  for (auto& t : x) t = (V)((double)(rng() % 2001) / 1000.0 - 1.0);
  for (auto& t : y0) t = (V)((double)(rng() % 2001) / 1000.0 - 1.0);
  const double alpha = 0.8, beta = 0.7;
  auto run = [&](const char* what, auto&& op) {
    std::printf("  %s (index %zu bytes, value %zu bytes)\n", what, sizeof(I), sizeof(V));
    std::vector<V> y = y0;
    op((V)alpha, x.data(), (V)beta, y.data());
    check_y(what, A, x, y0, alpha, beta, y);
  };
  run("SpOps_csr", [&](V a, const V* xx, V b, V* yy) { SpOps_csr(a, A, xx, b, yy); });
  run("SpOps_csr again (cached)", [&](V a, const V* xx, V b, V* yy) { SpOps_csr(a, A, xx, b, yy); });
  // values changed in place between calls: the default cache mode keeps the
  // pattern on the device but re-reads A.values, as the reference does
  {
    std::vector<V> saved(A.values, A.values + A.num_nnzs);
    for (I k = 0; k < A.num_nnzs; ++k) A.values[k] = (V)(-2.5 * (double)A.values[k] + 0.125 * (double)(k % 7));
    run("SpOps_csr after an in-place value edit", [&](V a, const V* xx, V b, V* yy) { SpOps_csr(a, A, xx, b, yy); });
    spops_b200::set_cache(true);  // whole device copies: an edit needs invalidate()
    spops_b200::invalidate(A.row_offset);
    run("SpOps_csr, full cache", [&](V a, const V* xx, V b, V* yy) { SpOps_csr(a, A, xx, b, yy); });
    std::copy(saved.begin(), saved.end(), A.values);
    spops_b200::invalidate(A.row_offset);
    run("SpOps_csr, full cache after invalidate", [&](V a, const V* xx, V b, V* yy) { SpOps_csr(a, A, xx, b, yy); });
    spops_b200::set_cache_mode(spops_b200::CacheMode::Pattern);
    EXPECT(spops_b200::cache_mode() == spops_b200::CacheMode::Pattern, "cache mode back to the default");
  }

  // COO both ways
  COO_Matrix<I, V> coo = csr_to_coo(A);
  EXPECT(coo.num_nnzs == A.num_nnzs, "csr_to_coo nnz");
  bool rows_ok = true;
  for (I r = 0; r < n; ++r)
    for (I k = A.row_offset[r]; k < A.row_offset[r + 1]; ++k)
      rows_ok = rows_ok && coo.row_index[k] == r && coo.col_index[k] == A.col_index[k] && coo.values[k] == A.values[k];
  EXPECT(rows_ok, "csr_to_coo arrays");
  run("SpOps_coo", [&](V a, const V* xx, V b, V* yy) { SpOps_coo(a, coo, xx, b, yy); });
  CSR_Matrix<I, V> back = coo_to_csr(coo);
  bool same = back.num_nnzs == A.num_nnzs;
  for (I r = 0; same && r <= n; ++r) same = back.row_offset[r] == A.row_offset[r];
  for (I k = 0; same && k < A.num_nnzs; ++k) same = back.col_index[k] == A.col_index[k] && back.values[k] == A.values[k];
  EXPECT(same, "coo_to_csr round trip");
  // compact: a row with duplicates in file order 5, 3, 5, 7 (7 cancels) -> 3, 5
  {
    COO_Matrix<I, V> d;
    std::memset(static_cast<void*>(&d), 0, sizeof(d));
    d.num_rows = 2;
    d.num_cols = 8;
    d.num_nnzs = 5;
    I ri[5] = {1, 1, 1, 1, 1}, cj[5] = {5, 3, 5, 7, 7};
    V vv[5] = {(V)1, (V)2, (V)4, (V)1.5, (V)-1.5};
    d.row_index = ri;
    d.col_index = cj;
    d.values = vv;
    CSR_Matrix<I, V> c = coo_to_csr(d, true);
    EXPECT(c.num_nnzs == 2 && c.row_offset[1] == 0 && c.row_offset[2] == 2, "compact sizes");
    EXPECT(c.col_index[0] == 3 && c.col_index[1] == 5 && c.values[0] == (V)2 && c.values[1] == (V)5,
           "compact order: reverse first appearance, zeros dropped");
    delete_host_matrix(c);
  }

  ELL_Matrix<I, V> ell = csr_to_ell(A, RowMajor);
  I widest = 0;
  for (I r = 0; r < n; ++r) widest = std::max(widest, (I)(A.row_offset[r + 1] - A.row_offset[r]));
  bool ell_ok = ell.max_row_width == widest;
  for (I r = 0; ell_ok && r < n; ++r) {
    const I len = A.row_offset[r + 1] - A.row_offset[r];
    for (I k = 0; ell_ok && k < ell.max_row_width; ++k) {
      const I c = ell.col_index[(int64_t)r * ell.max_row_width + k];
      ell_ok = k < len ? c == A.col_index[A.row_offset[r] + k] : c == (I)-1;
    }
  }
  EXPECT(ell_ok, "csr_to_ell row-major layout");
  run("SpOps_ell", [&](V a, const V* xx, V b, V* yy) { SpOps_ell(a, ell, xx, b, yy); });

  S_ELL_Matrix<I, V> sell = csr_to_sell(A, nullptr, 4, 4);
  EXPECT(sell.chunk_num == (n + 3) / 4, "csr_to_sell chunk_num");
  run("SpOps_sell", [&](V a, const V* xx, V b, V* yy) { SpOps_sell(a, sell, xx, b, yy); });

  SELL_C_Sigma_Matrix<I, V> scs = csr_to_sell_c_sigma(A, nullptr, 512, 32, 1);
  std::vector<int> seen(n, 0);
  for (I r = 0; r < n; ++r) seen[scs.reorder[r]]++;
  EXPECT(std::count(seen.begin(), seen.end(), 1) == n, "sell_c_sigma reorder is a permutation");
  bool desc = true;  // within each slice of 512 stored rows, lengths do not increase
  for (I r = 1; r < n; ++r)
    if (r % 512) {
      const I a0 = scs.reorder[r - 1], a1 = scs.reorder[r];
      desc = desc && (A.row_offset[a0 + 1] - A.row_offset[a0]) >= (A.row_offset[a1 + 1] - A.row_offset[a1]);
    }
  EXPECT(desc, "sell_c_sigma slices sorted by length");
  run("SpOps_sell_c_sigma", [&](V a, const V* xx, V b, V* yy) { SpOps_sell_c_sigma(a, scs, xx, b, yy); });
  // the same struct uploaded from its host arrays (as a struct a caller built)
  spops_b200::invalidate(scs.reorder);
  run("SpOps_sell_c_sigma from host arrays", [&](V a, const V* xx, V b, V* yy) { SpOps_sell_c_sigma(a, scs, xx, b, yy); });

  SELL_C_R_Matrix<I, V> scr = csr_to_sell_c_R(A, nullptr, 32, 1);
  run("SpOps_sell_c_R", [&](V a, const V* xx, V b, V* yy) { SpOps_sell_c_R(a, scr, xx, b, yy); });
  spops_b200::invalidate(scr.reorder);
  run("SpOps_sell_c_R from host arrays", [&](V a, const V* xx, V b, V* yy) { SpOps_sell_c_R(a, scr, xx, b, yy); });

  BSR_Matrix<I, V> bsr = csr_to_bsr(A, (I)4, (I)4);
  EXPECT(bsr.blockDim_r == 4 && bsr.blockDim_c == 4 && bsr.row_ptr[bsr.mb] == bsr.nnzb, "csr_to_bsr shape");
  run("SpOps_bsr", [&](V a, const V* xx, V b, V* yy) { SpOps_bsr(a, bsr, xx, b, yy); });
  spops_b200::invalidate(bsr.row_ptr);
  run("SpOps_bsr from host arrays", [&](V a, const V* xx, V b, V* yy) { SpOps_bsr(a, bsr, xx, b, yy); });

  CSR5_Matrix<I, uint32_t, V> c5 = csr_to_csr5<I, uint32_t, V>(A, nullptr);
  EXPECT(c5.omega == 32 && c5.sigma == 16, "csr5 tile shape");
  run("SpOps_csr5", [&](V a, const V* xx, V b, V* yy) { SpOps_csr5(a, c5, xx, b, yy); });

  // DIA on a banded matrix
  CSR_Matrix<I, V> B = random_csr<I, V>(n, n, 9, true);
  DIA_Matrix<I, V> dia = csr_to_dia(B, (I)MAX_DIAG_NUM, nullptr, (I)4);
  EXPECT(dia.complete_ndiags >= 1 && dia.complete_ndiags <= 9, "csr_to_dia diagonals");
  {
    std::vector<V> xb(n), yb0(n), yb;
    for (I r = 0; r < n; ++r) {
      xb[r] = (V)((double)((r * 37) % 101) / 50.0 - 1.0);
      yb0[r] = (V)((double)((r * 11) % 13) / 6.0 - 1.0);
    }
    yb = yb0;
    SpOps_dia((V)alpha, dia, xb.data(), (V)beta, yb.data());
    check_y("SpOps_dia", B, xb, yb0, alpha, beta, yb);
    spops_b200::invalidate(dia.diag_offsets);
    yb = yb0;
    SpOps_dia((V)alpha, dia, xb.data(), (V)beta, yb.data());
    check_y("SpOps_dia from host arrays", B, xb, yb0, alpha, beta, yb);
  }

  // upload on every call, then back to the default mode
  spops_b200::set_cache(false);
  run("SpOps_csr without cache", [&](V a, const V* xx, V b, V* yy) { SpOps_csr(a, A, xx, b, yy); });
  spops_b200::set_cache_mode(spops_b200::CacheMode::Pattern);

  delete_host_matrix(back);
  delete_host_matrix(coo);
  delete_host_matrix(ell);
  delete_host_matrix(sell);
  delete_host_matrix(scs);
  delete_host_matrix(scr);
  delete_host_matrix(bsr);
  delete_host_matrix(c5);
  delete_host_matrix(dia);
  delete_host_matrix(B);
  delete_host_matrix(A);
}

void lsh_checks() {
  // 64 rows in 4 groups of identical patterns: every group must end up together
  std::vector<long long> rp(1, 0), ci;
  for (int r = 0; r < 64; ++r) {
    const int g = r % 4;
    for (int k = 0; k < 12; ++k) ci.push_back(g * 100 + k * 3);
    rp.push_back((long long)ci.size());
  }
  std::vector<uint64_t> sig = minhash_signatures_flat<long long>(rp.data(), ci.data(), 64, 64, 7);
  EXPECT(sig.size() == 64 * 64, "minhash size");
  bool same = true;
  for (int k = 0; k < 64; ++k) same = same && sig[(size_t)0 * 64 + k] == sig[(size_t)4 * 64 + k];
  EXPECT(same, "identical rows share signatures");
  auto pairs = lsh_candidate_pairs_vector<long long, double>(rp.data(), ci.data(), 64, 64, 16, 7, true);
  EXPECT(!pairs.empty(), "lsh pairs found");
  bool within = true;
  for (auto& p : pairs) within = within && (p.i % 4) == (p.j % 4) && p.i < p.j && p.score == 1.0;
  EXPECT(within, "pairs only inside groups, score 1");
  std::vector<long long> perm, offs;
  hierarchical_clustering_v0_fast<long long, double>(rp.data(), ci.data(), 64, pairs, 8LL, perm, offs);
  EXPECT(perm.size() == 64 && offs.front() == 0 && offs.back() == 64, "clustering shape");
  bool grouped = true;
  for (size_t c = 0; c + 1 < offs.size(); ++c) {
    EXPECT(offs[c + 1] - offs[c] <= 8, "cluster size cap");
    for (long long t = offs[c]; t < offs[c + 1]; ++t) grouped = grouped && perm[t] % 4 == perm[offs[c]] % 4;
  }
  EXPECT(grouped, "clusters inside groups");
}

// Row-wise SpGEMM and top-k against a direct host product on a small matrix.
void spgemm_checks() {
  // A: 6 x 5; B = A^T (5 x 6)
  std::vector<long long> rp = {0, 2, 4, 5, 8, 8, 10}, ci = {0, 3, 1, 3, 2, 0, 1, 4, 3, 4};
  std::vector<double> v = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10};
  CSR_Matrix<long long, double> A{};
  A.num_rows = 6;
  A.num_cols = 5;
  A.num_nnzs = 10;
  A.row_offset = rp.data();
  A.col_index = ci.data();
  A.values = v.data();
  std::vector<double> dense(30, 0.0);
  for (long long r = 0; r < 6; ++r)
    for (long long e = rp[r]; e < rp[r + 1]; ++e) dense[(size_t)(r * 5 + ci[e])] = v[e];
  std::vector<long long> trp(6, 0), tci;
  std::vector<double> tv;
  for (long long c = 0; c < 5; ++c) {
    for (long long r = 0; r < 6; ++r)
      if (dense[(size_t)(r * 5 + c)] != 0.0) {
        tci.push_back(r);
        tv.push_back(dense[(size_t)(r * 5 + c)]);
      }
    trp[(size_t)c + 1] = (long long)tci.size();
  }
  CSR_Matrix<long long, double> B{};
  B.num_rows = 5;
  B.num_cols = 6;
  B.num_nnzs = (long long)tci.size();
  B.row_offset = trp.data();
  B.col_index = tci.data();
  B.values = tv.data();
  CSR_Matrix<long long, double> C{};
  LeSpGEMM<true, long long, double>(A, B, C, 2);
  EXPECT(C.num_rows == 6 && C.num_cols == 6 && C.kernel_flag == 2, "LeSpGEMM shape");
  bool ok = true;
  for (long long i = 0; i < 6; ++i)
    for (long long e = C.row_offset[i]; e < C.row_offset[i + 1]; ++e) {
      double s = 0;
      for (long long k = 0; k < 5; ++k) s += dense[(size_t)(i * 5 + k)] * dense[(size_t)(C.col_index[e] * 5 + k)];
      ok = ok && std::fabs(s - C.values[e]) <= 1e-12 * std::fabs(s) && s != 0.0;
      if (e > C.row_offset[i]) ok = ok && C.col_index[e] > C.col_index[e - 1];
    }
  EXPECT(ok, "LeSpGEMM values and ascending columns");
  EXPECT(C.row_offset[5] == C.row_offset[4], "empty row stays empty");
  delete_host_matrix(C);
  CSR_Matrix<long long, double> T{};
  HashSpGEMMTopK<long long, double>(A, T, 2LL);
  bool topk = T.num_rows == 6;
  for (long long i = 0; i < 6 && topk; ++i) {
    topk = T.row_offset[i + 1] - T.row_offset[i] <= 2;
    for (long long e = T.row_offset[i]; e < T.row_offset[i + 1]; ++e) {
      topk = topk && T.col_index[e] != i && T.values[e] > 0.0 && T.values[e] <= 1.0;
      if (e > T.row_offset[i]) topk = topk && T.values[e] <= T.values[e - 1];
    }
  }
  EXPECT(topk, "HashSpGEMMTopK rows: at most k, no diagonal, similarity descending");
  delete_host_matrix(T);
}

// A small symmetric Matrix Market file read into host structs.
void mtx_checks() {
  const char* path = "shim_test_matrix.mtx";
  FILE* f = std::fopen(path, "w");
  EXPECT(f != nullptr, "temporary file");
  if (!f) return;
  std::fprintf(f, "%%%%MatrixMarket matrix coordinate real symmetric\n%% comment\n3 3 4\n");
  std::fprintf(f, "1 1 2.5\n2 1 -1e-3\n3 2 0.1\n3 3 4\n");
  std::fclose(f);
  COO_Matrix<int, double> coo = read_coo_matrix<int, double>(path);
  EXPECT(coo.num_nnzs == 6 && coo.row_index[1] == 1 && coo.col_index[1] == 0 && coo.row_index[2] == 0 &&
             coo.col_index[2] == 1 && coo.values[2] == -1e-3,
         "read_coo_matrix expands the symmetric entries in file order");
  CSR_Matrix<long long, float> csr = read_csr_matrix<long long, float>(path, true);
  // compacting lists a row's columns in reverse order of first appearance
  // (include/sparse_operation.h:22 threads them through a linked list)
  EXPECT(csr.num_rows == 3 && csr.num_nnzs == 6 && csr.row_offset[3] == 6 && csr.col_index[0] == 1 &&
             csr.values[0] == -1e-3f && csr.col_index[1] == 0 && csr.values[1] == 2.5f,
         "read_csr_matrix shape and values");
  delete_host_matrix(coo);
  delete_host_matrix(csr);
  std::remove(path);
}

// the feature class on a 300 x 200 general file: 300 rows make 256 row
// blocks (44 of two rows), 200 columns one column per block
void feature_checks() {
  const char* path = "shim_test_features.mtx";
  FILE* f = std::fopen(path, "w");
  EXPECT(f != nullptr, "temporary file");
  if (!f) return;
  std::vector<int> rr, cc;
  for (int r = 0; r < 300; ++r)
    for (int k = 0; k < 1 + r % 5; ++k) {
      rr.push_back(r);
      cc.push_back((r * 7 + k * 31) % 200);
    }
  std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n300 200 %d\n", (int)rr.size());
  for (size_t i = 0; i < rr.size(); ++i) std::fprintf(f, "%d %d %d.5\n", rr[i] + 1, cc[i] + 1, (int)(i % 9) - 4);
  std::fclose(f);
  // the row distance the reference's CalculateTilesExtraFeatures computes
  double dist = 0.0;
  for (size_t i = 0; i < rr.size();) {
    size_t j = i;
    while (j < rr.size() && rr[j] == rr[i]) ++j;
    dist += (double)(cc[j - 1] - cc[i]) / (double)(j - i);
    i = j;
  }
  dist /= 300.0;
  MTX<int, double> m(7);
  EXPECT(m.MtxLoad(path) && m.CalculateFeatures() && m.CalculateTilesExtraFeatures(path), "MTX calls");
  m.FeaturesPrint();
  m.ExtraFeaturesPrint();
  const spops_features_t& s = m.features();
  const spops_tile_features_t& t = m.tile_features();
  const double nnz = (double)rr.size();
  EXPECT(m.getRowNum() == 300 && m.getColNum() == 200 && s.nnz == (int64_t)rr.size() && m.getMatName() ==
                                                                                             "shim_test_features",
         "MTX shape and name");
  EXPECT(t.num_blocks == 256 && t.rows_per_block == 1 && t.rows_mod == 44 && t.cols_per_block == 0 &&
             t.cols_mod == 200,
         "MTX tile grid");
  EXPECT(t.uniq_r == 1.0 && t.pot_reuse_r == nnz / 300.0 && std::fabs(t.distance_per_row - dist) <= 1e-12 * 300,
         "MTX tile extra features");
  EXPECT(!m.FeaturesWrite("shim_test_features_out"), "MTX FeaturesWrite (false when written, as the reference)");
  FILE* g = std::fopen("shim_test_features_out/shim_test_features/shim_test_features.features", "r");
  EXPECT(g != nullptr, "MTX .features file");
  if (g) std::fclose(g);
  std::remove(path);
}

// the rest of the reference's API on a small file: read_<fmt>_matrix gives
// the same y as the CSR read; sum_csr_duplicates, csr_transpose,
// csr_to_binary_pattern, minhash_estimated_jaccard, the thread controls
void api_checks() {
  const char* path = "shim_test_api.mtx";
  FILE* f = std::fopen(path, "w");
  EXPECT(f != nullptr, "temporary file");
  if (!f) return;
  const int n = 600;
  std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n%d %d %d\n", n, n, 3 * n - 2);
  for (int r = 0; r < n; ++r)
    for (int c = r - 1; c <= r + 1; ++c)
      if (c >= 0 && c < n) std::fprintf(f, "%d %d %g\n", r + 1, c + 1, c == r ? 4.0 : -1.0 - 0.001 * r);
  std::fclose(f);
  std::vector<double> x(n), y0(n, 0.5), yc(n), y(n);
  for (int i = 0; i < n; ++i) x[i] = 0.01 * (i % 97) - 0.3;
  CSR_Matrix<int, double> csr = read_csr_matrix<int, double>(path);
  yc = y0;
  SpOps_csr(1.0, csr, x.data(), 0.5, yc.data());
  auto same_y = [&](const char* what, auto&& op) {
    y = y0;
    op(y.data());
    double worst = 0;
    for (int i = 0; i < n; ++i) worst = std::max(worst, std::fabs(y[i] - yc[i]));
    EXPECT(worst <= 1e-12, what);
  };
  ELL_Matrix<int, double> ell = read_ell_matrix<int, double>(path);
  EXPECT(ell.num_rows == n && ell.max_row_width == 3 && ell.kernel_flag == KERNEL_FLAG, "read_ell_matrix shape");
  same_y("read_ell_matrix y", [&](double* yy) { SpOps_ell(1.0, ell, x.data(), 0.5, yy); });
  S_ELL_Matrix<int, double> sell = read_sell_matrix<int, double>(path, 4, 1);
  same_y("read_sell_matrix y", [&](double* yy) { SpOps_sell(1.0, sell, x.data(), 0.5, yy); });
  SELL_C_Sigma_Matrix<int, double> scs = read_sell_c_sigma_matrix<int, double>(path, 64, 8, 1);
  same_y("read_sell_c_sigma_matrix y", [&](double* yy) { SpOps_sell_c_sigma(1.0, scs, x.data(), 0.5, yy); });
  SELL_C_R_Matrix<int, double> scr = read_sell_c_R_matrix<int, double>(path, 8, 1);
  same_y("read_sell_c_R_matrix y", [&](double* yy) { SpOps_sell_c_R(1.0, scr, x.data(), 0.5, yy); });
  DIA_Matrix<int, double> dia = read_dia_matrix<int, double>(path, 16, 1);
  EXPECT(dia.complete_ndiags == 3, "read_dia_matrix diagonals");
  same_y("read_dia_matrix y", [&](double* yy) { SpOps_dia(1.0, dia, x.data(), 0.5, yy); });
  BSR_Matrix<int, double> bsr = read_bsr_matrix<int, double>(path, 4, 4);
  same_y("read_bsr_matrix y", [&](double* yy) { SpOps_bsr(1.0, bsr, x.data(), 0.5, yy); });
  delete_ell_matrix(ell);
  delete_s_ell_matrix(sell);
  delete_s_ell_c_sigma_matrix(scs);
  delete_s_ell_c_R_matrix(scr);
  delete_dia_matrix(dia);
  delete_bsr_matrix(bsr);
  // csr_transpose of the tridiagonal matrix: entry (c, r) of the result is
  // entry (r, c) of the input
  CSR_Matrix<int, double> t = csr_transpose(csr);
  bool tr_ok = t.num_rows == n && t.num_nnzs == csr.num_nnzs;
  for (int r = 0; tr_ok && r < n; ++r)
    for (int k = csr.row_offset[r]; k < csr.row_offset[r + 1]; ++k) {
      const int c = csr.col_index[k];
      bool found = false;
      for (int q = t.row_offset[c]; q < t.row_offset[c + 1]; ++q)
        found = found || (t.col_index[q] == r && t.values[q] == csr.values[k]);
      tr_ok = tr_ok && found;
    }
  EXPECT(tr_ok, "csr_transpose entries");
  std::vector<int> perm(n);
  for (int i = 0; i < n; ++i) perm[i] = (i * 7 + 3) % n;  // 7 is prime to 600
  CSR_Matrix<int, double> ro = csr_reorder_rows(csr, perm);
  bool ro_ok = ro.num_rows == n && ro.num_nnzs == csr.num_nnzs;
  for (int i = 0; ro_ok && i < n; ++i) {
    const int p = perm[i], len = csr.row_offset[p + 1] - csr.row_offset[p];
    ro_ok = ro.row_offset[i + 1] - ro.row_offset[i] == len;
    for (int k = 0; ro_ok && k < len; ++k)
      ro_ok = ro.col_index[ro.row_offset[i] + k] == csr.col_index[csr.row_offset[p] + k] &&
              ro.values[ro.row_offset[i] + k] == csr.values[csr.row_offset[p] + k];
  }
  EXPECT(ro_ok, "csr_reorder_rows");
  delete_csr_matrix(ro);
  CSR_Matrix<int, double> bp = csr_to_binary_pattern(csr);
  EXPECT(bp.num_nnzs == csr.num_nnzs && bp.values[0] == 1.0 && bp.col_index[5] == csr.col_index[5],
         "csr_to_binary_pattern");
  // the clustered LeSpGEMM flow (test/test_spgemm_hc_lsh.cpp) against the
  // row-wise LeSpGEMM: clusters of 8 rows, C = A * A^T
  {
    std::vector<int> offs;
    for (int r = 0; r < n; r += 8) offs.push_back(r);
    offs.push_back(n);
    CSR_VlengthCluster<int, double> acl = csr_to_vlength_cluster(csr, offs);
    EXPECT(acl.rows == (int)offs.size() - 1 && acl.cluster_sz[0] == 8 && acl.max_cluster_sz == 256,
           "csr_to_vlength_cluster shape");
    CSR_VlengthCluster<int, double> ccl;
    std::memset(static_cast<void*>(&ccl), 0, sizeof(ccl));
    LeSpGEMM_VLength<true>(acl, t, ccl, 3);
    CSR_Matrix<int, double> c1 = vlength_cluster2csr(ccl), c2;
    LeSpGEMM<true>(csr, t, c2, 1);
    bool same = c1.num_rows == c2.num_rows && c1.num_nnzs == c2.num_nnzs;
    for (int r = 0; same && r <= n; ++r) same = c1.row_offset[r] == c2.row_offset[r];
    for (int k = 0; same && k < c1.num_nnzs; ++k)
      same = c1.col_index[k] == c2.col_index[k] && std::fabs(c1.values[k] - c2.values[k]) <= 1e-12 * (1 + std::fabs(c2.values[k]));
    EXPECT(same, "LeSpGEMM_VLength = row-wise LeSpGEMM");
    // kernel 2 (array accumulator) keeps every structural column: the same C
    // as the row-wise product; kernel 1 (hash, sorted) the same again here
    for (int kf : {1, 2}) {
      CSR_VlengthCluster<int, double> ck;
      std::memset(static_cast<void*>(&ck), 0, sizeof(ck));
      LeSpGEMM_VLength<true>(acl, t, ck, kf);
      CSR_Matrix<int, double> c3 = vlength_cluster2csr(ck);
      bool same_k = c3.num_rows == c2.num_rows && c3.num_nnzs == c2.num_nnzs;
      for (int r = 0; same_k && r <= n; ++r) same_k = c3.row_offset[r] == c2.row_offset[r];
      for (int k = 0; same_k && k < c3.num_nnzs; ++k)
        same_k = c3.col_index[k] == c2.col_index[k] &&
                 std::fabs(c3.values[k] - c2.values[k]) <= 1e-12 * (1 + std::fabs(c2.values[k]));
      EXPECT(same_k, kf == 1 ? "LeSpGEMM_VLength kernel 1 = row-wise" : "LeSpGEMM_VLength kernel 2 = row-wise");
      delete_host_matrix(ck);
      delete_csr_matrix(c3);
    }
    delete_vlength_cluster_matrix(acl);
    delete_host_matrix(ccl);
    delete_csr_matrix(c1);
    delete_csr_matrix(c2);
  }
  delete_csr_matrix(t);
  delete_csr_matrix(bp);
  delete_csr_matrix(csr);
  // sum_csr_duplicates: row 1 in file order 5, 3, 5, 7, 7 (7 cancels) -> 3, 5
  int rp[3] = {0, 1, 6}, ci[6] = {2, 5, 3, 5, 7, 7};
  double vv[6] = {1.0, 1.0, 2.0, 4.0, 1.5, -1.5};
  sum_csr_duplicates(2, 8, rp, ci, vv);
  EXPECT(rp[1] == 1 && rp[2] == 3 && ci[0] == 2 && ci[1] == 3 && ci[2] == 5 && vv[1] == 2.0 && vv[2] == 5.0,
         "sum_csr_duplicates");
  const uint64_t sa[4] = {1, 2, 3, 4}, sb[4] = {1, 9, 3, 8};
  EXPECT(minhash_estimated_jaccard(sa, sb, 4) == 0.5 && minhash_estimated_jaccard(sa, sb, 0) == 0.0,
         "minhash_estimated_jaccard");
  Le_set_thread_num(3);
  EXPECT(Le_get_thread_num() == 3 && Le_get_thread_id() == 0 && Le_get_core_num() >= 1, "thread controls");
  std::remove(path);
}

int main() {
  std::setvbuf(stdout, nullptr, _IONBF, 0);
  try {
    run_all<int, double>();
    run_all<int, float>();
    run_all<long long, double>();
    lsh_checks();
    spgemm_checks();
    mtx_checks();
    feature_checks();
    api_checks();
  } catch (const std::exception& e) {
    std::printf("exception: %s\n", e.what());
    return 2;
  }
  if (failures) {
    std::printf("%d failure(s)\n", failures);
    return 1;
  }
  std::printf("shim OK\n");
  return 0;
}
