// Seeded synthetic sparse-matrix generators for the benchmark workloads.
//
// The reference's own inputs are SuiteSparse matrices that are not available
// here, so every workload is a seeded synthetic matrix with the stated shape,
// size and value distribution.  Each generator is a pure function of its
// arguments: row r draws from its own counter-based stream
// (splitmix64(seed, stream, r)), so the output does not depend on how many
// host threads fill it.  Rows are emitted with strictly increasing column
// indices, as a Matrix Market file sorted by (row, col) would give after
// read_csr_matrix (reference utils/sparse_io.cpp:190).
//
// Two-pass API: *_rowlen fills per-row lengths; the caller turns them into a
// row pointer and allocates; *_fill writes columns and values.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

inline uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

// Small per-row generator: splitmix64 sequence keyed by (seed, stream, row).
struct Rng {
  uint64_t s;
  Rng(uint64_t seed, uint64_t stream, uint64_t row) {
    s = mix64(seed ^ mix64(stream * 0x632be59bd9b4e019ULL ^ mix64(row + 0x1234567ULL)));
  }
  uint64_t next() {
    s += 0x9e3779b97f4a7c15ULL;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
  uint64_t below(uint64_t n) { return (uint64_t)(((unsigned __int128)next() * n) >> 64); }
  double normal() {  // Box-Muller, one value per call
    double u1 = uniform(), u2 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586476925 * u2);
  }
  int64_t poisson(double lam) {  // Knuth for small means, normal approximation above 64
    if (lam > 64.0) {
      double v = std::floor(lam + std::sqrt(lam) * normal() + 0.5);
      return v < 0 ? 0 : (int64_t)v;
    }
    double L = std::exp(-lam), p = 1.0;
    int64_t k = 0;
    do { ++k; p *= uniform(); } while (p > L);
    return k - 1;
  }
};

template <typename F>
void parallel_rows(int64_t n, F f) {
  unsigned nt = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  if (n < 4096) nt = 1;
  std::vector<std::thread> th;
  int64_t per = (n + nt - 1) / nt;
  for (unsigned t = 0; t < nt; ++t) {
    int64_t a = (int64_t)t * per, b = std::min<int64_t>(n, a + per);
    if (a >= b) break;
    th.emplace_back([=]() { for (int64_t r = a; r < b; ++r) f(r); });
  }
  for (auto& x : th) x.join();
}

// `len` distinct values drawn uniformly from [0, range), sorted ascending.
template <typename I>
void distinct_sorted(Rng& g, int64_t len, int64_t range, I* out) {
  std::vector<int64_t> v;
  v.reserve(len + 8);
  while ((int64_t)v.size() < len) {
    while ((int64_t)v.size() < len) v.push_back((int64_t)g.below((uint64_t)range));
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
  }
  for (int64_t k = 0; k < len; ++k) out[k] = (I)v[k];
}

template <typename I>
void write_sorted_unique(std::vector<int64_t>& v, I* out) {
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end()), v.end());
  for (size_t k = 0; k < v.size(); ++k) out[k] = (I)v[k];
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------- vectors
void synth_uniform_f64(int64_t n, uint64_t seed, double lo, double hi, double* out) {
  parallel_rows((n + 1023) / 1024, [&](int64_t blk) {
    Rng g(seed, 7, (uint64_t)blk);
    int64_t a = blk * 1024, b = std::min<int64_t>(n, a + 1024);
    for (int64_t i = a; i < b; ++i) out[i] = lo + (hi - lo) * g.uniform();
  });
}

void synth_normal_f64(int64_t n, uint64_t seed, double* out) {
  parallel_rows((n + 1023) / 1024, [&](int64_t blk) {
    Rng g(seed, 8, (uint64_t)blk);
    int64_t a = blk * 1024, b = std::min<int64_t>(n, a + 1024);
    for (int64_t i = a; i < b; ++i) out[i] = g.normal();
  });
}

// ------------------------------------------------- 2D 5-point Laplacian
// n = nx*ny rows, row r = (i, j) with r = i*ny + j; diagonal 4, neighbours -1.
int64_t synth_laplacian_nnz(int64_t nx, int64_t ny) {
  return 5 * nx * ny - 2 * nx - 2 * ny;
}

void synth_laplacian_fill_i32(int64_t nx, int64_t ny, int32_t* rp, int32_t* ci, double* v) {
  int64_t k = 0;
  rp[0] = 0;
  for (int64_t i = 0; i < nx; ++i)
    for (int64_t j = 0; j < ny; ++j) {
      int64_t r = i * ny + j;
      if (i > 0) { ci[k] = (int32_t)(r - ny); v[k++] = -1.0; }
      if (j > 0) { ci[k] = (int32_t)(r - 1); v[k++] = -1.0; }
      ci[k] = (int32_t)r; v[k++] = 4.0;
      if (j < ny - 1) { ci[k] = (int32_t)(r + 1); v[k++] = -1.0; }
      if (i < nx - 1) { ci[k] = (int32_t)(r + ny); v[k++] = -1.0; }
      rp[r + 1] = (int32_t)k;
    }
}

// ------------------------------------------------------ power-law rows
// Row length round(lognormal(mu, sigma)) clipped to [lo, hi] (and to ncols).
void synth_powerlaw_rowlen(int64_t n, int64_t ncols, double mu, double sigma, int64_t lo, int64_t hi,
                           uint64_t seed, int64_t* len) {
  parallel_rows(n, [&](int64_t r) {
    Rng g(seed, 1, (uint64_t)r);
    double L = std::floor(std::exp(mu + sigma * g.normal()) + 0.5);
    int64_t l = (int64_t)std::min<double>(std::max<double>(L, (double)lo), (double)hi);
    len[r] = std::min<int64_t>(l, ncols);
  });
}

// Columns uniform without replacement over [0, ncols), values N(0,1).
void synth_powerlaw_fill_i32(int64_t n, int64_t ncols, uint64_t seed, const int64_t* rp, int32_t* ci,
                             double* v) {
  parallel_rows(n, [&](int64_t r) {
    Rng g(seed, 2, (uint64_t)r);
    int64_t a = rp[r], L = rp[r + 1] - rp[r];
    distinct_sorted(g, L, ncols, ci + a);
    for (int64_t k = 0; k < L; ++k) v[a + k] = g.normal();
  });
}

// ---------------------------------------------- banded-plus-random rows
// Row length Poisson(mean) (at least 1); half of the draws within |i-j| <= band,
// half uniform; duplicates removed, so a row can come out shorter than drawn.
void synth_banded_rowlen(int64_t n, double mean, int64_t band, uint64_t seed, int64_t* len) {
  parallel_rows(n, [&](int64_t r) {
    Rng g(seed, 3, (uint64_t)r);
    int64_t L = std::max<int64_t>(1, g.poisson(mean));
    L = std::min<int64_t>(L, n);
    std::vector<int64_t> c;
    c.reserve(L);
    for (int64_t k = 0; k < L; ++k) {
      if (k & 1) {
        c.push_back((int64_t)g.below((uint64_t)n));
      } else {
        int64_t lo = std::max<int64_t>(0, r - band), hi = std::min<int64_t>(n - 1, r + band);
        c.push_back(lo + (int64_t)g.below((uint64_t)(hi - lo + 1)));
      }
    }
    std::sort(c.begin(), c.end());
    len[r] = (int64_t)(std::unique(c.begin(), c.end()) - c.begin());
  });
}

void synth_banded_fill_i32(int64_t n, double mean, int64_t band, uint64_t seed, const int64_t* rp,
                           int32_t* ci, double* v) {
  parallel_rows(n, [&](int64_t r) {
    Rng g(seed, 3, (uint64_t)r);
    int64_t L = std::max<int64_t>(1, g.poisson(mean));
    L = std::min<int64_t>(L, n);
    std::vector<int64_t> c;
    c.reserve(L);
    for (int64_t k = 0; k < L; ++k) {
      if (k & 1) {
        c.push_back((int64_t)g.below((uint64_t)n));
      } else {
        int64_t lo = std::max<int64_t>(0, r - band), hi = std::min<int64_t>(n - 1, r + band);
        c.push_back(lo + (int64_t)g.below((uint64_t)(hi - lo + 1)));
      }
    }
    write_sorted_unique(c, ci + rp[r]);
    Rng gv(seed, 4, (uint64_t)r);
    for (int64_t k = rp[r]; k < rp[r + 1]; ++k) v[k] = gv.normal();
  });
}

// --------------------------------------------- symmetric-pattern graph
// Half-degree draws: row i proposes round(lognormal(mu,sigma)/2) neighbours
// uniformly; the pattern is the union of proposals and their mirrors, so the
// mean degree is about exp(mu + sigma^2/2).  Produced as a COO edge list of
// proposals (i, j) with i != j; the caller symmetrises and deduplicates.
void synth_graph_proposals_count(int64_t n, double mu, double sigma, uint64_t seed, int64_t* cnt) {
  parallel_rows(n, [&](int64_t r) {
    Rng g(seed, 5, (uint64_t)r);
    double d = std::floor(std::exp(mu + sigma * g.normal()) * 0.5 + 0.5);
    cnt[r] = std::min<int64_t>(std::max<int64_t>((int64_t)d, 1), n - 1);
  });
}

void synth_graph_proposals_fill(int64_t n, uint64_t seed, const int64_t* off, int64_t* dst) {
  parallel_rows(n, [&](int64_t r) {
    Rng g(seed, 6, (uint64_t)r);
    for (int64_t k = off[r]; k < off[r + 1]; ++k) {
      int64_t j;
      do { j = (int64_t)g.below((uint64_t)n); } while (j == r);
      dst[k] = j;
    }
  });
}

// Values U[lo, hi] per stored entry, entry k of row r from row r's stream.
void synth_row_uniform_values(int64_t n, uint64_t seed, const int64_t* rp, double lo, double hi,
                              double* v) {
  parallel_rows(n, [&](int64_t r) {
    Rng g(seed, 9, (uint64_t)r);
    for (int64_t k = rp[r]; k < rp[r + 1]; ++k) v[k] = lo + (hi - lo) * g.uniform();
  });
}

// ------------------------------------------ planted column communities
// Row r belongs to community c_r (uniform over ncomm); its length is
// round(lognormal(mu, sigma)) clipped to [1, ncols]; each draw lands in the
// community's column block [c_r*w, (c_r+1)*w) with probability p_in, else
// uniformly over all columns; duplicates removed.  Values N(0,1).
static void planted_cols(int64_t r, int64_t ncols, int64_t ncomm, double mu, double sigma, double p_in,
                         uint64_t seed, std::vector<int64_t>& c) {
  Rng g(seed, 10, (uint64_t)r);
  int64_t w = ncols / ncomm;
  int64_t comm = (int64_t)g.below((uint64_t)ncomm);
  double Ld = std::floor(std::exp(mu + sigma * g.normal()) + 0.5);
  int64_t L = (int64_t)std::min<double>(std::max<double>(Ld, 1.0), (double)ncols);
  c.clear();
  c.reserve(L);
  for (int64_t k = 0; k < L; ++k) {
    if (g.uniform() < p_in)
      c.push_back(comm * w + (int64_t)g.below((uint64_t)w));
    else
      c.push_back((int64_t)g.below((uint64_t)ncols));
  }
  std::sort(c.begin(), c.end());
  c.erase(std::unique(c.begin(), c.end()), c.end());
}

void synth_planted_rowlen(int64_t n, int64_t ncols, int64_t ncomm, double mu, double sigma, double p_in,
                          uint64_t seed, int64_t* len) {
  parallel_rows(n, [&](int64_t r) {
    std::vector<int64_t> c;
    planted_cols(r, ncols, ncomm, mu, sigma, p_in, seed, c);
    len[r] = (int64_t)c.size();
  });
}

void synth_planted_fill_i64(int64_t n, int64_t ncols, int64_t ncomm, double mu, double sigma, double p_in,
                            uint64_t seed, const int64_t* rp, int64_t* ci, double* v) {
  parallel_rows(n, [&](int64_t r) {
    std::vector<int64_t> c;
    planted_cols(r, ncols, ncomm, mu, sigma, p_in, seed, c);
    for (size_t k = 0; k < c.size(); ++k) ci[rp[r] + (int64_t)k] = c[k];
    Rng gv(seed, 11, (uint64_t)r);
    for (int64_t k = rp[r]; k < rp[r + 1]; ++k) v[k] = gv.normal();
  });
}

// ---------------------------------------------- grouped rows
// Rows come in contiguous groups of `group` rows; group g draws from the
// column block [(g mod (ncols / width)) * width, ... + width) with
// probability p_in, else uniformly over all columns; row length
// round(lognormal(mu, sigma)) clipped to [1, width]; duplicates removed.
// Rows of a group share most of their columns, so MinHash-LSH pairs them,
// and C = A A^T has dense group x group blocks.  Values N(0, 1).
static void grouped_cols(int64_t r, int64_t ncols, int64_t group, int64_t width, double mu, double sigma,
                         double p_in, uint64_t seed, std::vector<int64_t>& c) {
  Rng g(seed, 12, (uint64_t)r);
  const int64_t nblocks = std::max<int64_t>(1, ncols / width);
  const int64_t blk = (r / group) % nblocks;
  double Ld = std::floor(std::exp(mu + sigma * g.normal()) + 0.5);
  int64_t L = (int64_t)std::min<double>(std::max<double>(Ld, 1.0), (double)width);
  c.clear();
  c.reserve(L);
  for (int64_t k = 0; k < L; ++k) {
    if (g.uniform() < p_in)
      c.push_back(blk * width + (int64_t)g.below((uint64_t)width));
    else
      c.push_back((int64_t)g.below((uint64_t)ncols));
  }
  std::sort(c.begin(), c.end());
  c.erase(std::unique(c.begin(), c.end()), c.end());
}

void synth_grouped_rowlen(int64_t n, int64_t ncols, int64_t group, int64_t width, double mu, double sigma,
                          double p_in, uint64_t seed, int64_t* len) {
  parallel_rows(n, [&](int64_t r) {
    std::vector<int64_t> c;
    grouped_cols(r, ncols, group, width, mu, sigma, p_in, seed, c);
    len[r] = (int64_t)c.size();
  });
}

void synth_grouped_fill_i64(int64_t n, int64_t ncols, int64_t group, int64_t width, double mu, double sigma,
                            double p_in, uint64_t seed, const int64_t* rp, int64_t* ci, double* v) {
  parallel_rows(n, [&](int64_t r) {
    std::vector<int64_t> c;
    grouped_cols(r, ncols, group, width, mu, sigma, p_in, seed, c);
    for (size_t k = 0; k < c.size(); ++k) ci[rp[r] + (int64_t)k] = c[k];
    Rng gv(seed, 13, (uint64_t)r);
    for (int64_t k = rp[r]; k < rp[r + 1]; ++k) v[k] = gv.normal();
  });
}

}  // extern "C"
