// Matrix Market files read on the device.
//
// Replaces read_coo_matrix / read_csr_matrix (reference utils/sparse_io.cpp:
// 26-214) with mm_read_banner and mm_read_mtx_crd_size (utils/mmio.cpp:
// 144-283).  The rules kept from them:
//   * banner "%%MatrixMarket matrix coordinate <field> <symmetry>" (any case
//     after the first word); field real, integer or pattern; symmetry general,
//     symmetric, skew-symmetric or hermitian as mm_is_valid allows (only
//     "symmetric" is expanded: every off-diagonal entry (r, c, v) is followed
//     by (c, r, v), in file order);
//   * lines starting with '%' before the size line are skipped; the size line
//     gives rows, cols, nnz (on a blank line the next three numbers are read);
//   * then nnz entries "row col value" ("row col" for pattern, value 1) as
//     scanf("%d %d %lf") reads them: whitespace-separated tokens, 1-based
//     indices, each value converted to double correctly rounded (decimal.cuh)
//     and then cast to the value type; tokens after the nnz-th entry are
//     ignored;
//   * a file with zero rows gives an empty matrix (0 x 0).
// The CSR form without the duplicate summation (compact = 0) is built straight
// from the placed entries: row counts, a scan for the row offsets, and a
// stable sort by row (skipped when the entries already come row by row), so
// entries keep their file order within a row as the reference's counting sort
// does (include/sparse_conversion.h:37-99).  With the summation it is the
// device coo_to_csr (coo_csr.cu).
//
// From a path, the banner and size line are read from a prefix and the
// entries part goes to the device in 4 MiB chunks: reader threads pread into
// pinned buffers kept by the context, and each upload overlaps the next
// chunk's read.  From bytes in host memory it is one copy.
// Device steps: one select over
// byte positions finds the token starts (a non-space after a space); one
// thread per entry parses its row, column and value; tokens that the fast
// conversions leave open (values within 2^-93 of a rounding midpoint, rare)
// are listed and finished by big_round in a second pass; a scan places the
// symmetric copies.
#include <cub/cub.cuh>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstdio>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "decimal.cuh"
#include "spops_internal.h"

namespace spops {
namespace {

inline unsigned grid_for(int64_t work, int threads = 256) {
  int64_t g = (work + threads - 1) / threads;
  return (unsigned)(g < 1 ? 1 : g);
}

__host__ __device__ __forceinline__ bool is_space(char c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f';
}

struct TokenStart {
  const char* t;
  __device__ bool operator()(int64_t i) const { return !is_space(t[i]) && (i == 0 || is_space(t[i - 1])); }
};

__device__ __forceinline__ const char* token_end(const char* p, const char* end) {
  while (p < end && !is_space(*p)) ++p;
  return p;
}

// errors: bit 0 syntax, bit 1 index out of range; first[] = first bad entry
struct ParseOut {
  int64_t* r;
  int64_t* c;
  double* v;
  unsigned long long* open_count;  // entries left to the exact pass
  int64_t* open_list;
  double* open_cand;
  int* err;
  unsigned long long* first_bad;
};

__global__ void parse_entries_kernel(const char* __restrict__ text, int64_t len, const int64_t* __restrict__ starts,
                                     int64_t nnz, int per, int64_t rows, int64_t cols,
                                     const dec::Pow10* __restrict__ tab, ParseOut o) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= nnz) return;
  const char* end = text + len;
  const char* t0 = text + starts[e * per];
  const char* t1 = text + starts[e * per + 1];
  int64_t r = 0, c = 0;
  bool ok = dec::parse_int64(t0, token_end(t0, end), &r) && dec::parse_int64(t1, token_end(t1, end), &c);
  int bad = ok ? 0 : 1;
  if (ok && (r < 1 || r > rows || c < 1 || c > cols)) bad = 2;
  double v = 1.0;
  if (!bad && per == 3) {
    const char* t2 = text + starts[e * per + 2];
    dec::Decimal d;
    if (!dec::scan_decimal(t2, token_end(t2, end), &d)) {
      bad = 1;
    } else {
      double cand = 0;
      if (!dec::fast_value(d, tab, &v, &cand)) {
        const unsigned long long k = atomicAdd(o.open_count, 1ULL);
        o.open_list[k] = e;
        o.open_cand[k] = cand;
      }
    }
  }
  if (bad) {
    atomicOr(o.err, bad);
    atomicMin(o.first_bad, (unsigned long long)e);
    return;
  }
  o.r[e] = r - 1;
  o.c[e] = c - 1;
  o.v[e] = v;
}

// the exact pass: one thread per open value (large local integers)
__global__ void __launch_bounds__(32) exact_values_kernel(const char* __restrict__ text, int64_t len,
                                                          const int64_t* __restrict__ starts, int per,
                                                          const int64_t* __restrict__ list,
                                                          const double* __restrict__ cand, int64_t m,
                                                          double* __restrict__ v, int* err,
                                                          unsigned long long* first_bad) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= m) return;
  const int64_t e = list[k];
  const char* t2 = text + starts[e * per + 2];
  dec::Big L, R;
  double out = 0;
  if (!dec::big_round(t2, token_end(t2, text + len), cand[k], &out, L, R)) {
    atomicOr(err, 1);
    atomicMin(first_bad, (unsigned long long)e);
    return;
  }
  v[e] = out;
}

__global__ void copies_kernel(const int64_t* __restrict__ r, const int64_t* __restrict__ c, int64_t nnz, bool symm,
                              int64_t* __restrict__ cnt) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e < nnz) cnt[e] = (symm && r[e] != c[e]) ? 2 : 1;
}

// CSR straight from the placed entries (read_csr_matrix without a COO
// handle): per-row counts, and whether the entries already come row by row.
template <typename I>
__global__ void csr_count_kernel(const I* __restrict__ ro, int64_t total, unsigned long long* __restrict__ cnt,
                                 int* __restrict__ unsorted) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= total) return;
  atomicAdd(cnt + (int64_t)ro[k], 1ULL);
  if (k > 0 && ro[k] < ro[k - 1]) *unsorted = 1;
}

template <typename I>
__global__ void csr_rowptr_kernel(const unsigned long long* __restrict__ scan, int64_t n1, I* __restrict__ rp) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r < n1) rp[r] = (I)scan[r];
}

__global__ void csr_iota_kernel(int64_t* __restrict__ a, int64_t m) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < m) a[i] = i;
}

template <typename I, typename V>
__global__ void csr_gather_kernel(const int64_t* __restrict__ perm, const I* __restrict__ ci, const V* __restrict__ v,
                                  int64_t m, I* __restrict__ co, V* __restrict__ vo) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= m) return;
  co[i] = ci[perm[i]];
  vo[i] = v[perm[i]];
}

template <typename I, typename V>
__global__ void place_kernel(const int64_t* __restrict__ r, const int64_t* __restrict__ c,
                             const double* __restrict__ v, const int64_t* __restrict__ pos, int64_t nnz, bool symm,
                             I* __restrict__ ro, I* __restrict__ co, V* __restrict__ vo) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= nnz) return;
  const int64_t p = pos[e];
  const V val = (V)v[e];  // read as double, then cast, as the reference does
  ro[p] = (I)r[e];
  co[p] = (I)c[e];
  vo[p] = val;
  if (symm && r[e] != c[e]) {
    ro[p + 1] = (I)c[e];
    co[p + 1] = (I)r[e];
    vo[p + 1] = val;
  }
}

const std::vector<dec::Pow10>& pow10_table() {
  static std::vector<dec::Pow10> t;
  static std::once_flag once;
  std::call_once(once, [] { t = dec::make_pow10_table(); });
  return t;
}

std::string lower_str(std::string s) {
  for (auto& ch : s) ch = (char)((ch >= 'A' && ch <= 'Z') ? ch + 32 : ch);
  return s;
}

struct Header {
  bool pattern = false, symmetric = false;
  int64_t rows = 0, cols = 0, nnz = 0;
  size_t data = 0;  // offset of the entries
};

// banner and size line (mm_read_banner, mm_read_mtx_crd_size)
spops_status_t read_header(const char* s, size_t n, Header* h) {
  size_t eol = 0;
  while (eol < n && s[eol] != '\n') ++eol;
  std::vector<std::string> tok;
  {
    size_t i = 0;
    while (i < eol && tok.size() < 5) {
      while (i < eol && is_space(s[i])) ++i;
      size_t j = i;
      while (j < eol && !is_space(s[j])) ++j;
      if (j > i) tok.emplace_back(s + i, j - i);
      i = j;
    }
  }
  if (tok.size() != 5) return fail(SPOPS_ERR_INVALID, "Matrix Market: the banner line has fewer than 5 words");
  if (tok[0].compare(0, 14, "%%MatrixMarket") != 0) return fail(SPOPS_ERR_INVALID, "Matrix Market: no %%%%MatrixMarket banner");
  const std::string mtx = lower_str(tok[1]), crd = lower_str(tok[2]), field = lower_str(tok[3]),
                    symm = lower_str(tok[4]);
  if (mtx != "matrix") return fail(SPOPS_ERR_UNSUPPORTED, "Matrix Market: object '%s' is not 'matrix'", mtx.c_str());
  if (crd != "coordinate" && crd != "array")
    return fail(SPOPS_ERR_UNSUPPORTED, "Matrix Market: format '%s'", crd.c_str());
  if (field != "real" && field != "complex" && field != "pattern" && field != "integer")
    return fail(SPOPS_ERR_UNSUPPORTED, "Matrix Market: field '%s'", field.c_str());
  if (symm != "general" && symm != "symmetric" && symm != "hermitian" && symm != "skew-symmetric")
    return fail(SPOPS_ERR_UNSUPPORTED, "Matrix Market: symmetry '%s'", symm.c_str());
  // mm_is_valid
  if ((crd == "array" && field == "pattern") || (field == "real" && symm == "hermitian") ||
      (field == "pattern" && (symm == "hermitian" || symm == "skew-symmetric")))
    return fail(SPOPS_ERR_INVALID, "Matrix Market: invalid type '%s %s %s'", crd.c_str(), field.c_str(), symm.c_str());
  if (crd != "coordinate" || field == "complex")
    return fail(SPOPS_ERR_UNSUPPORTED, "Matrix Market: only sparse real, integer or pattern coordinate matrices");
  h->pattern = field == "pattern";
  h->symmetric = symm == "symmetric";
  // comment lines, then the size line
  size_t p = eol < n ? eol + 1 : n;
  while (p < n && s[p] == '%') {
    while (p < n && s[p] != '\n') ++p;
    if (p < n) ++p;
  }
  size_t le = p;
  while (le < n && s[le] != '\n') ++le;
  auto read_ints = [&](size_t from, size_t to, int64_t* out, int want, size_t* stop) {
    int got = 0;
    size_t i = from;
    while (got < want) {
      while (i < to && is_space(s[i])) ++i;
      if (i >= to) break;
      size_t j = i;
      while (j < to && !is_space(s[j])) ++j;
      int64_t v = 0;
      if (!dec::parse_int64(s + i, s + j, &v)) break;
      out[got++] = v;
      i = j;
    }
    *stop = i;
    return got;
  };
  int64_t dims[3] = {0, 0, 0};
  size_t stop = 0;
  if (read_ints(p, le, dims, 3, &stop) == 3) {
    h->data = le < n ? le + 1 : n;  // the rest of the size line is not read
  } else {
    if (read_ints(le < n ? le + 1 : n, n, dims, 3, &stop) != 3)
      return fail(SPOPS_ERR_INVALID, "Matrix Market: no 'rows cols nnz' line");
    h->data = stop;
  }
  if (dims[0] < 0 || dims[1] < 0 || dims[2] < 0) return fail(SPOPS_ERR_INVALID, "Matrix Market: negative size");
  h->rows = dims[0];
  h->cols = dims[1];
  h->nnz = dims[2];
  return SPOPS_OK;
}

// The entries part of the file (len bytes) is in dtext on the device,
// written by work already queued on ctx->stream.
template <typename I, typename V>
spops_status_t read_t(Context* ctx, PoolBuf& dtext, int64_t len, const Header& H, Matrix** out, bool direct_csr) {
  cudaStream_t st = ctx->stream;
  const int per = H.pattern ? 2 : 3;
  const int64_t nnz = H.nnz;
  Trace tr("mtx");
  PoolBuf starts(ctx), nsel(ctx), tmp(ctx), tab(ctx), r(ctx), c(ctx), v(ctx), cnt(ctx), pos(ctx), misc(ctx),
      olist(ctx), ocand(ctx);
  // token starts
  int64_t ntok = 0;
  SPOPS_TRY(nsel.alloc(8));
  SPOPS_TRY(starts.alloc((size_t)std::max<int64_t>(nnz * per, 1) * 8));
  if (len > 0 && nnz > 0) {
    // every token start (at most (len + 1) / 2 of them); the first nnz * per are the entries
    PoolBuf all(ctx);
    SPOPS_TRY(all.alloc((size_t)((len + 1) / 2 + 1) * 8));
    cub::CountingInputIterator<int64_t> it(0);
    size_t tb = 0;
    SPOPS_CUDA(cub::DeviceSelect::If(nullptr, tb, it, all.as<int64_t>(), nsel.as<int64_t>(), len,
                                     TokenStart{dtext.as<char>()}, st));
    SPOPS_TRY(tmp.alloc(tb + 256));
    SPOPS_CUDA(cub::DeviceSelect::If(tmp.p, tb, it, all.as<int64_t>(), nsel.as<int64_t>(), len,
                                     TokenStart{dtext.as<char>()}, st));
    SPOPS_CUDA(cudaMemcpyAsync(&ntok, nsel.p, 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
    if (ntok < nnz * per)
      return fail(SPOPS_ERR_INVALID, "Matrix Market: %lld entries announced, %lld numbers found", (long long)nnz,
                  (long long)ntok);
    SPOPS_CUDA(cudaMemcpyAsync(starts.p, all.p, (size_t)(nnz * per) * 8, cudaMemcpyDeviceToDevice, st));
    tr.mark(st, "token select");
  } else if (nnz > 0) {
    return fail(SPOPS_ERR_INVALID, "Matrix Market: %lld entries announced, none found", (long long)nnz);
  }
  // parse
  const auto& T = pow10_table();
  SPOPS_TRY(tab.alloc(T.size() * sizeof(dec::Pow10)));
  SPOPS_CUDA(cudaMemcpyAsync(tab.p, T.data(), T.size() * sizeof(dec::Pow10), cudaMemcpyHostToDevice, st));
  const size_t nz1 = (size_t)std::max<int64_t>(nnz, 1);
  SPOPS_TRY(r.alloc(nz1 * 8));
  SPOPS_TRY(c.alloc(nz1 * 8));
  SPOPS_TRY(v.alloc(nz1 * 8));
  SPOPS_TRY(olist.alloc(nz1 * 8));
  SPOPS_TRY(ocand.alloc(nz1 * 8));
  SPOPS_TRY(misc.alloc(64));
  SPOPS_CUDA(cudaMemsetAsync(misc.p, 0, 64, st));
  unsigned long long* open_count = misc.as<unsigned long long>();
  int* err = reinterpret_cast<int*>(misc.as<char>() + 8);
  unsigned long long* first_bad = misc.as<unsigned long long>() + 2;
  SPOPS_CUDA(cudaMemsetAsync(first_bad, 0xff, 8, st));
  ParseOut o{r.as<int64_t>(), c.as<int64_t>(), v.as<double>(), open_count, olist.as<int64_t>(),
             ocand.as<double>(), err, first_bad};
  if (nnz > 0) {
    parse_entries_kernel<<<grid_for(nnz), 256, 0, st>>>(dtext.as<char>(), len, starts.as<int64_t>(), nnz, per, H.rows,
                                                        H.cols, tab.as<dec::Pow10>(), o);
    SPOPS_LAUNCH_CHECK();
  }
  unsigned long long hm[3] = {0, 0, 0};
  SPOPS_CUDA(cudaMemcpyAsync(hm, misc.p, 24, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  tr.mark(st, "parse entries");
  const int64_t nopen = (int64_t)hm[0];
  if (nopen > 0) {
    exact_values_kernel<<<grid_for(nopen, 32), 32, 0, st>>>(dtext.as<char>(), len, starts.as<int64_t>(), per,
                                                             olist.as<int64_t>(), ocand.as<double>(), nopen,
                                                             v.as<double>(), err, first_bad);
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cudaMemcpyAsync(hm, misc.p, 24, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
  }
  const int e = (int)(hm[1] & 0xffffffffULL);
  if (e) {
    const long long bad = (long long)hm[2];
    if (e & 1) return fail(SPOPS_ERR_INVALID, "Matrix Market: entry %lld is not 'row col%s'", bad + 1,
                           H.pattern ? "" : " value");
    return fail(SPOPS_ERR_INVALID, "Matrix Market: entry %lld has an index outside %lld x %lld", bad + 1,
                (long long)H.rows, (long long)H.cols);
  }
  // symmetric copies and the typed COO arrays
  SPOPS_TRY(cnt.alloc((size_t)(nnz + 1) * 8));
  SPOPS_TRY(pos.alloc((size_t)(nnz + 1) * 8));
  SPOPS_CUDA(cudaMemsetAsync(cnt.p, 0, (size_t)(nnz + 1) * 8, st));
  if (nnz > 0) {
    copies_kernel<<<grid_for(nnz), 256, 0, st>>>(r.as<int64_t>(), c.as<int64_t>(), nnz, H.symmetric,
                                                 cnt.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
  }
  size_t sb = 0;
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, sb, cnt.as<int64_t>(), pos.as<int64_t>(), nnz + 1, st));
  SPOPS_TRY(tmp.alloc(sb + 256));
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, sb, cnt.as<int64_t>(), pos.as<int64_t>(), nnz + 1, st));
  int64_t total = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&total, pos.as<int64_t>() + nnz, 8, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  if (direct_csr && H.rows > 0) {  // CSR in file order within rows, no COO handle
    PoolBuf prow(ctx), tc(ctx), tv(ctx), cnt2(ctx), scan(ctx), perm_in(ctx), perm(ctx), skey(ctx), tmp2(ctx);
    const size_t t1 = (size_t)std::max<int64_t>(total, 1), n1 = (size_t)H.rows + 1;
    SPOPS_TRY(prow.alloc(t1 * sizeof(I)));
    SPOPS_TRY(tc.alloc(t1 * sizeof(I)));
    SPOPS_TRY(tv.alloc(t1 * sizeof(V)));
    SPOPS_TRY(cnt2.alloc((n1 + 1) * 8));
    SPOPS_TRY(scan.alloc((n1 + 1) * 8));
    SPOPS_CUDA(cudaMemsetAsync(cnt2.p, 0, (n1 + 1) * 8, st));
    int* unsorted = reinterpret_cast<int*>(cnt2.as<unsigned long long>() + n1);
    if (nnz > 0) {
      place_kernel<I, V><<<grid_for(nnz), 256, 0, st>>>(r.as<int64_t>(), c.as<int64_t>(), v.as<double>(),
                                                        pos.as<int64_t>(), nnz, H.symmetric, prow.as<I>(), tc.as<I>(),
                                                        tv.as<V>());
      csr_count_kernel<I><<<grid_for(total), 256, 0, st>>>(prow.as<I>(), total, cnt2.as<unsigned long long>(),
                                                           unsorted);
      SPOPS_LAUNCH_CHECK();
    }
    size_t sb2 = 0;
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, sb2, cnt2.as<unsigned long long>(),
                                             scan.as<unsigned long long>(), (int64_t)n1, st));
    int rbits = 1;  // row keys are below rows
    while (rbits < 62 && (int64_t(1) << rbits) < H.rows) ++rbits;
    size_t ss2 = 0;
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, ss2, prow.as<I>(), prow.as<I>(), perm_in.as<int64_t>(),
                                               perm.as<int64_t>(), (int64_t)t1, 0, rbits, st));
    SPOPS_TRY(tmp2.alloc(std::max(sb2, ss2) + 256));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp2.p, sb2, cnt2.as<unsigned long long>(),
                                             scan.as<unsigned long long>(), (int64_t)n1, st));
    int hu = 0;
    SPOPS_CUDA(cudaMemcpyAsync(&hu, unsorted, 4, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
    tr.mark(st, "place + row counts");
    Matrix* C = new spops_matrix_s();
    C->ctx = ctx;
    C->format = SPOPS_FMT_CSR;
    C->itype = sizeof(I) == 4 ? SPOPS_INDEX_I32 : SPOPS_INDEX_I64;
    C->vtype = sizeof(V) == 8 ? SPOPS_VALUE_F64 : SPOPS_VALUE_F32;
    C->rows = H.rows;
    C->cols = H.cols;
    C->nnz = total;
    // the result's arrays reuse blocks earlier results of this context released
    spops_status_t s2 = C->row.alloc_cached(ctx, n1 * sizeof(I));
    if (s2 == SPOPS_OK) s2 = C->col.alloc_cached(ctx, t1 * sizeof(I));
    if (s2 == SPOPS_OK) s2 = C->val.alloc_cached(ctx, t1 * sizeof(V));
    if (s2 == SPOPS_OK) {
      csr_rowptr_kernel<I><<<grid_for((int64_t)n1), 256, 0, st>>>(scan.as<unsigned long long>(), (int64_t)n1,
                                                                 C->row.as<I>());
      if (total > 0 && !hu) {  // already row by row: the placed order is the CSR order
        SPOPS_CUDA(cudaMemcpyAsync(C->col.p, tc.p, (size_t)total * sizeof(I), cudaMemcpyDeviceToDevice, st));
        SPOPS_CUDA(cudaMemcpyAsync(C->val.p, tv.p, (size_t)total * sizeof(V), cudaMemcpyDeviceToDevice, st));
      } else if (total > 0) {  // stable sort by row keeps file order within a row
        if (perm_in.alloc(t1 * 8) != SPOPS_OK || perm.alloc(t1 * 8) != SPOPS_OK || skey.alloc(t1 * sizeof(I)) != SPOPS_OK)
          s2 = fail(SPOPS_ERR_ALLOC, "Matrix Market: sort buffers");
        if (s2 == SPOPS_OK) {
          csr_iota_kernel<<<grid_for(total), 256, 0, st>>>(perm_in.as<int64_t>(), total);
          SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(tmp2.p, ss2, prow.as<I>(), skey.as<I>(), perm_in.as<int64_t>(),
                                                     perm.as<int64_t>(), total, 0, rbits, st));
          csr_gather_kernel<I, V><<<grid_for(total), 256, 0, st>>>(perm.as<int64_t>(), tc.as<I>(), tv.as<V>(), total,
                                                                   C->col.as<I>(), C->val.as<V>());
        }
      }
      if (s2 == SPOPS_OK && cudaGetLastError() != cudaSuccess) s2 = fail(SPOPS_ERR_CUDA, "Matrix Market: CSR build");
      if (s2 == SPOPS_OK && cudaStreamSynchronize(st) != cudaSuccess) s2 = fail(SPOPS_ERR_CUDA, "Matrix Market: stream");
    }
    if (s2 != SPOPS_OK) {
      C->release_all();
      delete static_cast<spops_matrix_s*>(C);
      return s2;
    }
    tr.mark(st, "CSR arrays");
    *out = C;
    return SPOPS_OK;
  }
  Matrix* A = new spops_matrix_s();
  A->ctx = ctx;
  A->format = SPOPS_FMT_COO;
  A->itype = sizeof(I) == 4 ? SPOPS_INDEX_I32 : SPOPS_INDEX_I64;
  A->vtype = sizeof(V) == 8 ? SPOPS_VALUE_F64 : SPOPS_VALUE_F32;
  A->rows = H.rows;
  A->cols = H.cols;
  A->nnz = total;
  spops_status_t s = A->row.alloc((size_t)std::max<int64_t>(total, 1) * sizeof(I));
  if (s == SPOPS_OK) s = A->col.alloc((size_t)std::max<int64_t>(total, 1) * sizeof(I));
  if (s == SPOPS_OK) s = A->val.alloc((size_t)std::max<int64_t>(total, 1) * sizeof(V));
  if (s == SPOPS_OK && nnz > 0) {
    place_kernel<I, V><<<grid_for(nnz), 256, 0, st>>>(r.as<int64_t>(), c.as<int64_t>(), v.as<double>(),
                                                      pos.as<int64_t>(), nnz, H.symmetric, A->row.as<I>(),
                                                      A->col.as<I>(), A->val.as<V>());
    if (cudaGetLastError() != cudaSuccess) s = fail(SPOPS_ERR_CUDA, "Matrix Market: place launch failed");
  }
  tr.mark(st, "copies + COO arrays");
  if (s == SPOPS_OK) s = coo_analyse(ctx, A);
  if (s == SPOPS_OK && cudaStreamSynchronize(st) != cudaSuccess) s = fail(SPOPS_ERR_CUDA, "Matrix Market: stream error");
  tr.mark(st, "COO analysis");
  if (s != SPOPS_OK) {
    A->release_all();
    delete static_cast<spops_matrix_s*>(A);
    return s;
  }
  *out = A;
  return SPOPS_OK;
}

spops_status_t check_header(const Header& H, spops_index_t itype) {
  if (itype == SPOPS_INDEX_I32 && (H.rows > INT32_MAX || H.cols > INT32_MAX))
    return fail(SPOPS_ERR_TOO_LARGE, "Matrix Market: %lld x %lld does not fit int32 indices", (long long)H.rows,
                (long long)H.cols);
  return SPOPS_OK;
}

spops_status_t read_typed(Context* ctx, PoolBuf& dtext, int64_t len, const Header& H, spops_index_t itype,
                          spops_value_t vtype, Matrix** out, bool direct_csr) {
  const bool i32 = itype == SPOPS_INDEX_I32, f64 = vtype == SPOPS_VALUE_F64;
  if (i32 && f64) return read_t<int32_t, double>(ctx, dtext, len, H, out, direct_csr);
  if (i32) return read_t<int32_t, float>(ctx, dtext, len, H, out, direct_csr);
  if (f64) return read_t<int64_t, double>(ctx, dtext, len, H, out, direct_csr);
  return read_t<int64_t, float>(ctx, dtext, len, H, out, direct_csr);
}

// the file's bytes in host memory
spops_status_t parse_coo(Context* ctx, const char* text, size_t n, spops_index_t itype, spops_value_t vtype,
                         Matrix** out, bool direct_csr = false) {
  Header H;
  SPOPS_TRY(read_header(text, n, &H));
  SPOPS_TRY(check_header(H, itype));
  const int64_t len = (int64_t)(n - H.data);
  Trace tr("mtx");
  ArenaScope scope(ctx);  // this call's temporaries come from the arena
  PoolBuf dtext(ctx);
  SPOPS_TRY(dtext.alloc((size_t)std::max<int64_t>(len, 1)));
  if (len > 0) SPOPS_CUDA(cudaMemcpyAsync(dtext.p, text + H.data, (size_t)len, cudaMemcpyHostToDevice, ctx->stream));
  tr.mark(ctx->stream, "upload from host memory");
  return read_typed(ctx, dtext, len, H, itype, vtype, out, direct_csr);
}

// File chunks go to the device through pinned buffers: kReaders threads each
// pread their chunks (every kReaders-th one) into their two buffers in turn
// and queue the upload; a buffer is refilled once its previous upload ended.
constexpr size_t kChunk = size_t(4) << 20;
constexpr int kReaders = 4;

spops_status_t ensure_file_stage(Context* ctx) {
  if (!ctx->file_stage.empty()) return SPOPS_OK;
  for (int i = 0; i < 2 * kReaders; ++i) {
    void* b = nullptr;
    cudaEvent_t e = nullptr;
    if (cudaHostAlloc(&b, kChunk, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      break;
    }
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      cudaFreeHost(b);
      break;
    }
    ctx->file_stage.push_back(b);
    ctx->file_events.push_back(e);
  }
  if ((int)ctx->file_stage.size() == 2 * kReaders) return SPOPS_OK;
  for (cudaEvent_t e : ctx->file_events) cudaEventDestroy(e);
  for (void* b : ctx->file_stage) cudaFreeHost(b);
  ctx->file_events.clear();
  ctx->file_stage.clear();
  return fail(SPOPS_ERR_ALLOC, "Matrix Market: pinned staging buffers could not be allocated");
}

bool pread_all(int fd, char* dst, size_t n, int64_t off) {
  size_t got = 0;
  while (got < n) {
    const ssize_t r = ::pread(fd, dst + got, n - got, (off_t)(off + (int64_t)got));
    if (r < 0 && errno == EINTR) continue;
    if (r <= 0) return false;
    got += (size_t)r;
  }
  return true;
}

struct FileCloser {
  int fd;
  ~FileCloser() {
    if (fd >= 0) ::close(fd);
  }
};

spops_status_t read_path(Context* ctx, const char* path, spops_index_t itype, spops_value_t vtype, Matrix** out,
                         bool direct_csr = false) {
  Trace tr("mtx");
  const int fd = ::open(path, O_RDONLY | O_CLOEXEC);
  if (fd < 0) return fail(SPOPS_ERR_INVALID, "Matrix Market: unable to open file: %s", path);
  FileCloser closer{fd};
  struct stat sb;
  if (::fstat(fd, &sb) != 0 || sb.st_size < 0) return fail(SPOPS_ERR_INVALID, "Matrix Market: read error: %s", path);
  const int64_t size = (int64_t)sb.st_size;
  // the banner and size line from a prefix, grown until they end inside it
  Header H;
  std::string pre;
  for (int64_t want = 65536;; want *= 4) {
    const int64_t m = std::min(size, want);
    pre.resize((size_t)m);
    if (m > 0 && !pread_all(fd, &pre[0], (size_t)m, 0))
      return fail(SPOPS_ERR_INVALID, "Matrix Market: read error: %s", path);
    Header h;
    const spops_status_t s = read_header(pre.data(), (size_t)m, &h);
    if (m == size) {
      SPOPS_TRY(s);
      H = h;
      break;
    }
    if (s == SPOPS_OK && (int64_t)h.data < m) {
      H = h;
      break;
    }
  }
  SPOPS_TRY(check_header(H, itype));
  const int64_t len = size - (int64_t)H.data;
  ArenaScope scope(ctx);  // this call's temporaries come from the arena
  PoolBuf dtext(ctx);
  SPOPS_TRY(dtext.alloc((size_t)std::max<int64_t>(len, 1)));
  tr.mark(ctx->stream, "open + header + text buffer");
  if (len > 0) {
    SPOPS_TRY(ensure_file_stage(ctx));
    tr.mark(ctx->stream, "pinned staging");
    const int64_t nchunks = (len + (int64_t)kChunk - 1) / (int64_t)kChunk;
    const int nt = (int)std::min<int64_t>(kReaders, nchunks);
    std::atomic<int> bad{0};  // 1: read error, 2: CUDA error
    char* dst = dtext.as<char>();
    auto reader = [&](int w) {
      if (nt > 1 && cudaSetDevice(ctx->device) != cudaSuccess) {
        bad = 2;
        return;
      }
      int turn = 0;
      for (int64_t k = w; k < nchunks && !bad; k += nt, ++turn) {
        const int b = 2 * w + (turn & 1);
        char* buf = static_cast<char*>(ctx->file_stage[b]);
        const int64_t off = k * (int64_t)kChunk;
        const size_t n = (size_t)std::min<int64_t>((int64_t)kChunk, len - off);
        if (cudaEventSynchronize(ctx->file_events[b]) != cudaSuccess) {
          bad = 2;
          return;
        }
        if (!pread_all(fd, buf, n, (int64_t)H.data + off)) {
          bad = 1;
          return;
        }
        if (cudaMemcpyAsync(dst + off, buf, n, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
            cudaEventRecord(ctx->file_events[b], ctx->stream) != cudaSuccess) {
          bad = 2;
          return;
        }
      }
    };
    if (nt == 1) {
      reader(0);
    } else {
      std::vector<std::thread> th;
      for (int w = 0; w < nt; ++w) th.emplace_back(reader, w);
      for (auto& t : th) t.join();
    }
    tr.mark(ctx->stream, "file read + upload");
    if (bad == 1) return fail(SPOPS_ERR_INVALID, "Matrix Market: read error: %s", path);
    if (bad == 2) {
      cudaStreamSynchronize(ctx->stream);
      return fail(SPOPS_ERR_CUDA, "Matrix Market: upload failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
  }
  return read_typed(ctx, dtext, len, H, itype, vtype, out, direct_csr);
}

spops_status_t check_types(spops_index_t itype, spops_value_t vtype) {
  if ((itype != SPOPS_INDEX_I32 && itype != SPOPS_INDEX_I64) || (vtype != SPOPS_VALUE_F32 && vtype != SPOPS_VALUE_F64))
    return fail(SPOPS_ERR_INVALID, "Matrix Market: bad index or value type");
  return SPOPS_OK;
}

spops_status_t coo_to_csr_out(Context* ctx, Matrix* coo, int32_t compact, spops_matrix_t* csr) {
  if (coo->format == SPOPS_FMT_CSR) {  // built directly (compact = 0)
    *csr = static_cast<spops_matrix_s*>(coo);
    return SPOPS_OK;
  }
  spops_status_t s;
  if (coo->rows == 0) {  // read_csr_matrix: a matrix with no rows is 0 x 0
    Matrix* C = new spops_matrix_s();
    C->ctx = ctx;
    C->format = SPOPS_FMT_CSR;
    C->itype = coo->itype;
    C->vtype = coo->vtype;
    s = C->row.alloc(16);
    if (s == SPOPS_OK) s = C->col.alloc(16);
    if (s == SPOPS_OK) s = C->val.alloc(16);
    if (s == SPOPS_OK) SPOPS_CUDA(cudaMemsetAsync(C->row.p, 0, 16, ctx->stream));
    if (s == SPOPS_OK) s = csr_analyse(ctx, C);
    if (s != SPOPS_OK) {
      C->release_all();
      delete static_cast<spops_matrix_s*>(C);
    } else {
      *csr = static_cast<spops_matrix_s*>(C);
    }
  } else {
    Trace tr("mtx");
    s = spops_coo_to_csr(static_cast<spops_context_s*>(ctx), static_cast<spops_matrix_s*>(coo), compact, csr);
    tr.mark(ctx->stream, "coo_to_csr");
  }
  Trace tr("mtx");
  coo->release_all();
  delete static_cast<spops_matrix_s*>(coo);
  tr.mark(ctx->stream, "release COO");
  return s;
}

}  // namespace
}  // namespace spops

using namespace spops;

extern "C" {

spops_status_t spops_mtx_parse_coo(spops_context_t ctx, const char* text, int64_t len, spops_index_t itype,
                                   spops_value_t vtype, spops_matrix_t* coo) {
  if (!ctx || !text || !coo || len < 0) return fail(SPOPS_ERR_INVALID, "spops_mtx_parse_coo: null argument");
  SPOPS_TRY(check_types(itype, vtype));
  DeviceGuard g(ctx->device);
  Matrix* A = nullptr;
  SPOPS_TRY(parse_coo(ctx, text, (size_t)len, itype, vtype, &A));
  *coo = static_cast<spops_matrix_s*>(A);
  return SPOPS_OK;
}

spops_status_t spops_mtx_read_coo(spops_context_t ctx, const char* path, spops_index_t itype, spops_value_t vtype,
                                  spops_matrix_t* coo) {
  if (!ctx || !path || !coo) return fail(SPOPS_ERR_INVALID, "spops_mtx_read_coo: null argument");
  SPOPS_TRY(check_types(itype, vtype));
  DeviceGuard g(ctx->device);
  Matrix* A = nullptr;
  SPOPS_TRY(read_path(ctx, path, itype, vtype, &A));
  *coo = static_cast<spops_matrix_s*>(A);
  return SPOPS_OK;
}

spops_status_t spops_mtx_parse_csr(spops_context_t ctx, const char* text, int64_t len, spops_index_t itype,
                                   spops_value_t vtype, int32_t compact, spops_matrix_t* csr) {
  if (!ctx || !text || !csr || len < 0) return fail(SPOPS_ERR_INVALID, "spops_mtx_parse_csr: null argument");
  SPOPS_TRY(check_types(itype, vtype));
  DeviceGuard g(ctx->device);
  Matrix* A = nullptr;
  SPOPS_TRY(parse_coo(ctx, text, (size_t)len, itype, vtype, &A, compact == 0));
  return coo_to_csr_out(ctx, A, compact, csr);
}

spops_status_t spops_mtx_read_csr(spops_context_t ctx, const char* path, spops_index_t itype, spops_value_t vtype,
                                  int32_t compact, spops_matrix_t* csr) {
  if (!ctx || !path || !csr) return fail(SPOPS_ERR_INVALID, "spops_mtx_read_csr: null argument");
  SPOPS_TRY(check_types(itype, vtype));
  DeviceGuard g(ctx->device);
  Matrix* A = nullptr;
  SPOPS_TRY(read_path(ctx, path, itype, vtype, &A, compact == 0));
  return coo_to_csr_out(ctx, A, compact, csr);
}

}  // extern "C"
