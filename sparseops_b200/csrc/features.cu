// Structure features of a CSR matrix on the device, and the format selector.
//
// Features: the non-tile part of the reference's MTX::CalculateFeatures
// (src/sparse_features.cpp:643-775) over the per-entry statistics its
// MtxLoad gathers for a general real matrix (:336-478), computed from a CSR
// handle instead of a Matrix Market file:
//   one thread per row walks the row in storage order (as the file is read):
//     row count, lower / upper / diagonal counts, the diagonal-dominance sum
//     (+|a_ii|, -|a_ij|, in entry order), the largest |a| on and off the
//     diagonal, the row's log10 range with the reference's clamping (max
//     starts at 0, min starts at 0 and only falls), and per entry the column
//     count, column log10 range and diagonal-offset flag;
//   counts -> min / max / mean / variance (deterministic cub reductions);
//   P-ratio and Gini from the sorted counts (the P search is exact: the same
//   double expressions as the reference, evaluated for every prefix);
//   symmetry by a bisection per mirror: with ascending rows, column by
//   column over a transpose pattern the handle already holds (a warp bisects
//   row c of A for every entry of column c), else row by row on the CSR's
//   own arrays; rows in any other order through sorted (row, col) keys.
// The selector (spops_select_format) applies rules to the features or times
// the candidate formats.
#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "spops_internal.h"

namespace spops {
namespace {

inline unsigned grid_of(int64_t work, int threads = 256) {
  int64_t g = (work + threads - 1) / threads;
  return (unsigned)(g < 1 ? 1 : g);
}

struct Totals {
  unsigned long long lower, upper, diagonal, dominant, close, has_diag, has_off;
  unsigned long long max_diag_bits, max_off_bits;  // |a| >= 0: bit order = value order
  unsigned long long row_var_bits, col_var_bits;   // ranges >= 0; has_* flags below
  unsigned long long has_row_var, has_col_var;
};

__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* a, double v) {
  atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

// sums and maxima of one block's rows, then one global atomic per block
// and field (the totals are few addresses that every row would hit)
__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ unsigned long long warp_max(unsigned long long v) {
  for (int o = 16; o; o >>= 1) {
    const unsigned long long u = __shfl_xor_sync(0xffffffffu, v, o);
    v = u > v ? u : v;
  }
  return v;
}
enum { kLower, kUpper, kDiagonal, kDominant, kClose, kHasDiag, kHasOff, kMaxDiag, kMaxOff, kRowVar, kHasRowVar,
       kColVar, kHasColVar, kFields };
__device__ __forceinline__ unsigned long long* total_field(Totals* t, int f) {
  switch (f) {
    case kLower: return &t->lower;
    case kUpper: return &t->upper;
    case kDiagonal: return &t->diagonal;
    case kDominant: return &t->dominant;
    case kClose: return &t->close;
    case kHasDiag: return &t->has_diag;
    case kHasOff: return &t->has_off;
    case kMaxDiag: return &t->max_diag_bits;
    case kMaxOff: return &t->max_off_bits;
    case kRowVar: return &t->row_var_bits;
    case kHasRowVar: return &t->has_row_var;
    case kColVar: return &t->col_var_bits;
    default: return &t->has_col_var;
  }
}
// fields kMaxDiag .. kColVar combine by max (non-negative doubles as bits),
// the flags by max too, the counts by sum
__device__ __forceinline__ bool is_max_field(int f) { return f >= kHasDiag; }

// per-thread values into the block's shared totals, then to the device
__device__ void flush_totals(const unsigned long long (&v)[kFields], unsigned long long* sh, Totals* tot) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int f = 0; f < kFields; ++f) {
    const unsigned long long w = is_max_field(f) ? warp_max(v[f]) : warp_sum(v[f]);
    if (lane == 0 && w) {
      if (is_max_field(f)) atomicMax(&sh[f], w); else atomicAdd(&sh[f], w);
    }
  }
  __syncthreads();
  if (threadIdx.x < kFields && sh[threadIdx.x]) {
    const int f = threadIdx.x;
    if (is_max_field(f)) atomicMax(total_field(tot, f), sh[f]); else atomicAdd(total_field(tot, f), sh[f]);
  }
}

// A warp per row (rows w, w + W, ... for warp w of W): lanes take the
// row's entries for the counts, maxima, log10 ranges, diagonal offsets and
// column statistics, which do not depend on the order; the diagonal-dominance
// sum is added by lane 0 in entry order, as the reference adds it.
template <typename I, typename V>
__global__ void __launch_bounds__(256) row_pass_kernel(const I* __restrict__ rp, const I* __restrict__ ci,
                                                       const V* __restrict__ val, int64_t n, int64_t ncols,
                                                       int64_t close_thr, int64_t* __restrict__ row_cnt,
                                                       unsigned long long* __restrict__ col_cnt,
                                                       unsigned long long* __restrict__ col_max_bits,
                                                       unsigned long long* __restrict__ col_negmin_bits,
                                                       unsigned char* __restrict__ diag_seen,
                                                       Totals* __restrict__ tot) {
  __shared__ unsigned long long sh[kFields];
  if (threadIdx.x < kFields) sh[threadIdx.x] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t W = (int64_t)gridDim.x * (blockDim.x >> 5);
  unsigned long long v[kFields] = {};
  double maxd = -1.0, maxo = -1.0;  // this lane's largest |a| on / off the diagonal
  for (int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < n; r += W) {
    const int64_t s = rp[r], e = rp[r + 1];
    unsigned long long dg = 0;
    double rmax = 0.0, rmin = 0.0;
    for (int64_t k = s + lane; k < e; k += 32) {
      const int64_t c = (int64_t)ci[k];
      const double a = fabs((double)val[k]);
      const int64_t d = c - r;
      diag_seen[d + n - 1] = 1;
      if ((d < 0 ? -d : d) <= close_thr) ++v[kClose];
      if (d == 0) {
        ++dg;
        maxd = a > maxd ? a : maxd;
      } else {
        if (d < 0) ++v[kLower]; else ++v[kUpper];
        maxo = a > maxo ? a : maxo;
      }
      const double l = log10(a);
      if (rmax < l) rmax = l;
      if (a > 0.0 && rmin > l) rmin = l;
      atomicAdd(col_cnt + c, 1ULL);
      if (l > 0.0) atomic_max_nonneg(col_max_bits + c, l);
      if (a > 0.0 && l < 0.0) atomic_max_nonneg(col_negmin_bits + c, -l);
    }
    v[kDiagonal] += dg;
    // the row's diagonal count and log10 range over the warp
    const unsigned long long row_dg = warp_sum(dg);
    for (int o = 16; o; o >>= 1) {
      rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
      rmin = fmin(rmin, __shfl_xor_sync(0xffffffffu, rmin, o));
    }
    if (lane == 0) {
      double dom = 0.0;
      for (int64_t k = s; k < e; ++k) {
        const double a = fabs((double)val[k]);
        if ((int64_t)ci[k] == r) dom += a; else dom -= a;
      }
      row_cnt[r] = e - s;
      if (dom > 0.0) ++v[kDominant];
      if (row_dg) v[kHasDiag] = 1;
      if ((unsigned long long)(e - s) > row_dg) v[kHasOff] = 1;
      if (rmin != 0.0) {
        const unsigned long long b = (unsigned long long)__double_as_longlong(rmax - rmin);
        v[kRowVar] = b > v[kRowVar] ? b : v[kRowVar];
        v[kHasRowVar] = 1;
      }
    }
  }
  if (maxd >= 0.0) v[kMaxDiag] = (unsigned long long)__double_as_longlong(maxd);
  if (maxo >= 0.0) v[kMaxOff] = (unsigned long long)__double_as_longlong(maxo);
  flush_totals(v, sh, tot);
}

__global__ void col_var_kernel(const unsigned long long* __restrict__ col_max_bits,
                               const unsigned long long* __restrict__ col_negmin_bits, int64_t ncols,
                               Totals* __restrict__ tot) {
  __shared__ unsigned long long sh[kFields];
  if (threadIdx.x < kFields) sh[threadIdx.x] = 0;
  __syncthreads();
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  unsigned long long v[kFields] = {};
  if (c < ncols) {
    const double mn = -__longlong_as_double((long long)col_negmin_bits[c]);
    if (mn != 0.0) {
      const double mx = __longlong_as_double((long long)col_max_bits[c]);
      v[kColVar] = (unsigned long long)__double_as_longlong(mx - mn);
      v[kHasColVar] = 1;
    }
  }
  flush_totals(v, sh, tot);
}

__global__ void count_flags_kernel(const unsigned char* __restrict__ f, int64_t m, unsigned long long* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool on = i < m && f[i];
  const unsigned b = __ballot_sync(0xffffffffu, on);
  if ((threadIdx.x & 31) == 0 && b) atomicAdd(out, (unsigned long long)__popc(b));
}

__global__ void to_i64_kernel(const unsigned long long* __restrict__ a, int64_t m, int64_t* __restrict__ b) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < m) b[i] = (int64_t)a[i];
}

struct SqDev {
  double mean;
  __host__ __device__ double operator()(int64_t c) const {
    const double d = (double)c - mean;
    return d * d;
  }
};

struct NonZero {
  __host__ __device__ int64_t operator()(int64_t c) const { return c ? 1 : 0; }
};

// smallest prefix (from the largest counts) whose row share plus entry share
// reaches 1, with the reference's expressions: p = count / length,
// q = taken entries / nnz, stop when p + q >= 1.  Both shares and their
// rounded sum grow with the prefix, so the first prefix that stops is found
// by bisection; *best stays ~0 when none does.
__global__ void p_ratio_kernel(const int64_t* __restrict__ cum, int64_t len, int64_t nnz,
                               unsigned long long* __restrict__ best) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  auto stops = [&](int64_t q) {
    const int64_t taken = cum[len - 1] - (len - q - 1 >= 0 ? cum[len - q - 1] : 0);
    const double p_tmp = (double)q / (double)len;
    const double one_minus_p = (double)taken / (double)nnz;
    return !(p_tmp + one_minus_p < 1.0);
  };
  int64_t lo = 1, hi = len + 1;  // the answer is in [lo, hi); hi = len + 1: none
  while (lo < hi) {
    const int64_t mid = lo + (hi - lo) / 2;
    if (stops(mid)) hi = mid; else lo = mid + 1;
  }
  *best = lo <= len ? (unsigned long long)lo : ~0ULL;
}

struct Trap {
  const int64_t* cum;
  __host__ __device__ double operator()(int64_t i) const { return (double)(cum[i] + cum[i + 1]) / 2.0; }
};

// symmetric pairs: entry (r, c), r != c, whose mirror (c, r) exists, and with
// the same value printed with six decimals (sign kept, as the text is).
// The keys are the CSR's (row, col) pairs sorted, which only reorders each
// row's columns: the mirror (c, r) can only sit in row c's segment
// [rp[c], rp[c+1]), searched by bisection.  Matches are counted per warp.
template <typename I, typename V>
__global__ void symm_kernel(const I* __restrict__ rp, const uint64_t* __restrict__ keys, const V* __restrict__ vals,
                            int64_t m, unsigned long long* __restrict__ pat, unsigned long long* __restrict__ same) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool hit = false, eq = false;
  if (t < m) {
    const uint64_t k = keys[t];
    const uint64_t r = k >> 32, c = k & 0xffffffffu;
    if (r != c) {
      const uint64_t want = (c << 32) | r;
      int64_t lo = (int64_t)rp[c], hi = (int64_t)rp[c + 1];
      const int64_t end = hi;
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (keys[mid] < want) lo = mid + 1; else hi = mid;
      }
      if (lo < end && keys[lo] == want) {
        hit = true;
        const double a = (double)vals[t], b = (double)vals[lo];
        eq = signbit(a) == signbit(b) && rint(fabs(a) * 1e6) == rint(fabs(b) * 1e6);
      }
    }
  }
  const unsigned bh = __ballot_sync(0xffffffffu, hit), be = __ballot_sync(0xffffffffu, eq);
  if ((threadIdx.x & 31) == 0) {
    if (bh) atomicAdd(pat, (unsigned long long)__popc(bh));
    if (be) atomicAdd(same, (unsigned long long)__popc(be));
  }
}

// The same counts for rows whose columns strictly ascend, taken column by
// column: the entries (r, c) of column c are row c of A^T (trp, tri; perm
// gives each one's position in A), and the mirror (c, r) of each can only be
// in row c of A.  A warp takes row c and every lane bisects that same row of
// A for its own r, so the warp's probes share the row's few cache lines
// instead of every entry fetching its own from DRAM.  The warps stride over
// the rows and add their counts once at the end.
template <typename I, typename V>
__global__ void __launch_bounds__(256) symm_by_column_kernel(const I* __restrict__ rp, const I* __restrict__ ci,
                                                             const V* __restrict__ vals, const I* __restrict__ trp,
                                                             const I* __restrict__ tri,
                                                             const int64_t* __restrict__ perm, int64_t n,
                                                             unsigned long long* __restrict__ pat,
                                                             unsigned long long* __restrict__ same) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  unsigned long long hits = 0, eqs = 0;
  for (int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; c < n; c += nw) {
    const int64_t s = (int64_t)rp[c], e = (int64_t)rp[c + 1];
    const int64_t t1 = (int64_t)trp[c + 1];
    for (int64_t t = (int64_t)trp[c] + lane; t < t1; t += 32) {
      const int64_t r = (int64_t)tri[t];
      if (r == c) continue;
      int64_t lo = s, hi = e;
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if ((int64_t)ci[mid] < r) lo = mid + 1; else hi = mid;
      }
      if (lo < e && (int64_t)ci[lo] == r) {
        ++hits;
        const double a = (double)vals[perm[t]], b = (double)vals[lo];
        if (signbit(a) == signbit(b) && rint(fabs(a) * 1e6) == rint(fabs(b) * 1e6)) ++eqs;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    hits += __shfl_down_sync(0xffffffffu, hits, o);
    eqs += __shfl_down_sync(0xffffffffu, eqs, o);
  }
  if (lane == 0) {
    if (hits) atomicAdd(pat, hits);
    if (eqs) atomicAdd(same, eqs);
  }
}

// The same counts for rows whose columns strictly ascend, with no transpose
// and no copy: a warp takes row r, each lane an entry (r, c), and bisects
// row c of the CSR's own column array for r (4-byte probes, nothing to
// allocate).  The warps stride over the rows and add their counts at the end.
template <typename I, typename V>
__global__ void __launch_bounds__(256) symm_by_row_kernel(const I* __restrict__ rp, const I* __restrict__ ci,
                                                          const V* __restrict__ vals, int64_t n,
                                                          unsigned long long* __restrict__ pat,
                                                          unsigned long long* __restrict__ same) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  unsigned long long hits = 0, eqs = 0;
  for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; r < n; r += nw) {
    const int64_t k1 = (int64_t)rp[r + 1];
    for (int64_t k = (int64_t)rp[r] + lane; k < k1; k += 32) {
      const int64_t c = (int64_t)ci[k];
      if (c == r) continue;
      const int64_t end = (int64_t)rp[c + 1];
      int64_t lo = (int64_t)rp[c], hi = end;
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if ((int64_t)ci[mid] < r) lo = mid + 1; else hi = mid;
      }
      if (lo < end && (int64_t)ci[lo] == r) {
        ++hits;
        const double a = (double)vals[k], b = (double)vals[lo];
        if (signbit(a) == signbit(b) && rint(fabs(a) * 1e6) == rint(fabs(b) * 1e6)) ++eqs;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    hits += __shfl_down_sync(0xffffffffu, hits, o);
    eqs += __shfl_down_sync(0xffffffffu, eqs, o);
  }
  if (lane == 0) {
    if (hits) atomicAdd(pat, hits);
    if (eqs) atomicAdd(same, eqs);
  }
}

// flags[0] = 1 when some row's columns are not strictly ascending
template <typename I>
__global__ void rows_unsorted_kernel(const I* __restrict__ rp, const I* __restrict__ ci, int64_t n,
                                     unsigned int* __restrict__ flag) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int64_t s = (int64_t)rp[r], e = (int64_t)rp[r + 1];
  for (int64_t k = s + 1; k < e; ++k)
    if (ci[k] <= ci[k - 1]) {
      *flag = 1;
      return;
    }
}

template <typename I, typename V>
__global__ void symm_keys_kernel(const I* __restrict__ rp, const I* __restrict__ ci, const V* __restrict__ val,
                                 int64_t n, uint64_t* __restrict__ keys, V* __restrict__ vals) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  for (int64_t k = (int64_t)rp[r] + lane; k < (int64_t)rp[r + 1]; k += 32) {
    keys[k] = ((uint64_t)r << 32) | (uint64_t)(uint32_t)ci[k];
    vals[k] = val[k];
  }
}

// count statistics of one of the two count vectors (rows or columns)
struct CountStats {
  int64_t nz = 0, mn = 0, mx = 0;
  double ave = 0, sq = 0, var = 0, p = 0, gini = 0;
};

spops_status_t count_stats(Context* ctx, const int64_t* cnt, int64_t len, int64_t nnz, CountStats* out) {
  cudaStream_t st = ctx->stream;
  CountStats s;
  if (len <= 0) {
    *out = s;
    return SPOPS_OK;
  }
  PoolBuf sorted(ctx), cum(ctx), red(ctx), best(ctx), tmp(ctx);
  SPOPS_TRY(sorted.alloc((size_t)len * 8));
  SPOPS_TRY(cum.alloc((size_t)len * 8));
  SPOPS_TRY(red.alloc(64));
  SPOPS_TRY(best.alloc(8));
  size_t b1 = 0, b2 = 0, b3 = 0, b4 = 0, b5 = 0;
  int64_t* rd = red.as<int64_t>();
  double* rdd = reinterpret_cast<double*>(rd + 4);
  cub::TransformInputIterator<int64_t, NonZero, const int64_t*> nzit(cnt, NonZero());
  cub::TransformInputIterator<double, SqDev, const int64_t*> sqit(cnt, SqDev{(double)nnz / (double)len});
  cub::CountingInputIterator<int64_t> idx(0);
  cub::TransformInputIterator<double, Trap, cub::CountingInputIterator<int64_t>> trap(idx, Trap{cum.as<int64_t>()});
  SPOPS_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, b1, cnt, sorted.as<int64_t>(), len, 0, 64, st));
  SPOPS_CUDA(cub::DeviceScan::InclusiveSum(nullptr, b2, sorted.as<int64_t>(), cum.as<int64_t>(), len, st));
  SPOPS_CUDA(cub::DeviceReduce::Sum(nullptr, b3, nzit, rd, len, st));
  SPOPS_CUDA(cub::DeviceReduce::Sum(nullptr, b4, sqit, rdd, len, st));
  SPOPS_CUDA(cub::DeviceReduce::Sum(nullptr, b5, trap, rdd + 1, len > 1 ? len - 1 : 1, st));
  SPOPS_TRY(tmp.alloc(std::max({b1, b2, b3, b4, b5}) + 256));
  SPOPS_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, b1, cnt, sorted.as<int64_t>(), len, 0, 64, st));
  SPOPS_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, b2, sorted.as<int64_t>(), cum.as<int64_t>(), len, st));
  SPOPS_CUDA(cub::DeviceReduce::Sum(tmp.p, b3, nzit, rd, len, st));
  SPOPS_CUDA(cub::DeviceReduce::Sum(tmp.p, b4, sqit, rdd, len, st));
  SPOPS_CUDA(cudaMemsetAsync(rdd + 1, 0, 8, st));
  if (len > 1) SPOPS_CUDA(cub::DeviceReduce::Sum(tmp.p, b5, trap, rdd + 1, len - 1, st));
  SPOPS_CUDA(cudaMemsetAsync(best.p, 0xff, 8, st));
  p_ratio_kernel<<<1, 32, 0, st>>>(cum.as<int64_t>(), len, nnz, best.as<unsigned long long>());
  SPOPS_LAUNCH_CHECK();
  int64_t h_nz = 0, h_min = 0, h_max = 0;
  double h_var = 0, h_trap = 0;
  unsigned long long h_best = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&h_nz, rd, 8, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaMemcpyAsync(&h_min, sorted.as<int64_t>(), 8, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaMemcpyAsync(&h_max, sorted.as<int64_t>() + len - 1, 8, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaMemcpyAsync(&h_var, rdd, 8, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaMemcpyAsync(&h_trap, rdd + 1, 8, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaMemcpyAsync(&h_best, best.p, 8, cudaMemcpyDeviceToHost, st));
  int64_t first = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&first, cum.as<int64_t>(), 8, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  s.nz = h_nz;
  s.mn = h_min;
  s.mx = h_max;
  s.ave = (double)nnz / (double)len;
  s.sq = h_var;
  s.var = h_var / (double)len;
  s.p = h_best == ~0ULL ? 1.0 : (double)(int64_t)h_best / (double)len;
  const double area_b = (double)(first + 0) / 2.0 + h_trap;
  const double area_total = (double)nnz * (double)len / 2.0;
  s.gini = (area_total - area_b) / area_total;
  *out = s;
  return SPOPS_OK;
}

template <typename I, typename V>
spops_status_t features_t(Context* ctx, Matrix* A, spops_features_t* f) {
  cudaStream_t st = ctx->stream;
  const int64_t n = A->rows, nc = A->cols, nnz = A->nnz;
  std::memset(f, 0, sizeof(*f));
  f->rows = n;
  f->cols = nc;
  f->nnz = nnz;
  if (n <= 0 || nc <= 0) return SPOPS_OK;
  const int64_t ndl = n + nc - 1;
  PoolBuf rcnt(ctx), ccnt(ctx), cmax(ctx), cmin(ctx), seen(ctx), tot(ctx), ccnt64(ctx);
  SPOPS_TRY(rcnt.alloc((size_t)n * 8));
  SPOPS_TRY(ccnt.alloc((size_t)nc * 8));
  SPOPS_TRY(cmax.alloc((size_t)nc * 8));
  SPOPS_TRY(cmin.alloc((size_t)nc * 8));
  SPOPS_TRY(ccnt64.alloc((size_t)nc * 8));
  SPOPS_TRY(seen.alloc((size_t)ndl));
  SPOPS_TRY(tot.alloc(sizeof(Totals) + 64));
  SPOPS_CUDA(cudaMemsetAsync(ccnt.p, 0, (size_t)nc * 8, st));
  SPOPS_CUDA(cudaMemsetAsync(cmax.p, 0, (size_t)nc * 8, st));  // 0.0
  SPOPS_CUDA(cudaMemsetAsync(cmin.p, 0, (size_t)nc * 8, st));  // -min = 0.0
  SPOPS_CUDA(cudaMemsetAsync(seen.p, 0, (size_t)ndl, st));
  SPOPS_CUDA(cudaMemsetAsync(tot.p, 0, sizeof(Totals) + 64, st));
  Totals* T = tot.as<Totals>();
  unsigned long long* ndiag_d = reinterpret_cast<unsigned long long*>(tot.as<char>() + sizeof(Totals));
  row_pass_kernel<I, V><<<(unsigned)std::min<int64_t>((n + 7) / 8, (int64_t)ctx->num_sms * 8), 256, 0, st>>>(A->row.as<I>(), A->col.as<I>(), A->val.as<V>(), n, nc,
                                                    ndl / 20, rcnt.as<int64_t>(), ccnt.as<unsigned long long>(),
                                                    cmax.as<unsigned long long>(), cmin.as<unsigned long long>(),
                                                    seen.as<unsigned char>(), T);
  SPOPS_LAUNCH_CHECK();
  col_var_kernel<<<grid_of(nc), 256, 0, st>>>(cmax.as<unsigned long long>(), cmin.as<unsigned long long>(), nc, T);
  count_flags_kernel<<<grid_of(ndl), 256, 0, st>>>(seen.as<unsigned char>(), ndl, ndiag_d);
  to_i64_kernel<<<grid_of(nc), 256, 0, st>>>(ccnt.as<unsigned long long>(), nc, ccnt64.as<int64_t>());
  SPOPS_LAUNCH_CHECK();
  CountStats rs, cs;
  SPOPS_TRY(count_stats(ctx, rcnt.as<int64_t>(), n, nnz, &rs));
  SPOPS_TRY(count_stats(ctx, ccnt64.as<int64_t>(), nc, nnz, &cs));
  Totals h;
  unsigned long long h_ndiag = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&h, T, sizeof(Totals), cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaMemcpyAsync(&h_ndiag, ndiag_d, 8, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  f->nnz_lower = (int64_t)h.lower;
  f->nnz_upper = (int64_t)h.upper;
  f->nnz_diagonal = (int64_t)h.diagonal;
  f->ndiags = (int64_t)h_ndiag;
  f->nnz_ratio = (double)nnz / ((double)n * (double)nc);
  f->diag_close_ratio = (double)h.close / (double)nnz;
  f->min_nnz_row = rs.mn;
  f->max_nnz_row = rs.mx;
  f->nz_row_ratio = (double)rs.nz / (double)n;
  f->ave_nnz_row = rs.ave;
  f->var_nnz_row = rs.var;
  f->std_nnz_row = std::sqrt(rs.var);
  f->p_ratio_row = rs.p;
  f->gini_row = rs.gini;
  f->min_nnz_col = cs.mn;
  f->max_nnz_col = cs.mx;
  f->nz_col_ratio = (double)cs.nz / (double)nc;
  f->ave_nnz_col = cs.ave;
  f->var_nnz_col = cs.var;
  f->std_nnz_col = std::sqrt(cs.var);
  f->p_ratio_col = cs.p;
  f->gini_col = cs.gini;
  f->diagonal_dominant_ratio = (double)h.dominant / (double)std::min(n, nc);
  auto as_d = [](unsigned long long b) {
    double d;
    std::memcpy(&d, &b, 8);
    return d;
  };
  f->max_value_diagonal = h.has_diag ? as_d(h.max_diag_bits) : -DBL_MAX;
  f->max_value_offdiag = h.has_off ? as_d(h.max_off_bits) : -DBL_MAX;
  f->row_variability = h.has_row_var ? as_d(h.row_var_bits) : -1.0;
  f->col_variability = h.has_col_var ? as_d(h.col_var_bits) : -1.0;
  // symmetry (square matrices)
  if (n == nc && nnz > 0) {
    if (n > (int64_t)0xffffffffLL) return fail(SPOPS_ERR_UNSUPPORTED, "features: more than 2^32 rows");
    PoolBuf k0(ctx), k1(ctx), v0(ctx), v1(ctx), cntb(ctx), tmp(ctx);
    SPOPS_TRY(cntb.alloc(32));
    SPOPS_CUDA(cudaMemsetAsync(cntb.p, 0, 32, st));
    // rows whose columns already ascend need no sort: the keys are in order
    unsigned int* unsorted = reinterpret_cast<unsigned int*>(cntb.as<unsigned long long>() + 1) + 2;
    SPOPS_CUDA(cudaMemsetAsync(unsorted, 0, 4, st));
    rows_unsorted_kernel<I><<<grid_of(n), 256, 0, st>>>(A->row.as<I>(), A->col.as<I>(), n, unsorted);
    SPOPS_LAUNCH_CHECK();
    unsigned int h_unsorted = 0;
    SPOPS_CUDA(cudaMemcpyAsync(&h_unsorted, unsorted, 4, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
    unsigned long long* c2 = cntb.as<unsigned long long>();
    const int64_t sblocks = std::min<int64_t>((n + 7) / 8, (int64_t)ctx->num_sms * 8);
    if (!h_unsorted && A->tr.ready) {
      // column by column over the transpose pattern the handle already keeps
      // (built by the tile features, A^T x or the adjoint).  It is not built
      // for this count alone: building it costs more than the search it saves.
      symm_by_column_kernel<I, V><<<(unsigned)sblocks, 256, 0, st>>>(
          A->row.as<I>(), A->col.as<I>(), A->val.as<V>(), A->tr.rp.as<I>(), A->tr.ri.as<I>(),
          A->tr.perm.as<int64_t>(), n, c2, c2 + 1);
      SPOPS_LAUNCH_CHECK();
    } else if (!h_unsorted) {  // row by row on the CSR arrays themselves
      symm_by_row_kernel<I, V><<<(unsigned)sblocks, 256, 0, st>>>(A->row.as<I>(), A->col.as<I>(), A->val.as<V>(),
                                                                   n, c2, c2 + 1);
      SPOPS_LAUNCH_CHECK();
    } else {  // the (row, col) keys sorted, then a bisection per mirror
      SPOPS_TRY(k0.alloc((size_t)nnz * 8));
      SPOPS_TRY(k1.alloc((size_t)nnz * 8));
      SPOPS_TRY(v0.alloc((size_t)nnz * sizeof(V)));
      SPOPS_TRY(v1.alloc((size_t)nnz * sizeof(V)));
      symm_keys_kernel<I, V><<<grid_of(n * 32), 256, 0, st>>>(A->row.as<I>(), A->col.as<I>(), A->val.as<V>(), n,
                                                              k0.as<uint64_t>(), v0.as<V>());
      SPOPS_LAUNCH_CHECK();
      int end_bit = 32;  // the row half of the key holds n - 1 at most
      while (end_bit < 64 && ((uint64_t)(n - 1) >> (end_bit - 32)) != 0) ++end_bit;
      size_t b = 0;
      SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b, k0.as<uint64_t>(), k1.as<uint64_t>(), v0.as<V>(),
                                                 v1.as<V>(), nnz, 0, end_bit, st));
      SPOPS_TRY(tmp.alloc(b + 256));
      SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, b, k0.as<uint64_t>(), k1.as<uint64_t>(), v0.as<V>(),
                                                 v1.as<V>(), nnz, 0, end_bit, st));
      symm_kernel<I, V><<<grid_of(nnz), 256, 0, st>>>(A->row.as<I>(), k1.as<uint64_t>(), v1.as<V>(), nnz, c2, c2 + 1);
      SPOPS_LAUNCH_CHECK();
    }
    unsigned long long hc[2] = {0, 0};
    SPOPS_CUDA(cudaMemcpyAsync(hc, c2, 16, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
    const double off = (double)(nnz - f->nnz_diagonal);
    f->pattern_symm = (double)hc[0] / off;
    f->value_symm = (double)hc[1] / off;
  }
  return SPOPS_OK;
}

}  // namespace

spops_status_t count_summary(Context* ctx, const int64_t* cnt, int64_t len, int64_t nnz, CountSummary* out) {
  CountStats s;
  SPOPS_TRY(count_stats(ctx, cnt, len, nnz, &s));
  out->nz = s.nz;
  out->mn = s.mn;
  out->mx = s.mx;
  out->ave = s.ave;
  out->sq = s.sq;
  out->p = s.p;
  out->gini = s.gini;
  return SPOPS_OK;
}

spops_status_t csr_features(Context* ctx, Matrix* A, spops_features_t* f) {
  if (A->format != SPOPS_FMT_CSR) return fail(SPOPS_ERR_INVALID, "features: needs a CSR matrix");
  if (!A->plan.ready) SPOPS_TRY(csr_analyse(ctx, A));  // validates the pattern
  const bool i32 = A->itype == SPOPS_INDEX_I32, f64 = A->vtype == SPOPS_VALUE_F64;
  if (i32 && f64) return features_t<int32_t, double>(ctx, A, f);
  if (i32) return features_t<int32_t, float>(ctx, A, f);
  if (f64) return features_t<int64_t, double>(ctx, A, f);
  return features_t<int64_t, float>(ctx, A, f);
}

}  // namespace spops

using namespace spops;

extern "C" {

spops_status_t spops_matrix_features(spops_context_t ctx, spops_matrix_t csr, spops_features_t* features) {
  if (!ctx || !csr || !features) return fail(SPOPS_ERR_INVALID, "spops_matrix_features: null argument");
  DeviceGuard g(ctx->device);
  return csr_features(ctx, csr, features);
}

spops_status_t spops_select_format(spops_context_t ctx, spops_matrix_t csr, int32_t mode, spops_format_t* format,
                                   spops_format_params_t* params, double* ms) {
  if (!ctx || !csr || !format || !params) return fail(SPOPS_ERR_INVALID, "spops_select_format: null argument");
  if (csr->format != SPOPS_FMT_CSR) return fail(SPOPS_ERR_INVALID, "spops_select_format: needs a CSR matrix");
  DeviceGuard g(ctx->device);
  spops_features_t f;
  SPOPS_TRY(csr_features(ctx, csr, &f));
  std::memset(params, 0, sizeof(*params));
  if (ms) *ms = 0.0;
  const int64_t mn = std::min(f.rows, f.cols);
  const bool dia_dense = f.ndiags > 0 && (double)f.nnz >= 0.5 * (double)f.ndiags * (double)mn;
  if (mode == 2) {  // learned: the fitted decision tree (csrc/selector.cpp)
    tree_select(f, format, params);
    return SPOPS_OK;
  }
  if (mode == 0) {
    if (f.ndiags <= 64 && dia_dense) {
      *format = SPOPS_FMT_DIA;
      params->alignment = 1;
    } else {
      *format = SPOPS_FMT_CSR;
    }
    return SPOPS_OK;
  }
  // timed: each candidate runs a few SpMVs on the context stream
  struct Cand {
    spops_format_t f;
    spops_format_params_t p;
  };
  std::vector<Cand> cands;
  auto add = [&](spops_format_t fm, int64_t chunk, int64_t sigma, int32_t layout) {
    Cand c;
    std::memset(&c.p, 0, sizeof(c.p));
    c.f = fm;
    c.p.chunk = chunk;
    c.p.sigma = sigma;
    c.p.alignment = 1;
    c.p.layout = layout;
    cands.push_back(c);
  };
  add(SPOPS_FMT_CSR, 0, 0, 0);
  add(SPOPS_FMT_SELL_C_R, 32, 0, SPOPS_COL_MAJOR);
  add(SPOPS_FMT_SELL_C_SIGMA, 32, 4096, SPOPS_COL_MAJOR);
  add(SPOPS_FMT_CSR5, 0, 0, 0);
  if (f.ndiags <= 10240 && (double)f.nnz >= 0.25 * (double)f.ndiags * (double)mn) add(SPOPS_FMT_DIA, 0, 0, 0);
  const size_t vs = csr->vsize();
  DevBuf x, y;
  SPOPS_TRY(x.alloc((size_t)std::max<int64_t>(f.cols, 1) * vs));
  SPOPS_TRY(y.alloc((size_t)std::max<int64_t>(f.rows, 1) * vs));
  cudaStream_t st = ctx->stream;
  SPOPS_CUDA(cudaMemsetAsync(x.p, 0, x.bytes, st));
  cudaEvent_t e0, e1;
  SPOPS_CUDA(cudaEventCreate(&e0));
  SPOPS_CUDA(cudaEventCreate(&e1));
  double best = -1.0;
  spops_status_t result = SPOPS_OK;
  for (const Cand& c : cands) {
    spops_matrix_t M = csr;
    if (c.f != SPOPS_FMT_CSR) {
      spops_format_params_t p = c.p;
      if (spops_convert(ctx, csr, c.f, &p, &M) != SPOPS_OK) continue;  // e.g. too large: not a candidate
    }
    spops_status_t s = SPOPS_OK;
    for (int w = 0; w < 2 && s == SPOPS_OK; ++w) s = spops_spmv(ctx, 1.0, M, x.p, 0.0, y.p);
    float t = 0.f;
    if (s == SPOPS_OK) {
      cudaEventRecord(e0, st);
      for (int r = 0; r < 5 && s == SPOPS_OK; ++r) s = spops_spmv(ctx, 1.0, M, x.p, 0.0, y.p);
      cudaEventRecord(e1, st);
      cudaEventSynchronize(e1);
      cudaEventElapsedTime(&t, e0, e1);
    }
    if (M != csr) spops_matrix_destroy(M);
    if (s != SPOPS_OK) {
      result = s;
      break;
    }
    const double per = t / 5.0;
    if (best < 0 || per < best) {
      best = per;
      *format = c.f;
      *params = c.p;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (result != SPOPS_OK) return result;
  if (ms) *ms = best;
  return SPOPS_OK;
}

}  // extern "C"
