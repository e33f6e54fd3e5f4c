// Adjoint kernels of y = alpha*A*x + beta*y for a CSR matrix A:
//   dL/dx      = alpha * A^T g      (transpose SpMV)
//   dL/dA_ij   = alpha * g_i * x_j  on A's pattern (SDDMM)
// The reference has no differentiation; the transpose it offers is
// csr_transpose (include/sparse_conversion.h:2066-2108: CSR -> COO -> swap ->
// counting sort, then SpOps_csr), which the oracle restates for grad_x.
//
// Transpose, atomic-free: once per pattern a stable radix sort of the column
// indices gives perm (entry of A at each position of A^T) together with the
// row indices, and a histogram + scan gives A^T's row offsets; A^T's values
// are gathered through perm whenever A's values change (spops_matrix_touch /
// spops_csr_set_values).  A^T g then runs the ordinary CSR kernel on that
// matrix, so it needs no atomics and is deterministic.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "csr_tile.cuh"
#include "device_util.cuh"
#include "spops_internal.h"

namespace spops {
namespace {

inline unsigned grid_for(int64_t work, int threads = 256) {
  int64_t g = (work + threads - 1) / threads;
  return (unsigned)(g < 1 ? 1 : g);
}

template <typename I>
__global__ void expand_rows_kernel(const I* __restrict__ rp, int64_t n, I* __restrict__ row) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  for (int64_t k = (int64_t)rp[r] + lane; k < (int64_t)rp[r + 1]; k += 32) row[k] = (I)r;
}

template <typename I>
__global__ void count_cols_kernel(const I* __restrict__ ci, int64_t nnz, unsigned long long* __restrict__ cnt) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += stride)
    atomicAdd(cnt + ci[k], 1ULL);
}

template <typename I>
__global__ void cast_kernel(const unsigned long long* __restrict__ in, int64_t m, I* __restrict__ out) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < m) out[k] = (I)in[k];
}

__global__ void iota64_kernel(int64_t* __restrict__ a, int64_t m) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < m) a[k] = k;
}

template <typename I>
__global__ void gather_index_kernel(const int64_t* __restrict__ perm, const I* __restrict__ src, int64_t m,
                                    I* __restrict__ dst) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < m) dst[k] = src[perm[k]];
}

template <typename V>
__global__ void gather_values_kernel(const int64_t* __restrict__ perm, const V* __restrict__ src, int64_t m,
                                     V* __restrict__ dst) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < m) dst[k] = src[perm[k]];
}

// out[k] = alpha * g[row(k)] * x[col(k)], over the CSR plan's segments.
template <typename I, typename V>
__global__ void __launch_bounds__(256) sddmm_kernel(const I* __restrict__ rp, const I* __restrict__ ci,
                                                    const V* __restrict__ g, const V* __restrict__ x,
                                                    V* __restrict__ out, V alpha, const CsrSeg* __restrict__ segs,
                                                    int64_t nseg) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t j = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; j < nseg; j += nwarps) {
    const CsrSeg d = segs[j];
    if (d.chunk >= 0) {
      const V gi = alpha * g[d.r0];
      for (int64_t k = d.p0 + lane; k < d.p1; k += 32) out[k] = gi * ld_gather(x + ld_stream(ci + k));
    } else {
      const int nr = d.nr;
      int t = 32 / (nr > 0 ? nr : 1);
      t = t >= 32 ? 32 : t >= 16 ? 16 : t >= 8 ? 8 : t >= 4 ? 4 : t >= 2 ? 2 : 1;
      const int groups = 32 / t, grp = lane / t, sub = lane % t;
      for (int rb = 0; rb < nr; rb += groups) {
        const int rr = rb + grp;
        if (rr < nr) {
          const int64_t r = d.r0 + rr;
          const V gi = alpha * g[r];
          for (int64_t k = (int64_t)rp[r] + sub; k < (int64_t)rp[r + 1]; k += t)
            out[k] = gi * ld_gather(x + ld_stream(ci + k));
        }
      }
    }
  }
}

template <typename I, typename V>
spops_status_t build_transpose_t(Context* ctx, Matrix* A) {
  TransposeData& T = A->tr;
  cudaStream_t st = ctx->stream;
  const int64_t n = A->rows, nc = A->cols, nnz = A->nnz;
  size_t cub_sort = 0, cub_scan = 0;
  // columns are in [0, nc): the stable sort needs only their low bits
  int col_bits = 1;
  while (col_bits < 8 * (int)sizeof(I) - 1 && ((nc - 1) >> col_bits) > 0) ++col_bits;
  {
    I* k = nullptr;
    int64_t* v = nullptr;
    unsigned long long* u = nullptr;
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, cub_sort, k, k, v, v, (int64_t)(nnz > 0 ? nnz : 1), 0,
                                               col_bits, st));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cub_scan, u, u, (int64_t)(nc + 1), st));
  }
  const size_t nz = (size_t)(nnz > 0 ? nnz : 1), nc1 = (size_t)nc + 1;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t need = al(nz * sizeof(I)) * 2 + al(nz * 8) + al(nc1 * 8) * 2 + std::max(cub_sort, cub_scan);
  SPOPS_TRY(ctx->scratch_reserve(need));
  char* base = ctx->scratch.as<char>();
  size_t off = 0;
  auto take = [&](size_t b) { char* p = base + off; off += al(b); return p; };
  I* keys_out = reinterpret_cast<I*>(take(nz * sizeof(I)));
  I* rows = reinterpret_cast<I*>(take(nz * sizeof(I)));
  int64_t* idx = reinterpret_cast<int64_t*>(take(nz * 8));
  unsigned long long* cnt = reinterpret_cast<unsigned long long*>(take(nc1 * 8));
  unsigned long long* scan = reinterpret_cast<unsigned long long*>(take(nc1 * 8));
  void* cub_tmp = take(std::max(cub_sort, cub_scan));

  T.release();
  // large arrays: reuse blocks earlier results of this context released
  SPOPS_TRY(T.rp.alloc_cached(ctx, nc1 * sizeof(I)));
  SPOPS_TRY(T.ri.alloc_cached(ctx, nz * sizeof(I)));
  SPOPS_TRY(T.perm.alloc_cached(ctx, nz * 8));
  SPOPS_TRY(T.val.alloc_cached(ctx, nz * sizeof(V)));
  SPOPS_CUDA(cudaMemsetAsync(cnt, 0, nc1 * 8, st));
  if (nnz > 0) {
    count_cols_kernel<I><<<std::min<unsigned>(grid_for(nnz), 8192u), 256, 0, st>>>(A->col.as<I>(), nnz, cnt);
    iota64_kernel<<<grid_for(nnz), 256, 0, st>>>(idx, nnz);
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(cub_tmp, cub_sort, A->col.as<I>(), keys_out, idx, T.perm.as<int64_t>(),
                                               nnz, 0, col_bits, st));
    expand_rows_kernel<I><<<grid_for(n * 32), 256, 0, st>>>(A->row.as<I>(), n, rows);
    gather_index_kernel<I><<<grid_for(nnz), 256, 0, st>>>(T.perm.as<int64_t>(), rows, nnz, T.ri.as<I>());
    SPOPS_LAUNCH_CHECK();
  }
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(cub_tmp, cub_scan, cnt, scan, (int64_t)nc1, st));
  cast_kernel<I><<<grid_for((int64_t)nc1), 256, 0, st>>>(scan, (int64_t)nc1, T.rp.as<I>());
  SPOPS_LAUNCH_CHECK();
  // the CSR handle of A^T borrows the arrays above
  Matrix* V_ = new Matrix();
  V_->ctx = ctx;
  V_->format = SPOPS_FMT_CSR;
  V_->itype = A->itype;
  V_->vtype = A->vtype;
  V_->rows = nc;
  V_->cols = n;
  V_->nnz = nnz;
  V_->row.borrow(T.rp.p, T.rp.bytes);
  V_->col.borrow(T.ri.p, T.ri.bytes);
  V_->val.borrow(T.val.p, T.val.bytes);
  T.view = V_;
  spops_status_t s = csr_analyse(ctx, V_);
  if (s != SPOPS_OK) {
    T.release();
    return s;
  }
  T.ready = true;
  T.values_fresh = false;
  return SPOPS_OK;
}

// ---- source-row bands of the transpose.  A row of A^T lists its source rows
// in ascending order (the transpose's sort is stable), so the entries of
// each band of source rows are one subrange of it, found by bisection.
struct BandStarts {
  int64_t v[TransposeData::kMaxBands + 1];  // band b: source rows [v[b], v[b + 1])
};
struct BandPtrs {
  const void* rp[TransposeData::kMaxBands];
  void* ri[TransposeData::kMaxBands];
  int64_t* perm[TransposeData::kMaxBands];
};

template <typename I>
__device__ __forceinline__ int64_t first_source_at(const I* __restrict__ tri, int64_t s, int64_t e, int64_t r0) {
  while (s < e) {
    const int64_t m = (s + e) >> 1;
    if ((int64_t)tri[m] < r0) s = m + 1; else e = m;
  }
  return s;
}

// cnt[b * (nc + 1) + c] = entries of row c of A^T in band b
template <typename I>
__global__ void band_count_kernel(const I* __restrict__ trp, const I* __restrict__ tri, int64_t nc, int nb,
                                  BandStarts bs, unsigned long long* __restrict__ cnt) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const int64_t e = (int64_t)trp[c + 1];
  int64_t p = (int64_t)trp[c];
  for (int b = 0; b < nb; ++b) {
    const int64_t q = b + 1 < nb ? first_source_at(tri, p, e, bs.v[b + 1]) : e;
    cnt[(int64_t)b * (nc + 1) + c] = (unsigned long long)(q - p);
    p = q;
  }
}

// A warp per row c of A^T copies each band's subrange of the row (source
// rows and positions in A) to that band's arrays at the band's row offset.
template <typename I>
__global__ void band_fill_kernel(const I* __restrict__ trp, const I* __restrict__ tri,
                                 const int64_t* __restrict__ perm, int64_t nc, int nb, BandStarts bs, BandPtrs P) {
  const int64_t c = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= nc) return;
  const int64_t e = (int64_t)trp[c + 1];
  int64_t p = (int64_t)trp[c];
  for (int b = 0; b < nb; ++b) {
    const int64_t q = b + 1 < nb ? first_source_at(tri, p, e, bs.v[b + 1]) : e;
    const int64_t d = (int64_t)static_cast<const I*>(P.rp[b])[c] - p;
    I* ri = static_cast<I*>(P.ri[b]);
    for (int64_t k = p + lane; k < q; k += 32) {
      ri[d + k] = tri[k];
      P.perm[b][d + k] = perm[k];
    }
    p = q;
  }
}

void release_bands(TransposeData& T) {
  for (int b = 0; b < T.nbands; ++b) {
    if (T.bview[b]) {
      T.bview[b]->release_all();
      delete T.bview[b];
      T.bview[b] = nullptr;
    }
    T.brp[b].release();
    T.bri[b].release();
    T.bperm[b].release();
  }
  T.nbands = 0;
}

// The bands of A's transpose (built after the transpose, once per pattern
// and band count): row ranges of A with about nnz / nb entries each.
template <typename I, typename V>
spops_status_t build_bands_t(Context* ctx, Matrix* A, int nb) {
  TransposeData& T = A->tr;
  cudaStream_t st = ctx->stream;
  const int64_t n = A->rows, nc = A->cols, nnz = A->nnz;
  release_bands(T);
  std::vector<I> rp_h((size_t)n + 1);
  SPOPS_CUDA(cudaMemcpyAsync(rp_h.data(), A->row.p, ((size_t)n + 1) * sizeof(I), cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  BandStarts bs{};
  for (int b = 1; b < nb; ++b) {  // first row starting at or after entry b * nnz / nb
    const I target = (I)(nnz / nb * b + (nnz % nb) * b / nb);
    bs.v[b] = std::max<int64_t>(bs.v[b - 1], std::lower_bound(rp_h.begin(), rp_h.end(), target) - rp_h.begin());
    if (bs.v[b] > n) bs.v[b] = n;
  }
  bs.v[nb] = n;
  const size_t stride = (size_t)nc + 1;
  PoolBuf cnt(ctx), scan(ctx), tmp(ctx);
  SPOPS_TRY(cnt.alloc((size_t)nb * stride * 8));
  SPOPS_TRY(scan.alloc(stride * 8));
  size_t cub_b = 0;
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cub_b, (unsigned long long*)nullptr,
                                           (unsigned long long*)nullptr, (int64_t)stride, st));
  SPOPS_TRY(tmp.alloc(cub_b + 256));
  SPOPS_CUDA(cudaMemsetAsync(cnt.p, 0, (size_t)nb * stride * 8, st));
  band_count_kernel<I><<<grid_for(nc), 256, 0, st>>>(T.rp.as<I>(), T.ri.as<I>(), nc, nb, bs,
                                                      cnt.as<unsigned long long>());
  SPOPS_LAUNCH_CHECK();
  unsigned long long nnzb[TransposeData::kMaxBands] = {};
  T.nbands = nb;  // from here on release_bands frees what was allocated
  for (int b = 0; b < nb; ++b) {
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, cub_b, cnt.as<unsigned long long>() + b * stride,
                                             scan.as<unsigned long long>(), (int64_t)stride, st));
    SPOPS_TRY(T.brp[b].alloc(stride * sizeof(I)));
    cast_kernel<I><<<grid_for((int64_t)stride), 256, 0, st>>>(scan.as<unsigned long long>(), (int64_t)stride,
                                                               T.brp[b].as<I>());
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cudaMemcpyAsync(&nnzb[b], scan.as<unsigned long long>() + nc, 8, cudaMemcpyDeviceToHost, st));
  }
  SPOPS_CUDA(cudaStreamSynchronize(st));
  BandPtrs P{};
  for (int b = 0; b < nb; ++b) {
    const size_t m = (size_t)(nnzb[b] > 0 ? nnzb[b] : 1);
    SPOPS_TRY(T.bri[b].alloc(m * sizeof(I)));
    SPOPS_TRY(T.bperm[b].alloc(m * 8));
    P.rp[b] = T.brp[b].p;
    P.ri[b] = T.bri[b].p;
    P.perm[b] = T.bperm[b].as<int64_t>();
  }
  if (nc > 0) {
    band_fill_kernel<I><<<grid_for(nc * 32), 256, 0, st>>>(T.rp.as<I>(), T.ri.as<I>(), T.perm.as<int64_t>(), nc, nb,
                                                           bs, P);
    SPOPS_LAUNCH_CHECK();
  }
  for (int b = 0; b < nb; ++b) {  // CSR handles of the bands (values read through perm, never from val)
    if (nnzb[b] == 0) continue;    // an empty band: no handle, no launch
    Matrix* V_ = new Matrix();
    V_->ctx = ctx;
    V_->format = SPOPS_FMT_CSR;
    V_->itype = A->itype;
    V_->vtype = A->vtype;
    V_->rows = nc;
    V_->cols = n;
    V_->nnz = (int64_t)nnzb[b];
    V_->row.borrow(T.brp[b].p, T.brp[b].bytes);
    V_->col.borrow(T.bri[b].p, T.bri[b].bytes);
    V_->val.borrow(T.val.p, (size_t)(nnzb[b] > 0 ? nnzb[b] : 1) * sizeof(V));
    T.bview[b] = V_;
    const spops_status_t s = csr_analyse(ctx, V_);
    if (s != SPOPS_OK) {
      release_bands(T);
      return s;
    }
  }
  return SPOPS_OK;
}

// bands for A^T x through perm: the context's setting, or as many as keep
// each band's values within 64 MB once A's values pass 96 MB
int adjoint_band_count(const Context* ctx, const Matrix* A) {
  if (ctx->adjoint_bands > 0) return ctx->adjoint_bands;
  const int64_t bytes = A->nnz * (int64_t)A->vsize();
  if (bytes <= ((int64_t)96 << 20)) return 1;
  const int64_t nb = (bytes + ((int64_t)64 << 20) - 1) / ((int64_t)64 << 20);
  return (int)std::min<int64_t>(nb, TransposeData::kMaxBands);
}

// The same SDDMM over the SpMV's tile plan (32 lanes x 8 consecutive
// entries per tile): each lane loads its 8 columns with one vector load and
// issues their 8 x gathers together, finds the row of its first entry from
// the tile's row-start flags (as the tile SpMV does) and steps the row at
// each flag.  Same products as sddmm_kernel, in the same arithmetic.
template <typename I, typename V>
__global__ void __launch_bounds__(256) sddmm_tile_kernel(const I* __restrict__ rp, int64_t n, int64_t nnz,
                                                         const I* __restrict__ ci,
                                                         const int64_t* __restrict__ tile_row,
                                                         const uint8_t* __restrict__ flags_all, int64_t tiles,
                                                         const V* __restrict__ g, const V* __restrict__ x,
                                                         V* __restrict__ out, V alpha, bool vec_out) {
  constexpr int K = 8;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;  // lanes below this one
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t t = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; t < tiles; t += nw) {
    const int64_t el = t * (32 * K) + (int64_t)lane * K;
    I c[K];
    if (el + K <= nnz) {
      load_run<I, K>(ci + el, c);
    } else {
#pragma unroll
      for (int b = 0; b < K; ++b) c[b] = el + b < nnz ? ci[el + b] : I(0);
    }
    V xv[K];
#pragma unroll
    for (int b = 0; b < K; ++b) xv[b] = ld_gather(x + c[b]);
    const uint32_t flags = flags_all[t * 32 + lane];
    const int64_t tr = tile_row[t];
    int64_t row;
    if (tr >= 0) {
      const int cnt = __popc(flags);
      int excl = 0;
#pragma unroll
      for (int bit = 0; bit < 4; ++bit) excl += __popc(__ballot_sync(0xffffffffu, (cnt >> bit) & 1) & lt) << bit;
      const int first0 = (int)(__ballot_sync(0xffffffffu, flags & 1u) & 1u);
      row = tr + excl + (int)(flags & 1u) - first0;
    } else {
      row = row_holding(rp, n, el < nnz ? el : nnz - 1);
    }
    V gi = (el < nnz && row < n) ? alpha * g[row] : V(0);
    V o[K];
#pragma unroll
    for (int b = 0; b < K; ++b) {
      if (b > 0 && ((flags >> b) & 1u)) {
        ++row;
        if (tr < 0)
          while (row + 1 < n && rp[row] == rp[row + 1]) ++row;  // skip empty rows
        gi = row < n ? alpha * g[row] : V(0);
      }
      o[b] = gi * xv[b];
    }
    if (vec_out && el + K <= nnz) {  // whole 32-byte sectors: one store request per sector
      store_run<V, K>(out + el, o);
    } else {
#pragma unroll
      for (int b = 0; b < K; ++b)
        if (el + b < nnz) out[el + b] = o[b];
    }
  }
}

template <typename I, typename V>
spops_status_t refresh_values_t(Context* ctx, Matrix* A) {
  TransposeData& T = A->tr;
  if (A->nnz > 0) {
    gather_values_kernel<V><<<grid_for(A->nnz), 256, 0, ctx->stream>>>(T.perm.as<int64_t>(), A->val.as<V>(), A->nnz,
                                                                       T.val.as<V>());
    SPOPS_LAUNCH_CHECK();
  }
  T.values_fresh = true;
  return SPOPS_OK;
}

template <typename I, typename V>
spops_status_t sddmm_t(Context* ctx, Matrix* A, double alpha, const void* g, const void* x, void* out) {
  const CsrPlan& P = A->plan;
  if (P.nblocks == 0) return SPOPS_OK;
  if (ctx->csr_variant == 0 && csr_tile_usable(A, 0)) {  // the tile plan the default SpMV uses
    if (!P.tiles.ready || P.tiles.k != 8) SPOPS_TRY(csr_tile_analyse(ctx, A, 8));
    const CsrTiles& D = A->plan.tiles;
    int64_t grid = (int64_t)ctx->num_sms * 8;
    const int64_t need = (D.tiles + 7) / 8;
    if (grid > need) grid = need;
    if (grid > 0) {
      sddmm_tile_kernel<I, V><<<(unsigned)grid, 256, 0, ctx->stream>>>(
          A->row.as<I>(), A->rows, A->nnz, A->col.as<I>(), D.tile_row.as<int64_t>(), D.flags.as<uint8_t>(), D.tiles,
          static_cast<const V*>(g), static_cast<const V*>(x), static_cast<V*>(out), (V)alpha,
          ((uintptr_t)out % 32) == 0);
      SPOPS_LAUNCH_CHECK();
    }
    return SPOPS_OK;
  }
  int64_t grid = (int64_t)ctx->num_sms * 8;
  const int64_t need = (P.nblocks + 7) / 8;
  if (grid > need) grid = need;
  sddmm_kernel<I, V><<<(unsigned)grid, 256, 0, ctx->stream>>>(A->row.as<I>(), A->col.as<I>(),
                                                              static_cast<const V*>(g), static_cast<const V*>(x),
                                                              static_cast<V*>(out), (V)alpha, P.seg.as<CsrSeg>(),
                                                              P.nblocks);
  SPOPS_LAUNCH_CHECK();
  return SPOPS_OK;
}

#define SPOPS_DISPATCH2(A, FN, ...)                                                             \
  (((A)->itype == SPOPS_INDEX_I32)                                                              \
       ? (((A)->vtype == SPOPS_VALUE_F64) ? FN<int32_t, double>(__VA_ARGS__) : FN<int32_t, float>(__VA_ARGS__)) \
       : (((A)->vtype == SPOPS_VALUE_F64) ? FN<int64_t, double>(__VA_ARGS__) : FN<int64_t, float>(__VA_ARGS__)))

}  // namespace

void TransposeData::release() {
  release_bands(*this);
  rp.release();
  ri.release();
  perm.release();
  val.release();
  if (view) {
    view->release_all();
    delete view;
    view = nullptr;
  }
  ready = false;
  values_fresh = false;
}

spops_status_t csr_spmv_transpose(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  if (A->format != SPOPS_FMT_CSR) return fail(SPOPS_ERR_UNSUPPORTED, "transpose SpMV needs a CSR matrix");
  if (!A->plan.ready) SPOPS_TRY(csr_analyse(ctx, A));
  if (!A->tr.ready) SPOPS_TRY(SPOPS_DISPATCH2(A, build_transpose_t, ctx, A));
  Matrix* V_ = A->tr.view;
  if (!A->tr.values_fresh && ctx->csr_variant == 0 && csr_tile_usable(V_, 0) &&
      ((uintptr_t)A->tr.perm.p % 64) == 0) {
    // values changed since the last refresh (an optimizer step): read A's
    // values through the permutation inside the SpMV; the reordered copy is
    // refreshed only when something asks for it (csr_transpose_view)
    if (!V_->plan.ready) SPOPS_TRY(csr_analyse(ctx, V_));
    const int nb = adjoint_band_count(ctx, A);
    if (nb > 1) {
      // one band of source rows at a time: its slice of A's values stays in
      // L2 while the band's gathers run; the bands add into y in band order
      if (A->tr.nbands != nb) SPOPS_TRY(SPOPS_DISPATCH2(A, build_bands_t, ctx, A, nb));
      bool first = true;  // the first band run applies beta, the others add
      for (int b = 0; b < nb; ++b) {
        if (!A->tr.bview[b]) continue;
        SPOPS_TRY(csr_tile_spmv_indirect(ctx, A->tr.bview[b], A->tr.bperm[b].as<int64_t>(), A->val.p, alpha, x,
                                         first ? beta : 1.0, y));
        first = false;
      }
      if (!first) return SPOPS_OK;
    }
    return csr_tile_spmv_indirect(ctx, V_, A->tr.perm.as<int64_t>(), A->val.p, alpha, x, beta, y);
  }
  if (!A->tr.values_fresh) SPOPS_TRY(SPOPS_DISPATCH2(A, refresh_values_t, ctx, A));
  return csr_spmv(ctx, V_, alpha, x, beta, y);
}

spops_status_t csr_transpose_view(Context* ctx, Matrix* A, Matrix** view) {
  if (A->format != SPOPS_FMT_CSR) return fail(SPOPS_ERR_UNSUPPORTED, "transpose needs a CSR matrix");
  if (!A->plan.ready) SPOPS_TRY(csr_analyse(ctx, A));
  if (!A->tr.ready) SPOPS_TRY(SPOPS_DISPATCH2(A, build_transpose_t, ctx, A));
  if (!A->tr.values_fresh) SPOPS_TRY(SPOPS_DISPATCH2(A, refresh_values_t, ctx, A));
  *view = A->tr.view;
  return SPOPS_OK;
}

spops_status_t csr_sddmm(Context* ctx, Matrix* A, double alpha, const void* g, const void* x, void* out) {
  if (A->format != SPOPS_FMT_CSR) return fail(SPOPS_ERR_UNSUPPORTED, "SDDMM needs a CSR matrix");
  if (!A->plan.ready) SPOPS_TRY(csr_analyse(ctx, A));
  return SPOPS_DISPATCH2(A, sddmm_t, ctx, A, alpha, g, x, out);
}

}  // namespace spops
