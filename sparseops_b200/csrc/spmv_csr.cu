// Kernel choice (spops_set_option "csr_variant"): the tile kernel of
// spmv_csr_tile.cu (entries per lane / resident blocks per SM / next tile
// prefetched) 0 = 8/3/yes (default), 1 = 8/4/no, 5 = 4/4/no, 6 = 8/5/no, used
// when the arrays are aligned for its vector loads; the segment kernel below
// (entries per lane per load round / blocks per SM) 2 = 8/4, 3 = 4/6, 4 = 16/2.
// CSR SpMV y = alpha*A*x + beta*y for sm_100a.
//
// Replaces SpOps_csr (reference src/spmv_csr.cpp:165-185), whose variants are
// a per-row OpenMP loop (93-121) and an nnz-balanced row partition per thread
// (137-162).  The B200 design keeps the nnz balancing at the granularity of a
// warp: the entry stream is cut into SEGMENTS of about kCap entries, and each
// warp streams its segments with coalesced evict-first loads while many warps
// per SM keep enough bytes in flight to cover HBM latency.
//
// Analysis (once per matrix pattern, csr_analyse):
//   a new segment starts where a row's first entry crosses a multiple of kCap
//   entries, every kRowCap rows, and around every LONG row (> kCap entries).
//   A segment of short rows therefore holds fewer than 2*kCap entries and at
//   most kRowCap rows; a long row is split into ceil(len/kCap) chunks, each
//   its own segment.  The column indices are checked once against [0, cols)
//   and the row offsets for monotonicity, so the kernel never gathers outside x.
//
// SpMV: by default the tile kernel of spmv_csr_tile.cu, which keeps products
// in registers; this file's segment kernel (csr_warp_kernel) stages them in
// shared memory and serves unaligned arrays, the batched persistent kernel and
// multi-RHS.  Either way the summation order depends only on the matrix, so
// results are bit-reproducible run to run.
#include <cub/cub.cuh>

#include "device_util.cuh"
#include "spops_internal.h"
#include "warp_work.cuh"

namespace spops {
namespace {

constexpr int kBlock = 256;                 // 8 warps, each on its own segments
constexpr int kCap = kCsrCap;               // entries per long-row chunk; short segments < 2*kCap
constexpr int kRowCap = kCsrRowCap;         // rows per short segment at most
// Kernel choice (spops_set_option "csr_variant"): 0 / 1 the tile kernel of
// spmv_csr_tile.cu with 8 / 4 entries per lane (the default, when the arrays
// are aligned for its vector loads); 2 / 3 / 4 the segment kernel below with
// (entries per lane per load round, resident blocks per SM) = 8/4, 4/6, 16/2.

// ------------------------------------------------------------ analysis
template <typename I>
__global__ void validate_kernel(const I* __restrict__ rp, const I* __restrict__ ci, int64_t n, int64_t nnz,
                                int64_t ncols, int* __restrict__ bad) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r <= n; r += stride) {
    const int64_t a = rp[r];
    if (a < 0 || a > nnz || (r > 0 && (int64_t)rp[r - 1] > a) || (r == 0 && a != 0) || (r == n && a != nnz))
      atomicOr(bad, 1);
  }
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nnz; k += stride) {
    const int64_t c = ci[k];
    if (c < 0 || c >= ncols) atomicOr(bad, 2);
  }
}

template <typename I>
__global__ void plan_count_kernel(const I* __restrict__ rp, int64_t n, int64_t* __restrict__ nblk) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int64_t s = rp[r], e = rp[r + 1];
  const int64_t len = e - s;
  const bool is_long = len > kCap;
  bool flag = true;
  if (r > 0) {
    const int64_t sp = rp[r - 1];
    const bool prev_long = (s - sp) > kCap;
    flag = is_long || prev_long || (s / kCap) != (sp / kCap) || (r % kRowCap) == 0;
  }
  nblk[r] = flag ? (is_long ? (len + kCap - 1) / kCap : 1) : 0;
}

template <typename I>
__global__ void plan_fill_kernel(const I* __restrict__ rp, int64_t n, const int64_t* __restrict__ nblk,
                                 const int64_t* __restrict__ boff, int64_t* __restrict__ blk_row,
                                 int* __restrict__ blk_chunk, int64_t nblocks) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r == 0) blk_row[nblocks] = n;
  if (r >= n) return;
  const int64_t cnt = nblk[r];
  if (cnt == 0) return;
  const bool is_long = (int64_t)(rp[r + 1] - rp[r]) > kCap;
  const int64_t o = boff[r];
  for (int64_t c = 0; c < cnt; ++c) {
    blk_row[o + c] = r;
    blk_chunk[o + c] = is_long ? (int)c : -1;
  }
}

__global__ void count_long_kernel(const int* __restrict__ blk_chunk, int64_t nblocks,
                                  unsigned long long* __restrict__ nlong) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b < nblocks && blk_chunk[b] == 0) atomicAdd(nlong, 1ULL);
}

template <typename I>
__global__ void plan_seg_kernel(const I* __restrict__ rp, const int64_t* __restrict__ blk_row,
                                const int* __restrict__ blk_chunk, int64_t nblocks, CsrSeg* __restrict__ seg) {
  const int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b >= nblocks) return;
  const int64_t r0 = blk_row[b];
  const int c = blk_chunk[b];
  CsrSeg d;
  d.r0 = r0;
  d.chunk = c;
  if (c < 0) {
    const int64_t r1 = blk_row[b + 1];
    d.p0 = rp[r0];
    d.p1 = rp[r1];
    d.nr = (int32_t)(r1 - r0);
  } else {
    const int64_t s = rp[r0], e = rp[r0 + 1];
    d.p0 = s + (int64_t)c * kCap;
    d.p1 = (d.p0 + kCap < e) ? d.p0 + kCap : e;
    d.nr = (int32_t)((e - s + kCap - 1) / kCap);  // chunks of this long row
  }
  seg[b] = d;
}

// ------------------------------------------------------------ the kernel
// One warp per segment, grid-stride over segments.  A short segment (< 2*kCap
// entries, <= kRowCap rows) is loaded with coalesced evict-first loads, kItems
// entries per lane per round with every gather of the round issued before any
// is used; the products go to the warp's shared-memory slice and t = 32/nr
// lanes reduce each row with shuffles.  A long-row chunk (kCap entries) is
// summed in registers; the chunk sum goes to partial[] and the last chunk of
// the row to finish adds all of them (fixed tree) and writes y.
template <typename I, typename V, int kItems, int kMinBlocks>
__global__ void __launch_bounds__(kBlock, kMinBlocks) csr_warp_kernel(
    const I* __restrict__ ci, const V* __restrict__ val, const I* __restrict__ rp, const V* __restrict__ x,
    V* __restrict__ y, V alpha, V beta, bool beta_zero, const CsrSeg* __restrict__ segs, int64_t nseg,
    V* __restrict__ partial, int* __restrict__ counter) {
  __shared__ V prod_all[kBlock / 32][2 * kCap];
  const int lane = threadIdx.x & 31;
  V* prod = prod_all[threadIdx.x >> 5];
  const int64_t nwarps = (int64_t)gridDim.x * (kBlock / 32);
  for (int64_t j = blockIdx.x * (int64_t)(kBlock / 32) + (threadIdx.x >> 5); j < nseg; j += nwarps)
    csr_segment_spmv<I, V, kItems>(segs[j], j, ci, val, rp, x, y, alpha, beta, beta_zero, prod, partial, counter,
                                   lane);
}

template <typename I>
spops_status_t analyse_t(Context* ctx, Matrix* A) {
  CsrPlan& P = A->plan;
  const int64_t n = A->rows;
  const I* rp = A->row.as<I>();
  cudaStream_t st = ctx->stream;
  size_t cub_bytes = 0;
  int64_t* dummy = nullptr;
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, dummy, dummy, (int64_t)(n > 0 ? n : 1), st));
  const size_t arr = ((size_t)(n > 0 ? n : 1) * sizeof(int64_t) + 255) & ~(size_t)255;
  SPOPS_TRY(ctx->scratch_reserve(2 * arr + 256 + cub_bytes));
  char* base = ctx->scratch.as<char>();
  int64_t* nblk = reinterpret_cast<int64_t*>(base);
  int64_t* boff = reinterpret_cast<int64_t*>(base + arr);
  int* bad = reinterpret_cast<int*>(base + 2 * arr);
  void* cub_tmp = base + 2 * arr + 256;

  // validate the pattern once: the kernels index x with these columns
  SPOPS_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), st));
  {
    const int64_t work = (n + 1 > A->nnz ? n + 1 : A->nnz);
    int64_t grid = (work + 255) / 256;
    if (grid > 8 * ctx->num_sms * 8) grid = 8 * ctx->num_sms * 8;
    if (grid < 1) grid = 1;
    validate_kernel<I><<<(unsigned)grid, 256, 0, st>>>(rp, A->col.as<I>(), n, A->nnz, A->cols, bad);
    SPOPS_LAUNCH_CHECK();
  }
  int hbad = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st));

  int64_t nblocks = 0;
  if (n > 0) {
    const int threads = 256;
    const int64_t grid = (n + threads - 1) / threads;
    plan_count_kernel<I><<<(unsigned)grid, threads, 0, st>>>(rp, n, nblk);
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(cub_tmp, cub_bytes, nblk, boff, n, st));
    int64_t last_off = 0, last_cnt = 0;
    SPOPS_CUDA(cudaMemcpyAsync(&last_off, boff + n - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaMemcpyAsync(&last_cnt, nblk + n - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
    nblocks = last_off + last_cnt;
  } else {
    SPOPS_CUDA(cudaStreamSynchronize(st));
  }
  if (hbad) {
    return fail(SPOPS_ERR_INVALID, "CSR pattern invalid: %s%s", (hbad & 1) ? "row offsets not monotone in [0,nnz] " : "",
                (hbad & 2) ? "column index outside [0,cols)" : "");
  }
  P.release();
  P.cap = kCap;
  P.nblocks = nblocks;
  const size_t nb1 = (size_t)(nblocks > 0 ? nblocks : 1);
  SPOPS_TRY(P.blk_row.alloc((size_t)(nblocks + 1) * sizeof(int64_t)));
  SPOPS_TRY(P.blk_chunk.alloc(nb1 * sizeof(int)));
  SPOPS_TRY(P.seg.alloc(nb1 * sizeof(CsrSeg)));
  SPOPS_TRY(P.partial.alloc(nb1 * sizeof(double)));
  SPOPS_TRY(P.counter.alloc(nb1 * sizeof(int)));
  SPOPS_CUDA(cudaMemsetAsync(P.counter.p, 0, P.counter.bytes, st));
  if (n > 0) {
    const int threads = 256;
    const int64_t grid = (n + threads - 1) / threads;
    plan_fill_kernel<I><<<(unsigned)grid, threads, 0, st>>>(rp, n, nblk, boff, P.blk_row.as<int64_t>(),
                                                            P.blk_chunk.as<int>(), nblocks);
    SPOPS_LAUNCH_CHECK();
    if (nblocks > 0) {
      plan_seg_kernel<I><<<(unsigned)((nblocks + 255) / 256), 256, 0, st>>>(
          rp, P.blk_row.as<int64_t>(), P.blk_chunk.as<int>(), nblocks, P.seg.as<CsrSeg>());
      unsigned long long* nl = reinterpret_cast<unsigned long long*>(nblk);  // scratch reuse
      SPOPS_CUDA(cudaMemsetAsync(nl, 0, 8, st));
      count_long_kernel<<<(unsigned)((nblocks + 255) / 256), 256, 0, st>>>(P.blk_chunk.as<int>(), nblocks, nl);
      SPOPS_LAUNCH_CHECK();
      unsigned long long hl = 0;
      SPOPS_CUDA(cudaMemcpyAsync(&hl, nl, 8, cudaMemcpyDeviceToHost, st));
      SPOPS_CUDA(cudaStreamSynchronize(st));
      P.nlong = (int64_t)hl;
    }
  } else {
    SPOPS_CUDA(cudaMemsetAsync(P.blk_row.p, 0, sizeof(int64_t), st));
  }
  P.ready = true;
  return SPOPS_OK;
}

template <typename I, typename V, int kItems, int kMinBlocks>
spops_status_t launch_warp(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  const CsrPlan& P = A->plan;
  static int blocks_per_sm = -1;  // per instantiation
  if (blocks_per_sm < 0) {
    int bps = 0;
    SPOPS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, csr_warp_kernel<I, V, kItems, kMinBlocks>,
                                                             kBlock, 0));
    blocks_per_sm = bps > 0 ? bps : 1;
  }
  int64_t grid = (int64_t)ctx->num_sms * blocks_per_sm;
  const int64_t need = (P.nblocks + kBlock / 32 - 1) / (kBlock / 32);
  if (grid > need) grid = need;
  csr_warp_kernel<I, V, kItems, kMinBlocks><<<(unsigned)grid, kBlock, 0, ctx->stream>>>(
      A->col.as<I>(), A->val.as<V>(), A->row.as<I>(), static_cast<const V*>(x), static_cast<V*>(y), (V)alpha,
      (V)beta, beta == 0.0, P.seg.as<CsrSeg>(), P.nblocks, P.partial.as<V>(), P.counter.as<int>());
  SPOPS_LAUNCH_CHECK();
  return SPOPS_OK;
}

template <typename I, typename V>
spops_status_t spmv_t(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  if (A->rows == 0) return SPOPS_OK;
  switch (ctx->csr_variant) {
    case 2: return launch_warp<I, V, 8, 4>(ctx, A, alpha, x, beta, y);
    case 3: return launch_warp<I, V, 4, 6>(ctx, A, alpha, x, beta, y);
    case 4: return launch_warp<I, V, 16, 2>(ctx, A, alpha, x, beta, y);
    case 7:
    case 8:
    case 9:
      if (csr_win_usable(A)) return csr_win_spmv(ctx, A, ctx->csr_variant, alpha, x, beta, y);
      return launch_warp<I, V, 8, 4>(ctx, A, alpha, x, beta, y);
    default: {
      if (csr_tile_usable(A, ctx->csr_variant)) return csr_tile_spmv(ctx, A, ctx->csr_variant, alpha, x, beta, y);
      return launch_warp<I, V, 8, 4>(ctx, A, alpha, x, beta, y);  // arrays not aligned for vector loads
    }
  }
}

}  // namespace

spops_status_t csr_analyse(Context* ctx, Matrix* A) {
  return A->itype == SPOPS_INDEX_I32 ? analyse_t<int32_t>(ctx, A) : analyse_t<int64_t>(ctx, A);
}

spops_status_t csr_spmv(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  if (!A->plan.ready) SPOPS_TRY(csr_analyse(ctx, A));
  const bool i32 = A->itype == SPOPS_INDEX_I32, f64 = A->vtype == SPOPS_VALUE_F64;
  if (i32 && f64) return spmv_t<int32_t, double>(ctx, A, alpha, x, beta, y);
  if (i32) return spmv_t<int32_t, float>(ctx, A, alpha, x, beta, y);
  if (f64) return spmv_t<int64_t, double>(ctx, A, alpha, x, beta, y);
  return spmv_t<int64_t, float>(ctx, A, alpha, x, beta, y);
}

}  // namespace spops
