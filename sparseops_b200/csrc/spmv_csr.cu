// CSR SpMV y = alpha*A*x + beta*y for sm_100a.
//
// Replaces SpOps_csr (reference src/spmv_csr.cpp:165-185), whose variants are
// a per-row OpenMP loop (93-121) and an nnz-balanced row partition per thread
// (137-162).  The B200 design keeps the nnz balancing but moves it to the
// granularity of a thread block and makes every matrix byte a coalesced,
// streaming load:
//
//   analysis (once per matrix, csr_analyse): rows are cut into SEGMENTS.  A
//   new segment starts where a row's first entry crosses a multiple of kCap
//   entries, every kRowCap rows, and around every LONG row (> kCap entries).
//   A segment of short rows therefore holds < 2*kCap entries; a long row is
//   split into ceil(len/kCap) chunks, one thread block each.
//
//   SpMV (one thread block per segment or chunk):
//     short segment: the block streams col/val of its contiguous entry range
//       (consecutive threads read consecutive entries, evict-first), gathers
//       x through the read-only path, and stores the products in shared
//       memory; then groups of t = 1..32 lanes (t chosen from the segment's
//       rows per block) reduce one row each with warp shuffles.
//     long-row chunk: block-strided products, deterministic block reduction,
//       the chunk sum goes to partial[b]; the last chunk to finish (arrival
//       counter) adds the partials in chunk order and writes y.
//   The summation order is fixed by the matrix alone, so results are
//   bit-reproducible run to run.
#include <cub/cub.cuh>

#include "device_util.cuh"
#include "spops_internal.h"

namespace spops {
namespace {

constexpr int kBlock = 256;
constexpr int kCap = 2048;                  // entries per chunk
constexpr int kRowCap = 1024;               // rows per short segment at most
constexpr int kItems = 2 * kCap / kBlock;   // entries per thread in a short segment (max)

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

template <typename I, typename V>
__global__ void __launch_bounds__(kBlock) csr_stream_kernel(
    const I* __restrict__ rp, const I* __restrict__ ci, const V* __restrict__ val, const V* __restrict__ x,
    V* __restrict__ y, V alpha, V beta, bool beta_zero, const int64_t* __restrict__ blk_row,
    const int* __restrict__ blk_chunk, V* __restrict__ partial, int* __restrict__ counter) {
  __shared__ V prod[2 * kCap];
  __shared__ V red[kBlock / 32];
  const int64_t b = blockIdx.x;
  const int64_t r0 = blk_row[b];
  const int chunk = blk_chunk[b];
  const int tid = threadIdx.x;

  if (chunk < 0) {
    // ---------------------------------------------------- short segment
    const int64_t r1 = blk_row[b + 1];
    const int64_t p0 = rp[r0];
    const int m = (int)((int64_t)rp[r1] - p0);
    const I* cseg = ci + p0;
    const V* vseg = val + p0;
    I c[kItems];
    V a[kItems];
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const int k = tid + it * kBlock;
      if (k < m) {
        c[it] = ld_stream(cseg + k);
        a[it] = ld_stream(vseg + k);
      }
    }
#pragma unroll
    for (int it = 0; it < kItems; ++it) {
      const int k = tid + it * kBlock;
      if (k < m) prod[k] = a[it] * ld_gather(x + c[it]);
    }
    __syncthreads();

    const int nr = (int)(r1 - r0);
    int t = kBlock / (nr > 0 ? nr : 1);
    t = t >= 32 ? 32 : t >= 16 ? 16 : t >= 8 ? 8 : t >= 4 ? 4 : t >= 2 ? 2 : 1;
    const int groups = kBlock / t;
    const int g = tid / t, lane = tid % t;
    for (int base = 0; base < nr; base += groups) {
      const int rr = base + g;
      V sum = V(0);
      if (rr < nr) {
        const int s = (int)((int64_t)rp[r0 + rr] - p0), e = (int)((int64_t)rp[r0 + rr + 1] - p0);
        for (int k = s + lane; k < e; k += t) sum += prod[k];
      }
      sum = warp_sum(sum, t);
      if (rr < nr && lane == 0) axpby_store(y + r0 + rr, sum, alpha, beta, beta_zero);
    }
  } else {
    // ------------------------------------------------- long-row chunk
    const int64_t s = rp[r0], e = rp[r0 + 1];
    const int64_t p0 = s + (int64_t)chunk * kCap;
    const int64_t p1 = (p0 + kCap < e) ? p0 + kCap : e;
    V sum = V(0);
    for (int64_t k = p0 + tid; k < p1; k += kBlock) sum += ld_stream(val + k) * ld_gather(x + ld_stream(ci + k));
    sum = block_sum(sum, red);
    if (tid == 0) {
      const int nchunks = (int)((e - s + kCap - 1) / kCap);
      const int64_t first = b - chunk;
      partial[b] = sum;
      __threadfence();
      const int prev = atomicAdd(counter + first, 1);
      if (prev == nchunks - 1) {
        __threadfence();
        V tot = V(0);
        for (int q = 0; q < nchunks; ++q) tot += ld_cg(partial + first + q);
        axpby_store(y + r0, tot, alpha, beta, beta_zero);
        counter[first] = 0;
      }
    }
  }
}

template <typename I>
spops_status_t analyse_t(Context* ctx, Matrix* A) {
  CsrPlan& P = A->plan;
  const int64_t n = A->rows;
  const I* rp = A->row.as<I>();
  cudaStream_t st = ctx->stream;
  // scratch: nblk[n], boff[n], total (int64), CUB temp
  size_t cub_bytes = 0;
  int64_t* dummy = nullptr;
  SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, cub_bytes, dummy, dummy, (int64_t)(n > 0 ? n : 1), st));
  const size_t arr = ((size_t)(n > 0 ? n : 1) * sizeof(int64_t) + 255) & ~(size_t)255;
  SPOPS_TRY(ctx->scratch_reserve(2 * arr + 256 + cub_bytes));
  char* base = ctx->scratch.as<char>();
  int64_t* nblk = reinterpret_cast<int64_t*>(base);
  int64_t* boff = reinterpret_cast<int64_t*>(base + arr);
  void* cub_tmp = base + 2 * arr + 256;
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
  }
  P.release();
  P.cap = kCap;
  P.nblocks = nblocks;
  SPOPS_TRY(P.blk_row.alloc((size_t)(nblocks + 1) * sizeof(int64_t)));
  SPOPS_TRY(P.blk_chunk.alloc((size_t)(nblocks > 0 ? nblocks : 1) * sizeof(int)));
  SPOPS_TRY(P.partial.alloc((size_t)(nblocks > 0 ? nblocks : 1) * sizeof(double)));
  SPOPS_TRY(P.counter.alloc((size_t)(nblocks > 0 ? nblocks : 1) * sizeof(int)));
  SPOPS_CUDA(cudaMemsetAsync(P.counter.p, 0, P.counter.bytes, st));
  if (n > 0) {
    const int threads = 256;
    const int64_t grid = (n + threads - 1) / threads;
    plan_fill_kernel<I><<<(unsigned)grid, threads, 0, st>>>(rp, n, nblk, boff, P.blk_row.as<int64_t>(),
                                                            P.blk_chunk.as<int>(), nblocks);
    SPOPS_LAUNCH_CHECK();
  } else {
    SPOPS_CUDA(cudaMemsetAsync(P.blk_row.p, 0, sizeof(int64_t), st));
  }
  P.ready = true;
  return SPOPS_OK;
}

template <typename I, typename V>
spops_status_t spmv_t(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  const CsrPlan& P = A->plan;
  if (P.nblocks == 0) return SPOPS_OK;
  if (P.nblocks > INT32_MAX) return fail(SPOPS_ERR_TOO_LARGE, "CSR SpMV: %lld row blocks", (long long)P.nblocks);
  csr_stream_kernel<I, V><<<(unsigned)P.nblocks, kBlock, 0, ctx->stream>>>(
      A->row.as<I>(), A->col.as<I>(), A->val.as<V>(), static_cast<const V*>(x), static_cast<V*>(y), (V)alpha,
      (V)beta, beta == 0.0, P.blk_row.as<int64_t>(), P.blk_chunk.as<int>(), P.partial.as<V>(),
      P.counter.as<int>());
  SPOPS_LAUNCH_CHECK();
  return SPOPS_OK;
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
