// CSR SpMV y = alpha*A*x + beta*y for sm_100a.
//
// Replaces SpOps_csr (reference src/spmv_csr.cpp:165-185), whose variants are
// a per-row OpenMP loop (93-121) and an nnz-balanced row partition per thread
// (137-162).  The B200 design keeps the nnz balancing, at the granularity of a
// SEGMENT of the entry stream, and streams every matrix byte with bulk copies
// (TMA, cp.async.bulk) so that several segments per SM are always in flight.
//
// Analysis (once per matrix pattern, csr_analyse):
//   rows are cut into segments.  A new segment starts where a row's first
//   entry crosses a multiple of kCap entries, every kRowCap rows, and around
//   every LONG row (> kCap entries).  A segment of short rows therefore holds
//   fewer than 2*kCap entries and at most kRowCap rows; a long row is split
//   into ceil(len/kCap) chunks, each its own segment.  The column indices are
//   checked once against [0, cols) and the row offsets for monotonicity, so
//   the kernels never gather outside x.
//
// SpMV, pipelined kernel (csr_pipe_kernel; persistent, ~2 blocks per SM):
//   each block walks segments b, b+G, b+2G, ... through an S-stage ring of
//   shared-memory buffers.  Thread 0 bulk-copies a segment's values, column
//   indices and row offsets (16-byte aligned windows; the unaligned tail of
//   the arrays is loaded with plain loads) and signals an mbarrier; all
//   threads wait on it (bounded), gather x through the read-only path and
//   reduce: short segments with t = 1..32 lanes per row and warp shuffles,
//   long-row chunks with a block reduction whose result goes to partial[];
//   the last chunk of a long row to finish (arrival counter) adds the
//   partials in chunk order.  The buffer is refilled with segment b + S*G as
//   soon as the block is done with it.
//   The summation order depends only on the matrix, so results are
//   bit-reproducible run to run.
// SpMV, plain kernel (csr_stream_kernel): the same segments without bulk
//   copies, one block per segment; used when the arrays are not 16-byte
//   aligned (borrowed pointers into the middle of a buffer).
#include <cub/cub.cuh>

#include "device_util.cuh"
#include "spops_internal.h"
#include "tma_util.cuh"

namespace spops {
namespace {

constexpr int kBlock = 256;
constexpr int kCap = 1024;                  // entries per chunk
constexpr int kRowCap = 512;                // rows per short segment at most
constexpr int kItems = 2 * kCap / kBlock;   // entries per thread in a short segment (plain kernel)
constexpr int kStages = 4;                  // pipelined kernel: buffers per block
constexpr int kEBuf = 2 * kCap + 8;         // entries per stage (16-byte aligned windows)
constexpr int kRBuf = kRowCap + 8;          // row offsets per stage

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

// ------------------------------------------------------ shared reduction
// Reduce the rows of a short segment whose products (or value/column pairs)
// live in shared memory.  `entry(k)` returns the product of local entry k,
// `row_start(rr)` the local offset of row rr (rr = 0..nr).
template <typename V, typename EntryF, typename RowF>
__device__ __forceinline__ void reduce_rows(int nr, int64_t r0, EntryF entry, RowF row_start, V* __restrict__ y,
                                            V alpha, V beta, bool beta_zero) {
  const int tid = threadIdx.x;
  int t = kBlock / (nr > 0 ? nr : 1);
  t = t >= 32 ? 32 : t >= 16 ? 16 : t >= 8 ? 8 : t >= 4 ? 4 : t >= 2 ? 2 : 1;
  const int groups = kBlock / t;
  const int g = tid / t, lane = tid % t;
  for (int base = 0; base < nr; base += groups) {
    const int rr = base + g;
    V s0 = V(0), s1 = V(0);
    if (rr < nr) {
      const int s = row_start(rr), e = row_start(rr + 1);
      int k = s + lane;
      for (; k + t < e; k += 2 * t) {
        s0 += entry(k);
        s1 += entry(k + t);
      }
      if (k < e) s0 += entry(k);
    }
    V sum = warp_sum(s0 + s1, t);
    if (rr < nr && lane == 0) axpby_store(y + r0 + rr, sum, alpha, beta, beta_zero);
  }
}

// Long-row chunk epilogue: record the chunk sum; the last chunk to arrive
// adds all chunk sums of the row in order and writes y.
template <typename V>
__device__ __forceinline__ void long_row_finish(V sum, int64_t b, int chunk, int nchunks, int64_t row,
                                                V* __restrict__ partial, int* __restrict__ counter,
                                                V* __restrict__ y, V alpha, V beta, bool beta_zero) {
  const int64_t first = b - chunk;
  partial[b] = sum;
  __threadfence();
  const int prev = atomicAdd(counter + first, 1);
  if (prev == nchunks - 1) {
    __threadfence();
    V tot = V(0);
    for (int q = 0; q < nchunks; ++q) tot += ld_cg(partial + first + q);
    axpby_store(y + row, tot, alpha, beta, beta_zero);
    counter[first] = 0;
  }
}

// ------------------------------------------------------ pipelined kernel
template <typename I, typename V>
struct PipeSmem {
  static constexpr size_t val_bytes = (size_t)kStages * kEBuf * sizeof(V);
  static constexpr size_t col_bytes = (size_t)kStages * kEBuf * sizeof(I);
  static constexpr size_t rp_bytes = (size_t)kStages * kRBuf * sizeof(I);
  static constexpr size_t bar_off = (val_bytes + col_bytes + rp_bytes + 15) & ~(size_t)15;
  static constexpr size_t total = bar_off + kStages * sizeof(uint64_t) + (kBlock / 32) * sizeof(V) + 16;
};

template <typename I, typename V>
__device__ __forceinline__ void pipe_issue(const CsrSeg& d, int s, const I* __restrict__ rp,
                                           const I* __restrict__ ci, const V* __restrict__ val, int64_t nnz,
                                           int64_t n, V* sval, I* scol, I* srp, uint64_t* bar) {
  int64_t ws = d.p0 & ~3LL, we = (d.p1 + 3) & ~3LL;
  const int64_t nnz4 = nnz & ~3LL;
  if (we > nnz4) we = nnz4;
  if (we < ws) we = ws;
  int64_t ra = 0, rb = 0;
  if (d.chunk < 0) {
    ra = d.r0 & ~3LL;
    rb = (d.r0 + d.nr + 1 + 3) & ~3LL;
    const int64_t n4 = (n + 1) & ~3LL;
    if (rb > n4) rb = n4;
    if (rb < ra) rb = ra;
  }
  const uint32_t eb = (uint32_t)(we - ws), rbn = (uint32_t)(rb - ra);
  mbar_arrive_expect_tx(bar, eb * (uint32_t)(sizeof(I) + sizeof(V)) + rbn * (uint32_t)sizeof(I));
  if (eb) {
    bulk_load(sval + (size_t)s * kEBuf, val + ws, eb * (uint32_t)sizeof(V), bar);
    bulk_load(scol + (size_t)s * kEBuf, ci + ws, eb * (uint32_t)sizeof(I), bar);
  }
  if (rbn) bulk_load(srp + (size_t)s * kRBuf, rp + ra, rbn * (uint32_t)sizeof(I), bar);
}

template <typename I, typename V>
__global__ void __launch_bounds__(kBlock) csr_pipe_kernel(
    const I* __restrict__ rp, const I* __restrict__ ci, const V* __restrict__ val, const V* __restrict__ x,
    V* __restrict__ y, V alpha, V beta, bool beta_zero, const CsrSeg* __restrict__ segs, int64_t nseg,
    int64_t nnz, int64_t n, V* __restrict__ partial, int* __restrict__ counter, int* __restrict__ err) {
  using L = PipeSmem<I, V>;
  extern __shared__ __align__(128) unsigned char smem[];
  V* sval = reinterpret_cast<V*>(smem);
  I* scol = reinterpret_cast<I*>(smem + L::val_bytes);
  I* srp = reinterpret_cast<I*>(smem + L::val_bytes + L::col_bytes);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::bar_off);
  V* red = reinterpret_cast<V*>(smem + L::bar_off + kStages * sizeof(uint64_t));
  const int tid = threadIdx.x;
  const int64_t G = gridDim.x;

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(bars + s, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      const int64_t j = blockIdx.x + s * G;
      if (j < nseg) pipe_issue<I, V>(segs[j], s, rp, ci, val, nnz, n, sval, scol, srp, bars + s);
    }
  }

  int64_t it = 0;
  for (int64_t j = blockIdx.x; j < nseg; j += G, ++it) {
    const int s = (int)(it % kStages);
    const uint32_t parity = (uint32_t)((it / kStages) & 1);
    const bool ok = mbar_wait(bars + s, parity);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) atomicOr(err, 1);
      return;
    }
    const CsrSeg d = segs[j];
    V* sv = sval + (size_t)s * kEBuf;
    I* sc = scol + (size_t)s * kEBuf;
    I* sr = srp + (size_t)s * kRBuf;
    const int64_t ws = d.p0 & ~3LL;
    int64_t we = (d.p1 + 3) & ~3LL;
    if (we > (nnz & ~3LL)) we = nnz & ~3LL;
    if (we < ws) we = ws;
    // entries beyond the last aligned 16-byte boundary of the arrays
    for (int64_t k = (we > d.p0 ? we : d.p0) + tid; k < d.p1; k += kBlock) {
      sv[k - ws] = val[k];
      sc[k - ws] = ci[k];
    }
    if (d.chunk < 0) {
      const int64_t ra = d.r0 & ~3LL;
      int64_t rb = (d.r0 + d.nr + 1 + 3) & ~3LL;
      if (rb > ((n + 1) & ~3LL)) rb = (n + 1) & ~3LL;
      if (rb < ra) rb = ra;
      for (int64_t r = (rb > d.r0 ? rb : d.r0) + tid; r <= d.r0 + d.nr; r += kBlock) {
        sr[r - ra] = rp[r];
      }
      __syncthreads();  // plain-loaded tails visible to all threads
      const int off0 = (int)(d.r0 - ra);
      const int64_t base = ws;
      reduce_rows<V>(
          d.nr, d.r0, [&](int k) { return sv[k] * ld_gather(x + sc[k]); },
          [&](int rr) { return (int)((int64_t)sr[off0 + rr] - base); }, y, alpha, beta, beta_zero);
    } else {
      __syncthreads();
      V sum = V(0);
      const int a = (int)(d.p0 - ws), e = (int)(d.p1 - ws);
      for (int k = a + tid; k < e; k += kBlock) sum += sv[k] * ld_gather(x + sc[k]);
      sum = block_sum(sum, red);
      if (tid == 0) long_row_finish(sum, j, d.chunk, d.nr, d.r0, partial, counter, y, alpha, beta, beta_zero);
    }
    __syncthreads();  // everyone is done with stage s
    if (tid == 0) {
      const int64_t jn = j + kStages * G;
      if (jn < nseg) {
        fence_proxy_async_smem();
        pipe_issue<I, V>(segs[jn], s, rp, ci, val, nnz, n, sval, scol, srp, bars + s);
      }
    }
  }
}

// ---------------------------------------------------------- plain kernel
template <typename I, typename V>
__global__ void __launch_bounds__(kBlock) csr_stream_kernel(
    const I* __restrict__ rp, const I* __restrict__ ci, const V* __restrict__ val, const V* __restrict__ x,
    V* __restrict__ y, V alpha, V beta, bool beta_zero, const CsrSeg* __restrict__ segs, V* __restrict__ partial,
    int* __restrict__ counter) {
  __shared__ V prod[2 * kCap];
  __shared__ V red[kBlock / 32];
  const int64_t b = blockIdx.x;
  const CsrSeg d = segs[b];
  const int tid = threadIdx.x;
  if (d.chunk < 0) {
    const int m = (int)(d.p1 - d.p0);
    const I* cseg = ci + d.p0;
    const V* vseg = val + d.p0;
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
    const int64_t p0 = d.p0;
    reduce_rows<V>(
        d.nr, d.r0, [&](int k) { return prod[k]; }, [&](int rr) { return (int)((int64_t)rp[d.r0 + rr] - p0); },
        y, alpha, beta, beta_zero);
  } else {
    V sum = V(0);
    for (int64_t k = d.p0 + tid; k < d.p1; k += kBlock) sum += ld_stream(val + k) * ld_gather(x + ld_stream(ci + k));
    sum = block_sum(sum, red);
    if (tid == 0) long_row_finish(sum, b, d.chunk, d.nr, d.r0, partial, counter, y, alpha, beta, beta_zero);
  }
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
      SPOPS_LAUNCH_CHECK();
    }
  } else {
    SPOPS_CUDA(cudaMemsetAsync(P.blk_row.p, 0, sizeof(int64_t), st));
  }
  // bulk copies need 16-byte aligned array bases
  auto al = [](const void* p) { return ((uintptr_t)p & 15) == 0; };
  P.pipelined = al(A->row.p) && al(A->col.p) && al(A->val.p);
  P.ready = true;
  return SPOPS_OK;
}

template <typename I, typename V>
spops_status_t spmv_t(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  const CsrPlan& P = A->plan;
  if (P.nblocks == 0) return SPOPS_OK;
  const bool bz = beta == 0.0;
  if (P.pipelined && !ctx->force_plain) {
    using L = PipeSmem<I, V>;
    static int blocks_per_sm = -1;  // per (I, V) instantiation
    if (blocks_per_sm < 0) {
      SPOPS_CUDA(cudaFuncSetAttribute(csr_pipe_kernel<I, V>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)L::total));
      int bps = 0;
      SPOPS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, csr_pipe_kernel<I, V>, kBlock, L::total));
      blocks_per_sm = bps > 0 ? bps : 1;
    }
    int64_t grid = (int64_t)ctx->num_sms * blocks_per_sm;
    if (grid > P.nblocks) grid = P.nblocks;
    SPOPS_TRY(ctx->ensure_errword());
    csr_pipe_kernel<I, V><<<(unsigned)grid, kBlock, L::total, ctx->stream>>>(
        A->row.as<I>(), A->col.as<I>(), A->val.as<V>(), static_cast<const V*>(x), static_cast<V*>(y), (V)alpha,
        (V)beta, bz, P.seg.as<CsrSeg>(), P.nblocks, A->nnz, A->rows, P.partial.as<V>(), P.counter.as<int>(),
        ctx->errword.as<int>());
    SPOPS_LAUNCH_CHECK();
    return SPOPS_OK;
  }
  if (P.nblocks > INT32_MAX) return fail(SPOPS_ERR_TOO_LARGE, "CSR SpMV: %lld segments", (long long)P.nblocks);
  csr_stream_kernel<I, V><<<(unsigned)P.nblocks, kBlock, 0, ctx->stream>>>(
      A->row.as<I>(), A->col.as<I>(), A->val.as<V>(), static_cast<const V*>(x), static_cast<V*>(y), (V)alpha,
      (V)beta, bz, P.seg.as<CsrSeg>(), P.partial.as<V>(), P.counter.as<int>());
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
