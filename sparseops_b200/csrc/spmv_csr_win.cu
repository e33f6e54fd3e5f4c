// CSR SpMV by column-sorted row windows (csr_variant 7, 8, 9).
//
// Why: on B200 a gather of x costs one L1 -> L2 request per distinct line a
// warp instruction touches, and the SM's request port serves about one per
// cycle.  Row-ordered kernels over a matrix with columns spread across a large
// x issue one request per entry.  Visiting a large block of entries in column
// order lets neighbouring lanes share lines: on the 4.2M-row power-law matrix
// (windows of ~700K entries) the x requests to L2 drop about 3x and the port
// falls from ~80 % to ~19 % busy.  The price is the scatter of products into
// the window's partial y in shared memory: FP64 shared-memory additions are
// compare-and-swap loops on sm_100a, and while x stays in L2 they cost more
// than the gathers saved (0.56 ms against 0.47 ms for the default tile
// kernel on that matrix).  The layout pays off when x is far larger than L2
// and the row-ordered gathers reach HBM.
//
// Layout (built once per matrix, csr_win_analyse):
//   windows     contiguous row ranges [win_row0[w], win_row0[w+1]) of at most
//               `cap` rows, balanced by entries, one (variant 7), two (8) or
//               four (9) per SM; a window's partial y fits in shared memory
//   tiles       a window's entries sorted by (column, row) and cut into tiles
//               of 32; tile t of window w is win_tile0[w] + local index
//   tbase[t]    first (smallest) column of tile t, or -1 - e when the tile's
//               columns span more than 65535 and are stored in full at
//               tesc[e*32 .. e*32+31]
//   tidx[t*32+l]  (local row << 16) | (column - tbase[t]); local row 0xFFFF
//               marks padding after a window's last entry
//   tval[t*32+l]  the entry's value, a copy refreshed after spops_csr_set_values
//               through tperm[t*32+l] (the entry's CSR index, -1 for padding)
// The SpMV reads 12 bytes per entry plus 4 per tile, as for the CSR arrays.
//
// SpMV (csr_win_kernel): one CTA per window; the window's partial sums live in
// shared memory (zeroed, accumulated with shared-memory atomics, then written
// as y = alpha*partial + beta*y with coalesced stores).  Warps stream their
// tiles with evict-first loads and gather x through L1.
//
// Summation order: the entries of a row are added in column order, but
// concurrent warps add to the same row in an order the hardware chooses, so
// results can differ from run to run at rounding level (the row-ordered
// variants 0-6 are bit-reproducible).
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "device_util.cuh"
#include "spops_internal.h"

namespace spops {
namespace {

constexpr uint32_t kPadRow = 0xFFFFu;
constexpr int kWinUnroll = 4;  // tiles in flight per warp

inline unsigned grid_of(int64_t work, int threads = 256) {
  int64_t g = (work + threads - 1) / threads;
  return (unsigned)(g < 1 ? 1 : g);
}

// last w with cut[w] <= v, for a sorted cut array of m + 1 entries
__device__ __forceinline__ int64_t upper_index(const int64_t* cut, int64_t m, int64_t v) {
  int64_t lo = 0, hi = m;
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (cut[mid] <= v) lo = mid; else hi = mid;
  }
  return lo;
}

// One warp per row: sort key (window, column) and the entry's index.
template <typename I>
__global__ void win_key_kernel(const I* __restrict__ rp, const I* __restrict__ ci, int64_t n,
                               const int64_t* __restrict__ win_row0, int64_t nwin, int cbits,
                               uint64_t* __restrict__ key, int32_t* __restrict__ ent) {
  const int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const int64_t w = upper_index(win_row0, nwin, r);
  const int64_t e0 = rp[r], e1 = rp[r + 1];
  for (int64_t k = e0 + lane; k < e1; k += 32) {
    key[k] = ((uint64_t)w << cbits) | (uint64_t)ci[k];
    ent[k] = (int32_t)k;
  }
}

// One thread per tile: window, first column, and whether the span needs the
// full-column escape.
__global__ void win_tile_kernel(const uint64_t* __restrict__ skey, uint64_t cmask, const int64_t* __restrict__ win_e0,
                                const int64_t* __restrict__ win_tile0, int64_t nwin, int64_t ntiles,
                                int32_t* __restrict__ tile_win, int64_t* __restrict__ tile_col,
                                int64_t* __restrict__ esc_flag) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= ntiles) return;
  const int64_t w = upper_index(win_tile0, nwin, t);
  const int64_t s0 = win_e0[w] + (t - win_tile0[w]) * 32;
  const int64_t s1 = std::min(s0 + 32, win_e0[w + 1]);
  const int64_t c0 = (int64_t)(skey[s0] & cmask), c1 = (int64_t)(skey[s1 - 1] & cmask);
  tile_win[t] = (int32_t)w;
  tile_col[t] = c0;
  esc_flag[t] = (c1 - c0 > 0xFFFF) ? 1 : 0;
}

// One thread per tile slot.
template <typename I, typename V>
__global__ void win_fill_kernel(const I* __restrict__ rp, const V* __restrict__ val, const uint64_t* __restrict__ skey,
                                const int32_t* __restrict__ sent, uint64_t cmask, const int64_t* __restrict__ win_row0,
                                const int64_t* __restrict__ win_e0, const int64_t* __restrict__ win_tile0,
                                const int32_t* __restrict__ tile_win, const int64_t* __restrict__ tile_col,
                                const int64_t* __restrict__ esc_flag, const int64_t* __restrict__ esc_idx,
                                int64_t ntiles, int32_t* __restrict__ tbase, uint32_t* __restrict__ tidx,
                                V* __restrict__ tval, int32_t* __restrict__ tperm, int32_t* __restrict__ tesc) {
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= ntiles * 32) return;
  const int64_t t = g >> 5;
  const int lane = (int)(g & 31);
  const int64_t w = tile_win[t];
  const int64_t s = win_e0[w] + (t - win_tile0[w]) * 32 + lane;
  const bool esc = esc_flag[t] != 0;
  const int64_t base = tile_col[t];
  uint32_t id = kPadRow << 16;
  V v = V(0);
  int64_t col = 0;
  int32_t k = -1;
  if (s < win_e0[w + 1]) {
    k = sent[s];
    col = (int64_t)(skey[s] & cmask);
    // row holding entry k inside the window's rows
    int64_t lo = win_row0[w], hi = win_row0[w + 1];
    while (hi - lo > 1) {
      const int64_t mid = (lo + hi) >> 1;
      if ((int64_t)rp[mid] <= k) lo = mid; else hi = mid;
    }
    id = ((uint32_t)(lo - win_row0[w]) << 16) | (esc ? 0u : (uint32_t)(col - base));
    v = val[k];
  }
  tidx[g] = id;
  tval[g] = v;
  tperm[g] = k;
  if (esc) tesc[esc_idx[t] * 32 + lane] = (int32_t)col;
  if (lane == 0) tbase[t] = esc ? (int32_t)(-1 - esc_idx[t]) : (int32_t)base;
}

// New values for an unchanged pattern: tval[g] = val[tperm[g]].
template <typename V>
__global__ void win_values_kernel(const V* __restrict__ val, const int32_t* __restrict__ tperm, int64_t slots,
                                  V* __restrict__ tval) {
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= slots) return;
  const int32_t k = tperm[g];
  tval[g] = k >= 0 ? val[k] : V(0);
}

template <typename V, int kThreads, int kPerSm>
__global__ void __launch_bounds__(kThreads, kPerSm) csr_win_kernel(
    const int64_t* __restrict__ win_row0, const int64_t* __restrict__ win_tile0, int64_t nwin,
    const int32_t* __restrict__ tbase, const uint32_t* __restrict__ tidx, const V* __restrict__ tval,
    const int32_t* __restrict__ tesc, const V* __restrict__ x, V alpha, V beta, bool beta_zero, V* __restrict__ y) {
  extern __shared__ __align__(16) unsigned char win_smem[];
  V* part = reinterpret_cast<V*>(win_smem);
  constexpr int kWarps = kThreads / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t w = blockIdx.x; w < nwin; w += gridDim.x) {
    const int64_t r0 = win_row0[w], rows = win_row0[w + 1] - r0;
    for (int64_t i = threadIdx.x; i < rows; i += kThreads) part[i] = V(0);
    __syncthreads();
    const int64_t t0 = win_tile0[w], t1 = win_tile0[w + 1];
    for (int64_t t = t0 + (int64_t)warp * kWinUnroll; t < t1; t += (int64_t)kWarps * kWinUnroll) {
      uint32_t id[kWinUnroll];
      V v[kWinUnroll];
      int32_t b[kWinUnroll];
#pragma unroll
      for (int u = 0; u < kWinUnroll; ++u) {
        const int64_t tt = t + u;
        if (tt < t1) {
          b[u] = __ldg(tbase + tt);
          id[u] = __ldcs(tidx + tt * 32 + lane);
          v[u] = ld_stream(tval + tt * 32 + lane);
        } else {
          b[u] = 0;
          id[u] = kPadRow << 16;
          v[u] = V(0);
        }
      }
      V xv[kWinUnroll];
#pragma unroll
      for (int u = 0; u < kWinUnroll; ++u) {
        xv[u] = V(0);
        if ((id[u] >> 16) != kPadRow) {
          const int64_t col = b[u] >= 0 ? (int64_t)b[u] + (int64_t)(id[u] & 0xFFFFu)
                                        : (int64_t)__ldg(tesc + (int64_t)(-1 - b[u]) * 32 + lane);
          xv[u] = ld_gather(x + col);
        }
      }
      // FP64 shared-memory additions are compare-and-swap loops on sm_100a;
      // they, not the gathers, bound this kernel when x fits in L2
#pragma unroll
      for (int u = 0; u < kWinUnroll; ++u)
        if ((id[u] >> 16) != kPadRow) atomicAdd(part + (id[u] >> 16), v[u] * xv[u]);
    }
    __syncthreads();
    for (int64_t i = threadIdx.x; i < rows; i += kThreads) axpby_store(y + r0 + i, part[i], alpha, beta, beta_zero);
    __syncthreads();
  }
}

int per_sm_of(int variant) { return variant == 9 ? 4 : (variant == 8 ? 2 : 1); }

// Greedy windows over the host row offsets: each closes once it holds its
// share of the remaining entries or reaches `cap` rows.
void make_windows(const std::vector<int64_t>& rp, int64_t n, int64_t cap, int64_t target_windows,
                  std::vector<int64_t>& row0) {
  row0.clear();
  row0.push_back(0);
  const int64_t nnz = rp[n];
  int64_t a = 0;
  while (a < n) {
    const int64_t left = std::max<int64_t>(1, target_windows - (int64_t)row0.size() + 1);
    const int64_t share = std::max<int64_t>(1, (nnz - rp[a] + left - 1) / left);
    int64_t b = a + 1;
    while (b < n && b - a < cap && rp[b] - rp[a] < share) ++b;
    row0.push_back(b);
    a = b;
  }
}

template <typename I, typename V>
spops_status_t analyse_t(Context* ctx, Matrix* A, int variant) {
  CsrWin& W = A->plan.win;
  W.release();
  cudaStream_t st = ctx->stream;
  const int64_t n = A->rows, nnz = A->nnz;
  const int per_sm = per_sm_of(variant);
  int smem_sm = 0, smem_blk = 0;
  SPOPS_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->device));
  SPOPS_CUDA(cudaDeviceGetAttribute(&smem_blk, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
  const int64_t budget = std::min<int64_t>(smem_blk, smem_sm / per_sm - 1024) - 64;
  const int64_t cap = std::min<int64_t>(budget / (int64_t)sizeof(V), (int64_t)kPadRow - 1);
  if (cap < 32) return fail(SPOPS_ERR_UNSUPPORTED, "csr windows: no shared memory for a window");
  // host row offsets
  std::vector<int64_t> hrp((size_t)n + 1);
  if (sizeof(I) == 8) {
    SPOPS_CUDA(cudaMemcpyAsync(hrp.data(), A->row.p, hrp.size() * 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
  } else {
    std::vector<int32_t> r32(hrp.size());
    SPOPS_CUDA(cudaMemcpyAsync(r32.data(), A->row.p, r32.size() * 4, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
    std::copy(r32.begin(), r32.end(), hrp.begin());
  }
  // the fewest whole waves of windows (a multiple of the resident CTAs) that
  // the greedy cut meets
  const int64_t slots = (int64_t)ctx->num_sms * per_sm;
  int64_t target = slots * std::max<int64_t>(1, (n + slots * cap - 1) / (slots * cap));
  std::vector<int64_t> row0;
  for (int tries = 0;; ++tries) {
    make_windows(hrp, n, cap, target, row0);
    if ((int64_t)row0.size() - 1 <= target || tries == 16) break;
    target += slots;
  }
  const int64_t nwin = (int64_t)row0.size() - 1;
  std::vector<int64_t> e0((size_t)nwin + 1), tile0((size_t)nwin + 1, 0);
  int64_t max_rows = 1;
  for (int64_t w = 0; w <= nwin; ++w) e0[w] = hrp[row0[w]];
  for (int64_t w = 0; w < nwin; ++w) {
    tile0[w + 1] = tile0[w] + (e0[w + 1] - e0[w] + 31) / 32;
    max_rows = std::max(max_rows, row0[w + 1] - row0[w]);
  }
  const int64_t ntiles = tile0[nwin];
  SPOPS_TRY(W.win_row0.alloc((size_t)(nwin + 1) * 8));
  SPOPS_TRY(W.win_tile0.alloc((size_t)(nwin + 1) * 8));
  SPOPS_TRY(W.tbase.alloc((size_t)std::max<int64_t>(ntiles, 1) * 4));
  SPOPS_TRY(W.tidx.alloc((size_t)std::max<int64_t>(ntiles, 1) * 32 * 4));
  SPOPS_TRY(W.tval.alloc((size_t)std::max<int64_t>(ntiles, 1) * 32 * sizeof(V)));
  SPOPS_TRY(W.tperm.alloc((size_t)std::max<int64_t>(ntiles, 1) * 32 * 4));
  SPOPS_CUDA(cudaMemcpyAsync(W.win_row0.p, row0.data(), (size_t)(nwin + 1) * 8, cudaMemcpyHostToDevice, st));
  SPOPS_CUDA(cudaMemcpyAsync(W.win_tile0.p, tile0.data(), (size_t)(nwin + 1) * 8, cudaMemcpyHostToDevice, st));
  int64_t nesc = 0;
  if (nnz > 0) {
    int cbits = 1;
    while (cbits < 62 && ((int64_t)1 << cbits) < A->cols) ++cbits;
    int wbits = 1;
    while (((int64_t)1 << wbits) < nwin) ++wbits;
    const uint64_t cmask = ((uint64_t)1 << cbits) - 1;
    PoolBuf key(ctx), skey(ctx), ent(ctx), sent(ctx), tmp(ctx), we0(ctx), twin(ctx), tcol(ctx), eflag(ctx), eidx(ctx);
    SPOPS_TRY(key.alloc((size_t)nnz * 8));
    SPOPS_TRY(skey.alloc((size_t)nnz * 8));
    SPOPS_TRY(ent.alloc((size_t)nnz * 4));
    SPOPS_TRY(sent.alloc((size_t)nnz * 4));
    win_key_kernel<I><<<grid_of(n * 32), 256, 0, st>>>(A->row.as<I>(), A->col.as<I>(), n, W.win_row0.as<int64_t>(),
                                                       nwin, cbits, key.as<uint64_t>(), ent.as<int32_t>());
    SPOPS_LAUNCH_CHECK();
    size_t tb = 0;
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, key.as<uint64_t>(), skey.as<uint64_t>(), ent.as<int32_t>(),
                                               sent.as<int32_t>(), nnz, 0, cbits + wbits, st));
    SPOPS_TRY(tmp.alloc(tb + 256));
    SPOPS_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, key.as<uint64_t>(), skey.as<uint64_t>(), ent.as<int32_t>(),
                                               sent.as<int32_t>(), nnz, 0, cbits + wbits, st));
    key.release();
    ent.release();
    SPOPS_TRY(we0.alloc((size_t)(nwin + 1) * 8));
    SPOPS_CUDA(cudaMemcpyAsync(we0.p, e0.data(), (size_t)(nwin + 1) * 8, cudaMemcpyHostToDevice, st));
    SPOPS_TRY(twin.alloc((size_t)ntiles * 4));
    SPOPS_TRY(tcol.alloc((size_t)ntiles * 8));
    SPOPS_TRY(eflag.alloc((size_t)ntiles * 8));
    SPOPS_TRY(eidx.alloc((size_t)(ntiles + 1) * 8));
    win_tile_kernel<<<grid_of(ntiles), 256, 0, st>>>(skey.as<uint64_t>(), cmask, we0.as<int64_t>(),
                                                    W.win_tile0.as<int64_t>(), nwin, ntiles, twin.as<int32_t>(),
                                                    tcol.as<int64_t>(), eflag.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
    size_t sb = 0;
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, sb, eflag.as<int64_t>(), eidx.as<int64_t>(), ntiles, st));
    SPOPS_TRY(tmp.alloc(sb + 256));
    SPOPS_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, sb, eflag.as<int64_t>(), eidx.as<int64_t>(), ntiles, st));
    int64_t last_idx = 0, last_flag = 0;
    SPOPS_CUDA(cudaMemcpyAsync(&last_idx, eidx.as<int64_t>() + ntiles - 1, 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaMemcpyAsync(&last_flag, eflag.as<int64_t>() + ntiles - 1, 8, cudaMemcpyDeviceToHost, st));
    SPOPS_CUDA(cudaStreamSynchronize(st));
    nesc = last_idx + last_flag;
    SPOPS_TRY(W.tesc.alloc((size_t)std::max<int64_t>(nesc, 1) * 32 * 4));
    win_fill_kernel<I, V><<<grid_of(ntiles * 32), 256, 0, st>>>(
        A->row.as<I>(), A->val.as<V>(), skey.as<uint64_t>(), sent.as<int32_t>(), cmask, W.win_row0.as<int64_t>(),
        we0.as<int64_t>(), W.win_tile0.as<int64_t>(), twin.as<int32_t>(), tcol.as<int64_t>(), eflag.as<int64_t>(),
        eidx.as<int64_t>(), ntiles, W.tbase.as<int32_t>(), W.tidx.as<uint32_t>(), W.tval.as<V>(),
        W.tperm.as<int32_t>(), W.tesc.as<int32_t>());
    SPOPS_LAUNCH_CHECK();
    SPOPS_CUDA(cudaStreamSynchronize(st));
  } else {
    SPOPS_TRY(W.tesc.alloc(128));
  }
  W.nwin = nwin;
  W.ntiles = ntiles;
  W.nesc = nesc;
  W.max_rows = max_rows;
  W.per_sm = per_sm;
  W.values_fresh = true;
  W.ready = true;
  return SPOPS_OK;
}

template <typename V, int kThreads, int kPerSm>
spops_status_t launch_win(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  const CsrWin& W = A->plan.win;
  const size_t smem = std::max<size_t>(16, (size_t)W.max_rows * sizeof(V));
  auto kern = csr_win_kernel<V, kThreads, kPerSm>;
  SPOPS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int64_t grid = std::min<int64_t>(W.nwin, (int64_t)ctx->num_sms * kPerSm);
  if (grid <= 0) return SPOPS_OK;
  kern<<<(unsigned)grid, kThreads, smem, ctx->stream>>>(
      W.win_row0.as<int64_t>(), W.win_tile0.as<int64_t>(), W.nwin, W.tbase.as<int32_t>(), W.tidx.as<uint32_t>(),
      W.tval.as<V>(), W.tesc.as<int32_t>(), static_cast<const V*>(x), (V)alpha, (V)beta, beta == 0.0,
      static_cast<V*>(y));
  SPOPS_LAUNCH_CHECK();
  return SPOPS_OK;
}

template <typename V>
spops_status_t spmv_win_t(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  switch (A->plan.win.per_sm) {
    case 4: return launch_win<V, 256, 4>(ctx, A, alpha, x, beta, y);
    case 2: return launch_win<V, 512, 2>(ctx, A, alpha, x, beta, y);
    default: return launch_win<V, 1024, 1>(ctx, A, alpha, x, beta, y);
  }
}

}  // namespace

void CsrWin::release() {
  win_row0.release(); win_tile0.release(); tbase.release(); tidx.release(); tval.release(); tperm.release();
  tesc.release();
  values_fresh = false;
  nwin = ntiles = nesc = 0;
  max_rows = 0;
  per_sm = 0;
  ready = false;
}

bool csr_win_usable(const Matrix* A) {
  return A->cols <= (int64_t)INT32_MAX && A->nnz <= (int64_t)INT32_MAX;
}

spops_status_t csr_win_spmv(Context* ctx, Matrix* A, int variant, double alpha, const void* x, double beta, void* y) {
  const bool i32 = A->itype == SPOPS_INDEX_I32, f64 = A->vtype == SPOPS_VALUE_F64;
  CsrWin& W = A->plan.win;
  if (!W.ready || W.per_sm != per_sm_of(variant)) {
    spops_status_t s;
    if (i32) s = f64 ? analyse_t<int32_t, double>(ctx, A, variant) : analyse_t<int32_t, float>(ctx, A, variant);
    else s = f64 ? analyse_t<int64_t, double>(ctx, A, variant) : analyse_t<int64_t, float>(ctx, A, variant);
    if (s != SPOPS_OK) {
      W.release();
      return s;
    }
  }
  if (!W.values_fresh) {  // spops_csr_set_values since the plan was built
    const int64_t slots = W.ntiles * 32;
    if (slots > 0) {
      if (f64)
        win_values_kernel<double><<<grid_of(slots), 256, 0, ctx->stream>>>(A->val.as<double>(), W.tperm.as<int32_t>(),
                                                                           slots, W.tval.as<double>());
      else
        win_values_kernel<float><<<grid_of(slots), 256, 0, ctx->stream>>>(A->val.as<float>(), W.tperm.as<int32_t>(),
                                                                          slots, W.tval.as<float>());
      SPOPS_LAUNCH_CHECK();
    }
    W.values_fresh = true;
  }
  return f64 ? spmv_win_t<double>(ctx, A, alpha, x, beta, y) : spmv_win_t<float>(ctx, A, alpha, x, beta, y);
}

}  // namespace spops
