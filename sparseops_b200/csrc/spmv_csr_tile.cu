// CSR SpMV by fixed tiles of entries, summed in registers (the default CSR
// kernel).
//
// The matrix stays in the caller's CSR arrays.  Entries are cut into tiles of
// 32*K consecutive entries; lane l of the warp that owns tile t sums entries
// [t*32K + l*K, +K) -- one 128- or 256-bit load for its columns and values,
// K gathers of x, and a running sum that is cut at every row start inside the
// run.  That is the tile-segmented sum of CSR5 (Liu & Vinter, ICS'15; the
// reference's SpOps_csr5, src/spmv_csr5.cpp:113-457) applied to the plain
// CSR layout: with vector loads each lane's run is already one contiguous
// load, so no transposed copy of the matrix is made, and the products never
// pass through shared memory (the round trip that bounds the segment kernel
// in spmv_csr.cu).
//
// Analysis (once per matrix, csr_tile_analyse):
//   flags[t*32 + l]  bit b set when entry t*32K + l*K + b starts a non-empty row
//   tile_row[t]      row holding the tile's first entry; negative (~row) when
//                    an empty row lies inside the tile ("slow" tile: lanes then
//                    find their rows from the row offsets instead of counting
//                    flags)
//   empty            list of empty rows (y = beta*y for them)
// SpMV (csr_tile_kernel + csr_tile_calibrate_kernel):
//   lane row   = tile_row + number of flags before the lane's first entry
//                (bit-sliced ballots, no shared memory)
//   in-lane    complete rows go straight to y
//   cross-lane heads (before a lane's first flag) are summed by a segmented
//              warp scan into the row of the previous flagged lane
//   cross-tile the row open at a tile's end (open_row, open_sum) receives the
//              heads (carry_in) of the following tiles up to the next tile
//              that starts a row -- a second small kernel, in tile order.
// Summation order depends only on the matrix: results are bit-reproducible.
#include <cub/cub.cuh>

#include <functional>
#include <vector>

#include "bulk_copy.cuh"
#include "csr_tile.cuh"
#include "device_util.cuh"
#include "spops_internal.h"

namespace spops {
namespace {

constexpr int kTileBlock = 256;

inline unsigned grid_of(int64_t work, int threads = 256) {
  int64_t g = (work + threads - 1) / threads;
  return (unsigned)(g < 1 ? 1 : g);
}

// One thread per tile: walk the tile's entries with a row cursor.
template <typename I, int K>
__global__ void tile_build_kernel(const I* __restrict__ rp, int64_t n, int64_t nnz, int64_t tiles,
                                  int64_t* __restrict__ tile_row, uint8_t* __restrict__ flags) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= tiles) return;
  constexpr int T = 32 * K;
  const int64_t e0 = t * T, e1 = (e0 + T < nnz) ? e0 + T : nnz;
  int64_t r = row_holding(rp, n, e0);
  const int64_t r0 = r;
  bool slow = false;
  uint32_t word = 0;  // flags of 4 lanes, written as one 32-bit word
  for (int64_t e = e0; e < e0 + T; ++e) {
    const int q = (int)(e - e0);
    if (e < e1) {
      int steps = 0;
      while ((int64_t)rp[r + 1] <= e) {
        ++r;
        ++steps;
      }
      if (steps > 1) slow = true;  // passed over an empty row inside the tile
      if ((int64_t)rp[r] == e) word |= 1u << (((q / K) & 3) * 8 + (q % K));
    }
    if ((q + 1) % (4 * K) == 0) {
      reinterpret_cast<uint32_t*>(flags)[t * 8 + q / (4 * K)] = word;
      word = 0;
    }
  }
  tile_row[t] = slow ? ~r0 : r0;
}

template <typename I>
__global__ void tile_empty_kernel(const I* __restrict__ rp, int64_t n, int64_t* __restrict__ list,
                                  unsigned long long* __restrict__ count) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r < n && rp[r] == rp[r + 1]) list[atomicAdd(count, 1ULL)] = r;
}

// One warp per tile, grid-stride over tiles.  kPipe: the next tile's columns,
// values and flags are loaded before this tile's gathers are used, so the
// streaming loads of one tile overlap the gathers of the previous one.
template <typename I, typename V, int K, int kMinBlocks, bool kPipe>
__global__ void __launch_bounds__(kTileBlock, kMinBlocks) csr_tile_kernel(
    const I* __restrict__ rp, int64_t n, int64_t nnz, const I* __restrict__ ci, const V* __restrict__ val,
    const int64_t* __restrict__ tile_row, const uint8_t* __restrict__ flags_all, int64_t t_begin, int64_t tiles,
    const V* __restrict__ x, V* __restrict__ y, V alpha, V beta, bool bz, V* __restrict__ carry_in,
    V* __restrict__ open_sum, int64_t* __restrict__ open_row) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (kTileBlock / 32);
  int64_t t = t_begin + blockIdx.x * (int64_t)(kTileBlock / 32) + (threadIdx.x >> 5);
  if (t >= tiles) return;
  I c[K];
  V a[K];
  uint32_t flags = 0;
  int64_t tr = 0;
  if (kPipe) {
    tile_load<I, V, K>(ci, val, nnz, t, lane, c, a);
    flags = flags_all[t * 32 + lane];
    tr = tile_row[t];
  }
  for (; t < tiles; t += nw) {
    if (!kPipe) {
      tile_load<I, V, K>(ci, val, nnz, t, lane, c, a);
      flags = flags_all[t * 32 + lane];
      tr = tile_row[t];
    }
    V p[K];
#pragma unroll
    for (int b = 0; b < K; ++b) p[b] = a[b] * ld_gather(x + c[b]);
    const uint32_t f = flags;
    const int64_t r0 = tr;
    if (kPipe && t + nw < tiles) {
      tile_load<I, V, K>(ci, val, nnz, t + nw, lane, c, a);
      flags = flags_all[(t + nw) * 32 + lane];
      tr = tile_row[t + nw];
    }
    tile_finish<I, V, K>(rp, n, nnz, t, lane, f, r0, p, y, alpha, beta, bz, carry_in, open_sum, open_row);
  }
}

// ---- staged form (csr_variant 10): the matrix stream by bulk copies
// Each warp owns a ring of S slots in shared memory; lane 0 fills a slot with
// one tile's columns, values and row-start flags by three bulk copies
// (cp.async.bulk, completing on the slot's mbarrier) S tiles ahead.  The
// lanes read their runs from the slot, so the only per-entry loads that go
// through the SM's L1 request port are the x gathers.  The gathers of the
// next tile are issued before this tile's products are summed (its columns
// are already in shared memory), so a warp keeps gathers in flight through
// the cross-lane row sums.  The summation order is that of csr_tile_kernel
// (results agree to rounding: the compiler may fuse a product into its sum in
// one kernel and not in the other).  The partial last tile, if any, is read
// with plain loads.
template <typename I, typename V>
struct alignas(16) StageSlot {
  I col[256];
  V val[256];
  uint8_t flags[32];
};

template <typename I, typename V, int S>
struct alignas(128) StageRing {
  StageSlot<I, V> slot[S];
  unsigned long long bar[S];
};

// A lane's 32-byte run from a slot, its two 16-byte halves read in an order
// that spreads the 32 lanes over all banks (8 lanes per 128 bytes).
__device__ __forceinline__ void slot_run32(const void* base, int lane, uint4& q0, uint4& q1) {
  const uint4* p = reinterpret_cast<const uint4*>(base);
  const int h = (lane >> 2) & 1;
  const uint4 a = p[h], b = p[h ^ 1];
  q0 = h ? b : a;
  q1 = h ? a : b;
}

// A lane's 64-byte run, its four 16-byte quarters read rotated by
// (lane >> 1) & 3 for the same reason.
__device__ __forceinline__ void slot_run64(const void* base, int lane, uint4 (&q)[4]) {
  const uint4* p = reinterpret_cast<const uint4*>(base);
  const int r = (lane >> 1) & 3;
  uint4 w0 = p[r], w1 = p[(r + 1) & 3], w2 = p[(r + 2) & 3], w3 = p[(r + 3) & 3];
  if (r & 1) {  // rotate right by one
    const uint4 t = w3;
    w3 = w2;
    w2 = w1;
    w1 = w0;
    w0 = t;
  }
  if (r & 2) {  // and by two
    uint4 t = w0;
    w0 = w2;
    w2 = t;
    t = w1;
    w1 = w3;
    w3 = t;
  }
  q[0] = w0;
  q[1] = w1;
  q[2] = w2;
  q[3] = w3;
}

template <typename T, int K>
__device__ __forceinline__ void slot_read(const T* base, int lane, T (&out)[K]) {
  static_assert(K * sizeof(T) == 32 || K * sizeof(T) == 64, "runs of 32 or 64 bytes");
  if constexpr (K * sizeof(T) == 32) {
    uint4 q[2];
    slot_run32(base + lane * K, lane, q[0], q[1]);
    memcpy(out, q, 32);
  } else {
    uint4 q[4];
    slot_run64(base + lane * K, lane, q);
    memcpy(out, q, 64);
  }
}

constexpr int kStageWarps = 4;

template <typename I, typename V, int S, int kMinBlocks>
__global__ void __launch_bounds__(kStageWarps * 32, kMinBlocks) csr_stage_kernel(
    const I* __restrict__ rp, int64_t n, int64_t nnz, const I* __restrict__ ci, const V* __restrict__ val,
    const int64_t* __restrict__ tile_row, const uint8_t* __restrict__ flags_all, int64_t tiles,
    const V* __restrict__ x, V* __restrict__ y, V alpha, V beta, bool bz, V* __restrict__ carry_in,
    V* __restrict__ open_sum, int64_t* __restrict__ open_row, int* __restrict__ err) {
  constexpr int K = 8;
  constexpr uint32_t kColB = 32 * K * sizeof(I), kValB = 32 * K * sizeof(V), kTx = kColB + kValB + 32;
  using Ring = StageRing<I, V, S>;
  extern __shared__ __align__(128) unsigned char stage_smem[];
  const int lane = threadIdx.x & 31;
  Ring& R = reinterpret_cast<Ring*>(stage_smem)[threadIdx.x >> 5];
  const int64_t nw = (int64_t)gridDim.x * kStageWarps;
  int64_t t = blockIdx.x * (int64_t)kStageWarps + (threadIdx.x >> 5);
  if (t >= tiles) return;
  const int64_t full = nnz / (32 * K);  // tiles [0, full) come by bulk copies
  const uint32_t bar0 = smem_u32(&R.bar[0]);
  if (lane == 0) {
#pragma unroll
    for (int s = 0; s < S; ++s) mbar_init(bar0 + 8 * s, 1);
    mbar_init_fence();
  }
  __syncwarp();
  uint32_t pend = 0, phase = 0;  // per slot: a copy in flight; the parity its completion has
  auto issue = [&](int64_t tt, int s) {
    if (tt < full) {
      pend |= 1u << s;
      if (lane == 0) {
        const uint32_t b = bar0 + 8 * s;
        mbar_arrive_expect(b, kTx);
        bulk_g2s(smem_u32(R.slot[s].col), ci + tt * (32 * K), kColB, b);
        bulk_g2s(smem_u32(R.slot[s].val), val + tt * (32 * K), kValB, b);
        bulk_g2s(smem_u32(R.slot[s].flags), flags_all + tt * 32, 32, b);
      }
    }
  };
  auto wait = [&](int s) {
    const bool ok = mbar_wait_bounded(bar0 + 8 * s, (phase >> s) & 1u);
    phase ^= 1u << s;
    pend &= ~(1u << s);
    return __all_sync(0xffffffffu, ok);
  };
  auto give_up = [&]() {  // a copy did not complete in time: flag it, let the others land, leave
    if (lane == 0) atomicOr(err, 1);
#pragma unroll
    for (int s = 0; s < S; ++s)
      if ((pend >> s) & 1u) mbar_wait_bounded(bar0 + 8 * s, (phase >> s) & 1u);
  };
#pragma unroll
  for (int q = 0; q < S; ++q)
    if (t + q * nw < tiles) issue(t + q * nw, q);
  I c[K];
  V xv[K], xn[K];
  auto columns = [&](int64_t tt, int s) {
    if (tt < full) {
      slot_read<I, K>(R.slot[s].col, lane, c);
    } else {
      const int64_t el = tt * (32 * K) + (int64_t)lane * K;
#pragma unroll
      for (int b = 0; b < K; ++b) c[b] = el + b < nnz ? ci[el + b] : I(0);
    }
  };
  int s = 0;
  if (t < full && !wait(0)) return give_up();
  columns(t, 0);
#pragma unroll
  for (int b = 0; b < K; ++b) xv[b] = ld_gather(x + c[b]);
  while (true) {
    const int64_t tn = t + nw;
    const int sn = s + 1 == S ? 0 : s + 1;
    const int64_t tr = tile_row[t];
    V a[K];
    uint32_t f;
    if (t < full) {
      slot_read<V, K>(R.slot[s].val, lane, a);
      f = R.slot[s].flags[lane];
    } else {
      const int64_t el = t * (32 * K) + (int64_t)lane * K;
#pragma unroll
      for (int b = 0; b < K; ++b) a[b] = el + b < nnz ? val[el + b] : V(0);
      f = flags_all[t * 32 + lane];
    }
    const bool more = tn < tiles;
    if (more) {
      if (tn < full && !wait(sn)) return give_up();
      columns(tn, sn);
#pragma unroll
      for (int b = 0; b < K; ++b) xn[b] = ld_gather(x + c[b]);
    }
    __syncwarp();  // every lane is done with slot s
    if (t + S * nw < tiles) {
      if (lane == 0) fence_proxy_async_smem();
      issue(t + S * nw, s);
    }
    V p[K];
#pragma unroll
    for (int b = 0; b < K; ++b) p[b] = a[b] * xv[b];
    tile_finish<I, V, K>(rp, n, nnz, t, lane, f, tr, p, y, alpha, beta, bz, carry_in, open_sum, open_row);
    if (!more) break;
    t = tn;
    s = sn;
#pragma unroll
    for (int b = 0; b < K; ++b) xv[b] = xn[b];
  }
}

// The same SpMV with each value read through a permutation: value e is
// vsrc[perm[e]].  For A^T g while A's values change every step: A^T's
// values are A's, reordered, and reading them through the permutation inside
// the SpMV skips writing and re-reading the reordered copy.  The products and
// their order are those of the plain kernel on the reordered copy.
template <typename I, typename V>
__global__ void __launch_bounds__(kTileBlock, 3) csr_tile_indirect_kernel(
    const I* __restrict__ rp, int64_t n, int64_t nnz, const I* __restrict__ ci, const int64_t* __restrict__ perm,
    const V* __restrict__ vsrc, const int64_t* __restrict__ tile_row, const uint8_t* __restrict__ flags_all,
    int64_t tiles, const V* __restrict__ x, V* __restrict__ y, V alpha, V beta, bool bz, V* __restrict__ carry_in,
    V* __restrict__ open_sum, int64_t* __restrict__ open_row) {
  constexpr int K = 8;
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (kTileBlock / 32);
  int64_t t = blockIdx.x * (int64_t)(kTileBlock / 32) + (threadIdx.x >> 5);
  if (t >= tiles) return;
  I c[K];
  int64_t pm[K];
  uint32_t flags = 0;
  int64_t tr = 0;
  auto load = [&](int64_t tt) {
    const int64_t el = tt * (32 * K) + (int64_t)lane * K;
    if (el + K <= nnz) {
      load_run<I, K>(ci + el, c);
      load_run<int64_t, K>(perm + el, pm);
    } else {
#pragma unroll
      for (int b = 0; b < K; ++b) {
        const bool in = el + b < nnz;
        c[b] = in ? ci[el + b] : I(0);
        pm[b] = in ? perm[el + b] : 0;
      }
    }
    flags = flags_all[tt * 32 + lane];
    tr = tile_row[tt];
  };
  load(t);
  for (; t < tiles; t += nw) {
    const int64_t el = t * (32 * K) + (int64_t)lane * K;
    V p[K];
#pragma unroll
    for (int b = 0; b < K; ++b) {
      const V a = el + b < nnz ? ld_gather(vsrc + pm[b]) : V(0);
      p[b] = a * ld_gather(x + c[b]);
    }
    const uint32_t f = flags;
    const int64_t r0 = tr;
    if (t + nw < tiles) load(t + nw);
    tile_finish<I, V, K>(rp, n, nnz, t, lane, f, r0, p, y, alpha, beta, bz, carry_in, open_sum, open_row);
  }
}

// Rows open at a tile's end receive the heads of the following tiles up to the
// first one that starts a row; empty rows get y = beta*y.  Tiles [t_begin,
// tiles) only: a range ends where a row starts, so no chain crosses it.
template <typename V>
__global__ void csr_tile_calibrate_kernel(int64_t t_begin, int64_t tiles, const V* __restrict__ carry_in,
                                          const V* __restrict__ open_sum, const int64_t* __restrict__ open_row,
                                          const int64_t* __restrict__ empty, int64_t nempty, V* __restrict__ y,
                                          V alpha, V beta, bool bz) {
  const int64_t t = t_begin + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < tiles) {
    const int64_t r = open_row[t];
    if (r < 0) return;
    V tot = open_sum[t];
    for (int64_t u = t + 1; u < tiles; ++u) {
      tot += carry_in[u];
      if (open_row[u] >= 0) break;
    }
    axpby_store(y + r, tot, alpha, beta, bz);
  } else if (t - tiles < nempty) {
    axpby_store(y + empty[t - tiles], V(0), alpha, beta, bz);
  }
}

// ---- multi-RHS with k = 4G on the same tile plan (csr_tile_spmm); the
// per-tile work is spmm_tile_groups (csr_tile.cuh)
template <typename I, typename V, int G>
__global__ void __launch_bounds__(kTileBlock, 2) csr_tile_spmm_kernel(
    const I* __restrict__ rp, int64_t n, int64_t nnz, const I* __restrict__ ci, const V* __restrict__ val,
    const int64_t* __restrict__ tile_row, const uint8_t* __restrict__ flags_all, int64_t tiles,
    const V* __restrict__ X, int64_t ldx, V* __restrict__ Y, int64_t ldy, V alpha, V beta, bool bz,
    V* __restrict__ carry_in, V* __restrict__ open_sum, int64_t* __restrict__ open_row) {
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (kTileBlock / 32);
  for (int64_t t = blockIdx.x * (int64_t)(kTileBlock / 32) + (threadIdx.x >> 5); t < tiles; t += nw)
    spmm_tile_groups<I, V, G>(rp, n, nnz, ci, val, tile_row, flags_all, t, X, ldx, Y, ldy, alpha, beta, bz,
                              carry_in, open_sum, open_row, lane);
}

template <typename V, int KC>
__global__ void csr_tile_calibrate_k_kernel(int64_t tiles, const V* __restrict__ carry_in,
                                            const V* __restrict__ open_sum, const int64_t* __restrict__ open_row,
                                            const int64_t* __restrict__ empty, int64_t nempty, V* __restrict__ Y,
                                            int64_t ldy, V alpha, V beta, bool bz) {
  spmm_calibrate<V, KC>(blockIdx.x * (int64_t)blockDim.x + threadIdx.x, tiles, carry_in, open_sum, open_row, empty,
                        nempty, Y, ldy, alpha, beta, bz);
}

template <typename I, typename V, int G>
spops_status_t spmm_tiles_t(Context* ctx, Matrix* A, double alpha, const void* X, int64_t ldx, double beta, void* Y,
                            int64_t ldy) {
  constexpr int KC = 4 * G;
  const CsrTiles& D = A->plan.tiles;
  const bool bz = beta == 0.0;
  PoolBuf cin(ctx), osum(ctx);
  const size_t nt1 = (size_t)(D.tiles > 0 ? D.tiles : 1);
  SPOPS_TRY(cin.alloc(nt1 * KC * sizeof(V)));
  SPOPS_TRY(osum.alloc(nt1 * KC * sizeof(V)));
  if (D.tiles > 0) {
    static int blocks_per_sm = -1;  // per instantiation
    if (blocks_per_sm < 0) {
      int bps = 0;
      SPOPS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, csr_tile_spmm_kernel<I, V, G>, kTileBlock, 0));
      blocks_per_sm = bps > 0 ? bps : 1;
    }
    int64_t grid = (int64_t)ctx->num_sms * blocks_per_sm;
    const int64_t need = (D.tiles + kTileBlock / 32 - 1) / (kTileBlock / 32);
    if (grid > need) grid = need;
    csr_tile_spmm_kernel<I, V, G><<<(unsigned)grid, kTileBlock, 0, ctx->stream>>>(
        A->row.as<I>(), A->rows, A->nnz, A->col.as<I>(), A->val.as<V>(), D.tile_row.as<int64_t>(),
        D.flags.as<uint8_t>(), D.tiles, static_cast<const V*>(X), ldx, static_cast<V*>(Y), ldy, (V)alpha, (V)beta,
        bz, cin.as<V>(), osum.as<V>(), D.open_row.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
  }
  if (D.tiles + D.nempty > 0) {
    csr_tile_calibrate_k_kernel<V, KC><<<grid_of(D.tiles + D.nempty), 256, 0, ctx->stream>>>(
        D.tiles, cin.as<V>(), osum.as<V>(), D.open_row.as<int64_t>(), D.empty.as<int64_t>(), D.nempty,
        static_cast<V*>(Y), ldy, (V)alpha, (V)beta, bz);
    SPOPS_LAUNCH_CHECK();
  }
  return SPOPS_OK;
}

template <typename I, typename V>
spops_status_t spmm_tiles_k(Context* ctx, Matrix* A, double alpha, const void* X, int64_t ldx, int64_t k,
                            double beta, void* Y, int64_t ldy) {
  if (k == 8) return spmm_tiles_t<I, V, 2>(ctx, A, alpha, X, ldx, beta, Y, ldy);
  if (k == 16) return spmm_tiles_t<I, V, 4>(ctx, A, alpha, X, ldx, beta, Y, ldy);
  return spmm_tiles_t<I, V, 8>(ctx, A, alpha, X, ldx, beta, Y, ldy);
}

// Boundaries of `parts` tile ranges for the pipelined host SpMV: range p
// starts at the first tile at or after p * tiles / parts whose first entry
// starts a row (so every row lies in one range), and rb[p] is that row.
template <typename I, int K>
__global__ void part_bounds_kernel(const I* __restrict__ rp, int64_t n, const uint8_t* __restrict__ flags,
                                   int64_t tiles, int parts, int64_t* __restrict__ tb, int64_t* __restrict__ rb) {
  const int p = threadIdx.x;
  if (p > parts) return;
  if (p == 0 || p == parts) {
    tb[p] = p == 0 ? 0 : tiles;
    rb[p] = p == 0 ? 0 : n;
    return;
  }
  int64_t t = tiles * p / parts;
  while (t < tiles && !(flags[t * 32] & 1u)) ++t;
  tb[p] = t;
  rb[p] = t < tiles ? row_holding(rp, n, t * (32 * K)) : n;
}

template <int K>
int64_t tiles_of(int64_t nnz) {
  return (nnz + 32 * K - 1) / (32 * K);
}

template <typename I, int K>
spops_status_t analyse_t(Context* ctx, Matrix* A) {
  CsrTiles& D = A->plan.tiles;
  cudaStream_t st = ctx->stream;
  const int64_t n = A->rows, nnz = A->nnz;
  D.release();
  D.k = K;
  D.tiles = tiles_of<K>(nnz);
  const size_t nt1 = (size_t)(D.tiles > 0 ? D.tiles : 1);
  SPOPS_TRY(D.tile_row.alloc(nt1 * 8));
  SPOPS_TRY(D.flags.alloc(nt1 * 32));
  SPOPS_TRY(D.carry_in.alloc(nt1 * 8));
  SPOPS_TRY(D.open_sum.alloc(nt1 * 8));
  SPOPS_TRY(D.open_row.alloc(nt1 * 8));
  SPOPS_TRY(D.empty.alloc((size_t)(n > 0 ? n : 1) * 8));
  if (D.tiles > 0 && n > 0) {
    tile_build_kernel<I, K><<<grid_of(D.tiles), 256, 0, st>>>(A->row.as<I>(), n, nnz, D.tiles,
                                                                D.tile_row.as<int64_t>(), D.flags.as<uint8_t>());
    SPOPS_LAUNCH_CHECK();
  }
  SPOPS_TRY(ctx->scratch_reserve(256));
  unsigned long long* cnt = ctx->scratch.as<unsigned long long>();
  SPOPS_CUDA(cudaMemsetAsync(cnt, 0, 8, st));
  if (n > 0) {
    tile_empty_kernel<I><<<grid_of(n), 256, 0, st>>>(A->row.as<I>(), n, D.empty.as<int64_t>(), cnt);
    SPOPS_LAUNCH_CHECK();
  }
  unsigned long long h = 0;
  SPOPS_CUDA(cudaMemcpyAsync(&h, cnt, 8, cudaMemcpyDeviceToHost, st));
  SPOPS_CUDA(cudaStreamSynchronize(st));
  D.nempty = (int64_t)h;
  D.ready = true;
  return SPOPS_OK;
}

// Tiles [t0, t1) and their calibration; the empty rows when `empty_rows`.
template <typename I, typename V, int K, int kMinBlocks, bool kPipe>
spops_status_t spmv_range(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y, int64_t t0,
                          int64_t t1, bool empty_rows) {
  const CsrTiles& D = A->plan.tiles;
  const bool bz = beta == 0.0;
  if (t1 > t0) {
    static int blocks_per_sm = -1;  // per instantiation
    if (blocks_per_sm < 0) {
      int bps = 0;
      SPOPS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, csr_tile_kernel<I, V, K, kMinBlocks, kPipe>,
                                                               kTileBlock, 0));
      blocks_per_sm = bps > 0 ? bps : 1;
    }
    int64_t grid = (int64_t)ctx->num_sms * blocks_per_sm;
    const int64_t need = (t1 - t0 + kTileBlock / 32 - 1) / (kTileBlock / 32);
    if (grid > need) grid = need;
    csr_tile_kernel<I, V, K, kMinBlocks, kPipe><<<(unsigned)grid, kTileBlock, 0, ctx->stream>>>(
        A->row.as<I>(), A->rows, A->nnz, A->col.as<I>(), A->val.as<V>(), D.tile_row.as<int64_t>(),
        D.flags.as<uint8_t>(), t0, t1, static_cast<const V*>(x), static_cast<V*>(y), (V)alpha, (V)beta, bz,
        D.carry_in.as<V>(), D.open_sum.as<V>(), D.open_row.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
  }
  const int64_t ne = empty_rows ? D.nempty : 0;
  if (t1 - t0 + ne > 0) {
    csr_tile_calibrate_kernel<V><<<grid_of(t1 - t0 + ne), 256, 0, ctx->stream>>>(
        t0, t1, D.carry_in.as<V>(), D.open_sum.as<V>(), D.open_row.as<int64_t>(), D.empty.as<int64_t>(), ne,
        static_cast<V*>(y), (V)alpha, (V)beta, bz);
    SPOPS_LAUNCH_CHECK();
  }
  return SPOPS_OK;
}

// The staged kernel over all tiles, then the calibration.
template <typename I, typename V, int S, int kMinBlocks>
spops_status_t spmv_stage_t(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  const CsrTiles& D = A->plan.tiles;
  const bool bz = beta == 0.0;
  const int64_t tiles = D.tiles;
  if (tiles > 0) {
    SPOPS_TRY(ctx->ensure_errword());
    constexpr size_t smem = kStageWarps * sizeof(StageRing<I, V, S>);
    static int blocks_per_sm = -1;  // per instantiation
    if (blocks_per_sm < 0) {
      SPOPS_CUDA(cudaFuncSetAttribute(csr_stage_kernel<I, V, S, kMinBlocks>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      int bps = 0;
      SPOPS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, csr_stage_kernel<I, V, S, kMinBlocks>,
                                                               kStageWarps * 32, smem));
      blocks_per_sm = bps > 0 ? bps : 1;
    }
    int64_t grid = (int64_t)ctx->num_sms * blocks_per_sm;
    const int64_t need = (tiles + kStageWarps - 1) / kStageWarps;
    if (grid > need) grid = need;
    csr_stage_kernel<I, V, S, kMinBlocks><<<(unsigned)grid, kStageWarps * 32, smem, ctx->stream>>>(
        A->row.as<I>(), A->rows, A->nnz, A->col.as<I>(), A->val.as<V>(), D.tile_row.as<int64_t>(),
        D.flags.as<uint8_t>(), tiles, static_cast<const V*>(x), static_cast<V*>(y), (V)alpha, (V)beta, bz,
        D.carry_in.as<V>(), D.open_sum.as<V>(), D.open_row.as<int64_t>(), ctx->errword.as<int>());
    SPOPS_LAUNCH_CHECK();
  }
  if (tiles + D.nempty > 0) {
    csr_tile_calibrate_kernel<V><<<grid_of(tiles + D.nempty), 256, 0, ctx->stream>>>(
        0, tiles, D.carry_in.as<V>(), D.open_sum.as<V>(), D.open_row.as<int64_t>(), D.empty.as<int64_t>(), D.nempty,
        static_cast<V*>(y), (V)alpha, (V)beta, bz);
    SPOPS_LAUNCH_CHECK();
  }
  return SPOPS_OK;
}

template <typename I, typename V, int K, int kMinBlocks, bool kPipe>
spops_status_t spmv_t(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y) {
  return spmv_range<I, V, K, kMinBlocks, kPipe>(ctx, A, alpha, x, beta, y, 0, A->plan.tiles.tiles, true);
}

// y in `parts` row ranges; after each range, done(r0, r1) with the stream
// position at which rows [r0, r1) of y are final.
template <typename I, typename V>
spops_status_t spmv_parts_t(Context* ctx, Matrix* A, double alpha, const void* x, double beta, void* y,
                            const std::vector<int64_t>& tb, const std::vector<int64_t>& rb,
                            const std::function<spops_status_t(int64_t, int64_t)>& done) {
  const int parts = (int)tb.size() - 1;
  for (int p = 0; p < parts; ++p) {
    if (rb[p + 1] <= rb[p] && tb[p + 1] <= tb[p] && p > 0) continue;
    SPOPS_TRY((spmv_range<I, V, 8, 3, true>(ctx, A, alpha, x, beta, y, tb[p], tb[p + 1], p == 0)));
    if (rb[p + 1] > rb[p]) SPOPS_TRY(done(rb[p], rb[p + 1]));
  }
  return SPOPS_OK;
}

template <typename I, typename V>
spops_status_t spmv_indirect_t(Context* ctx, Matrix* A, const int64_t* perm, const void* vsrc, double alpha,
                               const void* x, double beta, void* y) {
  const CsrTiles& D = A->plan.tiles;
  const bool bz = beta == 0.0;
  const int64_t tiles = D.tiles;
  if (tiles > 0) {
    static int blocks_per_sm = -1;  // per instantiation
    if (blocks_per_sm < 0) {
      int bps = 0;
      SPOPS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, csr_tile_indirect_kernel<I, V>, kTileBlock, 0));
      blocks_per_sm = bps > 0 ? bps : 1;
    }
    int64_t grid = (int64_t)ctx->num_sms * blocks_per_sm;
    const int64_t need = (tiles + kTileBlock / 32 - 1) / (kTileBlock / 32);
    if (grid > need) grid = need;
    csr_tile_indirect_kernel<I, V><<<(unsigned)grid, kTileBlock, 0, ctx->stream>>>(
        A->row.as<I>(), A->rows, A->nnz, A->col.as<I>(), perm, static_cast<const V*>(vsrc),
        D.tile_row.as<int64_t>(), D.flags.as<uint8_t>(), tiles, static_cast<const V*>(x), static_cast<V*>(y),
        (V)alpha, (V)beta, bz, D.carry_in.as<V>(), D.open_sum.as<V>(), D.open_row.as<int64_t>());
    SPOPS_LAUNCH_CHECK();
  }
  if (tiles + D.nempty > 0) {
    csr_tile_calibrate_kernel<V><<<grid_of(tiles + D.nempty), 256, 0, ctx->stream>>>(
        0, tiles, D.carry_in.as<V>(), D.open_sum.as<V>(), D.open_row.as<int64_t>(), D.empty.as<int64_t>(), D.nempty,
        static_cast<V*>(y), (V)alpha, (V)beta, bz);
    SPOPS_LAUNCH_CHECK();
  }
  return SPOPS_OK;
}

// Kernel shape by variant: (entries per lane, resident blocks, pipelined).
template <typename I, typename V>
spops_status_t dispatch(Context* ctx, Matrix* A, int variant, double alpha, const void* x, double beta, void* y) {
  switch (variant) {
    case 1: return spmv_t<I, V, 8, 4, false>(ctx, A, alpha, x, beta, y);
    case 5: return spmv_t<I, V, 4, 4, false>(ctx, A, alpha, x, beta, y);
    case 6: return spmv_t<I, V, 8, 5, false>(ctx, A, alpha, x, beta, y);
    case 10: return spmv_stage_t<I, V, 2, 6>(ctx, A, alpha, x, beta, y);
    default: return spmv_t<I, V, 8, 3, true>(ctx, A, alpha, x, beta, y);
  }
}

}  // namespace

void CsrTiles::release() {
  tile_row.release(); flags.release(); carry_in.release(); open_sum.release(); open_row.release(); empty.release();
  part_tb.clear();
  part_rb.clear();
  tiles = 0;
  nempty = 0;
  k = 0;
  ready = false;
}

int csr_tile_k(int variant) { return variant == 5 ? 4 : 8; }

bool csr_tile_usable(const Matrix* A, int variant) {
  // vector loads need each lane's run aligned: run bytes (capped at 32)
  const size_t k = (size_t)csr_tile_k(variant);
  const size_t ca = k * A->isize() >= 32 ? 32 : k * A->isize();
  const size_t va = k * A->vsize() >= 32 ? 32 : k * A->vsize();
  return ((uintptr_t)A->col.p % ca) == 0 && ((uintptr_t)A->val.p % va) == 0;
}

spops_status_t csr_tile_analyse(Context* ctx, Matrix* A, int k) {
  const bool i32 = A->itype == SPOPS_INDEX_I32;
  if (k == 8) return i32 ? analyse_t<int32_t, 8>(ctx, A) : analyse_t<int64_t, 8>(ctx, A);
  return i32 ? analyse_t<int32_t, 4>(ctx, A) : analyse_t<int64_t, 4>(ctx, A);
}

spops_status_t csr_tile_spmv_parts(Context* ctx, Matrix* A, int parts, double alpha, const void* x, double beta,
                                   void* y, const std::function<spops_status_t(int64_t, int64_t)>& done) {
  if (!A->plan.tiles.ready || A->plan.tiles.k != 8) SPOPS_TRY(csr_tile_analyse(ctx, A, 8));
  CsrTiles& D = A->plan.tiles;
  const bool i32 = A->itype == SPOPS_INDEX_I32, f64 = A->vtype == SPOPS_VALUE_F64;
  if ((int)D.part_tb.size() != parts + 1) {  // boundaries, once per matrix and part count
    SPOPS_TRY(ctx->scratch_reserve((size_t)(2 * parts + 2) * 8));
    int64_t* tb = ctx->scratch.as<int64_t>();
    int64_t* rb = tb + parts + 1;
    if (i32)
      part_bounds_kernel<int32_t, 8><<<1, 64, 0, ctx->stream>>>(A->row.as<int32_t>(), A->rows, D.flags.as<uint8_t>(),
                                                                D.tiles, parts, tb, rb);
    else
      part_bounds_kernel<int64_t, 8><<<1, 64, 0, ctx->stream>>>(A->row.as<int64_t>(), A->rows, D.flags.as<uint8_t>(),
                                                                D.tiles, parts, tb, rb);
    SPOPS_LAUNCH_CHECK();
    std::vector<int64_t> h((size_t)(2 * parts + 2));
    SPOPS_CUDA(cudaMemcpyAsync(h.data(), tb, h.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    SPOPS_CUDA(cudaStreamSynchronize(ctx->stream));
    D.part_tb.assign(h.begin(), h.begin() + parts + 1);
    D.part_rb.assign(h.begin() + parts + 1, h.end());
  }
  if (i32 && f64) return spmv_parts_t<int32_t, double>(ctx, A, alpha, x, beta, y, D.part_tb, D.part_rb, done);
  if (i32) return spmv_parts_t<int32_t, float>(ctx, A, alpha, x, beta, y, D.part_tb, D.part_rb, done);
  if (f64) return spmv_parts_t<int64_t, double>(ctx, A, alpha, x, beta, y, D.part_tb, D.part_rb, done);
  return spmv_parts_t<int64_t, float>(ctx, A, alpha, x, beta, y, D.part_tb, D.part_rb, done);
}

bool csr_tile_spmm_usable(const Matrix* A, const void* X, int64_t ldx, int64_t k) {
  const size_t vs = A->vsize();
  return (k == 8 || k == 16 || k == 32) && A->rows > 0 && A->nnz > 0 && csr_tile_usable(A, 0) &&
         ((uintptr_t)X % 32) == 0 && ((size_t)ldx * vs) % 32 == 0 && ldx >= k && ldx <= 2 * k;
}

spops_status_t csr_tile_spmm(Context* ctx, Matrix* A, double alpha, const void* X, int64_t ldx, int64_t k,
                             double beta, void* Y, int64_t ldy, bool* used) {
  *used = false;
  if (!csr_tile_spmm_usable(A, X, ldx, k) || ldy < k) return SPOPS_OK;
  if (!A->plan.tiles.ready || A->plan.tiles.k != 8) SPOPS_TRY(csr_tile_analyse(ctx, A, 8));
  *used = true;
  const bool i32 = A->itype == SPOPS_INDEX_I32, f64 = A->vtype == SPOPS_VALUE_F64;
  if (i32 && f64) return spmm_tiles_k<int32_t, double>(ctx, A, alpha, X, ldx, k, beta, Y, ldy);
  if (i32) return spmm_tiles_k<int32_t, float>(ctx, A, alpha, X, ldx, k, beta, Y, ldy);
  if (f64) return spmm_tiles_k<int64_t, double>(ctx, A, alpha, X, ldx, k, beta, Y, ldy);
  return spmm_tiles_k<int64_t, float>(ctx, A, alpha, X, ldx, k, beta, Y, ldy);
}

spops_status_t csr_tile_spmv_indirect(Context* ctx, Matrix* A, const int64_t* perm, const void* vsrc, double alpha,
                                      const void* x, double beta, void* y) {
  if (!A->plan.tiles.ready || A->plan.tiles.k != 8) SPOPS_TRY(csr_tile_analyse(ctx, A, 8));
  const bool i32 = A->itype == SPOPS_INDEX_I32, f64 = A->vtype == SPOPS_VALUE_F64;
  if (i32 && f64) return spmv_indirect_t<int32_t, double>(ctx, A, perm, vsrc, alpha, x, beta, y);
  if (i32) return spmv_indirect_t<int32_t, float>(ctx, A, perm, vsrc, alpha, x, beta, y);
  if (f64) return spmv_indirect_t<int64_t, double>(ctx, A, perm, vsrc, alpha, x, beta, y);
  return spmv_indirect_t<int64_t, float>(ctx, A, perm, vsrc, alpha, x, beta, y);
}

spops_status_t csr_tile_spmv(Context* ctx, Matrix* A, int variant, double alpha, const void* x, double beta,
                             void* y) {
  const int k = csr_tile_k(variant);
  if (!A->plan.tiles.ready || A->plan.tiles.k != k) SPOPS_TRY(csr_tile_analyse(ctx, A, k));
  const bool i32 = A->itype == SPOPS_INDEX_I32, f64 = A->vtype == SPOPS_VALUE_F64;
  if (i32 && f64) return dispatch<int32_t, double>(ctx, A, variant, alpha, x, beta, y);
  if (i32) return dispatch<int32_t, float>(ctx, A, variant, alpha, x, beta, y);
  if (f64) return dispatch<int64_t, double>(ctx, A, variant, alpha, x, beta, y);
  return dispatch<int64_t, float>(ctx, A, variant, alpha, x, beta, y);
}

}  // namespace spops
